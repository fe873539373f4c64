// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_d0_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    (void)la;
    if (lb == 0 && lc == 0) {
        k_rys_thread<0, 0, 0, 1, true, false, 1><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 1) {
        k_rys_thread<0, 0, 1, 1, true, false, 1><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 2) {
        k_rys_thread<0, 0, 2, 2, true, false, 1><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 3) {
        k_rys_thread<0, 0, 3, 2, true, false, 1><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 4) {
        k_rys_thread<0, 0, 4, 2, true, false, 1><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 5) {
        k_rys_thread<0, 0, 5, 3, true, false, 1><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lb == 0 && lc == 6) {
        k_rys_thread<0, 0, 6, 6, true, false, 1><<<dim3((unsigned)nblk, 6), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
