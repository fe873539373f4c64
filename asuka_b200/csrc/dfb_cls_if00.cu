// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_if00_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<0, 0, 0, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<0, 0, 1, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<0, 0, 2, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<0, 0, 3, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<0, 0, 4, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<0, 0, 5, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<0, 0, 6, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
