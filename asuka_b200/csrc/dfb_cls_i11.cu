// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_i11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<1, 1, 0, 1, false, false, 1, double, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<1, 1, 1, 1, false, false, 1, double, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<1, 1, 2, 2, false, false, 1, double, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<1, 1, 3, 3, false, false, 1, double, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<1, 1, 4, 4, false, false, 1, double, false><<<dim3((unsigned)nblk, 4), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<1, 1, 5, 6, false, false, 1, double, false><<<dim3((unsigned)nblk, 6), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<1, 1, 6, 7, false, false, 1, double, false><<<dim3((unsigned)nblk, 7), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
