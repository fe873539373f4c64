// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_if22_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<2, 2, 0, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<2, 2, 1, 2, false, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<2, 2, 2, 3, false, false, 1, float, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<2, 2, 3, 5, false, false, 1, float, false><<<dim3((unsigned)nblk, 5), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<2, 2, 4, 8, false, false, 1, float, false><<<dim3((unsigned)nblk, 8), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<2, 2, 5, 11, false, false, 1, float, false><<<dim3((unsigned)nblk, 11), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<2, 2, 6, 14, false, false, 1, float, false><<<dim3((unsigned)nblk, 14), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
