// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_if33_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<3, 3, 0, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<3, 3, 1, 3, false, false, 1, float, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<3, 3, 2, 6, false, false, 1, float, false><<<dim3((unsigned)nblk, 6), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<3, 3, 3, 10, false, false, 1, float, false><<<dim3((unsigned)nblk, 10), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<3, 3, 4, 15, false, false, 1, float, false><<<dim3((unsigned)nblk, 15), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<3, 3, 5, 21, false, false, 1, float, false><<<dim3((unsigned)nblk, 21), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<3, 3, 6, 28, false, false, 1, float, false><<<dim3((unsigned)nblk, 28), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
