// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_df30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<3, 0, 0, 1, true, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<3, 0, 1, 2, true, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<3, 0, 2, 2, true, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<3, 0, 3, 5, true, false, 1, float, false><<<dim3((unsigned)nblk, 5), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<3, 0, 4, 5, true, false, 1, float, false><<<dim3((unsigned)nblk, 5), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<3, 0, 5, 7, true, false, 1, float, false><<<dim3((unsigned)nblk, 7), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<3, 0, 6, 10, true, false, 1, float, false><<<dim3((unsigned)nblk, 10), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
