// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_df11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<1, 1, 0, 1, true, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<1, 1, 1, 2, true, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<1, 1, 2, 2, true, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<1, 1, 3, 4, true, false, 1, float, false><<<dim3((unsigned)nblk, 4), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<1, 1, 4, 4, true, false, 1, float, false><<<dim3((unsigned)nblk, 4), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<1, 1, 5, 11, true, false, 1, float, false><<<dim3((unsigned)nblk, 11), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<1, 1, 6, 14, true, false, 1, float, false><<<dim3((unsigned)nblk, 14), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
