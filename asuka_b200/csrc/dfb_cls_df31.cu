// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_df31_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        const long ng = (long)(smem / sizeof(double)) - 256L * 3;
        const size_t sm = sizeof(double) * (size_t)(rys_stage_offset(ng, 3) + rys_stage_doubles(g.tab.nint, 3));
        static size_t attr[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (sm > attr[dev & 63]) {
            cudaFuncSetAttribute(k_rys_thread<3, 1, 0, 1, true, false, 1, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            attr[dev & 63] = sm;
        }
        k_rys_thread<3, 1, 0, 1, true, false, 1, float, true><<<dim3((unsigned)nblk, 1), 128, sm, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        k_rys_thread<3, 1, 1, 3, true, false, 1, float, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<3, 1, 2, 6, true, false, 1, float, false><<<dim3((unsigned)nblk, 6), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<3, 1, 3, 10, true, false, 1, float, false><<<dim3((unsigned)nblk, 10), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<3, 1, 4, 15, true, false, 1, float, false><<<dim3((unsigned)nblk, 15), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<3, 1, 5, 21, true, false, 1, float, false><<<dim3((unsigned)nblk, 21), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<3, 1, 6, 28, true, false, 1, float, false><<<dim3((unsigned)nblk, 28), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
