// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_i21_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<2, 1, 0, 1, false, false, 1, double, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        const long ng = (long)(smem / sizeof(double)) - 256L * 3;
        const size_t sm = sizeof(double) * (size_t)(rys_stage_offset(ng, 3) + rys_stage_doubles(g.tab.nint, 3));
        static size_t attr[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (sm > attr[dev & 63]) {
            cudaFuncSetAttribute(k_rys_thread<2, 1, 1, 2, false, false, 1, double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            attr[dev & 63] = sm;
        }
        k_rys_thread<2, 1, 1, 2, false, false, 1, double, true><<<dim3((unsigned)nblk, 2), 128, sm, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<2, 1, 2, 2, false, false, 1, double, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<2, 1, 3, 3, false, false, 1, double, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<2, 1, 4, 8, false, false, 1, double, false><<<dim3((unsigned)nblk, 8), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<2, 1, 5, 7, false, false, 1, double, false><<<dim3((unsigned)nblk, 7), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<2, 1, 6, 28, false, false, 1, double, false><<<dim3((unsigned)nblk, 28), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
