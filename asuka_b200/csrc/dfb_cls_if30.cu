// Generated by gen_classes.py -- class-specialised Rys kernel instantiations.
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_if30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st) {
    if (lc == 0) {
        k_rys_thread<3, 0, 0, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 1) {
        const long ng = (long)(smem / sizeof(double)) - 256L * 3;
        const size_t sm = sizeof(double) * (size_t)(rys_stage_offset(ng, 3) + rys_stage_doubles(g.tab.nint, 3));
        static size_t attr[64];
        int dev = 0;
        cudaGetDevice(&dev);
        if (sm > attr[dev & 63]) {
            cudaFuncSetAttribute(k_rys_thread<3, 0, 1, 1, false, false, 1, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            attr[dev & 63] = sm;
        }
        k_rys_thread<3, 0, 1, 1, false, false, 1, float, true><<<dim3((unsigned)nblk, 1), 128, sm, st>>>(g);
        return 1;
    }
    if (lc == 2) {
        k_rys_thread<3, 0, 2, 1, false, false, 1, float, false><<<dim3((unsigned)nblk, 1), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 3) {
        k_rys_thread<3, 0, 3, 2, false, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 4) {
        k_rys_thread<3, 0, 4, 2, false, false, 1, float, false><<<dim3((unsigned)nblk, 2), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 5) {
        k_rys_thread<3, 0, 5, 3, false, false, 1, float, false><<<dim3((unsigned)nblk, 3), 128, smem, st>>>(g);
        return 1;
    }
    if (lc == 6) {
        k_rys_thread<3, 0, 6, 4, false, false, 1, float, false><<<dim3((unsigned)nblk, 4), 128, smem, st>>>(g);
        return 1;
    }
    return 0;
}
}  // namespace dfb
