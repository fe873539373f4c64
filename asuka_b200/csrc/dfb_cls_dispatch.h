// Generated by gen_classes.py -- dispatch over the class-specialised kernels.
#pragma once
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_i0_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i1_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i2_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i3_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d0_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d1_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d2_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d3_launch(int la, int lb, int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);

inline int tmpl_launch(int la, int lb, int lc, bool deriv, const TmplArgs& g, long nblk, size_t smem,
                       cudaStream_t st) {
    if (!deriv && la == 0) return dfb_cls_i0_launch(la, lb, lc, g, nblk, smem, st);
    if (!deriv && la == 1) return dfb_cls_i1_launch(la, lb, lc, g, nblk, smem, st);
    if (!deriv && la == 2) return dfb_cls_i2_launch(la, lb, lc, g, nblk, smem, st);
    if (!deriv && la == 3) return dfb_cls_i3_launch(la, lb, lc, g, nblk, smem, st);
    if (deriv && la == 0) return dfb_cls_d0_launch(la, lb, lc, g, nblk, smem, st);
    if (deriv && la == 1) return dfb_cls_d1_launch(la, lb, lc, g, nblk, smem, st);
    if (deriv && la == 2) return dfb_cls_d2_launch(la, lb, lc, g, nblk, smem, st);
    if (deriv && la == 3) return dfb_cls_d3_launch(la, lb, lc, g, nblk, smem, st);
    return 0;
}
}  // namespace dfb
