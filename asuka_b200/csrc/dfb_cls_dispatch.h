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

inline bool tmpl_has(int la, int lb, int lc, bool deriv) {
    static const int ki[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {2, 2, 6}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 1, 6}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}, {3, 2, 5}};
    static const int kd[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}};
    const int (*k)[3] = deriv ? kd : ki;
    const int n = deriv ? (int)(sizeof(kd) / sizeof(kd[0])) : (int)(sizeof(ki) / sizeof(ki[0]));
    for (int i = 0; i < n; ++i)
        if (k[i][0] == la && k[i][1] == lb && k[i][2] == lc) return true;
    return false;
}
}  // namespace dfb
