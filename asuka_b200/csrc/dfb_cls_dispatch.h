// Generated by gen_classes.py -- dispatch over the class-specialised kernels.
#pragma once
#include "dfb_rys_tmpl.cuh"

namespace dfb {
int dfb_cls_i00_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i10_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i20_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i21_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i22_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i31_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_i32_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if00_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if10_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if20_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if21_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if22_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if31_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if32_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_if33_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d00_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d10_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d20_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d21_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d22_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d31_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_d32_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df00_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df10_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df11_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df20_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df21_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df22_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df30_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df31_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);
int dfb_cls_df32_launch(int lc, const TmplArgs& g, long nblk, size_t smem, cudaStream_t st);

// f32: the mixed-precision variant (float recurrence tables and accumulators)
inline int tmpl_launch(int la, int lb, int lc, bool deriv, bool f32, const TmplArgs& g, long nblk,
                       size_t smem, cudaStream_t st) {
    if (!deriv && !f32 && la == 0 && lb == 0) return dfb_cls_i00_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 1 && lb == 0) return dfb_cls_i10_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 1 && lb == 1) return dfb_cls_i11_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 2 && lb == 0) return dfb_cls_i20_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 2 && lb == 1) return dfb_cls_i21_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 2 && lb == 2) return dfb_cls_i22_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 3 && lb == 0) return dfb_cls_i30_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 3 && lb == 1) return dfb_cls_i31_launch(lc, g, nblk, smem, st);
    if (!deriv && !f32 && la == 3 && lb == 2) return dfb_cls_i32_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 0 && lb == 0) return dfb_cls_if00_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 1 && lb == 0) return dfb_cls_if10_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 1 && lb == 1) return dfb_cls_if11_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 2 && lb == 0) return dfb_cls_if20_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 2 && lb == 1) return dfb_cls_if21_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 2 && lb == 2) return dfb_cls_if22_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 3 && lb == 0) return dfb_cls_if30_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 3 && lb == 1) return dfb_cls_if31_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 3 && lb == 2) return dfb_cls_if32_launch(lc, g, nblk, smem, st);
    if (!deriv && f32 && la == 3 && lb == 3) return dfb_cls_if33_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 0 && lb == 0) return dfb_cls_d00_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 1 && lb == 0) return dfb_cls_d10_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 1 && lb == 1) return dfb_cls_d11_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 2 && lb == 0) return dfb_cls_d20_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 2 && lb == 1) return dfb_cls_d21_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 2 && lb == 2) return dfb_cls_d22_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 3 && lb == 0) return dfb_cls_d30_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 3 && lb == 1) return dfb_cls_d31_launch(lc, g, nblk, smem, st);
    if (deriv && !f32 && la == 3 && lb == 2) return dfb_cls_d32_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 0 && lb == 0) return dfb_cls_df00_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 1 && lb == 0) return dfb_cls_df10_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 1 && lb == 1) return dfb_cls_df11_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 2 && lb == 0) return dfb_cls_df20_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 2 && lb == 1) return dfb_cls_df21_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 2 && lb == 2) return dfb_cls_df22_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 3 && lb == 0) return dfb_cls_df30_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 3 && lb == 1) return dfb_cls_df31_launch(lc, g, nblk, smem, st);
    if (deriv && f32 && la == 3 && lb == 2) return dfb_cls_df32_launch(lc, g, nblk, smem, st);
    return 0;
}

inline bool tmpl_has(int la, int lb, int lc, bool deriv, bool f32) {
    static const int ki[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {2, 2, 6}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 1, 6}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}, {3, 2, 5}};
    static const int kif[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {2, 2, 6}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 1, 6}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}, {3, 2, 4}, {3, 2, 5}, {3, 2, 6}, {3, 3, 0}, {3, 3, 1}, {3, 3, 2}, {3, 3, 3}, {3, 3, 4}, {3, 3, 5}, {3, 3, 6}};
    static const int kd[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}};
    static const int kdf[][3] = {{0, 0, 0}, {0, 0, 1}, {0, 0, 2}, {0, 0, 3}, {0, 0, 4}, {0, 0, 5}, {0, 0, 6}, {1, 0, 0}, {1, 0, 1}, {1, 0, 2}, {1, 0, 3}, {1, 0, 4}, {1, 0, 5}, {1, 0, 6}, {1, 1, 0}, {1, 1, 1}, {1, 1, 2}, {1, 1, 3}, {1, 1, 4}, {1, 1, 5}, {1, 1, 6}, {2, 0, 0}, {2, 0, 1}, {2, 0, 2}, {2, 0, 3}, {2, 0, 4}, {2, 0, 5}, {2, 0, 6}, {2, 1, 0}, {2, 1, 1}, {2, 1, 2}, {2, 1, 3}, {2, 1, 4}, {2, 1, 5}, {2, 1, 6}, {2, 2, 0}, {2, 2, 1}, {2, 2, 2}, {2, 2, 3}, {2, 2, 4}, {2, 2, 5}, {2, 2, 6}, {3, 0, 0}, {3, 0, 1}, {3, 0, 2}, {3, 0, 3}, {3, 0, 4}, {3, 0, 5}, {3, 0, 6}, {3, 1, 0}, {3, 1, 1}, {3, 1, 2}, {3, 1, 3}, {3, 1, 4}, {3, 1, 5}, {3, 1, 6}, {3, 2, 0}, {3, 2, 1}, {3, 2, 2}, {3, 2, 3}, {3, 2, 4}, {3, 2, 5}, {3, 2, 6}};
    const int (*k)[3] = deriv ? (f32 ? kdf : kd) : (f32 ? kif : ki);
    const int n = deriv ? (f32 ? (int)(sizeof(kdf) / sizeof(kdf[0])) : (int)(sizeof(kd) / sizeof(kd[0])))
                        : (f32 ? (int)(sizeof(kif) / sizeof(kif[0])) : (int)(sizeof(ki) / sizeof(ki[0])));
    for (int i = 0; i < n; ++i)
        if (k[i][0] == la && k[i][1] == lb && k[i][2] == lc) return true;
    return false;
}
}  // namespace dfb
