// Shared device helpers for the DF two-electron kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define DFB_LMAX 8                                 // highest shell l on either side
#define DFB_NROOTS_MAX 10                          // (4+4+8+1)/2+1 = 9 needed; table holds 10
#define DFB_WARPS_PER_BLOCK 4

namespace dfb {

__host__ __device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// number of Cartesian components over all l < L (tetrahedral numbers)
__host__ __device__ __forceinline__ int ncart_below(int L) { return L * (L + 1) * (L + 2) / 6; }

// position of (ex, ey, ez=l-ex-ey) inside shell l, x-major order (for x=l..0, for y=l-x..0)
__host__ __device__ __forceinline__ int cart_index(int ex, int ey, int l) {
    return ((l - ex) * (l - ex + 1)) / 2 + (l - ex - ey);
}

// Rys root/weight table: per root count n, NINT equal intervals of T in
// [0, tmax), 2n rows (n nodes then n weights), DEG+1 power-basis coefficients
// in u = 2(T/h - k) - 1, h = tmax/NINT.
struct RysTable {
    const double* coef;   // concatenated over n = 1..nmax
    const double* herm;   // per n: s_i^2 (n) then W_i (n), concatenated
    int offs[DFB_NROOTS_MAX + 1];   // coefficient offset of root count n
    int hoff[DFB_NROOTS_MAX + 1];   // hermite offset of root count n
    int nmax, nint, deg;
    double tmax;
    double inv_h;  // intervals per unit T (nint / tmax)
    int* err;      // device word: 0, or the code of the first bounded wait that gave up (dfb_rys_error)
};

// Task t -> (pair list index, aux list index).  grid > 0: pair-major grid with
// `grid` aux shells per pair; grid < 0: aux-major grid with -grid pairs per aux
// shell (a warp then shares one aux shell and walks consecutive pairs, which the
// caller sorts by primitive-pair count); grid == 0: explicit lists.
__device__ __forceinline__ void task_indices(long t, long grid, long& tp, long& ta) {
    if (grid > 0) {
        tp = t / grid;
        ta = t - tp * grid;
    } else if (grid < 0) {
        ta = t / (-grid);
        tp = t - ta * (-grid);
    } else {
        tp = t;
        ta = t;
    }
}

// Nodes x_i (in t^2) and weights w_i (sum w_i = F_0(T)) of the n-point Rys rule,
// written to x[i * xs] and w[i * xs].
__device__ __forceinline__ void rys_eval(const RysTable& tab, int n, double T, double* x, double* w, int xs = 1) {
    if (T >= tab.tmax) {
        const double* h = tab.herm + tab.hoff[n];
        const double rs = rsqrt(T);
        const double inv = rs * rs;
        for (int i = 0; i < n; ++i) {
            x[i * xs] = __ldg(h + i) * inv;
            w[i * xs] = __ldg(h + n + i) * rs;
        }
        return;
    }
    const double Th = T * tab.inv_h;
    int k = (int)Th;
    if (k > tab.nint - 1) k = tab.nint - 1;
    const double u = 2.0 * (Th - (double)k) - 1.0;
    const int stride = tab.deg + 1;
    const double* c = tab.coef + tab.offs[n] + (size_t)k * (2 * n) * stride;
    for (int r = 0; r < 2 * n; ++r) {
        const double* cr = c + r * stride;
        double acc = __ldg(cr + tab.deg);
        for (int d = tab.deg - 1; d >= 0; --d) acc = fma(acc, u, __ldg(cr + d));
        if (r < n)
            x[r * xs] = acc;
        else
            w[(r - n) * xs] = acc;
    }
}

}  // namespace dfb
