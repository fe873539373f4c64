// Rys-quadrature DF integrals and their derivative contraction on sm_100a.
//
// One warp owns one task (an AB shell pair -- or an aux self-pair for the
// metric -- times one aux shell C) at a time and walks every task of the
// launch's angular class in a persistent loop:
//
//   1. the 32 lanes take 32 primitive triplets at once and evaluate T, the
//      Rys nodes/weights (table lookup, FP64) and the prefactor;
//   2. for each primitive triplet, lanes (root, direction) build the 2D
//      recurrence tables G[a][b] (a <= la+lb(+1), b <= lc) in shared memory,
//      the x table pre-scaled by weight*prefactor;
//   3. every lane accumulates its share of the contracted intermediate
//      (e 0 | f) = sum Gx Gy Gz  (la <= |e| <= la+lb, f in shell c) in registers;
//   4. after all primitives the horizontal recurrence (e 0|f) -> (a b|f) runs
//      once per contracted task, and the tile goes straight to its final place
//      (3c tensor both (mu,nu) orders, or both halves of the metric).
//
// The derivative variant accumulates, per AO primitive pair, the plain sum U
// and the exponent-weighted sums 2a*S, 2b*S over |e| up to la+lb+1, then
// contracts d/dA = 2a (a+1) - a_x (a-1) and d/dB = 2b [(a+1,b) + AB (a,b)] -
// b_x (a,b-1) against the adjoint tile; d/dC follows from translational
// invariance.  Per-block partial gradients live in shared memory.
//
// Mathematics restated from the reference (asuka/cueri/_eri_rys_cpu.pyx
// :690-718 recurrences, :802-817 horizontal shift, :2650-2957 derivative
// contraction); roots come from a tabulated fit instead of the reference's
// per-call moment solver.

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/dfb.h"
#include "dfb_common.cuh"
#include "dfb_cls_dispatch.h"
#include "dfb_internal.h"

namespace dfb {

static const double kTwoPi52 = 2.0 * 3.141592653589793238462643383279502884 * 3.141592653589793238462643383279502884 *
                               1.772453850905516027298167483341145182;

struct ClassInfo {
    int la, lb, lc;
    int nr;          // Rys roots
    int nmax, mmax;  // G table extents
    int lmin, lmax;  // |e| range of the contracted intermediate
    int ne, nf, nef;
    int na, nb, nc;
    int gt;          // (nmax+1)*(mmax+1)
    int item;        // doubles per primitive-triplet record
};

// Fields of one primitive triplet's shared-memory record in the generic path (field f of
// lane j at items[32 f + j]): everything the per-root recurrence coefficients need, with the
// reciprocals taken once per triplet, then the nodes and the prefactor-scaled weights.
enum {
    DFB_REC_HINV = 0,  // 1 / (2 (p+q))
    DFB_REC_HP = 1,    // 1 / (2p)
    DFB_REC_HQ = 2,    // 1 / (2q)
    DFB_REC_PA = 3,    // P - A (3 fields)
    DFB_REC_QCP = 6,   // q/(p+q) (C - P) (3 fields)
    DFB_REC_PCP = 9,   // -p/(p+q) (C - P) (3 fields)
    DFB_REC_X = 12     // nodes (nr fields), then weights x prefactor (nr fields)
};

static ClassInfo make_class(int la, int lb, int lc, bool deriv) {
    ClassInfo c;
    c.la = la;
    c.lb = lb;
    c.lc = lc;
    c.nr = (la + lb + lc + (deriv ? 1 : 0)) / 2 + 1;
    c.nmax = la + lb + (deriv ? 1 : 0);
    c.mmax = lc;
    c.lmin = deriv ? (la > 0 ? la - 1 : 0) : la;
    c.lmax = c.nmax;
    c.ne = ncart_below(c.lmax + 1) - ncart_below(c.lmin);
    c.nf = ncart(lc);
    c.nef = c.ne * c.nf;
    c.na = ncart(la);
    c.nb = ncart(lb);
    c.nc = ncart(lc);
    c.gt = (c.nmax + 1) * (c.mmax + 1);
    c.item = DFB_REC_X + 2 * c.nr;
    return c;
}


__device__ __forceinline__ void decode_cart(int l, int idx, int& x, int& y, int& z) {
    int xx = l;
    while (idx > l - xx) {
        idx -= (l - xx + 1);
        --xx;
    }
    x = xx;
    y = l - xx - idx;
    z = idx;
}

__device__ __forceinline__ void decode_e(const ClassInfo& ci, int e, int& x, int& y, int& z) {
    int L = ci.lmin;
    while (e >= ncart(L)) {
        e -= ncart(L);
        ++L;
    }
    decode_cart(L, e, x, y, z);
}

__constant__ int c_ncbtab[2 * DFB_LMAX + 4];  // ncart_below(L), L = 0 .. 2 LMAX + 3


__constant__ double c_binomtab[DFB_LMAX + 2][DFB_LMAX + 2];

__device__ __forceinline__ void build_G(double* G, int nmax, int mmax, double g00, double C, double Cp, double B0,
                                        double B1, double B1p) {
    const int M = mmax + 1;
    G[0] = g00;
    if (nmax > 0) G[M] = C * g00;
    if (mmax > 0) G[1] = Cp * g00;
    for (int a = 2; a <= nmax; ++a) G[a * M] = B1 * (double)(a - 1) * G[(a - 2) * M] + C * G[(a - 1) * M];
    for (int b = 2; b <= mmax; ++b) G[b] = B1p * (double)(b - 1) * G[b - 2] + Cp * G[b - 1];
    if (nmax == 0 || mmax == 0) return;
    for (int a = 1; a <= nmax; ++a) {
        G[a * M + 1] = (double)a * B0 * G[(a - 1) * M] + Cp * G[a * M];
        for (int b = 2; b <= mmax; ++b)
            G[a * M + b] = B1p * (double)(b - 1) * G[a * M + b - 2] + (double)a * B0 * G[(a - 1) * M + b - 1] +
                           Cp * G[a * M + b - 1];
    }
}

// Phase 1 of the generic path: one warp per work unit (task, chunk of the
// (e, f) elements).  Lanes evaluate 32 primitive triplets' roots at once, lanes
// (root, direction) build the 2D recurrence tables in shared memory for one
// triplet at a time, and every lane accumulates KB elements of the chunk.  The
// contracted intermediate goes to the task's scratch slot: E (integrals) or
// U | WA | WB (derivative; flushed once per AO primitive pair).  Splitting the
// elements of a task over warps keeps the SMs busy for the heavy high-l classes,
// which have few tasks.
#ifndef DFB_ACC_MIN_BLOCKS
#define DFB_ACC_MIN_BLOCKS 3  // resident blocks per SM the accumulation kernel is compiled for
#endif
template <int KB, bool DERIV>
__global__ void __launch_bounds__(DFB_WARPS_PER_BLOCK * 32, DFB_ACC_MIN_BLOCKS)
    k_rys_acc(ClassInfo ci, dfb_pair_side_t ps, dfb_aux_side_t ax, const int* __restrict__ task_pair,
              const int* __restrict__ task_aux, long t0, long nt, long naux_grid, double* __restrict__ scratch,
              long slot, RysTable tab) {
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int per_warp = 32 * ci.item + ci.nr * 3 * ci.gt;
    double* items = smem + wib * per_warp;
    double* gtab = items + 32 * ci.item;
    const long gwarp = (long)blockIdx.x * DFB_WARPS_PER_BLOCK + wib;
    const long nwarps = (long)gridDim.x * DFB_WARPS_PER_BLOCK;
    const int chunk_elems = 32 * KB;
    const int nchunk = (ci.nef + chunk_elems - 1) / chunk_elems;
    const int M = ci.mmax + 1;
    // per element of the lane: offsets of its x, y and z factors inside one root's
    // three tables (y and z include the table stride); elements past the end read
    // entry 0 and are never stored
    int ox[KB], oy[KB], oz[KB];
    auto make_offsets = [&](int cbase) {
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            const int t = cbase + lane + 32 * k;
            ox[k] = oy[k] = oz[k] = 0;
            if (t < ci.nef) {
                const int e = t / ci.nf, f = t - (t / ci.nf) * ci.nf;
                int ex, ey, ez, fx, fy, fz;
                decode_e(ci, e, ex, ey, ez);
                decode_cart(ci.lc, f, fx, fy, fz);
                ox[k] = ex * M + fx;
                oy[k] = ci.gt + ey * M + fy;
                oz[k] = 2 * ci.gt + ez * M + fz;
            }
        }
    };
    if (nchunk == 1) make_offsets(0);
    const long nunits = nt * nchunk;

    for (long unit = gwarp; unit < nunits; unit += nwarps) {
        const long tl = unit / nchunk;
        const int ch = (int)(unit - tl * nchunk);
        const long task = t0 + tl;
        long tp, ta;
        task_indices(task, naux_grid, tp, ta);
        const int pair = task_pair[tp];
        const int C = task_aux[ta];
        const int shA = ps.shA[pair];
        double A[3], Cc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            A[d] = ps.cxyz[3 * shA + d];
            Cc[d] = ax.cxyz[3 * C + d];
        }
        const int p0 = ps.pstart[pair];
        const int nprimAB = ps.npair[pair];
        const int c0 = ax.pstart[C];
        const int nprimC = ax.nprim[C];
        const long nitems = (long)nprimAB * nprimC;
        double* E = scratch + tl * slot;
        const int cbase = ch * chunk_elems;
        if (nchunk > 1) make_offsets(cbase);
        double acc[KB];
#pragma unroll
        for (int k = 0; k < KB; ++k) {
            acc[k] = 0.0;
            const int t = cbase + lane + 32 * k;
            if (DERIV && t < ci.nef) {
                E[t] = 0.0;
                E[ci.nef + t] = 0.0;
                E[2 * ci.nef + t] = 0.0;
            }
        }

        for (long base = 0; base < nitems; base += 32) {
            const long j = base + lane;
            if (j < nitems) {
                const int iab = (int)(j / nprimC);
                const int ic = (int)(j - (long)iab * nprimC);
                const double p = ps.eta[p0 + iab];
                const double Pp[3] = {ps.Px[p0 + iab], ps.Py[p0 + iab], ps.Pz[p0 + iab]};
                const double q = ax.pexp[c0 + ic];
                const double rp = 1.0 / p, rq = ax.rexp[c0 + ic];
                // one reciprocal square root: 1/(p+q) = s^2, 1/(p q sqrt(p+q)) = rp rq s
                const double s = rsqrt(p + q);
                const double inv = s * s;
                const double qi = q * inv, pi = p * inv;
                double PQ2 = 0.0;
                double* it = items + lane;  // field f of this lane's record at it[32 f]
                it[32 * DFB_REC_HINV] = 0.5 * inv;
                it[32 * DFB_REC_HP] = 0.5 * rp;
                it[32 * DFB_REC_HQ] = 0.5 * rq;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const double cp = Cc[d] - Pp[d];
                    PQ2 += cp * cp;
                    it[32 * (DFB_REC_PA + d)] = Pp[d] - A[d];
                    it[32 * (DFB_REC_QCP + d)] = qi * cp;
                    it[32 * (DFB_REC_PCP + d)] = -pi * cp;
                }
                const double T = p * q * inv * PQ2;
                const double pref = kTwoPi52 * ps.cK[p0 + iab] * rp * (ax.pcoef[c0 + ic] * rq) * s;
                // nodes and weights straight into the lane's shared-memory record
                rys_eval(tab, ci.nr, T, it + 32 * DFB_REC_X, it + 32 * (DFB_REC_X + ci.nr), 32);
                for (int u = 0; u < ci.nr; ++u) it[32 * (DFB_REC_X + ci.nr + u)] *= pref;
            }
            __syncwarp();
            const int nb = (int)((nitems - base) < 32 ? (nitems - base) : 32);
            for (int jj = 0; jj < nb; ++jj) {
                const double* it = items + jj;
                if (lane < ci.nr * 3) {
                    const int u = lane / 3, d = lane - 3 * (lane / 3);
                    const double x = it[32 * (DFB_REC_X + u)];
                    const double B0 = x * it[32 * DFB_REC_HINV];
                    const double B1 = (1.0 - x) * it[32 * DFB_REC_HP] + B0;
                    const double B1p = (1.0 - x) * it[32 * DFB_REC_HQ] + B0;
                    const double Cd = it[32 * (DFB_REC_PA + d)] + x * it[32 * (DFB_REC_QCP + d)];
                    const double Cpd = x * it[32 * (DFB_REC_PCP + d)];
                    const double g00 = (d == 0) ? it[32 * (DFB_REC_X + ci.nr + u)] : 1.0;
                    build_G(gtab + (u * 3 + d) * ci.gt, ci.nmax, ci.mmax, g00, Cd, Cpd, B0, B1, B1p);
                }
                __syncwarp();
                // roots outer, elements inner: KB independent FMA chains per root
                const double* g = gtab;
                for (int u = 0; u < ci.nr; ++u, g += 3 * ci.gt) {
#pragma unroll
                    for (int k = 0; k < KB; ++k) acc[k] = fma(g[ox[k]] * g[oy[k]], g[oz[k]], acc[k]);
                }
                if (DERIV) {
                    const long gidx = base + jj;
                    if ((gidx + 1) % nprimC == 0) {
                        const int iab = (int)(gidx / nprimC);
                        const double a2 = 2.0 * ps.ea[p0 + iab];
                        const double b2 = 2.0 * ps.eb[p0 + iab];
#pragma unroll
                        for (int k = 0; k < KB; ++k) {
                            const int t = cbase + lane + 32 * k;
                            if (t < ci.nef) {
                                E[t] += acc[k];
                                E[ci.nef + t] += a2 * acc[k];
                                E[2 * ci.nef + t] += b2 * acc[k];
                                acc[k] = 0.0;
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (!DERIV) {
#pragma unroll
            for (int k = 0; k < KB; ++k) {
                if (cbase + lane + 32 * k < ci.nef) E[cbase + lane + 32 * k] = acc[k];
            }
        }
        __syncwarp();
    }
}

#define DFB_EPI_CHUNK 128  // tile elements per epilogue work unit
#define DFB_HRR_TERMS 64   // capacity of one horizontal-recurrence term list (lb <= 8 needs 48)

// Terms of the horizontal recurrence for one b: (a b|f) = sum_t coef_t (a + k_t, 0|f)
// over k_t <= b componentwise, coef_t = prod_d C(b_d, k_d) AB_d^(b_d - k_d).  The
// lanes of a warp build the list together in the warp's shared memory.
__device__ __forceinline__ int hrr_terms(int bx, int by, int bz, const double* AB, double* tc, int* tk, int lane) {
    const int ny = by + 1, nz = bz + 1;
    const int n = (bx + 1) * ny * nz;
    for (int t = lane; t < n; t += 32) {
        const int kx = t / (ny * nz);
        const int r = t - kx * ny * nz;
        const int ky = r / nz;
        const int kz = r - ky * nz;
        double c = c_binomtab[bx][kx] * c_binomtab[by][ky] * c_binomtab[bz][kz];
        for (int m = kx; m < bx; ++m) c *= AB[0];
        for (int m = ky; m < by; ++m) c *= AB[1];
        for (int m = kz; m < bz; ++m) c *= AB[2];
        tc[t] = c;
        tk[t] = kx | (ky << 8) | (kz << 16);
    }
    return n;
}

// Position of the Cartesian component (x, y, z) in the contracted intermediate
// (shells lmin..lmax, x-major inside a shell); ebase = -ncart_below(lmin).
__device__ __forceinline__ int e_pos(int x, int y, int z, int ebase) {
    const int L = x + y + z;
    return c_ncbtab[L] + ebase + (((L - x) * (L - x + 1)) >> 1) + (L - x - y);
}

// sum_t coef_t T[(a + k_t) nf + ic] for one table, and for two tables read at the same positions.
__device__ __forceinline__ double hrr_apply(const double* __restrict__ T, int nf, int ic, int ebase, int ax, int ay,
                                            int az, const double* tc, const int* tk, int n) {
    double s = 0.0;
    for (int t = 0; t < n; ++t) {
        const int k = tk[t];
        const int e = e_pos(ax + (k & 255), ay + ((k >> 8) & 255), az + (k >> 16), ebase);
        s = fma(tc[t], __ldg(T + e * nf + ic), s);
    }
    return s;
}

__device__ __forceinline__ void hrr_apply2(const double* __restrict__ T1, const double* __restrict__ T2, int nf, int ic,
                                           int ebase, int ax, int ay, int az, const double* tc, const int* tk, int n,
                                           double& s1, double& s2) {
    s1 = s2 = 0.0;
    for (int t = 0; t < n; ++t) {
        const int k = tk[t];
        const int e = e_pos(ax + (k & 255), ay + ((k >> 8) & 255), az + (k >> 16), ebase) * nf + ic;
        s1 = fma(tc[t], __ldg(T1 + e), s1);
        s2 = fma(tc[t], __ldg(T2 + e), s2);
    }
}

// Phase 2: one warp per (task, B component, chunk of the (A component, aux
// component) elements).  The lanes of a unit share b, so they share the term
// list of the horizontal recurrence (built once per unit in shared memory) and
// run its loops in lockstep.  The tile goes to its final place (integrals) or is
// contracted with the adjoint (derivative; per-block partial gradients in shared
// memory).
template <bool DERIV>
__global__ void __launch_bounds__(DFB_WARPS_PER_BLOCK * 32)
    k_rys_epi(ClassInfo ci, dfb_pair_side_t ps, dfb_aux_side_t ax, const int* __restrict__ task_pair,
              const int* __restrict__ task_aux, long t0, long nt, long naux_grid, int mode, double* __restrict__ out,
              long sP, long sM, long sN, const double* __restrict__ bar, long sbP, long sbM, long sbN,
              double* __restrict__ grad, int natm, int smem_grad, const double* __restrict__ scratch, long slot) {
    extern __shared__ double sgrad[];
    constexpr int NL = DERIV ? 4 : 1;  // term lists per warp: b, and b - 1_d for d = x, y, z
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int ngrad = (DERIV && smem_grad) ? natm * 3 : 0;
    double* tc = sgrad + ngrad + wib * NL * DFB_HRR_TERMS;
    int* tk = (int*)(sgrad + ngrad + DFB_WARPS_PER_BLOCK * NL * DFB_HRR_TERMS) + wib * NL * DFB_HRR_TERMS;
    const long gwarp = (long)blockIdx.x * DFB_WARPS_PER_BLOCK + wib;
    const long nwarps = (long)gridDim.x * DFB_WARPS_PER_BLOCK;
    if (DERIV && smem_grad) {
        for (int i = threadIdx.x; i < ngrad; i += blockDim.x) sgrad[i] = 0.0;
        __syncthreads();
    }
    const int ebase = -c_ncbtab[ci.lmin];
    const int nf = ci.nf;
    const int nac = ci.na * ci.nc;
    const int nsub = (nac + DFB_EPI_CHUNK - 1) / DFB_EPI_CHUNK;
    const int chunk = (((nac + nsub - 1) / nsub + 31) / 32) * 32;  // even chunks, whole passes of the warp
    const int nec = ci.nb * nsub;
    for (long unit = gwarp; unit < nt * nec; unit += nwarps) {
        const long tl = unit / nec;
        const int r = (int)(unit - tl * nec);
        const int ib = r / nsub;
        const int j0 = (r - ib * nsub) * chunk;
        const int j1 = (j0 + chunk < nac) ? j0 + chunk : nac;
        const long task = t0 + tl;
        long tp, ta;
        task_indices(task, naux_grid, tp, ta);
        const int pair = task_pair[tp];
        const int C = task_aux[ta];
        const int shA = ps.shA[pair];
        const int shB = ps.b_dummy ? -1 : ps.shB[pair];
        double AB[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) AB[d] = ps.cxyz[3 * shA + d] - (ps.b_dummy ? 0.0 : ps.cxyz[3 * shB + d]);
        const double* E = scratch + tl * slot;
        const int aoA = ps.aostart[shA];
        const int aoB = ps.b_dummy ? 0 : ps.aostart[shB];
        const int aoC = ax.aostart[C];
        double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};
        int b[3];
        decode_cart(ci.lb, ib, b[0], b[1], b[2]);
        __syncwarp();  // the previous unit's lanes are done with the lists
        const int n0 = hrr_terms(b[0], b[1], b[2], AB, tc, tk, lane);
        int nd[3] = {0, 0, 0};
        if (DERIV) {
            if (b[0] > 0) nd[0] = hrr_terms(b[0] - 1, b[1], b[2], AB, tc + DFB_HRR_TERMS, tk + DFB_HRR_TERMS, lane);
            if (b[1] > 0)
                nd[1] = hrr_terms(b[0], b[1] - 1, b[2], AB, tc + 2 * DFB_HRR_TERMS, tk + 2 * DFB_HRR_TERMS, lane);
            if (b[2] > 0)
                nd[2] = hrr_terms(b[0], b[1], b[2] - 1, AB, tc + 3 * DFB_HRR_TERMS, tk + 3 * DFB_HRR_TERMS, lane);
        }
        __syncwarp();
        for (int j = j0 + lane; j < j1; j += 32) {
            const int ia = j / ci.nc;
            const int ic = j - ia * ci.nc;
            int a[3];
            decode_cart(ci.la, ia, a[0], a[1], a[2]);
            if (!DERIV) {
                const double v = hrr_apply(E, nf, ic, ebase, a[0], a[1], a[2], tc, tk, n0);
                if (mode == 0) {
                    const long P = aoC + ic, mu = aoA + ia, nu = aoB + ib;
                    out[P * sP + mu * sM + nu * sN] = v;
                    out[P * sP + nu * sM + mu * sN] = v;
                } else {
                    const long Pa = aoA + ia, Qc = aoC + ic;
                    out[Qc * sP + Pa * sM] = v;
                    out[Pa * sP + Qc * sM] = v;
                }
            } else {
                double gam;
                if (mode == 0) {
                    gam = bar[(long)(aoC + ic) * sbP + (long)(aoA + ia) * sbM + (long)(aoB + ib) * sbN];
                } else {
                    gam = bar[(long)(aoA + ia) * sbP + (long)(aoC + ic) * sbM];
                }
                if (gam != 0.0) {
                    const double* U = E;
                    const double* WA = E + ci.nef;
                    const double* WB = E + 2 * ci.nef;
                    // (a b|c) of WB is shared by the three directions of the B derivative
                    const double wb0 = ps.b_dummy ? 0.0 : hrr_apply(WB, nf, ic, ebase, a[0], a[1], a[2], tc, tk, n0);
#pragma unroll 1
                    for (int d = 0; d < 3; ++d) {
                        const int ex = d == 0, ey = d == 1, ez = d == 2;
                        const int ad = d == 0 ? a[0] : (d == 1 ? a[1] : a[2]);
                        const int bd = d == 0 ? b[0] : (d == 1 ? b[1] : b[2]);
                        const double abd = d == 0 ? AB[0] : (d == 1 ? AB[1] : AB[2]);
                        double dA, dB;
                        // d/dA: 2a (a+1_d b|c) - a_d (a-1_d b|c); d/dB: 2b (a+1_d b|c) + AB_d 2b (a b|c) - b_d (a b-1_d|c)
                        hrr_apply2(WA, WB, nf, ic, ebase, a[0] + ex, a[1] + ey, a[2] + ez, tc, tk, n0, dA, dB);
                        if (ad > 0)
                            dA -= (double)ad * hrr_apply(U, nf, ic, ebase, a[0] - ex, a[1] - ey, a[2] - ez, tc, tk, n0);
                        if (ps.b_dummy) {
                            dB = 0.0;
                        } else {
                            dB += abd * wb0;
                            if (bd > 0) {
                                const int o = (d + 1) * DFB_HRR_TERMS;
                                const int n = d == 0 ? nd[0] : (d == 1 ? nd[1] : nd[2]);
                                dB -= (double)bd * hrr_apply(U, nf, ic, ebase, a[0], a[1], a[2], tc + o, tk + o, n);
                            }
                        }
                        if (d == 0) {
                            gA[0] += gam * dA;
                            gB[0] += gam * dB;
                        } else if (d == 1) {
                            gA[1] += gam * dA;
                            gB[1] += gam * dB;
                        } else {
                            gA[2] += gam * dA;
                            gB[2] += gam * dB;
                        }
                    }
                }
            }
        }
        if (DERIV) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                for (int s = 16; s > 0; s >>= 1) {
                    gA[d] += __shfl_xor_sync(0xffffffffu, gA[d], s);
                    gB[d] += __shfl_xor_sync(0xffffffffu, gB[d], s);
                }
            }
            if (lane == 0) {
                const bool offdiag = (mode == 0) ? (shA != shB) : (shA != C);
                const double fac = offdiag ? 2.0 : 1.0;
                const int atA = ps.atom[shA];
                const int atB = ps.b_dummy ? -1 : ps.atom[shB];
                const int atC = ax.atom[C];
                double* G = smem_grad ? sgrad : grad;
                for (int d = 0; d < 3; ++d) {
                    const double vA = fac * gA[d], vB = fac * gB[d];
                    atomicAdd(G + 3 * atA + d, vA);
                    if (atB >= 0) atomicAdd(G + 3 * atB + d, vB);
                    atomicAdd(G + 3 * atC + d, -(vA + vB));
                }
            }
        }
        __syncwarp();
    }
    if (DERIV && smem_grad) {
        __syncthreads();
        for (int i = threadIdx.x; i < ngrad; i += blockDim.x)
            if (sgrad[i] != 0.0) atomicAdd(grad + i, sgrad[i]);
    }
}

__global__ void k_pair_tables(const double* __restrict__ cxyz, const int* __restrict__ spstart_sh,
                              const int* __restrict__ nprim_sh, const double* __restrict__ pexp,
                              const double* __restrict__ pcoef, const int* __restrict__ sp_A,
                              const int* __restrict__ sp_B, const int* __restrict__ sp_pstart,
                              const int* __restrict__ pp_sp, const int* __restrict__ pp_local, long npp, int b_dummy,
                              double* eta, double* Px,
                              double* Py, double* Pz, double* cK, double* ea, double* eb) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npp) return;
    const int sp = pp_sp[i];
    const int A = sp_A[sp];
    const int local = pp_local ? pp_local[i] : (int)(i - sp_pstart[sp]);
    if (b_dummy) {
        const double a = pexp[spstart_sh[A] + local];
        eta[i] = a;
        Px[i] = cxyz[3 * A + 0];
        Py[i] = cxyz[3 * A + 1];
        Pz[i] = cxyz[3 * A + 2];
        cK[i] = pcoef[spstart_sh[A] + local];
        ea[i] = a;
        eb[i] = 0.0;
        return;
    }
    const int B = sp_B[sp];
    const int nB = nprim_sh[B];
    const int ia = local / nB, ib = local - (local / nB) * nB;
    const double a = pexp[spstart_sh[A] + ia], b = pexp[spstart_sh[B] + ib];
    const double ca = pcoef[spstart_sh[A] + ia], cb = pcoef[spstart_sh[B] + ib];
    const double p = a + b, inv = 1.0 / p, mu = a * b * inv;
    double AB2 = 0.0;
    double P[3];
    for (int d = 0; d < 3; ++d) {
        const double Ad = cxyz[3 * A + d], Bd = cxyz[3 * B + d];
        AB2 += (Ad - Bd) * (Ad - Bd);
        P[d] = (a * Ad + b * Bd) * inv;
    }
    eta[i] = p;
    Px[i] = P[0];
    Py[i] = P[1];
    Pz[i] = P[2];
    cK[i] = (ca * cb) * exp(-mu * AB2);
    ea[i] = a;
    eb[i] = b;
}

// ---------------------------------------------------------------- host side

struct DeviceTable {
    bool ready = false;
    double* coef = nullptr;
    double* herm = nullptr;
    int* err = nullptr;  // staging wait error word (RysTable::err)
    RysTable tab;
};
static DeviceTable g_tables[64];
static bool g_binom_ready[64];

static int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

// Scratch policy of the generic path: one slot (nef or 3 nef doubles) per task
// of a batch; batches of up to DFB_SCRATCH_TASKS tasks, or fewer when the
// caller's scratch is smaller (the fixed scratch of dfb_rys_int_noalloc).
#define DFB_SCRATCH_TASKS 16384L

template <int KB, bool DERIV>
static int launch_rys(const ClassInfo& ci, const dfb_pair_side_t* ps, const dfb_aux_side_t* ax,
                      const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode, double* out,
                      long sP, long sM, long sN, const double* bar, long sbP, long sbM, long sbN, double* grad, int natm,
                      double* scratch, long scratch_doubles, cudaStream_t st, int query_only, long* need,
                      int fit_grid_to_scratch = 0) {
    const int dev = current_device();
    const long slot = (DERIV ? 3L : 1L) * ci.nef;
    if (query_only) {
        *need = (ntask < DFB_SCRATCH_TASKS ? (ntask > 0 ? ntask : 1) : DFB_SCRATCH_TASKS) * slot;
        return DFB_OK;
    }
    if (ntask == 0) return DFB_OK;
    if (scratch == nullptr || scratch_doubles < slot)
        return set_error(fit_grid_to_scratch ? DFB_ERR_UNSUPPORTED : DFB_ERR_INVALID,
                         "class (%d,%d,%d) needs %ld scratch doubles per task, the scratch holds %ld", ci.la, ci.lb,
                         ci.lc, slot, scratch_doubles);
    const int smem_grad = (DERIV && natm * 3 <= 4096) ? 1 : 0;
    const size_t smem_acc = sizeof(double) * ((size_t)DFB_WARPS_PER_BLOCK * (32 * ci.item + ci.nr * 3 * ci.gt));
    const size_t smem_epi = (smem_grad ? sizeof(double) * natm * 3 : 0) +
                            (sizeof(double) + sizeof(int)) * DFB_WARPS_PER_BLOCK * (DERIV ? 4 : 1) * DFB_HRR_TERMS;
    auto kacc = k_rys_acc<KB, DERIV>;
    auto kepi = k_rys_epi<DERIV>;
    if (smem_acc > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kacc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_acc);
        if (e != cudaSuccess) return set_cuda_error("cudaFuncSetAttribute", e);
    }
    int occ_acc = 0, occ_epi = 0, nsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_acc, kacc, DFB_WARPS_PER_BLOCK * 32, smem_acc);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_epi, kepi, DFB_WARPS_PER_BLOCK * 32, smem_epi);
    if (e != cudaSuccess) return set_cuda_error("occupancy", e);
    if (occ_acc < 1 || occ_epi < 1)
        return set_error(DFB_ERR_UNSUPPORTED, "class (%d,%d,%d) does not fit on an SM", ci.la, ci.lb, ci.lc);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int nchunk = (ci.nef + 32 * KB - 1) / (32 * KB);
    const long batch = scratch_doubles / slot;
    for (long t0 = 0; t0 < ntask; t0 += batch) {
        const long nt = (ntask - t0) < batch ? (ntask - t0) : batch;
        long b1 = (nt * nchunk + DFB_WARPS_PER_BLOCK - 1) / DFB_WARPS_PER_BLOCK;
        if (b1 > (long)occ_acc * nsm) b1 = (long)occ_acc * nsm;
        kacc<<<(unsigned)b1, DFB_WARPS_PER_BLOCK * 32, smem_acc, st>>>(ci, *ps, *ax, task_pair, task_aux, t0, nt,
                                                                          naux_grid, scratch, slot,
                                                                          g_tables[dev].tab);
        const long nec = (long)ci.nb * ((ci.na * ci.nc + DFB_EPI_CHUNK - 1) / DFB_EPI_CHUNK);
        long b2 = (nt * nec + DFB_WARPS_PER_BLOCK - 1) / DFB_WARPS_PER_BLOCK;
        if (b2 > (long)occ_epi * nsm) b2 = (long)occ_epi * nsm;
        kepi<<<(unsigned)b2, DFB_WARPS_PER_BLOCK * 32, smem_epi, st>>>(ci, *ps, *ax, task_pair, task_aux, t0, nt,
                                                                          naux_grid, mode, out, sP, sM, sN, bar, sbP,
                                                                          sbM, sbN, grad, natm, smem_grad, scratch,
                                                                          slot);
        count_launches(2);
        e = cudaGetLastError();
        if (e != cudaSuccess) return set_cuda_error("k_rys launch", e);
    }
    return DFB_OK;
}

template <bool DERIV>
static int dispatch_rys(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* ax,
                        const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode, double* out,
                        long sP, long sM, long sN, const double* bar, long sbP, long sbM, long sbN, double* grad, int natm,
                        double* scratch, long scratch_doubles, cudaStream_t st, int query_only, long* need,
                        int fit_grid_to_scratch = 0, int f32 = 0) {
    if (la < 0 || lb < 0 || lc < 0 || la > DFB_LMAX || lb > DFB_LMAX || lc > DFB_LMAX)
        return set_error(DFB_ERR_UNSUPPORTED, "angular momentum out of range (la=%d lb=%d lc=%d, max %d)", la, lb, lc,
                         DFB_LMAX);
    if (lb > la) return set_error(DFB_ERR_INVALID, "pairs must be l-ordered (la >= lb)");
    if (!query_only && ntask > 0 && (!ax->pexp || !ax->pcoef || !ax->rexp))
        return set_error(DFB_ERR_INVALID, "aux side without exponents, coefficients or reciprocal exponents");
    const ClassInfo ci = make_class(la, lb, lc, DERIV);
    if (ci.nr > DFB_NROOTS_MAX) return set_error(DFB_ERR_UNSUPPORTED, "too many Rys roots (%d)", ci.nr);
    const int dev = current_device();
    if (!query_only && !g_tables[dev].ready)
        return set_error(DFB_ERR_NOT_INITIALISED, "Rys table not uploaded on device %d", dev);
    if (!g_binom_ready[dev]) {
        double h[DFB_LMAX + 2][DFB_LMAX + 2];
        for (int n = 0; n < DFB_LMAX + 2; ++n)
            for (int k = 0; k < DFB_LMAX + 2; ++k) {
                double v = 0.0;
                if (k <= n) {
                    v = 1.0;
                    for (int i = 1; i <= k; ++i) v = v * (double)(n - k + i) / (double)i;
                }
                h[n][k] = v;
            }
        cudaError_t e = cudaMemcpyToSymbol(c_binomtab, h, sizeof(h));
        if (e != cudaSuccess) return set_cuda_error("binomial table upload", e);
        int nb[2 * DFB_LMAX + 4];
        for (int L = 0; L < 2 * DFB_LMAX + 4; ++L) nb[L] = ncart_below(L);
        e = cudaMemcpyToSymbol(c_ncbtab, nb, sizeof(nb));
        if (e != cudaSuccess) return set_cuda_error("index table upload", e);
        g_binom_ready[dev] = true;
    }
    if (!query_only && ntask > 0 && getenv("DFB_DISABLE_TMPL") == nullptr) {
        TmplArgs g;
        g.ps = *ps;
        g.ax = *ax;
        g.task_pair = task_pair;
        g.task_aux = task_aux;
        g.ntask = ntask;
        g.naux_grid = naux_grid;
        g.mode = mode;
        g.out = out;
        g.sP = sP;
        g.sM = sM;
        g.sN = sN;
        g.bar = bar;
        g.sbP = sbP;
        g.sbM = sbM;
        g.sbN = sbN;
        g.grad = grad;
        g.natm = natm;
        g.smem_grad = (DERIV && natm * 3 <= 4096) ? 1 : 0;
        g.tab = g_tables[dev].tab;
        const size_t smem = (g.smem_grad ? sizeof(double) * natm * 3 : 0) + sizeof(double) * 128 * 2 * ci.nr;
        const long nblk = (ntask + 127) / 128;
        if (nblk > 2147483647L) return set_error(DFB_ERR_INVALID, "too many tasks in one class launch");
        if (tmpl_launch(la, lb, lc, DERIV, f32 != 0, g, nblk, smem, st)) {
            count_launches(1);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return set_cuda_error("k_rys_thread launch", e);
            return DFB_OK;
        }
    }
    // scratch is needed only when one of the two component types runs this class on the generic kernel
    if (query_only && getenv("DFB_DISABLE_TMPL") == nullptr && tmpl_has(la, lb, lc, DERIV, false) &&
        tmpl_has(la, lb, lc, DERIV, true)) {
        *need = 0;
        return DFB_OK;
    }
    const int kb = (ci.nef + 31) / 32;
#define DFB_CASE(K)                                                                                              \
    if (kb <= K)                                                                                                 \
        return launch_rys<K, DERIV>(ci, ps, ax, task_pair, task_aux, ntask, naux_grid, mode, out, sP, sM, sN, bar, sbP, sbM, \
                                    sbN, grad, natm, scratch, scratch_doubles, st, query_only, need,      \
                                    fit_grid_to_scratch);
    DFB_CASE(1)
    DFB_CASE(2)
    DFB_CASE(4)
    DFB_CASE(8)
    DFB_CASE(16)
#undef DFB_CASE
    return launch_rys<16, DERIV>(ci, ps, ax, task_pair, task_aux, ntask, naux_grid, mode, out, sP, sM, sN, bar, sbP, sbM, sbN,
                                 grad, natm, scratch, scratch_doubles, st, query_only, need, fit_grid_to_scratch);
}

}  // namespace dfb

using namespace dfb;

extern "C" int dfb_rys_table_init(const double* coef, const int* offs, long ncoef, const double* herm,
                                  const int* hoffs, long nherm, int nmax, int nint, int deg, double tmax) {
    clear_error();
    if (nmax < 1 || nmax > DFB_NROOTS_MAX || nint < 1 || deg < 0 || !coef || !herm || !offs || !hoffs)
        return set_error(DFB_ERR_INVALID, "invalid Rys table description");
    if (deg != DFB_RYS_DEG)
        return set_error(DFB_ERR_INVALID, "Rys table degree %d, kernels are compiled for %d", deg, DFB_RYS_DEG);
    for (int n = 1; n <= nmax; ++n)
        if (offs[n] % 2 != 0) return set_error(DFB_ERR_INVALID, "Rys table blocks must be 16-byte aligned");
    const int dev = current_device();
    DeviceTable& t = g_tables[dev];
    if (t.ready) return DFB_OK;
    cudaError_t e = cudaMalloc(&t.coef, sizeof(double) * ncoef);
    if (e == cudaSuccess) e = cudaMalloc(&t.herm, sizeof(double) * nherm);
    if (e == cudaSuccess) e = cudaMalloc(&t.err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(t.err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(t.coef, coef, sizeof(double) * ncoef, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t.herm, herm, sizeof(double) * nherm, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return set_cuda_error("Rys table upload", e);
    t.tab.coef = t.coef;
    t.tab.herm = t.herm;
    t.tab.err = t.err;
    for (int n = 0; n <= DFB_NROOTS_MAX; ++n) {
        t.tab.offs[n] = (n >= 1 && n <= nmax) ? offs[n] : 0;
        t.tab.hoff[n] = (n >= 1 && n <= nmax) ? hoffs[n] : 0;
    }
    t.tab.nmax = nmax;
    t.tab.nint = nint;
    t.tab.deg = deg;
    t.tab.tmax = tmax;
    t.tab.inv_h = (double)nint / tmax;
    t.ready = true;
    return DFB_OK;
}

extern "C" int dfb_rys_error(int reset) {
    clear_error();
    const int dev = current_device();
    if (dev < 0 || dev >= 64 || !g_tables[dev].ready)
        return set_error(DFB_ERR_NOT_INITIALISED, "Rys table not uploaded on this device");
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, g_tables[dev].err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && reset && v != 0) e = cudaMemset(g_tables[dev].err, 0, sizeof(int));
    if (e != cudaSuccess) return set_cuda_error("dfb_rys_error", e);
    return v;
}

extern "C" int dfb_pair_tables(const double* cxyz, const int* shell_pstart, const int* shell_nprim,
                               const double* pexp, const double* pcoef, const int* sp_A, const int* sp_B,
                               const int* sp_pstart, const int* pp_sp, const int* pp_local, long npp, int b_dummy,
                               double* eta, double* Px,
                               double* Py, double* Pz, double* cK, double* ea, double* eb, void* stream) {
    clear_error();
    if (npp < 0) return set_error(DFB_ERR_INVALID, "npp < 0");
    if (npp == 0) return DFB_OK;
    const unsigned blocks = (unsigned)((npp + 255) / 256);
    k_pair_tables<<<blocks, 256, 0, (cudaStream_t)stream>>>(cxyz, shell_pstart, shell_nprim, pexp, pcoef, sp_A, sp_B,
                                                            sp_pstart, pp_sp, pp_local, npp, b_dummy, eta, Px, Py,
                                                            Pz, cK, ea, eb);
    count_launches(1);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error("k_pair_tables launch", e);
    return DFB_OK;
}

extern "C" int dfb_rys_int_prec(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* aux,
                                const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode,
                                int precision, double* out, long sP, long sM, long sN, double* scratch,
                                long scratch_doubles, void* stream) {
    clear_error();
    if (!ps || !aux || (ntask > 0 && (!task_pair || !task_aux || !out)) || (mode != 0 && mode != 1))
        return set_error(DFB_ERR_INVALID, "invalid arguments to dfb_rys_int");
    if (precision != DFB_PREC_FP64 && precision != DFB_PREC_MIXED)
        return set_error(DFB_ERR_INVALID, "unknown precision %d", precision);
    return dispatch_rys<false>(la, lb, lc, ps, aux, task_pair, task_aux, ntask, naux_grid, mode, out, sP, sM, sN, nullptr, 0, 0,
                               0, nullptr, 0, scratch, scratch_doubles, (cudaStream_t)stream, 0, nullptr, 0,
                               precision == DFB_PREC_MIXED);
}

extern "C" int dfb_rys_int(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* aux,
                           const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode, double* out, long sP,
                           long sM, long sN, double* scratch, long scratch_doubles, void* stream) {
    return dfb_rys_int_prec(la, lb, lc, ps, aux, task_pair, task_aux, ntask, naux_grid, mode, DFB_PREC_FP64, out, sP,
                            sM, sN, scratch, scratch_doubles, stream);
}

extern "C" int dfb_rys_deriv_prec(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* aux,
                                  const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode,
                                  int precision, const double* bar, long sbP, long sbM, long sbN, double* grad,
                                  int natm, double* scratch, long scratch_doubles, void* stream) {
    clear_error();
    if (!ps || !aux || (ntask > 0 && (!task_pair || !task_aux || !bar || !grad)) || (mode != 0 && mode != 1) ||
        natm < 1)
        return set_error(DFB_ERR_INVALID, "invalid arguments to dfb_rys_deriv");
    if (precision != DFB_PREC_FP64 && precision != DFB_PREC_MIXED)
        return set_error(DFB_ERR_INVALID, "unknown precision %d", precision);
    return dispatch_rys<true>(la, lb, lc, ps, aux, task_pair, task_aux, ntask, naux_grid, mode, nullptr, 0, 0, 0, bar, sbP, sbM,
                              sbN, grad, natm, scratch, scratch_doubles, (cudaStream_t)stream, 0, nullptr, 0,
                              precision == DFB_PREC_MIXED);
}

extern "C" int dfb_rys_deriv(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* aux,
                             const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode,
                             const double* bar,
                             long sbP, long sbM, long sbN, double* grad, int natm, double* scratch,
                             long scratch_doubles, void* stream) {
    return dfb_rys_deriv_prec(la, lb, lc, ps, aux, task_pair, task_aux, ntask, naux_grid, mode, DFB_PREC_FP64, bar,
                              sbP, sbM, sbN, grad, natm, scratch, scratch_doubles, stream);
}

extern "C" long dfb_rys_scratch_doubles(int la, int lb, int lc, long ntask, int deriv) {
    clear_error();
    long need = -1;
    dfb_pair_side_t ps;
    dfb_aux_side_t ax;
    memset(&ps, 0, sizeof(ps));
    memset(&ax, 0, sizeof(ax));
    int rc;
    if (deriv)
        rc = dispatch_rys<true>(la, lb, lc, &ps, &ax, nullptr, nullptr, ntask, 0, 0, nullptr, 0, 0, 0, nullptr, 0, 0, 0,
                                nullptr, 1, nullptr, 0, 0, 1, &need);
    else
        rc = dispatch_rys<false>(la, lb, lc, &ps, &ax, nullptr, nullptr, ntask, 0, 0, nullptr, 0, 0, 0, nullptr, 0, 0,
                                 0, nullptr, 1, nullptr, 0, 0, 1, &need);
    return rc == DFB_OK ? need : (long)rc;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of dfb_rys_int.
//
// Callers that cannot allocate device memory at the point where they need
// integrals -- a host framework that hands this library only its input and
// output buffers, code running under an external allocator that forbids new
// device allocations, or a plugin that must not touch the caller's memory
// pool -- cannot provide the scratch buffer dfb_rys_int requires for classes
// that run on the generic warp kernel.  This entry point uses a fixed scratch
// array that lives in the library's own device image instead.
//
// The array below is DFB_NOALLOC_SCRATCH_DOUBLES doubles (8 MiB) and every GPU
// that loads the library keeps it until the process exits.  Host code only
// sees a host-side stand-in for it, so its device address is looked up with
// cudaGetSymbolAddress on the first call on each device (with that device
// current) and cached; make that first call before any stream capture.  All
// calls share the array: each task overwrites the part it reads, so nothing
// needs clearing between calls, but calls that overlap on the GPU (different
// streams, or concurrent host threads) race on it and must be serialised by
// the caller.  The generic path needs one slot per task (the contracted
// intermediate: ne * nf doubles), so the class's tasks run in batches of
// floor(DFB_NOALLOC_SCRATCH_DOUBLES / slot) tasks, one accumulation and one
// epilogue launch per batch, in order on the caller's stream.  A class fails
// with DFB_ERR_UNSUPPORTED only when a single task's slot exceeds the array,
// which no class with l <= 8 on every centre does (the largest slot is about
// 38,000 doubles).
// ---------------------------------------------------------------------------

#define DFB_NOALLOC_SCRATCH_DOUBLES (1L << 20)
static __device__ __align__(256) double g_noalloc_scratch[DFB_NOALLOC_SCRATCH_DOUBLES];
static double* g_noalloc_ptr[64];

extern "C" int dfb_rys_int_noalloc(int la, int lb, int lc, const dfb_pair_side_t* ps, const dfb_aux_side_t* aux,
                                   const int* task_pair, const int* task_aux, long ntask, long naux_grid, int mode,
                                   double* out, long sP, long sM, long sN, void* stream) {
    clear_error();
    if (!ps || !aux || (ntask > 0 && (!task_pair || !task_aux || !out)) || (mode != 0 && mode != 1))
        return set_error(DFB_ERR_INVALID, "invalid arguments to dfb_rys_int_noalloc");
    const int dev = current_device();
    if (dev < 0 || dev >= 64) return set_error(DFB_ERR_INVALID, "device index %d out of range", dev);
    if (g_noalloc_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_cuda_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    return dispatch_rys<false>(la, lb, lc, ps, aux, task_pair, task_aux, ntask, naux_grid, mode, out, sP, sM, sN,
                               nullptr, 0, 0, 0, nullptr, 0, g_noalloc_ptr[dev], DFB_NOALLOC_SCRATCH_DOUBLES,
                               (cudaStream_t)stream, 0, nullptr, 1);
}
