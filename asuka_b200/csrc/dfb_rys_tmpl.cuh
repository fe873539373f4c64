// Class-specialised Rys kernels: one thread per (task, aux-component subset).
//
// For low and medium angular momenta the per-task work is dominated by the
// primitive loop (root evaluation, 2D recurrences, accumulation), so each
// thread owns one task -- an AB shell pair times one aux shell -- and keeps
// the recurrence tables and the contracted intermediate (e 0|f) in registers.
// LA, LB, LC, the root count and every loop bound are compile-time constants;
// every Cartesian component index is a template argument (integer_sequence
// folds), so all array indices are literal constants and the arrays live in
// registers.  Classes whose intermediate does not fit are split over FS
// threads, each owning a contiguous subset of the aux shell's Cartesian
// components (subset = blockIdx.y, uniform per block).
//
// Consecutive threads hold consecutive aux shells of the same AB pair (the
// task grid is pair-major and the aux list of a class is sorted by primitive
// count), so the pair-table reads of a warp are broadcasts and the primitive
// loops of a warp have similar trip counts.
//
// The derivative variant (DERIV) accumulates U = sum S, WA = sum 2a S and
// WB = sum 2b S over |e| in [LA-1, LA+LB+1] per primitive triplet and contracts
//   d/dA = 2a (a+1_d) - a_d (a-1_d),  d/dB = 2b [(a+1_d, b) + AB_d (a, b)] - b_d (a, b-1_d)
// with the adjoint tile; d/dC = -(d/dA + d/dB) (translational invariance).
#pragma once
#include <stdint.h>
#include <utility>

#include "../../include/dfb_types.h"
#include "dfb_common.cuh"

#define DFB_RYS_DEG 9  // polynomial degree of the Rys table (checked at upload)

namespace dfb {

__host__ __device__ constexpr int c_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int c_ncb(int L) { return L * (L + 1) * (L + 2) / 6; }

__host__ __device__ constexpr int c_cx(int l, int i) {
    int x = l;
    while (i > l - x) {
        i -= (l - x + 1);
        --x;
    }
    return x;
}
__host__ __device__ constexpr int c_cy(int l, int i) {
    int x = l;
    while (i > l - x) {
        i -= (l - x + 1);
        --x;
    }
    return l - x - i;
}
__host__ __device__ constexpr int c_cz(int l, int i) { return l - c_cx(l, i) - c_cy(l, i); }
__host__ __device__ constexpr int c_eidx(int LMIN, int x, int y, int z) {
    return c_ncb(x + y + z) - c_ncb(LMIN) + ((y + z) * (y + z + 1)) / 2 + z;
}
__host__ __device__ constexpr int c_eL(int LMIN, int e) {
    int L = LMIN;
    while (e >= c_ncart(L)) {
        e -= c_ncart(L);
        ++L;
    }
    return L;
}
__host__ __device__ constexpr int c_ex(int LMIN, int e) {
    return c_cx(c_eL(LMIN, e), e - (c_ncb(c_eL(LMIN, e)) - c_ncb(LMIN)));
}
__host__ __device__ constexpr int c_ey(int LMIN, int e) {
    return c_cy(c_eL(LMIN, e), e - (c_ncb(c_eL(LMIN, e)) - c_ncb(LMIN)));
}
__host__ __device__ constexpr int c_ez(int LMIN, int e) {
    return c_cz(c_eL(LMIN, e), e - (c_ncb(c_eL(LMIN, e)) - c_ncb(LMIN)));
}
__host__ __device__ constexpr double c_binom(int n, int k) {
    double v = 1.0;
    for (int i = 1; i <= k; ++i) v = v * (double)(n - k + i) / (double)i;
    return (k < 0 || k > n) ? 0.0 : v;
}

// Degree-9 polynomial in u by Estrin's scheme: five independent linear terms, then
// three levels of combination with u^2, u^4, u^8 -- a dependency depth of four
// fused multiply-adds instead of Horner's nine.
__device__ __forceinline__ double poly9(const double* c, double u, double u2, double u4, double u8) {
    const double p01 = fma(c[1], u, c[0]), p23 = fma(c[3], u, c[2]), p45 = fma(c[5], u, c[4]);
    const double p67 = fma(c[7], u, c[6]), p89 = fma(c[9], u, c[8]);
    const double q0 = fma(p23, u2, p01), q1 = fma(p67, u2, p45);
    return fma(p89, u8, fma(q1, u4, q0));
}

// Coefficient pair d of table function r for the row of interval k: global memory through the
// read-only cache, or the block's shared-memory copy of this root count's table (STAGED).
template <int NR, bool STAGED>
__device__ __forceinline__ double2 rys_coef2(const double* cnr, int k, int r, int d) {
    const double2* c = reinterpret_cast<const double2*>(cnr + (size_t)k * (2 * NR) * (DFB_RYS_DEG + 1)) +
                       r * ((DFB_RYS_DEG + 1) / 2) + d;
    if constexpr (STAGED)
        return *c;
    else
        return __ldg(c);
}

template <int NR, bool STAGED = false>
__device__ __forceinline__ void rys_eval_t(const RysTable& tab, const double* cnr, double T, double (&x)[NR],
                                           double (&w)[NR]) {
    if (T >= tab.tmax) {
        const double* h = tab.herm + tab.hoff[NR];
        const double rs = rsqrt(T);
        const double inv = rs * rs;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            x[i] = __ldg(h + i) * inv;
            w[i] = __ldg(h + NR + i) * rs;
        }
        return;
    }
    const double Th = T * tab.inv_h;
    int k = (int)Th;
    if (k > tab.nint - 1) k = tab.nint - 1;
    const double u = 2.0 * (Th - (double)k) - 1.0;
    constexpr int S = DFB_RYS_DEG + 1;
    static_assert(S == 10, "poly9 evaluates degree-9 tables");
    const double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4;
#pragma unroll
    for (int r = 0; r < 2 * NR; ++r) {
        double cf[S];
#pragma unroll
        for (int d = 0; d < S / 2; ++d) {
            const double2 v = rys_coef2<NR, STAGED>(cnr, k, r, d);
            cf[2 * d] = v.x;
            cf[2 * d + 1] = v.y;
        }
        const double acc = poly9(cf, u, u2, u4, u8);
        if (r < NR)
            x[r] = acc;
        else
            w[r - NR] = acc;
    }
}

// Same evaluation, two table functions at a time, results to a per-thread
// shared-memory slot r[0..NR) = nodes, r[NR..2NR) = weights (bounds the
// coefficient registers in flight); entry i sits at r[i * RS], so the slots of
// consecutive threads interleave and a warp's stores hit consecutive words.
template <int NR, int RS, bool STAGED = false>
__device__ __forceinline__ void rys_eval_smem(const RysTable& tab, const double* cnr, double T,
                                              double* __restrict__ r) {
    if (T >= tab.tmax) {
        const double* h = tab.herm + tab.hoff[NR];
        const double rs = rsqrt(T);
        const double inv = rs * rs;
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            r[i * RS] = __ldg(h + i) * inv;
            r[(NR + i) * RS] = __ldg(h + NR + i) * rs;
        }
        return;
    }
    const double Th = T * tab.inv_h;
    int k = (int)Th;
    if (k > tab.nint - 1) k = tab.nint - 1;
    const double u = 2.0 * (Th - (double)k) - 1.0;
    constexpr int S = DFB_RYS_DEG + 1;
    const double u2 = u * u, u4 = u2 * u2, u8 = u4 * u4;
#pragma unroll 1
    for (int f = 0; f < 2 * NR; f += 2) {
        double cf0[S], cf1[S];
#pragma unroll
        for (int d = 0; d < S / 2; ++d) {
            const double2 v0 = rys_coef2<NR, STAGED>(cnr, k, f, d);
            const double2 v1 = rys_coef2<NR, STAGED>(cnr, k, f + 1, d);
            cf0[2 * d] = v0.x;
            cf0[2 * d + 1] = v0.y;
            cf1[2 * d] = v1.x;
            cf1[2 * d + 1] = v1.y;
        }
        r[f * RS] = poly9(cf0, u, u2, u4, u8);
        r[(f + 1) * RS] = poly9(cf1, u, u2, u4, u8);
    }
}

// 2D recurrence tables of one root and direction in the component type R (double, or
// float for the mixed-precision kernels; the coefficients arrive already rounded to R).
template <int NM, int MM, typename R>
__device__ __forceinline__ void build_G_t(R (&G)[NM + 1][MM + 1], R g00, R C, R Cp, R B0, R B1, R B1p) {
    G[0][0] = g00;
#pragma unroll
    for (int a = 1; a <= NM; ++a) {
        R v = C * G[a - 1][0];
        if (a >= 2) v += B1 * (R)(a - 1) * G[a >= 2 ? a - 2 : 0][0];
        G[a][0] = v;
    }
#pragma unroll
    for (int b = 1; b <= MM; ++b) {
        R v = Cp * G[0][b - 1];
        if (b >= 2) v += B1p * (R)(b - 1) * G[0][b >= 2 ? b - 2 : 0];
        G[0][b] = v;
    }
#pragma unroll
    for (int a = 1; a <= NM; ++a) {
#pragma unroll
        for (int b = 1; b <= MM; ++b) {
            R v = (R)a * B0 * G[a - 1][b - 1] + Cp * G[a][b - 1];
            if (b >= 2) v += B1p * (R)(b - 1) * G[a][b >= 2 ? b - 2 : 0];
            G[a][b] = v;
        }
    }
}

struct TmplArgs {
    dfb_pair_side_t ps;
    dfb_aux_side_t ax;
    const int* task_pair;
    const int* task_aux;
    long ntask;
    long naux_grid;
    int mode;
    double* out;
    long sP, sM, sN;
    const double* bar;
    long sbP, sbM, sbN;
    double* grad;
    int natm;
    int smem_grad;
    RysTable tab;
};

static constexpr double kTwoPi52_t = 2.0 * 3.141592653589793238462643383279502884 *
                                     3.141592653589793238462643383279502884 * 1.772453850905516027298167483341145182;

// Compile-time description of one class, one component subset and one pass.
//   MODE 0: integrals            one accumulator  E  over |e| in [LA, LA+LB]
//   MODE 1: derivative, combined U, WA, WB        over |e| in [LA-1, LA+LB+1]
//   MODE 2: derivative, centre A U  over [LA-1, LA+LB-1], WA over [LA+1, LA+LB+1]
//   MODE 3: derivative, centre B U  over [LA, LA+LB-1],   WB over [LA, LA+LB+1]
// Centre C gets -(A + B) from the pass(es) that computed them.
// R: type of the recurrence tables and the accumulators (double; float in the
// mixed-precision kernels, where roots, weights, prefactors, the horizontal
// recurrence, the adjoint contraction and the gradient stay FP64).
template <int LA_, int LB_, int LC_, int FS_, int FSI_, int MODE_, typename R_ = double>
struct Cls {
    using R = R_;
    static constexpr int LA = LA_, LB = LB_, LC = LC_, FS = FS_, FSI = FSI_, MODE = MODE_;
    static constexpr bool DERIV = MODE > 0;
    static constexpr int NR = (LA + LB + LC + (DERIV ? 1 : 0)) / 2 + 1;
    static constexpr int NM = LA + LB + (DERIV ? 1 : 0);
    static constexpr int NF = c_ncart(LC);
    static constexpr int NFS = (NF + FS - 1) / FS;
    static constexpr int F0 = FSI * NFS;
    static constexpr int F1 = (F0 + NFS < NF) ? (F0 + NFS) : NF;
    static constexpr int NL = F1 - F0;
    static constexpr int NA = c_ncart(LA), NB = c_ncart(LB);
    static constexpr int NARR = MODE == 0 ? 1 : (MODE == 1 ? 3 : 2);
    // Angular range [lo(k), hi(k)] of the contracted intermediate accumulated in array k: only
    // what the epilogue reads.  Derivative (MODE 1, both centres): array 0 (weight 1) feeds the
    // (a-1, b) and (a, b-1) terms, array 1 (weight 2a) the (a+1, b) term, array 2 (weight 2b) the
    // (a, b+1) = (a+1, b) + AB (a, b) term.  MODE 2 / 3: the centre-A / centre-B halves.
    __host__ __device__ static constexpr int lo(int k) {
        return MODE == 0 ? LA
             : MODE == 1 ? (k == 0 ? (LA > 0 ? LA - 1 : 0) : (k == 1 ? LA + 1 : LA))
             : MODE == 2 ? (k == 0 ? (LA > 0 ? LA - 1 : 0) : LA + 1)
                         : LA;
    }
    __host__ __device__ static constexpr int hi(int k) {
        return MODE == 0 ? LA + LB
             : MODE == 1 ? (k == 0 ? LA + LB - 1 : NM)
             : MODE == 2 ? (k == 0 ? (LA > 0 ? LA + LB - 1 : -1) : LA + LB + 1)
                         : (k == 0 ? LA + LB - 1 : LA + LB + 1);
    }
    // weight of array k: 0 -> 1, 1 -> 2a, 2 -> 2b
    __host__ __device__ static constexpr int wt(int k) { return MODE == 1 ? k : (MODE == 2 ? (k == 0 ? 0 : 1) : (k == 0 ? 0 : 2)); }
    __host__ __device__ static constexpr int ne(int k) { return (k < NARR && hi(k) >= lo(k)) ? c_ncb(hi(k) + 1) - c_ncb(lo(k)) : 0; }
    static constexpr int NE0 = ne(0) > 0 ? ne(0) : 1, NE1 = ne(1) > 0 ? ne(1) : 1, NE2 = ne(2) > 0 ? ne(2) : 1;
    __host__ __device__ static constexpr int md(int d) {
        int m = 0;
        for (int f = F0; f < F1; ++f) {
            const int v = d == 0 ? c_cx(LC, f) : (d == 1 ? c_cy(LC, f) : c_cz(LC, f));
            m = v > m ? v : m;
        }
        return m;
    }
    static constexpr int MDX = md(0), MDY = md(1), MDZ = md(2);
    struct Acc {
        R a0[NE0][NL];
        R a1[NE1][NL];
        R a2[NE2][NL];
    };
    typedef R GtX[NM + 1][MDX + 1];
    typedef R GtY[NM + 1][MDY + 1];
    typedef R GtZ[NM + 1][MDZ + 1];
    typedef double ABt[3][LB + 2];

    template <int K>
    __device__ __forceinline__ static R& at(Acc& A, int e, int f) {
        if constexpr (K == 0) return A.a0[e][f];
        else if constexpr (K == 1) return A.a1[e][f];
        else return A.a2[e][f];
    }
    template <int K>
    __device__ __forceinline__ static double get(const Acc& A, int e, int f) {
        if constexpr (K == 0) return (double)A.a0[e][f];
        else if constexpr (K == 1) return (double)A.a1[e][f];
        else return (double)A.a2[e][f];
    }

    // accumulate element J = e*NL + f of array K for one root
    template <int K, int J>
    __device__ __forceinline__ static void acc_one(Acc& A, const GtX& Gx, const GtY& Gy, const GtZ& Gz, R a2, R b2) {
        constexpr int e = J / NL, f = J % NL;
        constexpr int ex = c_ex(lo(K), e), ey = c_ey(lo(K), e), ez = c_ez(lo(K), e);
        constexpr int fx = c_cx(LC, F0 + f), fy = c_cy(LC, F0 + f), fz = c_cz(LC, F0 + f);
        const R t = Gx[ex][fx] * Gy[ey][fy] * Gz[ez][fz];
        if constexpr (wt(K) == 0)
            at<K>(A, e, f) += t;
        else if constexpr (wt(K) == 1)
            at<K>(A, e, f) = fma(a2, t, at<K>(A, e, f));
        else
            at<K>(A, e, f) = fma(b2, t, at<K>(A, e, f));
    }
    template <int K, int... Js>
    __device__ __forceinline__ static void acc_arr(Acc& A, const GtX& Gx, const GtY& Gy, const GtZ& Gz, R a2, R b2,
                                                   std::integer_sequence<int, Js...>) {
        (acc_one<K, Js>(A, Gx, Gy, Gz, a2, b2), ...);
    }
    __device__ __forceinline__ static void acc_all(Acc& A, const GtX& Gx, const GtY& Gy, const GtZ& Gz, R a2, R b2) {
        acc_arr<0>(A, Gx, Gy, Gz, a2, b2, std::make_integer_sequence<int, ne(0) * NL>{});
        if constexpr (NARR > 1) acc_arr<1>(A, Gx, Gy, Gz, a2, b2, std::make_integer_sequence<int, ne(1) * NL>{});
        if constexpr (NARR > 2) acc_arr<2>(A, Gx, Gy, Gz, a2, b2, std::make_integer_sequence<int, ne(2) * NL>{});
    }
    __device__ __forceinline__ static void zero(Acc& A) {
#pragma unroll
        for (int e = 0; e < NE0; ++e)
#pragma unroll
            for (int f = 0; f < NL; ++f) A.a0[e][f] = R(0);
#pragma unroll
        for (int e = 0; e < NE1; ++e)
#pragma unroll
            for (int f = 0; f < NL; ++f) A.a1[e][f] = R(0);
#pragma unroll
        for (int e = 0; e < NE2; ++e)
#pragma unroll
            for (int f = 0; f < NL; ++f) A.a2[e][f] = R(0);
    }

    template <int N, int K>
    struct Binom {
        static constexpr double value = c_binom(N, K);
    };

    // (a b | f) from array K, all indices compile-time
    template <int K, int AX, int AY, int AZ, int BX, int BY, int BZ, int F, int KX, int KY, int KZ>
    __device__ __forceinline__ static double hrr_term(const Acc& A, const ABt& ABp) {
        constexpr double c = Binom<BX, KX>::value * Binom<BY, KY>::value * Binom<BZ, KZ>::value;
        constexpr int idx = c_eidx(lo(K), AX + KX, AY + KY, AZ + KZ);
        static_assert(idx >= 0 && idx < ne(K), "horizontal recurrence reads outside the accumulated range");
        return c * ABp[0][BX - KX] * ABp[1][BY - KY] * ABp[2][BZ - KZ] * get<K>(A, idx, F);
    }
    template <int K, int AX, int AY, int AZ, int BX, int BY, int BZ, int F, int... Ks>
    __device__ __forceinline__ static double hrr_sum(const Acc& A, const ABt& ABp, std::integer_sequence<int, Ks...>) {
        constexpr int NYZ = (BY + 1) * (BZ + 1);
        return (hrr_term<K, AX, AY, AZ, BX, BY, BZ, F, Ks / NYZ, (Ks / (BZ + 1)) % (BY + 1), Ks % (BZ + 1)>(A, ABp) +
                ...);
    }
    template <int K, int AX, int AY, int AZ, int BX, int BY, int BZ, int F>
    __device__ __forceinline__ static double hrr(const Acc& A, const ABt& ABp) {
        return hrr_sum<K, AX, AY, AZ, BX, BY, BZ, F>(
            A, ABp, std::make_integer_sequence<int, (BX + 1) * (BY + 1) * (BZ + 1)>{});
    }

    // output element J = (ia*NB + ib)*NL + f
    template <int J>
    __device__ __forceinline__ static void out_one(const Acc& A, const ABt& ABp, const TmplArgs& g, long aoA,
                                                   long aoB, long aoC) {
        constexpr int f = J % NL, ib = (J / NL) % NB, ia = J / (NL * NB);
        constexpr int ax = c_cx(LA, ia), ay = c_cy(LA, ia), az = c_cz(LA, ia);
        constexpr int bx = c_cx(LB, ib), by = c_cy(LB, ib), bz = c_cz(LB, ib);
        const double v = hrr<0, ax, ay, az, bx, by, bz, f>(A, ABp);
        const long P = aoC + F0 + f, mu = aoA + ia, nu = aoB + ib;
        if (g.mode == 0) {
            g.out[P * g.sP + mu * g.sM + nu * g.sN] = v;
            g.out[P * g.sP + nu * g.sM + mu * g.sN] = v;
        } else {
            g.out[P * g.sP + mu * g.sM] = v;
            g.out[mu * g.sP + P * g.sM] = v;
        }
    }
    template <int... Js>
    __device__ __forceinline__ static void out_all(const Acc& A, const ABt& ABp, const TmplArgs& g, long aoA,
                                                   long aoB, long aoC, std::integer_sequence<int, Js...>) {
        (out_one<Js>(A, ABp, g, aoA, aoB, aoC), ...);
    }

    // derivative of element J contracted with its adjoint value, direction D
    template <int J, int D>
    __device__ __forceinline__ static void der_dir(const Acc& A, const ABt& ABp, const double* AB, double gam,
                                                   double (&gA)[3], double (&gB)[3], bool bdummy) {
        constexpr int f = J % NL, ib = (J / NL) % NB, ia = J / (NL * NB);
        constexpr int ax = c_cx(LA, ia), ay = c_cy(LA, ia), az = c_cz(LA, ia);
        constexpr int bx = c_cx(LB, ib), by = c_cy(LB, ib), bz = c_cz(LB, ib);
        constexpr int ad = D == 0 ? ax : (D == 1 ? ay : az);
        constexpr int bd = D == 0 ? bx : (D == 1 ? by : bz);
        constexpr int px = ax + (D == 0), py = ay + (D == 1), pz = az + (D == 2);
        if constexpr (MODE == 1 || MODE == 2) {
            constexpr int KW = MODE == 1 ? 1 : 1;  // WA
            double dA = hrr<KW, px, py, pz, bx, by, bz, f>(A, ABp);
            if constexpr (ad > 0)
                dA -= (double)ad * hrr<0, ax - (D == 0), ay - (D == 1), az - (D == 2), bx, by, bz, f>(A, ABp);
            gA[D] = fma(gam, dA, gA[D]);
        }
        if constexpr (MODE == 1 || MODE == 3) {
            if (!bdummy) {
                constexpr int KW = MODE == 1 ? 2 : 1;  // WB
                double dB = hrr<KW, px, py, pz, bx, by, bz, f>(A, ABp) +
                            AB[D] * hrr<KW, ax, ay, az, bx, by, bz, f>(A, ABp);
                if constexpr (bd > 0)
                    dB -= (double)bd * hrr<0, ax, ay, az, bx - (D == 0), by - (D == 1), bz - (D == 2), f>(A, ABp);
                gB[D] = fma(gam, dB, gB[D]);
            }
        }
    }
    template <int J>
    __device__ __forceinline__ static void der_one(const Acc& A, const ABt& ABp, const double* AB,
                                                   const TmplArgs& g, long aoA, long aoB, long aoC, double (&gA)[3],
                                                   double (&gB)[3]) {
        constexpr int f = J % NL, ib = (J / NL) % NB, ia = J / (NL * NB);
        double gam;
        if (g.mode == 0)
            gam = g.bar[(aoC + F0 + f) * g.sbP + (aoA + ia) * g.sbM + (aoB + ib) * g.sbN];
        else
            gam = g.bar[(aoA + ia) * g.sbP + (aoC + F0 + f) * g.sbM];
        der_dir<J, 0>(A, ABp, AB, gam, gA, gB, g.ps.b_dummy);
        der_dir<J, 1>(A, ABp, AB, gam, gA, gB, g.ps.b_dummy);
        der_dir<J, 2>(A, ABp, AB, gam, gA, gB, g.ps.b_dummy);
    }
    template <int... Js>
    __device__ __forceinline__ static void der_all(const Acc& A, const ABt& ABp, const double* AB,
                                                   const TmplArgs& g, long aoA, long aoB, long aoC, double (&gA)[3],
                                                   double (&gB)[3], std::integer_sequence<int, Js...>) {
        (der_one<Js>(A, ABp, AB, g, aoA, aoB, aoC, gA, gB), ...);
    }
};

template <class CL, bool STAGED = false>
__device__ __forceinline__ void rys_thread_body(const TmplArgs& g, long task, double* sgrad, const double* cnr) {
    using R = typename CL::R;
    constexpr int NR = CL::NR, NM = CL::NM, LB = CL::LB;
    // per-thread root slot after the optional gradient buffer
    extern __shared__ double smem_all[];
    constexpr int RS = 128;  // threads per block: root slot entry i of thread t at sroot[i * 128]
    double* sroot = smem_all + ((CL::DERIV && g.smem_grad) ? g.natm * 3 : 0) + threadIdx.x;
    long tp, ta;
    task_indices(task, g.naux_grid, tp, ta);
    const int pair = g.task_pair[tp];
    const int C = g.task_aux[ta];
    const int shA = g.ps.shA[pair];
    const int shB = g.ps.b_dummy ? -1 : g.ps.shB[pair];
    if (CL::MODE == 3 && g.ps.b_dummy) return;  // no B centre
    double A[3], AB[3], Cc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        A[d] = g.ps.cxyz[3 * shA + d];
        const double Bd = g.ps.b_dummy ? 0.0 : g.ps.cxyz[3 * shB + d];
        AB[d] = A[d] - Bd;
        Cc[d] = g.ax.cxyz[3 * C + d];
    }
    const int p0 = g.ps.pstart[pair];
    const int nab = g.ps.npair[pair];
    const int c0 = g.ax.pstart[C];
    const int nc = g.ax.nprim[C];

    typename CL::Acc acc;
    CL::zero(acc);

    // No division in the primitive loops: 1/p once per primitive pair, 1/q from the aux
    // table, and one reciprocal square root s = (p+q)^(-1/2) per primitive triplet, with
    // 1/(p+q) = s^2 and the prefactor 2 pi^(5/2) / (p q sqrt(p+q)) = (2 pi^(5/2) cK / p) (cc / q) s.
    for (int iab = 0; iab < nab; ++iab) {
        const double p = g.ps.eta[p0 + iab];
        const double rp = 1.0 / p;
        const double cKr = kTwoPi52_t * g.ps.cK[p0 + iab] * rp;
        const double h_p = 0.5 * rp;
        const R a2 = CL::DERIV ? (R)(2.0 * g.ps.ea[p0 + iab]) : R(0);
        const R b2 = CL::DERIV ? (R)(2.0 * g.ps.eb[p0 + iab]) : R(0);
        const double Pp[3] = {g.ps.Px[p0 + iab], g.ps.Py[p0 + iab], g.ps.Pz[p0 + iab]};
        double PA[3], CP[3], PQ2 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            PA[d] = Pp[d] - A[d];
            CP[d] = Cc[d] - Pp[d];
            PQ2 += CP[d] * CP[d];
        }
        for (int ic = 0; ic < nc; ++ic) {
            const double q = g.ax.pexp[c0 + ic];
            const double rq = g.ax.rexp[c0 + ic];
            const double s = rsqrt(p + q);
            const double inv = s * s;
            const double T = p * q * inv * PQ2;
            const double pref = cKr * (g.ax.pcoef[c0 + ic] * rq) * s;
            // few roots: registers; more roots: shared-memory slot (bounds registers)
            constexpr int NRR = NR <= 2 ? NR : 1;
            double xr[NRR], wr[NRR];
            if constexpr (NR <= 2)
                rys_eval_t<NR, STAGED>(g.tab, cnr, T, xr, wr);
            else
                rys_eval_smem<NR, RS, STAGED>(g.tab, cnr, T, sroot);
            const double qi = q * inv, pi = p * inv;
            const double h_q = 0.5 * rq;
#pragma unroll
            for (int u = 0; u < NR; ++u) {
                double x, wu;
                if constexpr (NR <= 2) {
                    x = xr[u < NRR ? u : 0];
                    wu = wr[u < NRR ? u : 0];
                } else {
                    x = sroot[u * RS];
                    wu = sroot[(NR + u) * RS];
                }
                const double B0 = x * 0.5 * inv;
                const double B1 = (1.0 - x) * h_p + B0;
                const double B1p = (1.0 - x) * h_q + B0;
                typename CL::GtX Gx;
                typename CL::GtY Gy;
                typename CL::GtZ Gz;
                const R b0 = (R)B0, b1 = (R)B1, b1p = (R)B1p;
                build_G_t<NM, CL::MDX, R>(Gx, (R)(pref * wu), (R)(PA[0] + qi * x * CP[0]), (R)(-pi * x * CP[0]), b0,
                                          b1, b1p);
                build_G_t<NM, CL::MDY, R>(Gy, R(1), (R)(PA[1] + qi * x * CP[1]), (R)(-pi * x * CP[1]), b0, b1, b1p);
                build_G_t<NM, CL::MDZ, R>(Gz, R(1), (R)(PA[2] + qi * x * CP[2]), (R)(-pi * x * CP[2]), b0, b1, b1p);
                CL::acc_all(acc, Gx, Gy, Gz, a2, b2);
            }
        }
    }

    typename CL::ABt ABp;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ABp[d][0] = 1.0;
#pragma unroll
        for (int k = 1; k < LB + 2; ++k) ABp[d][k] = ABp[d][k - 1] * AB[d];
    }
    const long aoA = g.ps.aostart[shA];
    const long aoB = g.ps.b_dummy ? 0 : g.ps.aostart[shB];
    const long aoC = g.ax.aostart[C];
    constexpr int NOUT = CL::NA * CL::NB * CL::NL;
    if constexpr (!CL::DERIV) {
        CL::out_all(acc, ABp, g, aoA, aoB, aoC, std::make_integer_sequence<int, NOUT>{});
    } else {
        double gA[3] = {0.0, 0.0, 0.0}, gB[3] = {0.0, 0.0, 0.0};
        CL::der_all(acc, ABp, AB, g, aoA, aoB, aoC, gA, gB, std::make_integer_sequence<int, NOUT>{});
        const bool offdiag = (g.mode == 0) ? (shA != shB) : (shA != C);
        const double fac = offdiag ? 2.0 : 1.0;
        const int atA = g.ps.atom[shA];
        const int atB = g.ps.b_dummy ? -1 : g.ps.atom[shB];
        const int atC = g.ax.atom[C];
        double* G = g.smem_grad ? sgrad : g.grad;
        // With the aux-major task grid the lanes of a warp usually share the aux
        // shell, hence atom C: when all 32 lanes are converged and agree, reduce
        // over the warp first instead of 32 atomics on one address.
        const unsigned act = __activemask();
        const bool uniformC = (act == 0xffffffffu) && __all_sync(0xffffffffu, atC == __shfl_sync(0xffffffffu, atC, 0));
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double vA = fac * gA[d], vB = fac * gB[d];
            if (CL::MODE != 3) atomicAdd(G + 3 * atA + d, vA);
            if (CL::MODE != 2 && atB >= 0) atomicAdd(G + 3 * atB + d, vB);
            double vC = -(vA + vB);
            if (uniformC) {
                for (int s = 16; s > 0; s >>= 1) vC += __shfl_xor_sync(0xffffffffu, vC, s);
                if ((threadIdx.x & 31) == 0) atomicAdd(G + 3 * atC + d, vC);
            } else {
                atomicAdd(G + 3 * atC + d, vC);
            }
        }
    }
}

// grid.y enumerates (pass, component subset): SPLIT derivative classes run the
// centre-A pass on y < FS and the centre-B pass on FS <= y < 2 FS.
// MINB: resident 128-thread blocks per SM the register allocation must allow, chosen per class
// from measured timings (csrc/class_tuning.json, written by asuka_b200.tune_classes);
// DFB_THREAD_MIN_BLOCKS raises it for every class (the tuner's variant build).
#ifndef DFB_THREAD_MIN_BLOCKS
#define DFB_THREAD_MIN_BLOCKS 1
#endif

// Staging of the Rys coefficient table (STAGE): at block start one thread copies this root count's
// table (nint x 2 NR x 10 doubles: 30 KB per root) from global into shared memory with one bulk
// asynchronous copy (cp.async.bulk, completion counted on an mbarrier); the block's root
// evaluations then gather from shared memory instead of L1/L2.  Every wait on the mbarrier is
// bounded: a block whose wait gives up records an error code (dfb_rys_error), evaluates from the
// global table, and before it exits waits (bounded) once more for its copy in flight.
constexpr long RYS_WAIT_LIMIT = 1L << 22;

__device__ __forceinline__ uint32_t rys_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool rys_mbar_wait(uint32_t bar, uint32_t parity) {
    for (long it = 0; it < RYS_WAIT_LIMIT; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Doubles of the shared-memory table copy of root count nr, and its offset after the gradient
// buffer (ng doubles) and the root slots (128 x 2 nr doubles), rounded to 16 bytes.
__host__ __device__ constexpr long rys_stage_doubles(int nint, int nr) { return (long)nint * 2 * nr * (DFB_RYS_DEG + 1); }
__host__ __device__ constexpr long rys_stage_offset(long ng, int nr) { return (ng + 256L * nr + 1) & ~1L; }

template <int LA, int LB, int LC, int FS, bool DERIV, bool SPLIT, int MINB = 1, typename R = double,
          bool STAGE = false>
__global__ void __launch_bounds__(128, (DFB_THREAD_MIN_BLOCKS > MINB ? DFB_THREAD_MIN_BLOCKS : MINB))
    k_rys_thread(TmplArgs g) {
    extern __shared__ double sgrad[];
    const int ng = (DERIV && g.smem_grad) ? g.natm * 3 : 0;
    constexpr int NR = (LA + LB + LC + (DERIV ? 1 : 0)) / 2 + 1;
    const double* cnr = g.tab.coef + g.tab.offs[NR];
    [[maybe_unused]] bool staged = false;
    [[maybe_unused]] uint32_t bar = 0;
    if constexpr (STAGE) {
        __shared__ __align__(8) unsigned long long s_mbar;
        double* stab = sgrad + rys_stage_offset(ng, NR);
        const uint32_t bytes = (uint32_t)(rys_stage_doubles(g.tab.nint, NR) * sizeof(double));
        bar = rys_smem_u32(&s_mbar);
        staged = ((rys_smem_u32(stab) | (uint32_t)(uintptr_t)cnr) & 15u) == 0;  // uniform over the block
        if (staged) {
            if (threadIdx.x == 0) {
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
                asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
                                 "r"(rys_smem_u32(stab)), "l"(cnr), "r"(bytes), "r"(bar)
                             : "memory");
            }
        }
        if (DERIV && g.smem_grad) {
            for (int i = threadIdx.x; i < ng; i += blockDim.x) sgrad[i] = 0.0;
        }
        if (staged) {
            if (rys_mbar_wait(bar, 0)) {
                cnr = stab;
            } else {
                atomicCAS(g.tab.err, 0, 1);
                staged = false;  // evaluate from the global table; the copy is waited for at exit
            }
        }
        __syncthreads();
    } else if (DERIV && g.smem_grad) {
        for (int i = threadIdx.x; i < ng; i += blockDim.x) sgrad[i] = 0.0;
        __syncthreads();
    }
    constexpr int M0 = !DERIV ? 0 : (SPLIT ? 2 : 1);
    const long task = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (task < g.ntask) {
        switch (blockIdx.y) {
#define DFB_FSI(I)                                                                                              \
    case I:                                                                                                     \
        if constexpr (I < FS)                                                                                   \
            rys_thread_body<Cls<LA, LB, LC, FS, (I < FS ? I : 0), M0, R>, STAGE>(g, task, sgrad, cnr);         \
        else if constexpr (SPLIT && I < 2 * FS)                                                                 \
            rys_thread_body<Cls<LA, LB, LC, FS, (I >= FS && I < 2 * FS ? I - FS : 0), 3, R>, STAGE>(g, task,   \
                                                                                                   sgrad, cnr); \
        break;
            DFB_FSI(0) DFB_FSI(1) DFB_FSI(2) DFB_FSI(3) DFB_FSI(4) DFB_FSI(5) DFB_FSI(6) DFB_FSI(7)
            DFB_FSI(8) DFB_FSI(9) DFB_FSI(10) DFB_FSI(11) DFB_FSI(12) DFB_FSI(13) DFB_FSI(14) DFB_FSI(15)
            DFB_FSI(16) DFB_FSI(17) DFB_FSI(18) DFB_FSI(19) DFB_FSI(20) DFB_FSI(21) DFB_FSI(22) DFB_FSI(23)
            DFB_FSI(24) DFB_FSI(25) DFB_FSI(26) DFB_FSI(27) DFB_FSI(28) DFB_FSI(29) DFB_FSI(30) DFB_FSI(31)
            DFB_FSI(32) DFB_FSI(33) DFB_FSI(34) DFB_FSI(35) DFB_FSI(36) DFB_FSI(37) DFB_FSI(38) DFB_FSI(39)
            DFB_FSI(40) DFB_FSI(41) DFB_FSI(42) DFB_FSI(43) DFB_FSI(44) DFB_FSI(45) DFB_FSI(46) DFB_FSI(47)
            DFB_FSI(48) DFB_FSI(49) DFB_FSI(50) DFB_FSI(51) DFB_FSI(52) DFB_FSI(53) DFB_FSI(54) DFB_FSI(55)
#undef DFB_FSI
            default:
                break;
        }
    }
    if (DERIV && g.smem_grad) {
        __syncthreads();
        for (int i = threadIdx.x; i < ng; i += blockDim.x)
            if (sgrad[i] != 0.0) atomicAdd(g.grad + i, sgrad[i]);
    }
    if constexpr (STAGE) {
        // a copy whose wait gave up may still be landing in this block's shared memory
        if (!staged && ((rys_smem_u32(sgrad + rys_stage_offset(ng, NR)) | (uint32_t)(uintptr_t)(g.tab.coef + g.tab.offs[NR])) & 15u) == 0)
            if (!rys_mbar_wait(bar, 0)) atomicCAS(g.tab.err, 0, 2);
    }
}

}  // namespace dfb
