// FP64 dense kernel of the DF gradient: the 3c adjoint
//
//   Gamma[P] = Cw A_P Cw^T = U_P Cw^T,    U_P = Cw A_P,   A_P = d_P I - Z_P / 2 (symmetric)
//
// written as (nP, nao, nao).  The inner dimension is only nocc (tens), so the product is
// bound by writing Gamma (8 nP nao^2 bytes) and by the FP64 FMA pipe, not by reading U and Cw.
// Gamma_P is symmetric: one CTA computes one 64 x 64 tile (mt <= nt) of one P, 16 x 16 threads
// with 4 x 4 outputs each, operands staged in shared memory in k chunks of 32; the tile is
// staged in shared memory and written, and for an off-diagonal tile also its transpose, both
// row-contiguous.  In a diagonal tile the upper entries are mirrored onto the
// lower ones, so every Gamma_P is exactly symmetric.  About 0.57 of the full product's FMAs
// for nao = 416 (28 of 49 tiles).
//
// The reference forms this adjoint through its whitened-factor route (df_whiten_adjoint_Qmn,
// asuka/integrals/df_adjoint.py:172-235) with cuBLAS GEMMs; this build's adjoint formulation
// needs Gamma = Cw A_P Cw^T instead.

#include "../../include/dfb.h"
#include "dfb_internal.h"

namespace dfb {
namespace dense {

constexpr int GT = 64;       // tile edge
constexpr int KC = 64;       // k per shared-memory chunk
constexpr int NT = 256;      // threads per CTA (16 x 16)
constexpr int SK = GT + 2;   // row stride of the operand chunks (16-byte aligned rows)
constexpr int SC = GT + 1;   // row stride of the tile stage

// Position of tile column r (= 4 tx + 2 h + q: thread tx's pair h, element q) inside a row of
// the B chunk: the pairs of the 16 column threads are contiguous per h, so the 16-byte loads
// of a warp read 256 contiguous bytes (two wavefronts, no bank conflict).
__device__ __forceinline__ int bpos(int r) { return 32 * ((r >> 1) & 1) + 2 * (r >> 2) + (r & 1); }

__global__ void __launch_bounds__(NT, 3) k_gamma_sym(long nP, int nao, int nocc, const double* __restrict__ U,
                                                  long sUm, long sUp, const double* __restrict__ Cw,
                                                  double* __restrict__ out, int T) {
    extern __shared__ __align__(16) double smem[];  // sA (later the tile stage) | sB
    double* sA = smem;             // sA[c * SK + r] = U[P][mu0 + r][k0 + c]
    double* sB = smem + KC * SK;   // sB[c * SK + bpos(r)] = Cw[nu0 + r][k0 + c]
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    // upper-triangle tile (mt, nt), mt <= nt, of a T x T tile grid
    int idx = blockIdx.x, mt = 0;
    while (idx >= T - mt) {
        idx -= T - mt;
        ++mt;
    }
    const int nt = mt + idx;
    const int mu0 = mt * GT, nu0 = nt * GT;
    // staging: thread covers k column lc = tid % 64 of tile rows lr0 + 4 i (i < 16)
    const int lc = tid & (KC - 1), lr0 = tid / KC;
    // with nocc <= KC the Cw tile is the same for every P of this CTA: staged once
    const bool one_chunk = nocc <= KC;
    if (one_chunk) {
        const bool kin = lc < nocc;
#pragma unroll 4
        for (int i = 0; i < GT / (NT / KC); ++i) {
            const int r = lr0 + (NT / KC) * i;
            sB[lc * SK + bpos(r)] = (kin && nu0 + r < nao) ? Cw[(long)(nu0 + r) * nocc + lc] : 0.0;
        }
    }
    for (long P = blockIdx.y; P < nP; P += gridDim.y) {
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        const double* Up = U + P * sUp;
        for (int k0 = 0; k0 < nocc; k0 += KC) {
            __syncthreads();  // the previous chunk (or the previous P's tile stage) is consumed
            const bool kin = k0 + lc < nocc;
#pragma unroll 4
            for (int i = 0; i < GT / (NT / KC); ++i) {
                const int r = lr0 + (NT / KC) * i;
                sA[lc * SK + r] = (kin && mu0 + r < nao) ? Up[(long)(mu0 + r) * sUm + k0 + lc] : 0.0;
                if (!one_chunk)
                    sB[lc * SK + bpos(r)] = (kin && nu0 + r < nao) ? Cw[(long)(nu0 + r) * nocc + k0 + lc] : 0.0;
            }
            __syncthreads();
            const double* pa = sA + 4 * ty;
            const double* pb = sB + 2 * tx;
            auto step = [&](int c) {
                const double2 a01 = *reinterpret_cast<const double2*>(pa + c * SK);
                const double2 a23 = *reinterpret_cast<const double2*>(pa + c * SK + 2);
                const double2 b01 = *reinterpret_cast<const double2*>(pb + c * SK);
                const double2 b23 = *reinterpret_cast<const double2*>(pb + c * SK + 32);
                const double a[4] = {a01.x, a01.y, a23.x, a23.y};
                const double b[4] = {b01.x, b01.y, b23.x, b23.y};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
            };
            const int kc = (nocc - k0) < KC ? (nocc - k0) : KC;
#pragma unroll 8
            for (int c = 0; c < kc; ++c) step(c);
        }
        double* outP = out + P * (long)nao * nao;
        // stage the tile in shared memory, then write it and (off the diagonal) its transpose with
        // consecutive threads on consecutive columns: every store instruction fills whole sectors.
        // A diagonal tile writes its upper part (m <= n) and mirrors the strict upper part.
        __syncthreads();  // every thread is done reading sA
        double* sC = smem;  // sC[m * SC + n], over sA (sB stays)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) sC[(4 * ty + i) * SC + 4 * tx + j] = acc[i][j];
        __syncthreads();
        const int wc = tid & (GT - 1), wr0 = tid >> 6;  // column of this thread, first row
        const bool diag = mt == nt;
        if (nu0 + wc < nao) {
#pragma unroll 4
            for (int r = wr0; r < GT; r += NT / GT) {  // tile row r, column wc
                if (mu0 + r < nao && (!diag || r <= wc)) outP[(long)(mu0 + r) * nao + nu0 + wc] = sC[r * SC + wc];
            }
        }
        if (mu0 + wc < nao) {
#pragma unroll 4
            for (int r = wr0; r < GT; r += NT / GT) {  // transposed: output row nu0 + r, column mu0 + wc
                if (nu0 + r < nao && (!diag || wc < r)) outP[(long)(nu0 + r) * nao + mu0 + wc] = sC[wc * SC + r];
            }
        }
    }
}

}  // namespace dense
}  // namespace dfb

using namespace dfb;

extern "C" int dfb_gamma_sym(long nP, int nao, int nocc, const double* U, long sU_mu, long sU_P, const double* Cw,
                             double* out, void* stream) {
    clear_error();
    if (nP < 0 || nao < 0 || nocc < 0)
        return set_error(DFB_ERR_INVALID, "invalid sizes to dfb_gamma_sym (nP %ld, nao %d, nocc %d)", nP, nao, nocc);
    if (nP == 0 || nao == 0) return DFB_OK;
    if (nocc == 0) return set_error(DFB_ERR_INVALID, "nocc == 0: Gamma is zero (clear it instead)");
    if (!U || !Cw || !out || sU_mu < nocc || sU_P < 0)
        return set_error(DFB_ERR_INVALID, "invalid pointers or strides to dfb_gamma_sym");
    const int T = (nao + dense::GT - 1) / dense::GT;
    const long ntiles = (long)T * (T + 1) / 2;
    if (ntiles > 0x7fffffffL) return set_error(DFB_ERR_UNSUPPORTED, "nao %d too large", nao);
    // four P per CTA: the Cw tile is staged once per CTA, and many short CTAs keep the last wave small
    long gy = (nP + 3) / 4;
    if (gy > 65535) gy = 65535;
    if (gy < 1) gy = 1;
    const size_t smem = sizeof(double) * 2 * dense::KC * dense::SK;
    cudaError_t e = cudaFuncSetAttribute(dense::k_gamma_sym, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error("cudaFuncSetAttribute(k_gamma_sym)", e);
    dense::k_gamma_sym<<<dim3((unsigned)ntiles, (unsigned)gy), dense::NT, smem, (cudaStream_t)stream>>>(
        nP, nao, nocc, U, sU_mu, sU_P, Cw, out, T);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error("k_gamma_sym launch", e);
    return DFB_OK;
}
