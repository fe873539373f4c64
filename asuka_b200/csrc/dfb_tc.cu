// Split-BF16 GEMM on the fifth-generation tensor cores (tcgen05, sm_100a) for the
// mixed-precision DF contractions.
//
//   C[b] (+)= A[b] . B[b]^T      A: M x K, B: N x K, FP64 in, FP64 out
//
// Each FP64 operand element is split in registers into NT bfloat16 terms
// (x = t0 + t1 + t2, every term the rounded remainder of the previous ones: 8, 16,
// 24 significant bits) and written to shared memory in the UMMA canonical K-major
// layout.  One elected thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32)
// for the cross products whose order is at most 2^-16 relative (t0 t0; t0 t1, t1 t0;
// t0 t2, t1 t1, t2 t0), accumulating the leading product and the correction
// products in two separate FP32 accumulators in tensor memory; the epilogue reads
// both with tcgen05.ld and combines them in FP64.  FP32 accumulation runs over one
// k span per CTA (split-K); spans are combined with FP64 atomic adds.
//
// Operands are addressed through a two-level k index, k = kq * nk1 + k1, so strided
// views (the exchange update's W[Q, mu, i] with k = (Q, i), the transposed orbital
// matrix) need no copy.  Loads are plain (coalesced, vectorised where the k stride
// is 1), because the split happens in registers between the load and the store to
// shared memory; a 2-stage pipeline overlaps the loads and splits of one k chunk
// with the MMAs of the previous one.
//
// Every wait on an mbarrier is bounded: a wait that gives up records an error code
// (dfb_tc_error), the CTA skips its remaining work, waits (bounded) for its MMAs
// in flight, frees its tensor memory and exits.
//
// The reference runs these contractions as cuBLAS DGEMMs (FP64, or cuBLAS's FP64
// emulation in early SCF cycles): asuka/hf/cuda/ext/src/hf_df_jk_cuda_ext.cpp:231-598.

#include <cuda_bf16.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/dfb.h"
#include "dfb_internal.h"

namespace dfb {
namespace tc {

constexpr int BM = 128;       // UMMA M (cta_group::1): rows of the A tile = tensor-memory lanes
constexpr int BK = 32;        // k elements per pipeline stage (two UMMA k-steps of 16)
constexpr int NTHREADS = 128;  // 4 warps: all load and split, thread 0 issues, warp w reads lanes 32w..32w+31
constexpr int NSTAGE = 2;
constexpr long WAIT_LIMIT = 1L << 22;  // try_wait rounds before a wait gives up

__device__ int g_tc_error;  // 0, or the code of the first bounded wait that gave up

struct Operand {
    const double* p;
    long s_row, s_kq, s_k1, nk1, s_batch;
};

struct Args {
    Operand a, b;
    long M, N, K;
    double* C;
    long ldc, s_cbatch;
    int accumulate;  // 0: C = A B^T (one k span), 1: C += A B^T (FP64 atomic adds)
    int symmetric;   // A == B, M == N: tiles tn >= tm only, off-diagonal tiles also written transposed
    long kspan;      // k per CTA, a multiple of BK
    int ntm, ntn;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for phase `parity` of an mbarrier; false (and an error code) when it gives up
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int code) {
    for (long it = 0; it < WAIT_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicCAS(&g_tc_error, 0, code);
    return false;
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// UMMA shared-memory descriptor, K-major, no swizzle: core matrices of 8 rows x 16 bytes;
// LBO = byte distance of the two core matrices along k, SBO = of consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, absolute LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 accumulator, M = 128, N = n
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x = t0 + t1 + t2 (+ rounding below 2^-24 |x|): each term the bfloat16 rounding of what is left.
// The remainders are exact in FP32 (a bfloat16 term holds the leading 8 of the at most 24
// significant bits left), so after one rounding of x to FP32 the split runs in FP32.
template <int NT>
__device__ __forceinline__ void split_terms(double x, __nv_bfloat16 (&t)[NT]) {
    float r = (float)x;
#pragma unroll
    for (int i = 0; i < NT; ++i) {
        t[i] = __float2bfloat16_rn(r);
        r -= __bfloat162float(t[i]);
    }
}

// four consecutive k of one row: FP64 values, zero outside [0, kend) and rows >= nrow
__device__ __forceinline__ void load4(const Operand& o, long batch, long row, long nrow, long k, long kend,
                                      double (&v)[4]) {
    v[0] = v[1] = v[2] = v[3] = 0.0;
    if (row >= nrow || k >= kend) return;
    long ko = k / o.nk1;
    long ki = k - ko * o.nk1;
    const double* base = o.p + batch * o.s_batch + row * o.s_row;
    const double* q = base + ko * o.s_kq + ki * o.s_k1;
    if (o.s_k1 == 1 && ki + 3 < o.nk1 && k + 3 < kend && ((reinterpret_cast<uintptr_t>(q) & 15u) == 0)) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(q));
        const double2 b = __ldg(reinterpret_cast<const double2*>(q) + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
        return;
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        if (k + e < kend) v[e] = __ldg(base + ko * o.s_kq + ki * o.s_k1);
        if (++ki == o.nk1) {
            ki = 0;
            ++ko;
        }
    }
}

// byte offset of element (r, k) inside one term's tile: [r/8][k/8][r%8][k%8], BK = 32
__device__ __forceinline__ uint32_t tile_off(int r, int k) {
    return (uint32_t)((r >> 3) * (BK / 8) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

template <int NT>
__device__ __forceinline__ void store_split(uint8_t* tile, uint32_t term_bytes, int r, int k, const double (&v)[4]) {
    __nv_bfloat16 t[4][NT];
#pragma unroll
    for (int e = 0; e < 4; ++e) split_terms<NT>(v[e], t[e]);
    const uint32_t off = tile_off(r, k);
#pragma unroll
    for (int i = 0; i < NT; ++i) {
        uint2 w;
        w.x = (uint32_t)__bfloat16_as_ushort(t[0][i]) | ((uint32_t)__bfloat16_as_ushort(t[1][i]) << 16);
        w.y = (uint32_t)__bfloat16_as_ushort(t[2][i]) | ((uint32_t)__bfloat16_as_ushort(t[3][i]) << 16);
        *reinterpret_cast<uint2*>(tile + i * term_bytes + off) = w;
    }
}

template <int BN>
__host__ __device__ constexpr int tmem_cols() {
    return (2 * BN <= 32) ? 32 : (2 * BN <= 64) ? 64 : (2 * BN <= 128) ? 128 : (2 * BN <= 256) ? 256 : 512;
}

template <int BN, int NT>
__host__ __device__ constexpr int smem_bytes() {
    return NSTAGE * NT * (BM + BN) * BK * 2 + 64;
}

template <int BN, int NT>
__global__ void __launch_bounds__(NTHREADS) k_tc_gemm(Args g) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
    extern __shared__ __align__(1024) uint8_t smem[];
    constexpr uint32_t A_TERM = BM * BK * 2, B_TERM = BN * BK * 2;
    constexpr uint32_t STAGE = NT * (A_TERM + B_TERM);
    constexpr int TCOLS = tmem_cols<BN>();
    constexpr uint32_t IDESC = instr_desc_bf16(BN);
    constexpr uint32_t LBO = 128, SBO = (BK / 8) * 128;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + NSTAGE * STAGE);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + NSTAGE);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    // tile of this CTA
    int tm, tn;
    {
        int t = blockIdx.x;
        if (g.symmetric) {
            tm = 0;
            while (t >= g.ntn - tm) {
                t -= g.ntn - tm;
                ++tm;
            }
            tn = tm + t;
        } else {
            tm = t / g.ntn;
            tn = t - tm * g.ntn;
        }
    }
    const long batch = blockIdx.z;
    const long kbeg = (long)blockIdx.y * g.kspan;
    const long kend = (kbeg + g.kspan < g.K) ? kbeg + g.kspan : g.K;

    if (tid == 0) {
        mbar_init(smem_u32(&bars[0]), 1);
        mbar_init(smem_u32(&bars[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t acc_main = tmem, acc_corr = tmem + BN;

    uint32_t phase0 = 0, phase1 = 0;
    int pend0 = 0, pend1 = 0;  // commit outstanding on stage 0 / 1
    int stage = 0;
    bool first = true;
    int abort_local = 0;  // this thread's bounded wait gave up; made block-uniform by __syncthreads_or
    // Item (row, 4 consecutive k) of a thread: for its j-th item the warp covers 16 rows of one
    // 8-wide k octet -- lanes 0-7 rows 0-7 and lanes 8-15 the same rows' upper half of the
    // octet, lanes 16-31 the next 8 rows -- so a warp's 8-byte stores into the core-matrix
    // layout fill all 32 banks twice (two wavefronts, no conflict), and each pair of lanes reads
    // 64 contiguous bytes of a row.
    constexpr int NJA = BM * BK / 4 / NTHREADS, NJB = BN * BK / 4 / NTHREADS;
    const int lrow = (lane & 7) + 8 * (lane >> 4), lk = ((lane >> 3) & 1) * 4;
    auto item_a = [&](int j, int& r, int& k) {
        const int c = j * (NTHREADS / 32) + warp;
        r = (c % (BM / 16)) * 16 + lrow;
        k = (c / (BM / 16)) * 8 + lk;
    };
    auto item_b = [&](int j, int& r, int& k) {
        const int c = j * (NTHREADS / 32) + warp;
        r = (c % (BN / 16)) * 16 + lrow;
        k = (c / (BN / 16)) * 8 + lk;
    };
    for (long kc = kbeg; kc < kend; kc += BK) {
        // FP64 loads of this chunk (issued before waiting for the stage to free up)
        double va[NJA][4];
        double vb[NJB][4];
#pragma unroll
        for (int j = 0; j < NJA; ++j) {
            int r, k;
            item_a(j, r, k);
            load4(g.a, batch, (long)tm * BM + r, g.M, kc + k, kend, va[j]);
        }
#pragma unroll
        for (int j = 0; j < NJB; ++j) {
            int r, k;
            item_b(j, r, k);
            load4(g.b, batch, (long)tn * BN + r, g.N, kc + k, kend, vb[j]);
        }
        // the MMAs that last read this stage must be done
        if (stage == 0 && pend0) {
            if (!mbar_wait(smem_u32(&bars[0]), phase0, 1)) abort_local = 1;
            phase0 ^= 1;
            pend0 = 0;
        } else if (stage == 1 && pend1) {
            if (!mbar_wait(smem_u32(&bars[1]), phase1, 1)) abort_local = 1;
            phase1 ^= 1;
            pend1 = 0;
        }
        uint8_t* sa = smem + stage * STAGE;
        uint8_t* sb = sa + NT * A_TERM;
#pragma unroll
        for (int j = 0; j < NJA; ++j) {
            int r, k;
            item_a(j, r, k);
            store_split<NT>(sa, A_TERM, r, k, va[j]);
        }
#pragma unroll
        for (int j = 0; j < NJB; ++j) {
            int r, k;
            item_b(j, r, k);
            store_split<NT>(sb, B_TERM, r, k, vb[j]);
        }
        // generic-proxy stores -> visible to the tensor cores (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        fence_before_sync();
        if (__syncthreads_or(abort_local)) {
            abort_local = 1;
            break;
        }
        if (tid == 0) {
            fence_after_sync();
            const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sb);
#pragma unroll
            for (int ks = 0; ks < BK / 16; ++ks) {
                const uint32_t ko = ks * 2 * LBO;
                const uint32_t acc = (first && ks == 0) ? 0u : 1u;
                umma_bf16(acc_main, smem_desc(a0 + ko, LBO, SBO), smem_desc(b0 + ko, LBO, SBO), IDESC, acc);
                // correction products t_i t_j, i + j in [1, NT - 1]
                bool firstc = (first && ks == 0);
#pragma unroll
                for (int s = 1; s < NT; ++s)
#pragma unroll
                    for (int i = 0; i <= s; ++i) {
                        umma_bf16(acc_corr, smem_desc(a0 + i * A_TERM + ko, LBO, SBO),
                                  smem_desc(b0 + (s - i) * B_TERM + ko, LBO, SBO), IDESC, firstc ? 0u : 1u);
                        firstc = false;
                    }
            }
            umma_commit(smem_u32(&bars[stage]));
        }
        if (stage == 0)
            pend0 = 1;
        else
            pend1 = 1;
        stage ^= 1;
        first = false;
    }
    // drain: every commit of this CTA has arrived before tensor memory is read or freed
    if (pend0 && !mbar_wait(smem_u32(&bars[0]), phase0, 2)) abort_local = 1;
    if (pend1 && !mbar_wait(smem_u32(&bars[1]), phase1, 2)) abort_local = 1;
    const int aborted = __syncthreads_or(abort_local);
    fence_after_sync();
    if (!aborted && !first) {
        const long m = (long)tm * BM + warp * 32 + lane;
        double* Cb = g.C + batch * g.s_cbatch;
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v0[16], v1[16];
            const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
            tmem_ld16(acc_main + lane_base + c0, v0);
            tmem_ld16(acc_corr + lane_base + c0, v1);
            if (m < g.M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const long n = (long)tn * BN + c0 + i;
                    if (n >= g.N) break;
                    // symmetric products: the entries n <= m of the tile write both (m, n) and (n, m),
                    // so the result is exactly symmetric (n > m only occurs in off-diagonal tiles)
                    if (g.symmetric && tm == tn && n > m) continue;
                    const bool mirror = g.symmetric && n != m;
                    const double v = (double)v0[i] + (double)v1[i];
                    if (g.accumulate) {
                        atomicAdd(Cb + m * g.ldc + n, v);
                        if (mirror) atomicAdd(Cb + n * g.ldc + m, v);
                    } else {
                        Cb[m * g.ldc + n] = v;
                        if (mirror) Cb[n * g.ldc + m] = v;
                    }
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS) : "memory");
    }
}

template <int BN, int NT>
static int launch(const Args& g, long batch, cudaStream_t st) {
    auto k = k_tc_gemm<BN, NT>;
    constexpr int smem = smem_bytes<BN, NT>();
    // resident CTAs per SM x tensor-memory columns must fit the 512 columns of an SM, so that
    // tcgen05.alloc never waits on another CTA: pad the shared memory request when needed
    int dev = 0, smem_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    const int max_res = 512 / tmem_cols<BN>();
    int req = smem;
    if (smem_sm / (req + 1024) > max_res) req = smem_sm / (max_res + 1) - 1024 + 1;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, req);
    if (e != cudaSuccess) return set_cuda_error("cudaFuncSetAttribute(k_tc_gemm)", e);
    const long ntiles = g.symmetric ? (long)g.ntm * (g.ntm + 1) / 2 : (long)g.ntm * g.ntn;
    const long nsplit = (g.K + g.kspan - 1) / g.kspan;
    if (ntiles > 2147483647L || nsplit > 65535 || batch > 65535)
        return set_error(DFB_ERR_INVALID, "tensor-core GEMM grid too large (%ld tiles, %ld k spans, %ld batch)",
                         ntiles, nsplit, batch);
    k<<<dim3((unsigned)ntiles, (unsigned)nsplit, (unsigned)batch), NTHREADS, req, st>>>(g);
    count_launches(1);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error("k_tc_gemm launch", e);
    return DFB_OK;
}

template <int NT>
static int dispatch_bn(int bn, const Args& g, long batch, cudaStream_t st) {
    switch (bn) {
        case 32: return launch<32, NT>(g, batch, st);
        case 48: return launch<48, NT>(g, batch, st);
        case 64: return launch<64, NT>(g, batch, st);
        default: return launch<128, NT>(g, batch, st);
    }
}

}  // namespace tc
}  // namespace dfb

using namespace dfb;

extern "C" int dfb_tc_gemm(long M, long N, long K, long batch, const dfb_tc_operand_t* A, const dfb_tc_operand_t* B,
                           double* C, long ldc, long s_cbatch, int accumulate, int symmetric, int nterms, long kspan,
                           void* stream) {
    clear_error();
    if (M < 0 || N < 0 || K < 0 || batch < 0 || !A || !B || (M > 0 && N > 0 && batch > 0 && !C))
        return set_error(DFB_ERR_INVALID, "invalid arguments to dfb_tc_gemm");
    if (nterms != 2 && nterms != 3) return set_error(DFB_ERR_INVALID, "nterms must be 2 or 3 (got %d)", nterms);
    if (A->nk1 < 1 || B->nk1 < 1) return set_error(DFB_ERR_INVALID, "inner k extents must be >= 1");
    if (symmetric && (M != N || A->ptr != B->ptr))
        return set_error(DFB_ERR_INVALID, "symmetric products need A == B and M == N");
    if (M == 0 || N == 0 || batch == 0) return DFB_OK;
    if (K == 0) return set_error(DFB_ERR_INVALID, "K == 0: nothing to accumulate (clear C instead)");
    if (kspan <= 0) kspan = K;
    kspan = ((kspan + tc::BK - 1) / tc::BK) * tc::BK;
    if (!accumulate && kspan < K)
        return set_error(DFB_ERR_INVALID, "a k span shorter than K needs accumulate=1 (C += A B^T)");
    int bn = 128;
    const long nmin = N < 128 ? N : 128;
    if (nmin <= 32)
        bn = 32;
    else if (nmin <= 48)
        bn = 48;
    else if (nmin <= 64)
        bn = 64;
    if (symmetric) bn = 128;  // square tiles: the tile grids of m and n coincide
    tc::Args g;
    g.a = {A->ptr, A->s_row, A->s_kq, A->s_k1, A->nk1, A->s_batch};
    g.b = {B->ptr, B->s_row, B->s_kq, B->s_k1, B->nk1, B->s_batch};
    g.M = M;
    g.N = N;
    g.K = K;
    g.C = C;
    g.ldc = ldc;
    g.s_cbatch = s_cbatch;
    g.accumulate = accumulate;
    g.symmetric = symmetric;
    g.kspan = kspan;
    g.ntm = (int)((M + tc::BM - 1) / tc::BM);
    g.ntn = (int)((N + bn - 1) / bn);
    if (symmetric && g.ntm != g.ntn) return set_error(DFB_ERR_INVALID, "symmetric tiling mismatch");
    cudaStream_t st = (cudaStream_t)stream;
    return nterms == 3 ? tc::dispatch_bn<3>(bn, g, batch, st) : tc::dispatch_bn<2>(bn, g, batch, st);
}

extern "C" int dfb_tc_error(int reset) {
    clear_error();
    int v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, tc::g_tc_error, sizeof(int));
    if (e != cudaSuccess) return set_cuda_error("dfb_tc_error", e);
    if (reset && v != 0) {
        const int z = 0;
        e = cudaMemcpyToSymbol(tc::g_tc_error, &z, sizeof(int));
        if (e != cudaSuccess) return set_cuda_error("dfb_tc_error reset", e);
    }
    return v;
}
