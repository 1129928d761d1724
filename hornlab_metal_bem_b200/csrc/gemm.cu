// Trailing update of the blocked LU: A22 -= L21 * U12 (complex, planar),
// batched over matrices.  K = 16/32 inside a block column, 64 for the
// block's trailing matrix.
//
// CUDA-core path: 64 x 64 complex output tile per 256-thread CTA, 4 x 4
// complex outputs per thread, L and U chunks staged in shared memory by
// double-buffered cp.async and read with 128-bit broadcast loads; FP32 FMA gives the exact-FP32 products of
// LAPACK cgemm-based cgetrf.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "hbem_internal.h"

namespace hbem {
struct TcWorkspace;
namespace {

// C[start:n, col_start:col_end] -= L[start:n, k0:k0+kw] * U[k0:k0+kw, col_start:col_end]
// (kw a multiple of 16) for one 64 x 64 complex tile per CTA, K in chunks of
// 16 double-buffered through cp.async (the next chunk's loads
// are in flight while the current one is multiplied); 4 x 4 complex
// accumulators per thread.  L is stored transposed ([k][row]) with the row
// index XOR-swizzled by k, so the coalesced row-segment loads do not all
// land on one bank.
__global__ void __launch_bounds__(256) k_trailing_simt(float *a_re, float *a_im, long long lda, long long a_stride,
                                                       int n, int k0, int kw, int start, int col_start, int col_end) {
    constexpr int KC = 16;
    __shared__ __align__(16) float Lr[2][KC][64], Li[2][KC][64];
    __shared__ __align__(16) float Ur[2][KC][64], Ui[2][KC][64];
    const int mat = blockIdx.z;
    float *are = a_re + (size_t)mat * a_stride, *aim = a_im + (size_t)mat * a_stride;
    const int row0 = start + blockIdx.y * 64, col0 = col_start + blockIdx.x * 64;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    float cr[4][4], ci[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cr[i][j] = ci[i][j] = 0.f;
    auto load_chunk = [&](int kc, int sbuf) {
        for (int e = tid; e < 64 * KC; e += 256) {
            const int r = e / KC, kk = e - r * KC;
            const int gr = row0 + r;
            const bool ok = gr < n;
            const size_t off = ok ? (size_t)gr * lda + k0 + kc + kk : 0;
            const int rs = r ^ ((kk & 7) << 2);   // 16 k of one row on 8 banks instead of 1
            cp_async4(&Lr[sbuf][kk][rs], are + off, ok ? 4 : 0);
            cp_async4(&Li[sbuf][kk][rs], aim + off, ok ? 4 : 0);
        }
        for (int e = tid; e < 64 * KC; e += 256) {
            const int kk = e / 64, c = e - kk * 64;
            const int gc = col0 + c;
            const bool ok = gc < col_end;
            const size_t off = ok ? (size_t)(k0 + kc + kk) * lda + gc : 0;
            cp_async4(&Ur[sbuf][kk][c], are + off, ok ? 4 : 0);
            cp_async4(&Ui[sbuf][kk][c], aim + off, ok ? 4 : 0);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    };
    load_chunk(0, 0);
    int sbuf = 0;
    for (int kc = 0; kc < kw; kc += KC) {
        if (kc + KC < kw) {
            load_chunk(kc + KC, sbuf ^ 1);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            const int lo = (ty * 4) ^ ((kk & 7) << 2);   // XOR of a multiple of 4 keeps the float4 whole
            const float4 lr = *reinterpret_cast<const float4 *>(&Lr[sbuf][kk][lo]);
            const float4 li = *reinterpret_cast<const float4 *>(&Li[sbuf][kk][lo]);
            const float4 ur = *reinterpret_cast<const float4 *>(&Ur[sbuf][kk][tx * 4]);
            const float4 ui = *reinterpret_cast<const float4 *>(&Ui[sbuf][kk][tx * 4]);
            const float a_r[4] = {lr.x, lr.y, lr.z, lr.w}, a_i[4] = {li.x, li.y, li.z, li.w};
            const float b_r[4] = {ur.x, ur.y, ur.z, ur.w}, b_i[4] = {ui.x, ui.y, ui.z, ui.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    cr[i][j] = fmaf(a_r[i], b_r[j], cr[i][j]);
                    cr[i][j] = fmaf(-a_i[i], b_i[j], cr[i][j]);
                    ci[i][j] = fmaf(a_r[i], b_i[j], ci[i][j]);
                    ci[i][j] = fmaf(a_i[i], b_r[j], ci[i][j]);
                }
        }
        __syncthreads();
        sbuf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = row0 + ty * 4 + i;
        if (gr >= n) continue;
        const int gc = col0 + tx * 4;
        float *pr = are + (size_t)gr * lda + gc;
        float *pi = aim + (size_t)gr * lda + gc;
        if (gc + 3 < col_end && ((reinterpret_cast<uintptr_t>(pr) | reinterpret_cast<uintptr_t>(pi)) & 15) == 0) {
            float4 vr = *reinterpret_cast<float4 *>(pr), vi = *reinterpret_cast<float4 *>(pi);
            vr.x -= cr[i][0]; vr.y -= cr[i][1]; vr.z -= cr[i][2]; vr.w -= cr[i][3];
            vi.x -= ci[i][0]; vi.y -= ci[i][1]; vi.z -= ci[i][2]; vi.w -= ci[i][3];
            *reinterpret_cast<float4 *>(pr) = vr;
            *reinterpret_cast<float4 *>(pi) = vi;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (gc + j < col_end) {
                    pr[j] -= cr[i][j];
                    pi[j] -= ci[i][j];
                }
        }
    }
}

}  // namespace

int launch_trailing_tc(TcWorkspace *w, int n, int batch, int k0, int start, int col_start, int col_end, float *a_re,
                       float *a_im, long long lda, long long a_stride, int *status, cudaStream_t st,
                       int reserve_sms = 0);

// A[start:n, col_start:col_end] -= L[start:n, k0:k0+kw] U[k0:k0+kw, col_start:col_end] on the CUDA cores
int launch_trailing_simt(int n, int batch, int k0, int kw, int start, int col_start, int col_end, float *a_re,
                         float *a_im, long long lda, long long a_stride, cudaStream_t st) {
    const int m = n - start, w = col_end - col_start;
    if (m <= 0 || w <= 0) return HBEM_OK;
    if (kw % 16) return fail(HBEM_ERR_ARG, "trailing update: K must be a multiple of 16");
    dim3 grid((w + 63) / 64, (m + 63) / 64, batch);
    k_trailing_simt<<<grid, 256, 0, st>>>(a_re, a_im, lda, a_stride, n, k0, kw, start, col_start, col_end);
    HBEM_LAUNCH_CHECK("k_trailing_simt");
    return HBEM_OK;
}

int launch_trailing_update(int n, int batch, int k0, int kw, int start, int col_end, float *a_re, float *a_im,
                           long long lda, long long a_stride, TcWorkspace *tc, int *status, cudaStream_t st) {
    const int m = n - start, w = col_end - start;
    if (m <= 0 || w <= 0) return HBEM_OK;
    if (kw % 16) return fail(HBEM_ERR_ARG, "trailing update: K must be a multiple of 16");
    if (tc && kw == 64 && status)
        return launch_trailing_tc(tc, n, batch, k0, start, start, col_end, a_re, a_im, lda, a_stride, status, st);
    return launch_trailing_simt(n, batch, k0, kw, start, start, col_end, a_re, a_im, lda, a_stride, st);
}

}  // namespace hbem

// ===========================================================================
// Tensor-core trailing update (tcgen05, BF16x3 split products, FP32 TMEM
// accumulation) for the mixed-precision LU.
//
// The complex update C -= L U is one real GEMM: for a tile of 64 complex rows
// the 128 MMA rows are [Lr, -Li] (real part) and [Li, Lr] (imaginary part)
// against B = [Ur; Ui].  Each FP32 operand x is split into hi = bf16(x) and
// lo = bf16(x - hi); A B ~ Ah Bh + Ah Bl + Al Bh is a single K = 3 * 2 * 64
// = 384 contraction over the packed operands A3 = [Ah | Ah | Al] and
// B3^T = [Bh | Bl | Bh] (both K-major, written by k_pack_*), tiles of 64
// complex rows x 64 columns (k_trailing_tc: TMA ring, single-thread MMA
// issue into a 128 x 64 FP32 TMEM accumulator, C staged through shared
// memory by the epilogue warps).
// Every mbarrier wait is bounded; a timeout sets the status word and the CTA
// returns after releasing its TMEM.
// ===========================================================================
namespace hbem {
namespace {

constexpr int kTcM = 128;          // MMA rows per tile (64 complex rows: real and imaginary parts)
constexpr int kTcN = 64;           // columns per tile
constexpr int kTcKBlk = 64;        // bf16 elements per K-block (128 bytes)
constexpr int kTcK3 = 384;         // 3 x 2 x 64
constexpr int kTcKBlocks = kTcK3 / kTcKBlk;
constexpr int kTcStages = 4;       // operand ring
constexpr int kTcABytes = kTcM * kTcKBlk * 2;
constexpr int kTcBBytes = kTcN * kTcKBlk * 2;
constexpr int kTcStageBytes = kTcABytes + kTcBBytes;
constexpr int kTcCBytes = kTcM * kTcN * 4;   // one C tile staged in shared memory
constexpr int kTcThreads = 320;    // warp 0: MMA issuer, warp 1: TMA producer, warps 2-9: C tiles
constexpr size_t kTcSmem = (size_t)kTcStages * kTcStageBytes + 2 * kTcCBytes + 1024;
constexpr long long kSpinLimit = 1LL << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Bounded wait on an mbarrier phase; false after kSpinLimit polls or when
// another role has flagged a failure.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int *fail = nullptr) {
    for (long long it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (fail && (it & 1023) == 1023 && *fail) return false;
    }
    return false;
}

// K-major, 128-byte swizzle UMMA shared-memory descriptor: rows of 128 bytes
// in 8-row groups of 1024 bytes (stride byte offset 1024).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                           // leading byte offset (unused for SW128 K-major)
    d |= (uint64_t)(1024 >> 4) << 32;                 // stride byte offset
    d |= (uint64_t)1 << 46;                           // descriptor version (sm100)
    d |= (uint64_t)2 << 61;                           // layout: SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: BF16 A/B, FP32 accumulate, K-major A/B.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Barrier of the four C-tile warps that also ORs a predicate across them, so
// every warp takes the same branch afterwards.
__device__ __forceinline__ bool epi_bar_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 256, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred)
        : "memory");
    return r != 0;
}

struct TcTile {
    int mat, tm, tn;
};
__device__ __forceinline__ TcTile tc_tile(int t, int tiles_m, int tiles_n) {
    const int per = tiles_m * tiles_n;
    const int mat = t / per, rem = t - mat * per;
    return {mat, rem / tiles_n, rem - (rem / tiles_n) * tiles_n};
}

// Persistent trailing update: each CTA walks tiles b, b + G, b + 2G, ... of
// 64 complex rows x 64 columns (columns fastest, so consecutive tiles share
// their L panel in L2).
//   warp 1 (TMA producer): streams the six 64-wide K-blocks of A3 / B3 of
//     every tile through a 4-stage ring, running ahead across tiles;
//   warp 0 (MMA issuer): 4 x tcgen05.mma (M = 128, N = 64, K = 16) per block
//     into one of two TMEM accumulators, releases ring slots with
//     tcgen05.commit and signals "accumulator full";
//   warps 2-5 (C tiles): prefetch the next tile's C (real rows, then
//     imaginary rows) into one of two shared buffers with cp.async, drain the
//     finished accumulator into the current buffer (C - L U), hand the
//     accumulator back, and write the tile out with coalesced stores.
// Shared C layout: row r holds 16 groups of 4 columns, group g at position
// g ^ (r & 7) (aligned 16-byte copies, conflict-free float4 drain).  Every
// wait is bounded; a timeout sets *status and the roles stop, drain their
// copies, free TMEM and return.
__global__ void __launch_bounds__(kTcThreads, 1) k_trailing_tc(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB, float *a_re,
                                                                float *a_im, long long lda, long long a_stride, int n,
                                                                int start, int col_start, int col_end, int rows3,
                                                                int cols_pad,
                                                                int tiles_m, int tiles_n, int n_tiles, int *status) {
    extern __shared__ uint8_t s_raw[];
    __shared__ uint64_t s_full[kTcStages], s_empty[kTcStages];
    __shared__ uint64_t s_acc_full[2], s_acc_empty[2];
    __shared__ uint64_t s_done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(s_raw) + 1023) & ~(uintptr_t)1023);
    float *sC0 = reinterpret_cast<float *>(base + (size_t)kTcStages * kTcStageBytes);
    if (tid == 0) {
        s_fail = 0;
        for (int s = 0; s < kTcStages; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_empty[s])));
        }
        for (int b = 0; b < 2; ++b) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_acc_full[b])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 8;" ::"r"(smem_u32(&s_acc_empty[b])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_done)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(2 * kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;
    const int G = gridDim.x;
    const int my_tiles = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / G + 1 : 0;

    if (warp == 1) {
        // ---- TMA producer
        if (lane == 0) {
            int last_use[kTcStages];
            for (int s = 0; s < kTcStages; ++s) last_use[s] = -1;
            bool ok = true;
            long long g = 0;   // ring position
            for (int i = 0; i < my_tiles && ok; ++i) {
                const TcTile tt = tc_tile(blockIdx.x + i * G, tiles_m, tiles_n);
                const int row_a = tt.mat * rows3 + tt.tm * kTcM;
                const int row_b = tt.mat * cols_pad + tt.tn * kTcN;
                for (int kb = 0; kb < kTcKBlocks; ++kb, ++g) {
                    const int s = (int)(g % kTcStages);
                    const int u = (int)(g / kTcStages);
                    if (u > 0 && !mbar_wait(smem_u32(&s_empty[s]), (u - 1) & 1, &s_fail)) { ok = false; break; }
                    uint8_t *sa = base + (size_t)s * kTcStageBytes;
                    uint8_t *sb = sa + kTcABytes;
                    const uint32_t bar = smem_u32(&s_full[s]);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                                 "r"(kTcStageBytes)
                                 : "memory");
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                        ::"r"(smem_u32(sa)), "l"(reinterpret_cast<uint64_t>(&tmA)), "r"(kb * kTcKBlk), "r"(row_a),
                          "r"(bar)
                        : "memory");
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                        ::"r"(smem_u32(sb)), "l"(reinterpret_cast<uint64_t>(&tmB)), "r"(kb * kTcKBlk), "r"(row_b),
                          "r"(bar)
                        : "memory");
                    last_use[s] = u;
                }
            }
            if (!ok) {
                s_fail = 1;
                atomicExch(status, 3);
            }
            // every issued copy must land before the CTA may exit
            for (int s = 0; s < kTcStages; ++s)
                if (last_use[s] >= 0) mbar_wait(smem_u32(&s_full[s]), last_use[s] & 1);
        }
    } else if (warp == 0) {
        // ---- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = umma_idesc_bf16(kTcM, kTcN);
            bool ok = true;
            long long g = 0;
            for (int i = 0; i < my_tiles && ok; ++i) {
                const int b = i & 1;
                // the epilogue must have drained this accumulator (tile i - 2)
                if (i >= 2 && !mbar_wait(smem_u32(&s_acc_empty[b]), ((i >> 1) - 1) & 1, &s_fail)) {
                    ok = false;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_addr = tmem + (uint32_t)(b * kTcN);
                for (int kb = 0; kb < kTcKBlocks; ++kb, ++g) {
                    const int s = (int)(g % kTcStages);
                    const int u = (int)(g / kTcStages);
                    if (!mbar_wait(smem_u32(&s_full[s]), u & 1, &s_fail)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = smem_u32(base + (size_t)s * kTcStageBytes);
                    const uint32_t sb = sa + kTcABytes;
#pragma unroll
                    for (int kk = 0; kk < kTcKBlk / 16; ++kk) {
                        const uint64_t da = umma_desc_sw128(sa + kk * 32);
                        const uint64_t db = umma_desc_sw128(sb + kk * 32);
                        const uint32_t acc = (kb > 0 || kk > 0) ? 1u : 0u;
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                            ::"r"(acc_addr), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&s_empty[s]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&s_acc_full[b]))
                             : "memory");
            }
            if (!ok) {
                s_fail = 1;
                atomicExch(status, 1);
            }
            // completion of everything issued, before TMEM may be freed
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&s_done))
                         : "memory");
            mbar_wait(smem_u32(&s_done), 0);
        }
    } else {
        // ---- C tiles: 8 warps; thread et owns column group gq = et & 15 of
        // rows (et >> 4) + 16 it; warp pair (w, w + 4) shares TMEM lane
        // quarter w & 3 and drains columns [32 h, 32 h + 32), h = (w - 2) >> 2.
        const int et = tid - 64;   // 0..255
        const int q = warp & 3;
        const int h = (warp - 2) >> 2;
        const int gq = et & 15, r_first = et >> 4;
        auto sidx = [](int r, int c) { return r * kTcN + ((((c >> 2) ^ (r & 7)) << 2) | (c & 3)); };
        auto prefetch = [&](int t, float *sC) {
            const TcTile tt = tc_tile(t, tiles_m, tiles_n);
            const int row_c0 = start + tt.tm * 64, gcol = col_start + tt.tn * kTcN + 4 * gq;
            if (gcol >= col_end) {
                asm volatile("cp.async.commit_group;" ::: "memory");
                return;
            }
            const bool full4 = gcol + 3 < col_end;
            const float *mre = a_re + (size_t)tt.mat * a_stride + gcol, *mim = a_im + (size_t)tt.mat * a_stride + gcol;
#pragma unroll
            for (int it = 0; it < kTcM / 16; ++it) {
                const int r = r_first + 16 * it;
                const int grow = row_c0 + (r & 63);
                if (grow >= n) continue;
                const float *src = ((r < 64) ? mre : mim) + (size_t)grow * lda;
                const uint32_t dst = smem_u32(sC + sidx(r, 4 * gq));
                if (full4 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
                } else {
                    for (int j = 0; j < 4; ++j)
                        if (gcol + j < col_end)
                            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(
                                             smem_u32(sC + sidx(r, 4 * gq + j))),
                                         "l"(src + j)
                                         : "memory");
                }
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        if (my_tiles > 0) prefetch(blockIdx.x, sC0);
        for (int i = 0; i < my_tiles; ++i) {
            const int b = i & 1;
            float *sC = sC0 + (size_t)b * (kTcM * kTcN);
            if (i + 1 < my_tiles) {
                prefetch(blockIdx.x + (i + 1) * G, sC0 + (size_t)(b ^ 1) * (kTcM * kTcN));
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
            bool ok = true;
            if (!mbar_wait(smem_u32(&s_acc_full[b]), (i >> 1) & 1, &s_fail)) {
                ok = false;
                atomicExch(status, 2);
                s_fail = 1;
            }
            // the C tile's copies from every thread have landed; stop together on any failure
            if (epi_bar_or(!ok || s_fail != 0)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            {
                const int r = q * 32 + lane;
                const int c0 = 32 * h;
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                    "%13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
                    "[%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                      "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                      "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                      "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                      "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    float4 *p4 = reinterpret_cast<float4 *>(sC + sidx(r, c0 + 4 * jj));
                    float4 cv = *p4;
                    cv.x -= __uint_as_float(v[4 * jj]);
                    cv.y -= __uint_as_float(v[4 * jj + 1]);
                    cv.z -= __uint_as_float(v[4 * jj + 2]);
                    cv.w -= __uint_as_float(v[4 * jj + 3]);
                    *p4 = cv;
                }
            }
            // hand the accumulator back (one arrival per warp)
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&s_acc_empty[b])) : "memory");
            epi_bar();   // the whole tile is drained
            {
                const TcTile tt = tc_tile(blockIdx.x + i * G, tiles_m, tiles_n);
                const int row_c0 = start + tt.tm * 64, gcol = col_start + tt.tn * kTcN + 4 * gq;
                if (gcol < col_end) {
                    const bool full4 = gcol + 3 < col_end;
                    float *mre = a_re + (size_t)tt.mat * a_stride + gcol, *mim = a_im + (size_t)tt.mat * a_stride + gcol;
#pragma unroll
                    for (int it = 0; it < kTcM / 16; ++it) {
                        const int r = r_first + 16 * it;
                        const int grow = row_c0 + (r & 63);
                        if (grow >= n) continue;
                        float *dst = ((r < 64) ? mre : mim) + (size_t)grow * lda;
                        const float4 cv = *reinterpret_cast<const float4 *>(sC + sidx(r, 4 * gq));
                        if (full4 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
                            *reinterpret_cast<float4 *>(dst) = cv;
                        } else {
                            const float e4[4] = {cv.x, cv.y, cv.z, cv.w};
                            for (int j = 0; j < 4; ++j)
                                if (gcol + j < col_end) dst[j] = e4[j];
                        }
                    }
                }
            }
            epi_bar();   // buffer b may be refilled by the prefetch of tile i + 2
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTcN));
}

// Pack L21 (rows start..n, cols k0..k0+64) into A3 (K-major, bf16 hi/lo).
__global__ void k_pack_a(const float *a_re, const float *a_im, long long lda, long long a_stride, int n, int start,
                         int k0, int rows3, int rows_used, __nv_bfloat16 *A3) {
    const int mat = blockIdx.z;
    const int i = blockIdx.x * blockDim.y + threadIdx.y;  // complex row offset
    const int k = threadIdx.x;                            // 0..63
    const int m = n - start;
    if (i >= rows_used) return;                           // complex rows incl. tile padding
    float lr = 0.f, li = 0.f;
    if (i < m) {
        lr = a_re[(size_t)mat * a_stride + (size_t)(start + i) * lda + k0 + k];
        li = a_im[(size_t)mat * a_stride + (size_t)(start + i) * lda + k0 + k];
    }
    const int t = i >> 6, rl = i & 63;
    __nv_bfloat16 *re_row = A3 + ((size_t)mat * rows3 + (size_t)t * 128 + rl) * kTcK3;
    __nv_bfloat16 *im_row = re_row + (size_t)64 * kTcK3;
    auto put = [](__nv_bfloat16 *row, int k2, float x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        row[k2] = h;
        row[128 + k2] = h;
        row[256 + k2] = l;
    };
    put(re_row, k, lr);
    put(re_row, 64 + k, -li);
    put(im_row, k, li);
    put(im_row, 64 + k, lr);
}

// Pack U12 (rows k0..k0+64, cols start..col_end) into B3^T (K-major).
__global__ void k_pack_b(const float *a_re, const float *a_im, long long lda, long long a_stride, int start,
                         int col_end, int k0, int cols_pad, int cols_used, __nv_bfloat16 *B3) {
    const int mat = blockIdx.z;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;  // column offset
    const int k = blockIdx.y;                             // 0..63
    if (j >= cols_used) return;
    float ur = 0.f, ui = 0.f;
    if (start + j < col_end) {
        ur = a_re[(size_t)mat * a_stride + (size_t)(k0 + k) * lda + start + j];
        ui = a_im[(size_t)mat * a_stride + (size_t)(k0 + k) * lda + start + j];
    }
    __nv_bfloat16 *row = B3 + ((size_t)mat * cols_pad + j) * kTcK3;
    auto put = [&](int k2, float x) {
        const __nv_bfloat16 h = __float2bfloat16_rn(x);
        const __nv_bfloat16 l = __float2bfloat16_rn(x - __bfloat162float(h));
        row[k2] = h;
        row[128 + k2] = l;
        row[256 + k2] = h;
    };
    put(k, ur);
    put(64 + k, ui);
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

int make_map(CUtensorMap *map, void *ptr, long long rows, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(HBEM_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    const cuuint64_t dims[2] = {(cuuint64_t)kTcK3, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)kTcK3 * 2};
    const cuuint32_t box[2] = {(cuuint32_t)kTcKBlk, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(HBEM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return HBEM_OK;
}

}  // namespace

// Packed-operand workspace and tensor maps for one factorisation: sized for
// the first (largest) trailing update and reused by the later, smaller ones.
struct TcWorkspace {
    __nv_bfloat16 *A3 = nullptr, *B3 = nullptr;
    int rows3 = 0, cols_pad = 0, batch = 0;
    CUtensorMap ma, mb;
};

int tc_workspace_create(int n, int batch, TcWorkspace **out, cudaStream_t st) {
    *out = nullptr;
    auto *w = new TcWorkspace();
    w->rows3 = ((n + 63) / 64) * kTcM;
    w->cols_pad = ((n + kTcN - 1) / kTcN) * kTcN;
    w->batch = batch;
    cudaError_t e = cudaMallocAsync((void **)&w->A3, (size_t)batch * w->rows3 * kTcK3 * 2, st);
    if (e == cudaSuccess) e = cudaMallocAsync((void **)&w->B3, (size_t)batch * w->cols_pad * kTcK3 * 2, st);
    if (e != cudaSuccess) {
        if (w->A3) cudaFreeAsync(w->A3, st);
        delete w;
        return cuda_fail(e, "tensor-core workspace");
    }
    int rc = make_map(&w->ma, w->A3, (long long)batch * w->rows3, kTcM);
    if (rc == HBEM_OK) rc = make_map(&w->mb, w->B3, (long long)batch * w->cols_pad, kTcN);
    if (rc != HBEM_OK) {
        cudaFreeAsync(w->A3, st);
        cudaFreeAsync(w->B3, st);
        delete w;
        return rc;
    }
    *out = w;
    return HBEM_OK;
}

void tc_workspace_destroy(TcWorkspace *w, cudaStream_t st) {
    if (!w) return;
    cudaFreeAsync(w->A3, st);
    cudaFreeAsync(w->B3, st);
    delete w;
}

// Mixed-precision trailing update with K = 64 (one LU block); status
// receives 1/2 if a barrier wait timed out.  The persistent grid leaves
// reserve_sms SMs (at most half of them) to kernels on other streams.
// A[start:n, col_start:col_end] -= L[start:n, k0:k0+64] U[k0:k0+64, col_start:col_end] on the tensor cores
int launch_trailing_tc(TcWorkspace *w, int n, int batch, int k0, int start, int col_start, int col_end, float *a_re,
                       float *a_im, long long lda, long long a_stride, int *status, cudaStream_t st,
                       int reserve_sms) {
    const int m = n - start, wd = col_end - col_start;
    if (m <= 0 || wd <= 0) return HBEM_OK;
    const int tiles_m = (m + 63) / 64, tiles_n = (wd + kTcN - 1) / kTcN;
    // packed rows use the workspace's fixed per-matrix pitch (rows3 / cols_pad)
    {
        dim3 blk(64, 4), grd((tiles_m * 64 + 3) / 4, 1, batch);
        k_pack_a<<<grd, blk, 0, st>>>(a_re, a_im, lda, a_stride, n, start, k0, w->rows3, tiles_m * 64, w->A3);
        HBEM_LAUNCH_CHECK("k_pack_a");
    }
    {
        dim3 grd((tiles_n * kTcN + 127) / 128, 64, batch);
        k_pack_b<<<grd, 128, 0, st>>>(a_re, a_im, lda, a_stride, col_start, col_end, k0, w->cols_pad, tiles_n * kTcN,
                                      w->B3);
        HBEM_LAUNCH_CHECK("k_pack_b");
    }
    static int n_sm = 0;
    if (!n_sm) {
        int dev = 0;
        HBEM_CUDA(cudaGetDevice(&dev));
        HBEM_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
        HBEM_CUDA(cudaFuncSetAttribute(k_trailing_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    }
    const long long total = (long long)tiles_m * tiles_n * batch;
    if (total > 0x7fffffffLL) return fail(HBEM_ERR_ARG, "trailing update: too many tiles");
    const int ctas = n_sm - std::min(std::max(reserve_sms, 0), n_sm / 2);
    const int grid = (int)std::min<long long>(total, ctas);
    k_trailing_tc<<<grid, kTcThreads, kTcSmem, st>>>(w->ma, w->mb, a_re, a_im, lda, a_stride, n, start, col_start,
                                                    col_end, w->rows3, w->cols_pad, tiles_m, tiles_n, (int)total,
                                                    status);
    HBEM_LAUNCH_CHECK("k_trailing_tc");
    return HBEM_OK;
}

}  // namespace hbem
