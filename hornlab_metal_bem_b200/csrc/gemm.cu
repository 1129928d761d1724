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
int tc_workspace_k(const TcWorkspace *w);

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
    if (tc && kw == tc_workspace_k(tc) && status)
        return launch_trailing_tc(tc, n, batch, k0, start, start, col_end, a_re, a_im, lda, a_stride, status, st);
    return launch_trailing_simt(n, batch, k0, kw, start, start, col_end, a_re, a_im, lda, a_stride, st);
}

}  // namespace hbem

// ===========================================================================
// Tensor-core trailing update (tcgen05, split products, FP32 TMEM
// accumulation): BF16x3 for the mixed-precision LU, TF32x3 (FP32-class
// products: each split keeps 11 significant bits, so hi + lo carries 22 and
// the dropped lo x lo term is below 2^-22 of the product) for the plain LU.
//
// The complex update C -= L U is one real GEMM: for a tile of 64 complex rows
// the 128 MMA rows are [Lr, -Li] (real part) and [Li, Lr] (imaginary part)
// against B = [Ur; Ui] (K = 2 x 64).  Each FP32 operand x is split into
// hi = bf16(x) and lo = bf16(x - hi); A B ~ Ah Bh + Ah Bl + Al Bh.  The packed
// operands hold each split once, A2 = [Ah | Al] and B2^T = [Bh | Bl] (both
// K-major, 256 elements per row, written by k_pack_*); the three products are
// three MMA groups over the same shared-memory blocks.  A CTA takes work units
// of consecutive column tiles of one row block and keeps that row block's A2
// resident in shared memory while B2 streams through a ring (k_trailing_tc:
// TMA, single-thread MMA issue into two FP32 TMEM accumulators, C staged
// through shared memory by the epilogue warps).  Per variant (the same 224 KB
// of shared memory):
//   BF16x3: tiles of 64 complex rows x 64 columns, A2 64 KB (4 K-blocks of
//           128 bytes per row), ring of 6 x 16 KB, two 32 KB C tiles;
//   TF32x3 with K = 64 (and BF16x3 with K = 128): tiles of 64 complex rows x
//           32 columns, A2 128 KB (8 K-blocks), ring of 6 x 8 KB, three
//           16 KB C tiles (C prefetched two tiles ahead);
//   TF32x3 with K = 32 (two passes per 64-column LU block): the BF16x3
//           K = 64 shape (A2 64 KB, 64-column tiles, 6 x 16 KB ring, two
//           32 KB C tiles).
// Every mbarrier wait is bounded; a timeout sets the status word and the CTA
// returns after releasing its TMEM.
// ===========================================================================
namespace hbem {
namespace {

constexpr int kTcM = 128;          // MMA rows per tile (64 complex rows: real and imaginary parts)
constexpr int kTcABlk = kTcM * 128;  // one A K-block (128 bytes per row), 16 KB
constexpr int kTcThreads = 320;    // warp 0: MMA issuer, warp 1: TMA producer, warps 2-9: C tiles
constexpr long long kSpinLimit = 1LL << 24;

// Shapes of the variants (see above): operand format and KC, the complex K
// of one update (64: one LU block; 128: two blocks, BF16x3 only).
template <bool TF32, int KC>
struct TcCfg {
    static_assert(KC == 64 || (KC == 128 && !TF32) || (KC == 32 && TF32),
                  "tensor-core update: K = 64, 128 with BF16x3, or 32 with TF32x3");
    static constexpr int ES = TF32 ? 4 : 2;            // operand bytes
    static constexpr int EPB = 128 / ES;               // operand elements per 128-byte K-block
    static constexpr int K2 = 4 * KC;                  // packed elements per row: hi (real K = 2 KC), lo
    static constexpr int KBH = 2 * KC / EPB;           // K-blocks of one split
    static constexpr int N = KBH == 4 ? 32 : 64;       // columns per tile
    static constexpr int ABytes = 2 * KBH * kTcABlk;   // resident A2 of a row block
    static constexpr int BBlk = N * 128;               // one B K-block
    static constexpr int StageBytes = 2 * BBlk;        // ring stage: Bh and Bl of one K-block
    // B ring: one and a half 32-column tiles (K-block 4) / three 64-column tiles ahead
    static constexpr int Stages = 6;
    static constexpr int CBytes = kTcM * N * 4;        // one C tile staged in shared memory
    // C buffers: the 32-column tiles prefetch C two tiles ahead (one tile's
    // time is shorter than the HBM latency of its C), the 64-column ones one
    static constexpr int CBufs = N == 32 ? 3 : 2;
    static constexpr int Fmt = TF32 ? 2 : 1;           // instruction-descriptor operand format
    static constexpr size_t Smem =
        (size_t)ABytes + (size_t)Stages * StageBytes + (size_t)CBufs * CBytes + 1024;
    static_assert(Smem <= 227 * 1024, "tensor-core trailing update: shared memory");
};

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

// Instruction descriptor: FP32 accumulate, K-major A/B of operand format
// fmt (kind::f16 with 1 = BF16, kind::tf32 with 2 = TF32), M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n, int fmt) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Barrier of the eight C-tile warps (256 threads, named barrier 1) that also
// ORs a predicate across them, so every warp takes the same branch afterwards.
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

// Work unit u = (matrix, row block, chunk of at most `chunk` column tiles);
// this CTA's tiles in order: units blockIdx.x, + G, + 2G, ..., column tiles
// ascending inside a unit.
struct TcWalk {
    int u, tn, tn_end, mat, tm;
    bool valid;
    int tiles_m, tiles_n, n_chunks, chunk, n_units, G;
    __device__ void load() {
        valid = u < n_units;
        if (!valid) return;
        const int row = u / n_chunks, c = u - row * n_chunks;
        mat = row / tiles_m;
        tm = row - mat * tiles_m;
        tn = c * chunk;
        tn_end = min(tiles_n, tn + chunk);
    }
    __device__ TcWalk(int u0, int tiles_m_, int tiles_n_, int n_chunks_, int chunk_, int n_units_, int G_)
        : u(u0), tiles_m(tiles_m_), tiles_n(tiles_n_), n_chunks(n_chunks_), chunk(chunk_), n_units(n_units_),
          G(G_) {
        load();
    }
    __device__ bool last_of_unit() const { return tn + 1 == tn_end; }
    __device__ TcTile tile() const { return {mat, tm, tn}; }
    __device__ void advance() {
        if (++tn == tn_end) {
            u += G;
            load();
        }
    }
};

// Persistent trailing update over work units (see TcWalk).
//   warp 1 (TMA producer): per unit, the row block's 2 KBH A2 K-blocks into
//     the resident A buffer (after the MMAs of the previous unit released
//     it), then per tile the KBH K-blocks of B2 (Bh and Bl blocks per ring
//     stage), running ahead across tiles;
//   warp 0 (MMA issuer): per K-block, Ah Bh + Ah Bl + Al Bh as 3 x 4
//     tcgen05.mma (M = 128, N, 32 bytes of K each) into one of two TMEM
//     accumulators, releases ring slots with tcgen05.commit, signals
//     "accumulator full", and releases A after a unit's last tile;
//   warps 2-9 (C tiles): prefetch the next tile's C (real rows, then
//     imaginary rows) into one of two shared buffers with cp.async, drain the
//     finished accumulator into the current buffer (C - L U), hand the
//     accumulator back, and write the tile out with coalesced stores.
// Shared C layout: row r holds N / 4 groups of 4 columns, group g at position
// g ^ (r & 7) (aligned 16-byte copies, conflict-free float4 drain).  Every
// wait is bounded; a timeout sets *status and the roles stop, drain their
// copies, free TMEM and return.
template <bool TF32, int KC>
__global__ void __launch_bounds__(kTcThreads, 1) k_trailing_tc(const __grid_constant__ CUtensorMap tmA,
                                                                const __grid_constant__ CUtensorMap tmB, float *a_re,
                                                                float *a_im, long long lda, long long a_stride, int n,
                                                                int start, int col_start, int col_end, int rows3,
                                                                int cols_pad, int tiles_m, int tiles_n, int n_chunks,
                                                                int chunk, int n_units, int *status) {
    using Cfg = TcCfg<TF32, KC>;
    constexpr int kTcN = Cfg::N, kTcStages = Cfg::Stages, kTcStageBytes = Cfg::StageBytes, kTcABytes = Cfg::ABytes;
    constexpr int KBH = Cfg::KBH, EPB = Cfg::EPB;
    extern __shared__ uint8_t s_raw[];
    __shared__ uint64_t s_full[kTcStages], s_empty[kTcStages];
    __shared__ uint64_t s_acc_full[2], s_acc_empty[2];
    __shared__ uint64_t s_a_full, s_a_empty;
    __shared__ uint64_t s_done;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(s_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t *sA = base;
    uint8_t *ring = base + kTcABytes;
    float *sC0 = reinterpret_cast<float *>(ring + (size_t)kTcStages * kTcStageBytes);
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
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_a_full)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&s_a_empty)));
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

    if (warp == 1) {
        // ---- TMA producer
        if (lane == 0) {
            int last_use[kTcStages];
            for (int s = 0; s < kTcStages; ++s) last_use[s] = -1;
            bool ok = true;
            long long g = 0;   // ring position
            int units = 0;     // A loads issued
            TcWalk w(blockIdx.x, tiles_m, tiles_n, n_chunks, chunk, n_units, G);
            while (w.valid && ok) {
                // the previous unit's MMAs must be done with the resident A
                if (units > 0 && !mbar_wait(smem_u32(&s_a_empty), (units - 1) & 1, &s_fail)) {
                    ok = false;
                    break;
                }
                {
                    const uint32_t bar = smem_u32(&s_a_full);
                    const int row_a = w.mat * rows3 + w.tm * kTcM;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(kTcABytes)
                                 : "memory");
                    for (int kb = 0; kb < 2 * KBH; ++kb)
                        asm volatile(
                            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                            ::"r"(smem_u32(sA + (size_t)kb * kTcABlk)), "l"(reinterpret_cast<uint64_t>(&tmA)),
                              "r"(kb * EPB), "r"(row_a), "r"(bar)
                            : "memory");
                    ++units;
                }
                bool last;
                do {
                    const int row_b = w.mat * cols_pad + w.tn * kTcN;
                    for (int kh = 0; kh < KBH; ++kh, ++g) {
                        const int s = (int)(g % kTcStages);
                        const int u = (int)(g / kTcStages);
                        if (u > 0 && !mbar_wait(smem_u32(&s_empty[s]), (u - 1) & 1, &s_fail)) { ok = false; break; }
                        uint8_t *sb = ring + (size_t)s * kTcStageBytes;
                        const uint32_t bar = smem_u32(&s_full[s]);
                        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                                     "r"(kTcStageBytes)
                                     : "memory");
                        // Bh of this K-block, then Bl
                        asm volatile(
                            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                            ::"r"(smem_u32(sb)), "l"(reinterpret_cast<uint64_t>(&tmB)), "r"(kh * EPB),
                              "r"(row_b), "r"(bar)
                            : "memory");
                        asm volatile(
                            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                            ::"r"(smem_u32(sb + Cfg::BBlk)), "l"(reinterpret_cast<uint64_t>(&tmB)),
                              "r"((KBH + kh) * EPB), "r"(row_b), "r"(bar)
                            : "memory");
                        last_use[s] = u;
                    }
                    last = w.last_of_unit();
                    w.advance();
                } while (!last && ok);
            }
            if (!ok) {
                s_fail = 1;
                atomicExch(status, 3);
            }
            // every issued copy must land before the CTA may exit
            for (int s = 0; s < kTcStages; ++s)
                if (last_use[s] >= 0) mbar_wait(smem_u32(&s_full[s]), last_use[s] & 1);
            if (units > 0) mbar_wait(smem_u32(&s_a_full), (units - 1) & 1);
        }
    } else if (warp == 0) {
        // ---- MMA issuer
        if (lane == 0) {
            constexpr uint32_t idesc = umma_idesc(kTcM, kTcN, Cfg::Fmt);
            bool ok = true;
            long long g = 0;
            int i = 0;        // tiles
            int units = 0;
            TcWalk w(blockIdx.x, tiles_m, tiles_n, n_chunks, chunk, n_units, G);
            while (w.valid && ok) {
                if (!mbar_wait(smem_u32(&s_a_full), units & 1, &s_fail)) { ok = false; break; }
                const uint32_t a0 = smem_u32(sA);
                bool last;
                do {
                    const int b = i & 1;
                    // the epilogue must have drained this accumulator (tile i - 2)
                    if (i >= 2 && !mbar_wait(smem_u32(&s_acc_empty[b]), ((i >> 1) - 1) & 1, &s_fail)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t acc_addr = tmem + (uint32_t)(b * kTcN);
                    for (int kh = 0; kh < KBH; ++kh, ++g) {
                        const int s = (int)(g % kTcStages);
                        const int u = (int)(g / kTcStages);
                        if (!mbar_wait(smem_u32(&s_full[s]), u & 1, &s_fail)) { ok = false; break; }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint32_t sb = smem_u32(ring + (size_t)s * kTcStageBytes);
                        // (A block, B block): Ah Bh, Ah Bl, Al Bh of this K-block
                        const uint32_t pa[3] = {a0 + (uint32_t)(kh * kTcABlk), a0 + (uint32_t)(kh * kTcABlk),
                                                a0 + (uint32_t)((KBH + kh) * kTcABlk)};
                        const uint32_t pb[3] = {sb, sb + (uint32_t)Cfg::BBlk, sb};
#pragma unroll
                        for (int pr = 0; pr < 3; ++pr) {
#pragma unroll
                            for (int kk = 0; kk < 4; ++kk) {   // 32 bytes of K per instruction
                                const uint64_t da = umma_desc_sw128(pa[pr] + kk * 32);
                                const uint64_t db = umma_desc_sw128(pb[pr] + kk * 32);
                                const uint32_t acc = (kh > 0 || pr > 0 || kk > 0) ? 1u : 0u;
                                if (TF32)
                                    asm volatile(
                                        "{\n\t.reg .pred p;\n\t"
                                        "setp.ne.b32 p, %4, 0;\n\t"
                                        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                                        ::"r"(acc_addr), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                                        : "memory");
                                else
                                    asm volatile(
                                        "{\n\t.reg .pred p;\n\t"
                                        "setp.ne.b32 p, %4, 0;\n\t"
                                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                                        ::"r"(acc_addr), "l"(da), "l"(db), "r"(idesc), "r"(acc)
                                        : "memory");
                            }
                        }
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                         smem_u32(&s_empty[s]))
                                     : "memory");
                    }
                    if (!ok) break;
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_u32(&s_acc_full[b]))
                                 : "memory");
                    ++i;
                    last = w.last_of_unit();
                    w.advance();
                } while (!last);
                if (!ok) break;
                // A may be replaced once this unit's MMAs have completed
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&s_a_empty))
                             : "memory");
                ++units;
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
        // ---- C tiles: 8 warps; thread et owns column group gq = et % GQ (4
        // columns) of rows et / GQ + RS it; warp pair (w, w + 4) shares TMEM
        // lane quarter w & 3 and drains the columns [N/2 h, N/2 h + N/2),
        // h = (w - 2) >> 2.
        constexpr int GQ = kTcN / 4, RS = 256 / GQ, HALF = kTcN / 2;
        const int et = tid - 64;   // 0..255
        const int q = warp & 3;
        const int h = (warp - 2) >> 2;
        const int gq = et % GQ, r_first = et / GQ;
        auto sidx = [](int r, int c) { return r * kTcN + ((((c >> 2) ^ (r & 7)) << 2) | (c & 3)); };
        auto prefetch = [&](const TcTile tt, float *sC) {
            const int row_c0 = start + tt.tm * 64, gcol = col_start + tt.tn * kTcN + 4 * gq;
            if (gcol >= col_end) {
                asm volatile("cp.async.commit_group;" ::: "memory");
                return;
            }
            const bool full4 = gcol + 3 < col_end;
            const float *mre = a_re + (size_t)tt.mat * a_stride + gcol, *mim = a_im + (size_t)tt.mat * a_stride + gcol;
#pragma unroll
            for (int it = 0; it < kTcM / RS; ++it) {
                const int r = r_first + RS * it;
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
        constexpr int CB = Cfg::CBufs;
        TcWalk cur(blockIdx.x, tiles_m, tiles_n, n_chunks, chunk, n_units, G);
        TcWalk nxt = cur;
        for (int k = 0; k + 1 < CB && nxt.valid; ++k) {
            prefetch(nxt.tile(), sC0 + (size_t)k * (kTcM * kTcN));
            nxt.advance();
        }
        for (int i = 0; cur.valid; ++i) {
            const int b = i & 1;
            float *sC = sC0 + (size_t)(i % CB) * (kTcM * kTcN);
            if (nxt.valid) {
                // tile i + CB - 1 into the buffer tile i - 1 has written back
                prefetch(nxt.tile(), sC0 + (size_t)((i + CB - 1) % CB) * (kTcM * kTcN));
                nxt.advance();
                if constexpr (CB == 3) asm volatile("cp.async.wait_group 2;" ::: "memory");
                else asm volatile("cp.async.wait_group 1;" ::: "memory");
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
                const int c0 = HALF * h;
                uint32_t v[HALF];
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * kTcN + c0);
                if constexpr (HALF == 32)
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                        "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                        "%30, %31}, [%32];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                          "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                          "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                        : "r"(taddr));
                else
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                        "%12, %13, %14, %15}, [%16];"
                        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                          "=r"(v[14]), "=r"(v[15])
                        : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int jj = 0; jj < HALF / 4; ++jj) {
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
                const TcTile tt = cur.tile();
                const int row_c0 = start + tt.tm * 64, gcol = col_start + tt.tn * kTcN + 4 * gq;
                if (gcol < col_end) {
                    const bool full4 = gcol + 3 < col_end;
                    float *mre = a_re + (size_t)tt.mat * a_stride + gcol, *mim = a_im + (size_t)tt.mat * a_stride + gcol;
#pragma unroll
                    for (int it = 0; it < kTcM / RS; ++it) {
                        const int r = r_first + RS * it;
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
            epi_bar();   // this buffer may be refilled by the next iteration's prefetch
            cur.advance();
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kTcN));
}

// Operand splits: hi = x rounded to the operand format, lo = (x - hi) rounded
// (x - hi is exact in FP32).  TF32 rounding keeps 10 fraction bits, to
// nearest with ties away from zero: half the weight of the 13 dropped bits is
// added to the FP32 pattern before they are cleared (finite x).
__device__ __forceinline__ float tf32_round(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

template <bool TF32>
struct TcSplit;
template <>
struct TcSplit<false> {
    using T = __nv_bfloat16;
    __device__ static T hi(float x) { return __float2bfloat16_rn(x); }
    __device__ static float val(T h) { return __bfloat162float(h); }
    __device__ static void store2(T *p, T a, T b) {
        __nv_bfloat162 v;
        v.x = a;
        v.y = b;
        *reinterpret_cast<__nv_bfloat162 *>(p) = v;
    }
};
template <>
struct TcSplit<true> {
    using T = float;
    __device__ static T hi(float x) { return tf32_round(x); }
    __device__ static float val(T h) { return h; }
    __device__ static void store2(T *p, T a, T b) { *reinterpret_cast<float2 *>(p) = make_float2(a, b); }
};

// Pack L21 (rows start..n, cols k0..k0+KC) into A2 (K-major, hi/lo splits):
// real-part row [Lr | -Li], imaginary-part row [Li | Lr], hi then lo.
template <bool TF32, int KC>
__global__ void k_pack_a(const float *a_re, const float *a_im, long long lda, long long a_stride, int n, int start,
                         int k0, int rows3, int rows_used, typename TcSplit<TF32>::T *A2) {
    using S = TcSplit<TF32>;
    using T = typename S::T;
    constexpr int K2 = TcCfg<TF32, KC>::K2;
    const int mat = blockIdx.z;
    const int i = blockIdx.x * blockDim.y + threadIdx.y;  // complex row offset
    const int k = threadIdx.x;                            // 0..KC-1
    const int m = n - start;
    if (i >= rows_used) return;                           // complex rows incl. tile padding
    float lr = 0.f, li = 0.f;
    if (i < m) {
        lr = a_re[(size_t)mat * a_stride + (size_t)(start + i) * lda + k0 + k];
        li = a_im[(size_t)mat * a_stride + (size_t)(start + i) * lda + k0 + k];
    }
    const int t = i >> 6, rl = i & 63;
    T *re_row = A2 + ((size_t)mat * rows3 + (size_t)t * 128 + rl) * K2;
    T *im_row = re_row + (size_t)64 * K2;
    auto put = [](T *row, int k2, float x) {
        const T h = S::hi(x);
        row[k2] = h;
        row[2 * KC + k2] = S::hi(x - S::val(h));
    };
    put(re_row, k, lr);
    put(re_row, KC + k, -li);
    put(im_row, k, li);
    put(im_row, KC + k, lr);
}

// Pack U12 (rows k0..k0+KC, cols start..col_end) into B2^T (K-major, hi/lo
// splits): per column [hi Ur | hi Ui | lo Ur | lo Ui], KC entries each.
template <bool TF32, int KC>
__global__ void __launch_bounds__(256) k_pack_b(const float *a_re, const float *a_im, long long lda,
                                                long long a_stride, int start, int col_end, int k0, int cols_pad,
                                                int cols_used, typename TcSplit<TF32>::T *B2) {
    // 64 columns per CTA, CH = min(KC, 64) rows of U12 at a time: the CH x 64
    // block is read along its rows (coalesced), transposed in shared memory
    // and written into the packed K-major rows (consecutive threads,
    // consecutive pairs)
    using S = TcSplit<TF32>;
    using T = typename S::T;
    constexpr int K2 = TcCfg<TF32, KC>::K2;
    constexpr int CH = KC < 64 ? KC : 64, PAIRS = 2 * CH, JSTEP = 256 / PAIRS;
    __shared__ float s_ur[CH][65], s_ui[CH][65];
    const int mat = blockIdx.z;
    const int j0 = blockIdx.x * 64;
    const int tid = threadIdx.x;
    // pair p of a chunk covers its entries 2p, 2p + 1 of [hi Ur, hi Ui, lo Ur, lo Ui] (CH each)
    const int p = tid % PAIRS;
    const int kk = 2 * p;
    const int part = kk / CH, k = kk % CH;   // part: 0 hi Ur, 1 hi Ui, 2 lo Ur, 3 lo Ui
    for (int kc = 0; kc < KC; kc += CH) {
        const float *ure = a_re + (size_t)mat * a_stride + (size_t)(k0 + kc) * lda + start;
        const float *uim = a_im + (size_t)mat * a_stride + (size_t)(k0 + kc) * lda + start;
        if (kc) __syncthreads();   // the previous chunk's reads of s_ur / s_ui are done
        for (int e = tid; e < CH * 64; e += 256) {
            const int kr = e >> 6, jj = e & 63, j = j0 + jj;
            const bool in = start + j < col_end;
            s_ur[kr][jj] = in ? ure[(size_t)kr * lda + j] : 0.f;
            s_ui[kr][jj] = in ? uim[(size_t)kr * lda + j] : 0.f;
        }
        __syncthreads();
        for (int jj = tid / PAIRS; jj < 64; jj += JSTEP) {
            const int j = j0 + jj;
            if (j >= cols_used) break;
            const float x0 = (part & 1) ? s_ui[k][jj] : s_ur[k][jj];
            const float x1 = (part & 1) ? s_ui[k + 1][jj] : s_ur[k + 1][jj];
            T v0 = S::hi(x0), v1 = S::hi(x1);
            if (part >= 2) {
                v0 = S::hi(x0 - S::val(v0));
                v1 = S::hi(x1 - S::val(v1));
            }
            S::store2(B2 + ((size_t)mat * cols_pad + j) * K2 + part * KC + kc + k, v0, v1);
        }
    }
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

// Packed rows of k2 elements of es bytes; boxes of one 128-byte K-block x box_rows.
int make_map(CUtensorMap *map, void *ptr, long long rows, int box_rows, int es, int k2) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return fail(HBEM_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    const cuuint64_t dims[2] = {(cuuint64_t)k2, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)k2 * es};
    const cuuint32_t box[2] = {(cuuint32_t)(128 / es), (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ptr, dims,
                    strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(HBEM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return HBEM_OK;
}

}  // namespace

// Packed-operand workspace and tensor maps for one factorisation: sized for
// the first (largest) trailing update and reused by the later, smaller ones.
// tf32: TF32x3 operands (plain LU) instead of BF16x3 (mixed LU); kc: the
// complex K of one update (64; 128 for BF16x3; 32 for TF32x3, two passes per
// 64-column block).
struct TcWorkspace {
    void *A2 = nullptr, *B2 = nullptr;
    int rows3 = 0, cols_pad = 0, batch = 0, kc = 64;
    bool tf32 = false;
    CUtensorMap ma, mb;
};

int tc_workspace_create(int n, int batch, bool tf32, int kc, TcWorkspace **out, cudaStream_t st) {
    *out = nullptr;
    if (!(kc == 64 || (kc == 128 && !tf32) || (kc == 32 && tf32)))
        return fail(HBEM_ERR_ARG, "tensor-core update: K = 64, 128 with BF16x3, or 32 with TF32x3");
    auto *w = new TcWorkspace();
    const int es = tf32 ? 4 : 2, k2 = 4 * kc;
    const int tn = 2 * kc * es / 128 == 4 ? 32 : 64;   // the configuration's tile width (TcCfg::N)
    w->tf32 = tf32;
    w->kc = kc;
    w->rows3 = ((n + 63) / 64) * kTcM;
    w->cols_pad = ((n + tn - 1) / tn) * tn;
    w->batch = batch;
    cudaError_t e = cudaMallocAsync(&w->A2, (size_t)batch * w->rows3 * k2 * es, st);
    if (e == cudaSuccess) e = cudaMallocAsync(&w->B2, (size_t)batch * w->cols_pad * k2 * es, st);
    if (e != cudaSuccess) {
        if (w->A2) cudaFreeAsync(w->A2, st);
        delete w;
        return cuda_fail(e, "tensor-core workspace");
    }
    int rc = make_map(&w->ma, w->A2, (long long)batch * w->rows3, kTcM, es, k2);
    if (rc == HBEM_OK) rc = make_map(&w->mb, w->B2, (long long)batch * w->cols_pad, tn, es, k2);
    if (rc != HBEM_OK) {
        cudaFreeAsync(w->A2, st);
        cudaFreeAsync(w->B2, st);
        delete w;
        return rc;
    }
    *out = w;
    return HBEM_OK;
}

void tc_workspace_destroy(TcWorkspace *w, cudaStream_t st) {
    if (!w) return;
    cudaFreeAsync(w->A2, st);
    cudaFreeAsync(w->B2, st);
    delete w;
}

// The K one launch_trailing_tc call consumes: the workspace's K, or 64 for
// the TF32x3 K = 32 workspace, which runs two passes per call.
int tc_workspace_k(const TcWorkspace *w) { return w ? (w->tf32 && w->kc == 32 ? 64 : w->kc) : 0; }

namespace {

template <bool TF32, int KC>
int launch_trailing_tc_t(TcWorkspace *w, int n, int batch, int k0, int start, int col_start, int col_end,
                         float *a_re, float *a_im, long long lda, long long a_stride, int *status, cudaStream_t st,
                         int reserve_sms) {
    using Cfg = TcCfg<TF32, KC>;
    using T = typename TcSplit<TF32>::T;
    const int m = n - start, wd = col_end - col_start;
    const int tiles_m = (m + 63) / 64, tiles_n = (wd + Cfg::N - 1) / Cfg::N;
    // packed rows use the workspace's fixed per-matrix pitch (rows3 / cols_pad)
    {
        dim3 blk(KC, 256 / KC), grd((tiles_m * 64 + blk.y - 1) / blk.y, 1, batch);
        k_pack_a<TF32, KC><<<grd, blk, 0, st>>>(a_re, a_im, lda, a_stride, n, start, k0, w->rows3, tiles_m * 64,
                                                static_cast<T *>(w->A2));
        HBEM_LAUNCH_CHECK("k_pack_a");
    }
    {
        dim3 grd((tiles_n * Cfg::N + 63) / 64, 1, batch);
        k_pack_b<TF32, KC><<<grd, 256, 0, st>>>(a_re, a_im, lda, a_stride, col_start, col_end, k0, w->cols_pad,
                                                tiles_n * Cfg::N, static_cast<T *>(w->B2));
        HBEM_LAUNCH_CHECK("k_pack_b");
    }
    int n_sm = 0;
    {
        int dev = 0;
        HBEM_CUDA(cudaGetDevice(&dev));
        HBEM_CUDA(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
        const int rc = func_opt_in((const void *)k_trailing_tc<TF32, KC>, (int)Cfg::Smem);
        if (rc != HBEM_OK) return rc;
    }
    const int ctas = n_sm - std::min(std::max(reserve_sms, 0), n_sm / 2);
    // work units of `chunk` consecutive column tiles: about ten units per CTA
    // where the tiles allow (load balance), else one tile per unit
    const long long total = (long long)tiles_m * tiles_n * batch;
    long long want = total / (10LL * ctas);
    int chunk = (int)std::max(1LL, std::min<long long>(want, tiles_n));
    const int n_chunks = (tiles_n + chunk - 1) / chunk;
    chunk = (tiles_n + n_chunks - 1) / n_chunks;
    const long long units = (long long)batch * tiles_m * n_chunks;
    if (units > 0x7fffffffLL) return fail(HBEM_ERR_ARG, "trailing update: too many tiles");
    if ((long long)(n_chunks - 1) * chunk >= tiles_n) return fail(HBEM_ERR_STATE, "trailing update: empty work unit");
    const int grid = (int)std::min<long long>(units, ctas);
    k_trailing_tc<TF32, KC><<<grid, kTcThreads, Cfg::Smem, st>>>(w->ma, w->mb, a_re, a_im, lda, a_stride, n, start,
                                                                  col_start, col_end, w->rows3, w->cols_pad, tiles_m,
                                                                  tiles_n, n_chunks, chunk, (int)units, status);
    HBEM_LAUNCH_CHECK("k_trailing_tc");
    return HBEM_OK;
}

}  // namespace

// Tensor-core trailing update with the workspace's K (64: one LU block, 128:
// two), BF16x3 or TF32x3 by the workspace; status receives 1/2/3 if a
// barrier wait timed out.  The persistent grid leaves reserve_sms SMs (at
// most half of them) to kernels on other streams.
// A[start:n, col_start:col_end] -= L[start:n, k0:k0+K] U[k0:k0+K, col_start:col_end]
int launch_trailing_tc(TcWorkspace *w, int n, int batch, int k0, int start, int col_start, int col_end, float *a_re,
                       float *a_im, long long lda, long long a_stride, int *status, cudaStream_t st,
                       int reserve_sms) {
    if (n - start <= 0 || col_end - col_start <= 0) return HBEM_OK;
    if (w->tf32 && w->kc == 32) {
        // the 64 columns of an LU block as two K = 32 passes (C read and
        // written twice, each pass in the 64 KB-A, 64-column-tile shape)
        int rc = launch_trailing_tc_t<true, 32>(w, n, batch, k0, start, col_start, col_end, a_re, a_im, lda,
                                                a_stride, status, st, reserve_sms);
        if (rc != HBEM_OK) return rc;
        return launch_trailing_tc_t<true, 32>(w, n, batch, k0 + 32, start, col_start, col_end, a_re, a_im, lda,
                                              a_stride, status, st, reserve_sms);
    }
    if (w->tf32)
        return launch_trailing_tc_t<true, 64>(w, n, batch, k0, start, col_start, col_end, a_re, a_im, lda, a_stride,
                                              status, st, reserve_sms);
    if (w->kc == 128)
        return launch_trailing_tc_t<false, 128>(w, n, batch, k0, start, col_start, col_end, a_re, a_im, lda,
                                                a_stride, status, st, reserve_sms);
    return launch_trailing_tc_t<false, 64>(w, n, batch, k0, start, col_start, col_end, a_re, a_im, lda, a_stride,
                                           status, st, reserve_sms);
}

}  // namespace hbem
