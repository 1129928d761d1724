// Batched complex LU with partial pivoting and triangular solves on sm_100a,
// replacing LAPACK cgesv/cgetrf/cgetrs (reference main.swift:7834-7941,
// 8015-8020).  Matrices are planar (re, im) float32, row-major.
//
// Two-level right-looking blocked factorisation, batched over matrices:
//   for each 64-column block b0:
//     for each inner sub-panel c (64, 32 or 16 columns):
//       k_panel      : factor rows c..n of the sub-panel with partial pivoting
//                      (pivot = first max |re|+|im|, as LAPACK's icamax),
//                      staged in one CTA's shared memory when it fits, else
//                      spread over a 2/4/8/16-CTA cluster's shared memory
//                      (k_panel_cluster), else in L2;
//       k_swap_trsm  : swap + forward-solve the other columns of the block;
//       trailing     : update the block's remaining columns (K = 16/32);
//     k_swap_trsm    : the block's 64 swaps on all other columns and the
//                      64-row TRSM U12 = L11^-1 A12;
//     trailing       : A22 -= L21 U12 with K = 64.
// The solve applies the pivots then runs blocked forward / backward
// substitution: op(A) = A with n > 128 in 128-row block steps over many CTAs
// (k_trsv_*), A^T / A^H and small n in one CTA per right-hand side (k_getrs).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <cmath>
#include <string>
#include <vector>

#include "hbem_internal.h"

namespace hbem {

// A[start:n, start:col_end] -= A[start:n, k0:k0+kw] * A[k0:k0+kw, start:col_end]
struct TcWorkspace;
int tc_workspace_create(int n, int batch, bool tf32, int kc, TcWorkspace **out, cudaStream_t st);
void tc_workspace_destroy(TcWorkspace *w, cudaStream_t st);
int launch_trailing_update(int n, int batch, int k0, int kw, int start, int col_end, float *a_re, float *a_im,
                           long long lda, long long a_stride, TcWorkspace *tc, int *status, cudaStream_t st);
int launch_trailing_simt(int n, int batch, int k0, int kw, int start, int col_start, int col_end, float *a_re,
                         float *a_im, long long lda, long long a_stride, cudaStream_t st);
int launch_trailing_tc(TcWorkspace *w, int n, int batch, int k0, int start, int col_start, int col_end, float *a_re,
                       float *a_im, long long lda, long long a_stride, int *status, cudaStream_t st,
                       int reserve_sms = 0);

namespace {

constexpr int kPanelThreads = 512;

__device__ __forceinline__ float cabs1(float r, float i) { return fabsf(r) + fabsf(i); }

// The panel kernels' complex arithmetic with every rounding fixed (products
// that are not fused are __fmul_rn, the rest explicit fmaf), so the compiler
// cannot contract a*b - c*d either way and every panel kernel computes the
// same bits for the same element:
//   l = x / d as x * (1 / d):  inv = conj(d) / (d.re^2 + d.im^2);
//   x -= l * u.
__device__ __forceinline__ void pivot_inverse(float dr, float di, float &ir, float &ii) {
    const float den = 1.0f / fmaf(dr, dr, __fmul_rn(di, di));
    ir = __fmul_rn(dr, den);
    ii = __fmul_rn(-di, den);
}
__device__ __forceinline__ void cmul_fixed(float xr, float xi, float yr, float yi, float &zr, float &zi) {
    zr = fmaf(xr, yr, -__fmul_rn(xi, yi));
    zi = fmaf(xr, yi, __fmul_rn(xi, yr));
}
__device__ __forceinline__ void csub_mul_fixed(float &xr, float &xi, float lr, float li, float ur, float ui) {
    xr = __fsub_rn(xr, fmaf(lr, ur, -__fmul_rn(li, ui)));
    xi = __fsub_rn(xi, fmaf(lr, ui, __fmul_rn(li, ur)));
}

// Panel factorisation of rows k0..n-1 x nb columns (nb <= 32), worked in
// place through L2: the fallback for panels taller than a cluster's shared
// memory holds.  Per column j, three barrier-separated phases:
//   R (threads over rows)    : scale column j-1 by 1/pivot, local argmax of
//                              |re| + |im| in column j (first index on ties);
//   P (nb threads)           : pick the pivot, swap rows j <-> p, publish the
//                              pivot row;
//   E (threads over elements): A[r][c] -= (A[r][j] / pivot) * A[j][c], r, c > j.
__global__ void __launch_bounds__(kPanelThreads) k_panel(float *a_re, float *a_im, long long lda, long long a_stride,
                                                         int n, int k0, int nb, int *piv, long long piv_stride,
                                                         int *info) {
    __shared__ float s_v[kPanelThreads / 32];
    __shared__ int s_i[kPanelThreads / 32];
    __shared__ float s_pr[32], s_pi[32];
    const int b = blockIdx.x;
    int *pv = piv + (size_t)b * piv_stride;
    const int m = n - k0;  // panel rows
    // element (r, c) of the panel at global pitch lda
    const int P = (int)lda;
    float *pre = a_re + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    float *pim = a_im + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    // element-phase mapping: LPR lanes per row, RPW rows per warp instruction
    const int LPR = nb > 16 ? 32 : 16;
    const int c_off = lane & (LPR - 1);
    const int r_sub = lane / LPR;
    const int r_step = nw * (32 / LPR);
    int first_zero = 0;
    float ir = 0.f, ii = 0.f;  // 1 / pivot of the previous column
    for (int j = 0; j <= nb; ++j) {
        // ---- phase R
        float v = -1.f;
        int idx = 0x7fffffff;
        for (int r = j + tid; r < m; r += blockDim.x) {
            const int o = r * P;
            if (j > 0) {
                const float xr = pre[o + j - 1], xi = pim[o + j - 1];
                cmul_fixed(xr, xi, ir, ii, pre[o + j - 1], pim[o + j - 1]);
            }
            if (j < nb) {
                const float c = cabs1(pre[o + j], pim[o + j]);
                if (c > v) { v = c; idx = r; }
            }
        }
        if (j == nb) break;
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
        }
        if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
        __syncthreads();
        // ---- phase P
        if (tid < nb) {
            float bv = s_v[0];
            int p = s_i[0];
            for (int w = 1; w < nw; ++w) {
                const float ov = s_v[w];
                const int oi = s_i[w];
                if (ov > bv || (ov == bv && oi < p)) { bv = ov; p = oi; }
            }
            if (p >= m) p = j;  // column of NaNs: keep the diagonal, as icamax does
            const int c = tid;
            const float jr = pre[j * P + c], ji = pim[j * P + c];
            const float pr = pre[p * P + c], pi = pim[p * P + c];
            s_pr[c] = pr;
            s_pi[c] = pi;
            pre[j * P + c] = pr;
            pim[j * P + c] = pi;
            if (p != j) {
                pre[p * P + c] = jr;
                pim[p * P + c] = ji;
            }
            if (c == 0) pv[k0 + j] = k0 + p;
        }
        __syncthreads();
        const float dr = s_pr[j], di = s_pi[j];
        const bool zero = (dr == 0.f && di == 0.f);
        if (zero) {
            if (first_zero == 0) first_zero = k0 + j + 1;
            ir = 0.f;
            ii = 0.f;
        } else {
            pivot_inverse(dr, di, ir, ii);
        }
        // ---- phase E
        const int c = j + 1 + c_off;
        if (c < nb && !zero) {
            const float ur = s_pr[c], ui = s_pi[c];
            for (int r = j + 1 + warp * (32 / LPR) + r_sub; r < m; r += r_step) {
                const int o = r * P;
                const float xr = pre[o + j], xi = pim[o + j];
                float lr, li;
                cmul_fixed(xr, xi, ir, ii, lr, li);
                csub_mul_fixed(pre[o + c], pim[o + c], lr, li, ur, ui);
            }
        }
        __syncthreads();
    }
    if (tid == 0 && first_zero && info[b] == 0) info[b] = first_zero;
}

// Panel factorisation in one CTA's shared memory (pitch nb + 1, nb <= 64:
// a whole 64-column block when it fits), thread per row.  Per column j, two
// barrier-separated phases:
//   P (warp 0): reduce the per-warp argmax candidates of column j (first
//               index on ties, as icamax), swap rows j <-> p, publish the
//               pivot row;
//   E (threads over rows > j): scale the row's column-j entry by 1/pivot,
//               apply the rank-1 update to its columns > j and take the
//               argmax candidate of column j + 1 from the updated row.
// The arithmetic of every element is that of k_panel; the fused scaling,
// update and pivot search save one barrier and a pass per column, and a
// thread's columns are independent (rows at pitch nb + 1 keep consecutive
// threads on distinct banks).
__device__ __forceinline__ void argmax_warp(float &v, int &idx) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
}

constexpr int kPanelRowsThreads = 1024;   // one row per thread up to 1024 rows
__global__ void __launch_bounds__(kPanelRowsThreads) k_panel_rows(float *a_re, float *a_im, long long lda,
                                                              long long a_stride, int n, int k0, int nb, int *piv,
                                                              long long piv_stride, int *info) {
    extern __shared__ float s_panel[];
    __shared__ float s_v[kPanelRowsThreads / 32];
    __shared__ int s_i[kPanelRowsThreads / 32];
    __shared__ float s_pr[64], s_pi[64];   // nb <= 64
    const int b = blockIdx.x;
    int *pv = piv + (size_t)b * piv_stride;
    const int m = n - k0;
    const int P = nb + 1;
    float *pre = s_panel, *pim = s_panel + m * P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    float *gre = a_re + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    float *gim = a_im + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    for (int e = tid; e < m * nb; e += blockDim.x) {
        const int r = e / nb, j = e - r * nb;
        pre[r * P + j] = gre[(size_t)r * lda + j];
        pim[r * P + j] = gim[(size_t)r * lda + j];
    }
    __syncthreads();
    float v = -1.f;
    int idx = 0x7fffffff;
    for (int r = tid; r < m; r += blockDim.x) {
        const float c = cabs1(pre[r * P], pim[r * P]);
        if (c > v) { v = c; idx = r; }
    }
    argmax_warp(v, idx);
    if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
    __syncthreads();
    int first_zero = 0;
    for (int j = 0; j < nb; ++j) {
        // ---- phase P
        if (warp == 0) {
            float bv = lane < nw ? s_v[lane] : -1.f;
            int p = lane < nw ? s_i[lane] : 0x7fffffff;
            argmax_warp(bv, p);
            if (p >= m) p = j;  // column of NaNs: keep the diagonal, as icamax does
            for (int c = lane; c < nb; c += 32) {
                const float jr = pre[j * P + c], ji = pim[j * P + c];
                const float pr = pre[p * P + c], pi = pim[p * P + c];
                s_pr[c] = pr;
                s_pi[c] = pi;
                pre[j * P + c] = pr;
                pim[j * P + c] = pi;
                if (p != j) {
                    pre[p * P + c] = jr;
                    pim[p * P + c] = ji;
                }
            }
            if (lane == 0) pv[k0 + j] = k0 + p;
        }
        __syncthreads();
        const float dr = s_pr[j], di = s_pi[j];
        const bool zero = (dr == 0.f && di == 0.f);
        float ir = 0.f, ii = 0.f;
        if (zero) {
            if (first_zero == 0) first_zero = k0 + j + 1;
        } else {
            pivot_inverse(dr, di, ir, ii);
        }
        // ---- phase E
        v = -1.f;
        idx = 0x7fffffff;
        const bool next = j + 1 < nb;
        for (int r = j + 1 + tid; r < m; r += blockDim.x) {
            const int o = r * P;
            const float xr = pre[o + j], xi = pim[o + j];
            float lr, li;
            cmul_fixed(xr, xi, ir, ii, lr, li);
            pre[o + j] = lr;
            pim[o + j] = li;
            if (!zero) {
#pragma unroll 4
                for (int c = j + 1; c < nb; ++c) csub_mul_fixed(pre[o + c], pim[o + c], lr, li, s_pr[c], s_pi[c]);
            }
            if (next) {
                const float a = cabs1(pre[o + j + 1], pim[o + j + 1]);
                if (a > v) { v = a; idx = r; }
            }
        }
        if (next) {
            argmax_warp(v, idx);
            if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
        }
        __syncthreads();
    }
    for (int e = tid; e < m * nb; e += blockDim.x) {
        const int r = e / nb, j = e - r * nb;
        gre[(size_t)r * lda + j] = pre[r * P + j];
        gim[(size_t)r * lda + j] = pim[r * P + j];
    }
    if (tid == 0 && first_zero && info[b] == 0) info[b] = first_zero;
}

// A sub-panel of W = 16, 32 or 64 columns with its rows in registers: thread
// t holds rows t, t + T, ... (R of them, W complex values each, as (re, im)
// pairs) from the load to the write-back, so a column moves no row through
// shared memory.  The column loop is rolled two columns at a time (the code
// stays in the instruction cache); every row is rotated left by two places
// per step, so column j sits in register j mod 2 and the trailing columns
// follow it (after W columns the rows are back in order).  Per column j:
//   every warp reduces the per-warp argmax candidates itself (first index on
//   ties, as icamax); the owners of rows j and p publish those two rows (the
//   pivot row as (re, im, im, re) quadruples); one barrier; the two rows
//   change hands, every thread scales and updates its rows below j and takes
//   its candidate for column j + 1; a second barrier publishes the
//   candidates.
// The update x -= l u is three packed FP32 instructions (FMUL2, FFMA2,
// FADD2) whose halves round exactly as the scalar pivot_inverse /
// cmul_fixed / csub_mul_fixed of the shared-memory kernels (negations are
// exact), so the factors are the same bits.  Rows j < W < T live in slot 0
// of thread j.  For m <= R * T rows; dynamic shared memory m * (2W + 1)
// floats stages the coalesced load and store.
template <int W, int R, int T>
struct PanelRegs {
    static constexpr int NW = T / 32;
    float2 x[R][W];
    // column j in register B; `live` trailing columns in registers B+1 .. B+live
    template <int B>
    __device__ __forceinline__ void column(int j, int m, int k0, int tid, int lane, int warp, float *s_v, int *s_i,
                                           float4 *s_p, float2 *s_o, int *pv, int &first_zero) {
        float bv = lane < NW ? s_v[lane] : -1.f;
        int p = lane < NW ? s_i[lane] : 0x7fffffff;
        argmax_warp(bv, p);
        if (p >= m) p = j;  // column of NaNs: keep the diagonal, as icamax does
        const int po = p % T, ps = p / T;
        if (tid == j) {
#pragma unroll
            for (int c = 0; c < W; ++c) s_o[c] = x[0][c];
        }
        if (tid == po) {
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (s == ps) {
#pragma unroll
                    for (int c = 0; c < W; ++c) s_p[c] = make_float4(x[s][c].x, x[s][c].y, x[s][c].y, x[s][c].x);
                }
            pv[k0 + j] = k0 + p;
        }
        __syncthreads();
        if (tid == j) {
#pragma unroll
            for (int c = 0; c < W; ++c) {
                const float4 u = s_p[c];
                x[0][c] = make_float2(u.x, u.y);
            }
        }
        if (p != j && tid == po) {
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (s == ps) {
#pragma unroll
                    for (int c = 0; c < W; ++c) x[s][c] = s_o[c];
                }
        }
        const float4 d = s_p[B];
        const bool zero = (d.x == 0.f && d.y == 0.f);
        float ir = 0.f, ii = 0.f;
        if (zero) {
            if (first_zero == 0) first_zero = k0 + j + 1;
        } else {
            pivot_inverse(d.x, d.y, ir, ii);
        }
        const int live = W - 1 - j;
        bool act[R];
        float2 nl[R], pl[R];   // (-l.re, -l.re) and (l.im, -l.im)
#pragma unroll
        for (int s = 0; s < R; ++s) {
            const int r = tid + s * T;
            act[s] = r > j && r < m;
            float lr, li;
            cmul_fixed(x[s][B].x, x[s][B].y, ir, ii, lr, li);
            if (act[s]) x[s][B] = make_float2(lr, li);
            nl[s] = make_float2(-lr, -lr);
            pl[s] = make_float2(li, -li);
        }
        if (!zero) {
#pragma unroll
            for (int c = B + 1; c < W; ++c)
                if (c - B <= live) {
                    const float4 u = s_p[c];
                    const float2 u1 = make_float2(u.x, u.y), u2 = make_float2(u.z, u.w);
#pragma unroll
                    for (int s = 0; s < R; ++s)
                        if (act[s]) {
                            // x - (fma(lr, ur, -li ui), fma(lr, ui, li ur)) as x + fma(-l.re, u, (li ui, -li ur))
                            const float2 q = __ffma2_rn(nl[s], u1, __fmul2_rn(pl[s], u2));
                            x[s][c] = __fadd2_rn(x[s][c], q);
                        }
                }
        }
        float v = -1.f;
        int idx = 0x7fffffff;
        if (B + 1 < W && live > 0) {
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (act[s]) {
                    const float a = cabs1(x[s][B + 1].x, x[s][B + 1].y);
                    if (a > v) { v = a; idx = tid + s * T; }
                }
        }
        if (live > 0) {
            argmax_warp(v, idx);
            if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
        }
        __syncthreads();
    }
};

template <int W, int R, int T>
__global__ void __launch_bounds__(T, 1) k_panel_reg(float *a_re, float *a_im, long long lda, long long a_stride,
                                                    int n, int k0, int *piv, long long piv_stride, int *info) {
    constexpr int NW = T / 32, SP = 2 * W + 1;
    static_assert(T % 32 == 0 && NW <= 32 && T > W && (W == 16 || W == 32 || W == 64), "layout");
    __shared__ float s_v[NW];
    __shared__ int s_i[NW];
    __shared__ float4 s_p[W];   // pivot row (the new row j) as (re, im, im, re), rotated as the rows are
    __shared__ float2 s_o[W];   // old row j (the new row p)
    extern __shared__ float s_stage[];
    const int b = blockIdx.x;
    int *pv = piv + (size_t)b * piv_stride;
    const int m = n - k0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float *gre = a_re + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    float *gim = a_im + (size_t)b * a_stride + (size_t)k0 * lda + k0;
    // coalesced in and out through shared memory: a warp moves consecutive
    // (row, part, column) elements; pitch 2W + 1 keeps a thread's own row on
    // distinct banks from its neighbours'
    for (int e = tid; e < m * 2 * W; e += T) {
        const int r = e / (2 * W), k = e % (2 * W);
        cp_async4(&s_stage[r * SP + k], (k < W ? gre + k : gim + (k - W)) + (size_t)r * lda, 4);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    PanelRegs<W, R, T> P;
#pragma unroll
    for (int s = 0; s < R; ++s) {
        const int r = tid + s * T;
#pragma unroll
        for (int c = 0; c < W; ++c)
            P.x[s][c] = r < m ? make_float2(s_stage[r * SP + c], s_stage[r * SP + W + c]) : make_float2(0.f, 0.f);
    }
    float v = -1.f;
    int idx = 0x7fffffff;
#pragma unroll
    for (int s = 0; s < R; ++s) {
        const int r = tid + s * T;
        const float c = cabs1(P.x[s][0].x, P.x[s][0].y);
        if (r < m && c > v) { v = c; idx = r; }
    }
    argmax_warp(v, idx);
    if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
    __syncthreads();
    int first_zero = 0;
#pragma unroll 1
    for (int j = 0; j < W; j += 2) {
        P.template column<0>(j, m, k0, tid, lane, warp, s_v, s_i, s_p, s_o, pv, first_zero);
        P.template column<1>(j + 1, m, k0, tid, lane, warp, s_v, s_i, s_p, s_o, pv, first_zero);
        // rotate left by two: columns j + 2, j + 3 to registers 0, 1
#pragma unroll
        for (int s = 0; s < R; ++s) {
            const float2 t0 = P.x[s][0], t1 = P.x[s][1];
#pragma unroll
            for (int c = 0; c + 2 < W; ++c) P.x[s][c] = P.x[s][c + 2];
            P.x[s][W - 2] = t0;
            P.x[s][W - 1] = t1;
        }
    }
#pragma unroll
    for (int s = 0; s < R; ++s) {
        const int r = tid + s * T;
        if (r < m) {
#pragma unroll
            for (int c = 0; c < W; ++c) {
                s_stage[r * SP + c] = P.x[s][c].x;
                s_stage[r * SP + W + c] = P.x[s][c].y;
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < m * 2 * W; e += T) {
        const int r = e / (2 * W), k = e % (2 * W);
        (k < W ? gre + k : gim + (k - W))[(size_t)r * lda] = s_stage[r * SP + k];
    }
    if (tid == 0 && first_zero && info[b] == 0) info[b] = first_zero;
}

// Panel factorisation across a thread-block cluster, for panels too tall for
// one CTA's shared memory.  CTA q of the cluster owns panel rows
// [q R, (q+1) R) in its shared memory (pitch nb + 1), thread per row as in
// k_panel_rows.  Per column j, one cluster barrier:
//   before it, warp 0 of every CTA publishes its best candidate (value,
//   row) and a copy of that row, and CTA 0 a copy of row j, in buffers
//   double-buffered by column parity;
//   after it, every CTA picks the pivot from the CS candidates (same order
//   everywhere) and reads the pivot row, and the pivot row's owner the old
//   row j, from those buffers (DSMEM); owners then write row j := pivot row,
//   row p := old row j locally, and every CTA scales, updates and takes the
//   next column's candidate from its own rows below j in one pass.
// A buffer of parity j is rewritten only after the barrier of column j + 1,
// which every CTA reaches after its reads of column j.
template <int CS>
__global__ void __launch_bounds__(kPanelRowsThreads)
    k_panel_cluster(float *a_re, float *a_im, long long lda, long long a_stride, int n, int k0, int nb, int R,
                    int *piv, long long piv_stride, int *info) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ float s_panel[];
    __shared__ float s_v[kPanelRowsThreads / 32];
    __shared__ int s_i[kPanelRowsThreads / 32];
    __shared__ float s_cv[2];                 // this CTA's candidate (by column parity)
    __shared__ int s_ci[2];
    __shared__ float s_cr[2][64], s_cim[2][64];   // its row (nb <= 64)
    __shared__ float s_jr[2][64], s_jim[2][64];   // CTA 0: row j
    __shared__ float s_pr[64], s_pi[64];          // pivot row
    __shared__ float s_or[64], s_oi[64];          // old row j (used by the pivot row's owner)
    const int q = (int)cluster.block_rank();
    const int b = blockIdx.y;
    int *pv = piv + (size_t)b * piv_stride;
    const int m = n - k0;
    const int P = nb + 1;
    const int r0 = q * R, r1 = min(m, r0 + R);  // own panel rows
    const int nr = max(0, r1 - r0);
    float *pre = s_panel, *pim = s_panel + R * P;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    float *gre = a_re + (size_t)b * a_stride + (size_t)(k0 + r0) * lda + k0;
    float *gim = a_im + (size_t)b * a_stride + (size_t)(k0 + r0) * lda + k0;
    for (int e = tid; e < nr * nb; e += blockDim.x) {
        const int r = e / nb, j = e - r * nb;
        pre[r * P + j] = gre[(size_t)r * lda + j];
        pim[r * P + j] = gim[(size_t)r * lda + j];
    }
    __syncthreads();
    float v = -1.f;
    int idx = 0x7fffffff;
    for (int lr = tid; lr < nr; lr += blockDim.x) {
        const float c = cabs1(pre[lr * P], pim[lr * P]);
        if (c > v) { v = c; idx = r0 + lr; }
    }
    argmax_warp(v, idx);
    if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
    __syncthreads();
    int first_zero = 0;
    for (int j = 0; j < nb; ++j) {
        const int par = j & 1;
        // ---- publish this CTA's candidate (and, CTA 0, row j)
        if (warp == 0) {
            float cv = lane < nw ? s_v[lane] : -1.f;
            int ci = lane < nw ? s_i[lane] : 0x7fffffff;
            argmax_warp(cv, ci);
            if (lane == 0) { s_cv[par] = cv; s_ci[par] = ci; }
            for (int c = lane; c < nb; c += 32) {
                if (ci < m) {
                    s_cr[par][c] = pre[(ci - r0) * P + c];
                    s_cim[par][c] = pim[(ci - r0) * P + c];
                }
                if (q == 0) {
                    s_jr[par][c] = pre[(j - r0) * P + c];
                    s_jim[par][c] = pim[(j - r0) * P + c];
                }
            }
        }
        cluster.sync();
        // ---- pivot: warp 0 alone (lane c reads CTA c's candidate); the other
        // warps only need the pivot row, which they read after the barrier
        if (warp == 0) {
            float bv = -1.f;
            int p = 0x7fffffff;
            if (lane < CS) {
                bv = *cluster.map_shared_rank(&s_cv[par], lane);
                p = *cluster.map_shared_rank(&s_ci[par], lane);
            }
            argmax_warp(bv, p);
            if (p >= m) p = j;  // column of NaNs: keep the diagonal, as icamax does
            const int owner_p = p / R;
            for (int c = lane; c < nb; c += 32) {
                if (p == j) {
                    s_pr[c] = *cluster.map_shared_rank(&s_jr[par][c], 0);
                    s_pi[c] = *cluster.map_shared_rank(&s_jim[par][c], 0);
                } else {
                    s_pr[c] = *cluster.map_shared_rank(&s_cr[par][c], owner_p);
                    s_pi[c] = *cluster.map_shared_rank(&s_cim[par][c], owner_p);
                    if (q == owner_p) {
                        s_or[c] = *cluster.map_shared_rank(&s_jr[par][c], 0);
                        s_oi[c] = *cluster.map_shared_rank(&s_jim[par][c], 0);
                    }
                }
                if (q == 0) {   // row j (< 64 <= R) lives in CTA 0
                    pre[(j - r0) * P + c] = s_pr[c];
                    pim[(j - r0) * P + c] = s_pi[c];
                }
                if (q == owner_p && p != j) {
                    pre[(p - r0) * P + c] = s_or[c];
                    pim[(p - r0) * P + c] = s_oi[c];
                }
            }
            if (q == 0 && tid == 0) pv[k0 + j] = k0 + p;
        }
        __syncthreads();
        const float dr = s_pr[j], di = s_pi[j];
        const bool zero = (dr == 0.f && di == 0.f);
        float ir = 0.f, ii = 0.f;
        if (zero) {
            if (first_zero == 0) first_zero = k0 + j + 1;
        } else {
            pivot_inverse(dr, di, ir, ii);
        }
        // ---- E (own rows below j)
        v = -1.f;
        idx = 0x7fffffff;
        const bool next = j + 1 < nb;
        for (int lr = max(0, j + 1 - r0) + tid; lr < nr; lr += blockDim.x) {
            const int o = lr * P;
            const float xr = pre[o + j], xi = pim[o + j];
            float l_r, l_i;
            cmul_fixed(xr, xi, ir, ii, l_r, l_i);
            pre[o + j] = l_r;
            pim[o + j] = l_i;
            if (!zero) {
#pragma unroll 4
                for (int c = j + 1; c < nb; ++c) csub_mul_fixed(pre[o + c], pim[o + c], l_r, l_i, s_pr[c], s_pi[c]);
            }
            if (next) {
                const float a = cabs1(pre[o + j + 1], pim[o + j + 1]);
                if (a > v) { v = a; idx = r0 + lr; }
            }
        }
        if (next) {
            argmax_warp(v, idx);
            if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
        }
        // also orders the last column's scaling before the write-back
        __syncthreads();
    }
    for (int e = tid; e < nr * nb; e += blockDim.x) {
        const int r = e / nb, j = e - r * nb;
        gre[(size_t)r * lda + j] = pre[r * P + j];
        gim[(size_t)r * lda + j] = pim[r * P + j];
    }
    if (q == 0 && tid == 0 && first_zero && info[b] == 0) info[b] = first_zero;
    // no CTA may exit while another can still read its shared memory
    cluster.sync();
}

// Row swaps + forward substitution for a column range, staged in shared
// memory.  A CTA owns up to kSwapCols consecutive columns of
// [col_lo, col_hi) minus the panel [ex_lo, ex_lo + np).  The rows touched by
// the pivots of rows k0 .. k0+np-1 (the np block rows and at most np distinct
// rows below) are loaded once with coalesced reads, the swap sequence is
// replayed in shared memory, columns >= trsm_lo are solved with the unit-lower
// L11 = A[k0:k0+np, k0:k0+np] (np <= 64) in 16-row register chunks, and the
// touched rows are written back.
constexpr int kSwapCols = 64;
constexpr int kSwapThreads = 256;
constexpr size_t kSwapSmem = (size_t)(2 * 128 * (kSwapCols + 1) + 2 * 64 * 65) * sizeof(float);

__global__ void __launch_bounds__(kSwapThreads) k_swap_trsm(float *a_re, float *a_im, long long lda,
                                                            long long a_stride, int k0, int np, int col_lo,
                                                            int col_hi, int ex_lo, int ex_w, int trsm_lo,
                                                            const int *piv, long long piv_stride) {
    extern __shared__ float s_dyn[];
    constexpr int XP = kSwapCols + 1;
    float *Xr = s_dyn, *Xi = Xr + 128 * XP;           // [slot][col]
    float *Lr = Xi + 128 * XP, *Li = Lr + 64 * 65;     // [row][col] of L11
    __shared__ int s_slot[64];   // smem slot holding the partner row of pivot j
    __shared__ int s_row[128];   // global row of each slot (-1: unused)
    __shared__ int s_col[kSwapCols];
    const int b = blockIdx.y;
    float *are = a_re + (size_t)b * a_stride, *aim = a_im + (size_t)b * a_stride;
    const int *pv = piv ? piv + (size_t)b * piv_stride : nullptr;   // NULL: no interchanges, TRSM only
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ncols_total = col_hi - col_lo - ex_w;
    const int c_first = blockIdx.x * kSwapCols;
    const int ncols = min(kSwapCols, ncols_total - c_first);
    if (tid < kSwapCols) {
        int col = col_lo + c_first + tid;
        if (col >= ex_lo) col += ex_w;
        s_col[tid] = tid < ncols ? col : -1;
    }
    if (tid < 128) s_row[tid] = tid < np ? k0 + tid : -1;
    __shared__ int s_pv[64];
    if (tid < np) s_pv[tid] = pv ? pv[k0 + tid] : k0 + tid;
    __syncthreads();
    if (tid < np) {
        const int p = s_pv[tid];
        int slot;
        if (p < k0 + np) {
            slot = p - k0;
        } else {
            int first = tid;
            for (int j = 0; j < tid; ++j)
                if (s_pv[j] == p) { first = j; break; }
            slot = np + first;
            if (first == tid) s_row[slot] = p;
        }
        s_slot[tid] = slot;
    }
    // every global read is an asynchronous copy, all in flight together
    const bool any_trsm = trsm_lo < col_hi;
    if (any_trsm)
        for (int e = tid; e < np * np; e += blockDim.x) {
            const int r = e / np, c = e - r * np;
            cp_async4(&Lr[r * 65 + c], are + (size_t)(k0 + r) * lda + k0 + c, 4);
            cp_async4(&Li[r * 65 + c], aim + (size_t)(k0 + r) * lda + k0 + c, 4);
        }
    __syncthreads();
    // load touched rows: warps over slots, lanes over columns
    for (int sl = warp; sl < 128; sl += kSwapThreads / 32) {
        const int row = s_row[sl];
        if (row < 0) continue;
        for (int c = lane; c < ncols; c += 32) {
            cp_async4(&Xr[sl * XP + c], are + (size_t)row * lda + s_col[c], 4);
            cp_async4(&Xi[sl * XP + c], aim + (size_t)row * lda + s_col[c], 4);
        }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    if (tid < ncols) {
        const int c = tid;
        for (int j = 0; j < np; ++j) {
            const int sl = s_slot[j];
            if (sl != j) {
                const float tr = Xr[j * XP + c], ti = Xi[j * XP + c];
                Xr[j * XP + c] = Xr[sl * XP + c];
                Xi[j * XP + c] = Xi[sl * XP + c];
                Xr[sl * XP + c] = tr;
                Xi[sl * XP + c] = ti;
            }
        }
    }
    // TRSM X[0:np] = L11^-1 X[0:np] on the columns >= trsm_lo, in 16-row
    // blocks: row group 0 (threads 0..63, one per column) solves the block's
    // diagonal triangle in registers, then the four row groups update the
    // rows below it (row r by group r mod 4)
    if (any_trsm) {
        static_assert(kSwapCols == 64 && kSwapThreads == 256, "64 columns x 4 row groups");
        const int c = tid & 63, rg = tid >> 6;
        const bool col_on = c < ncols && s_col[c] >= trsm_lo;
        for (int q0 = 0; q0 < np; q0 += 16) {
            const int qn = min(16, np - q0);
            __syncthreads();
            if (rg == 0 && col_on) {
                float xr[16], xi[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (i < qn) { xr[i] = Xr[(q0 + i) * XP + c]; xi[i] = Xi[(q0 + i) * XP + c]; }
#pragma unroll
                for (int i = 1; i < 16; ++i)
                    if (i < qn) {
                        float sr = xr[i], si = xi[i];
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (j < i) {
                                const float lr = Lr[(q0 + i) * 65 + q0 + j], li = Li[(q0 + i) * 65 + q0 + j];
                                sr -= lr * xr[j] - li * xi[j];
                                si -= lr * xi[j] + li * xr[j];
                            }
                        xr[i] = sr;
                        xi[i] = si;
                    }
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (i < qn) { Xr[(q0 + i) * XP + c] = xr[i]; Xi[(q0 + i) * XP + c] = xi[i]; }
            }
            __syncthreads();
            if (col_on && q0 + qn < np) {
                float xr[16], xi[16];
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    if (i < qn) { xr[i] = Xr[(q0 + i) * XP + c]; xi[i] = Xi[(q0 + i) * XP + c]; }
                for (int r = q0 + qn + rg; r < np; r += 4) {
                    float sr = Xr[r * XP + c], si = Xi[r * XP + c];
#pragma unroll
                    for (int j = 0; j < 16; ++j)
                        if (j < qn) {
                            const float lr = Lr[r * 65 + q0 + j], li = Li[r * 65 + q0 + j];
                            sr -= lr * xr[j] - li * xi[j];
                            si -= lr * xi[j] + li * xr[j];
                        }
                    Xr[r * XP + c] = sr;
                    Xi[r * XP + c] = si;
                }
            }
        }
    }
    __syncthreads();
    for (int sl = warp; sl < 128; sl += kSwapThreads / 32) {
        const int row = s_row[sl];
        if (row < 0) continue;
        for (int c = lane; c < ncols; c += 32) {
            are[(size_t)row * lda + s_col[c]] = Xr[sl * XP + c];
            aim[(size_t)row * lda + s_col[c]] = Xi[sl * XP + c];
        }
    }
}

// ---------------------------------------------------------------------------
// Triangular solves, one CTA per (matrix, right-hand side): x staged in
// shared memory; 32-row diagonal blocks staged as a tile and solved by a
// register column sweep in warp 0; the block's contribution to every later
// row applied by one thread per row (op = A: the row's 32 contiguous factor
// entries; op = A^T / A^H: consecutive threads read consecutive columns of
// the block's factor rows).  Best when many matrices / right-hand sides
// fill the GPU; TR: 0 = A, 1 = A^T, 2 = A^H.
// ---------------------------------------------------------------------------
constexpr int kGetrsThreads = 512;

template <int TR>
__device__ __forceinline__ void op_at(const float *Ar, const float *Ai, long long lda, int i, int j, float &re,
                                      float &im) {
    if (TR == 0) {
        re = Ar[(size_t)i * lda + j];
        im = Ai[(size_t)i * lda + j];
    } else {
        re = Ar[(size_t)j * lda + i];
        im = TR == 2 ? -Ai[(size_t)j * lda + i] : Ai[(size_t)j * lda + i];
    }
}

// One triangular phase on x in shared memory: lower (blocks from the top) or
// upper (from the bottom), unit or non-unit diagonal.
template <bool LOWER, bool UNIT, int TR>
__device__ void getrs_phase(int n, const float *Ar, const float *Ai, long long lda, float *xr, float *xi, float *t_r,
                            float *t_i, float *wt_r, float *wt_i) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (n + 31) / 32;
    for (int q = 0; q < nblk; ++q) {
        const int b = LOWER ? q : nblk - 1 - q;
        const int j0 = b * 32, jb = min(32, n - j0);
        for (int e = tid; e < 32 * 32; e += blockDim.x) {
            // op = A: lanes along a factor row; op = A^T / A^H: lanes along the
            // factor row that holds an op-column (coalesced either way)
            const int r = TR == 0 ? (e >> 5) : (e & 31), c = TR == 0 ? (e & 31) : (e >> 5);
            float tr = 0.f, ti = 0.f;
            if (r < jb && c < jb && (LOWER ? c <= r : c >= r)) op_at<TR>(Ar, Ai, lda, j0 + r, j0 + c, tr, ti);
            t_r[r * 33 + c] = tr;
            t_i[r * 33 + c] = ti;
        }
        __syncthreads();
        if (warp == 0) {
            float vr = lane < jb ? xr[j0 + lane] : 0.f, vi = lane < jb ? xi[j0 + lane] : 0.f;
            for (int t = 0; t < jb; ++t) {
                const int j = LOWER ? t : jb - 1 - t;
                if (!UNIT && lane == j) {
                    const float dr = t_r[j * 33 + j], di = t_i[j * 33 + j];
                    const float den = 1.0f / (dr * dr + di * di);
                    const float yr = vr, yi = vi;
                    vr = (yr * dr + yi * di) * den;
                    vi = (yi * dr - yr * di) * den;
                }
                const float jr = __shfl_sync(0xffffffffu, vr, j), ji = __shfl_sync(0xffffffffu, vi, j);
                if (LOWER ? lane > j : lane < j) {
                    const float lr = t_r[lane * 33 + j], li = t_i[lane * 33 + j];
                    vr -= lr * jr - li * ji;
                    vi -= lr * ji + li * jr;
                }
            }
            if (lane < jb) { xr[j0 + lane] = vr; xi[j0 + lane] = vi; }
        }
        __syncthreads();
        // later rows: below the block (lower) or above it (upper)
        const int r0 = LOWER ? j0 + jb : 0, r1 = LOWER ? n : j0;
        const float cs = TR == 2 ? -1.f : 1.f;
        if (TR == 0 && wt_r) {
            // op = A: each warp takes 32 rows at a time, loads the 32 x jb block
            // row by row (one 128-byte line per load) into its own tile, then
            // lane r reduces row r from shared memory
            float *mr = wt_r + warp * (32 * 33), *mi = wt_i + warp * (32 * 33);
            for (int gb = r0 + warp * 32; gb < r1; gb += (blockDim.x >> 5) * 32) {
                const int nr = min(32, r1 - gb);
#pragma unroll 8
                for (int rr = 0; rr < 32; ++rr) {
                    float vr = 0.f, vi = 0.f;
                    if (rr < nr && lane < jb) {
                        vr = Ar[(size_t)(gb + rr) * lda + j0 + lane];
                        vi = Ai[(size_t)(gb + rr) * lda + j0 + lane];
                    }
                    mr[rr * 33 + lane] = vr;
                    mi[rr * 33 + lane] = vi;
                }
                __syncwarp();
                float pr = 0.f, pi = 0.f;
#pragma unroll 8
                for (int c = 0; c < 32; ++c) {
                    const float ar = mr[lane * 33 + c], ai = mi[lane * 33 + c];
                    const float x_r = xr[j0 + c], x_i = xi[j0 + c];
                    pr += ar * x_r - ai * x_i;
                    pi += ar * x_i + ai * x_r;
                }
                if (lane < nr) {
                    xr[gb + lane] -= pr;
                    xi[gb + lane] -= pi;
                }
                __syncwarp();
            }
            __syncthreads();
            continue;
        }
        for (int i = r0 + tid; i < r1; i += blockDim.x) {
            float pr = 0.f, pi = 0.f;
            if (TR == 0) {
                const float *rr = Ar + (size_t)i * lda + j0, *ri = Ai + (size_t)i * lda + j0;
#pragma unroll 8
                for (int c = 0; c < jb; ++c) {
                    const float ar = rr[c], ai = ri[c];
                    pr += ar * xr[j0 + c] - ai * xi[j0 + c];
                    pi += ar * xi[j0 + c] + ai * xr[j0 + c];
                }
            } else {
#pragma unroll 8
                for (int c = 0; c < jb; ++c) {
                    const float ar = Ar[(size_t)(j0 + c) * lda + i], ai = cs * Ai[(size_t)(j0 + c) * lda + i];
                    pr += ar * xr[j0 + c] - ai * xi[j0 + c];
                    pi += ar * xi[j0 + c] + ai * xr[j0 + c];
                }
            }
            xr[i] -= pr;
            xi[i] -= pi;
        }
        __syncthreads();
    }
}

template <int TR>
__global__ void __launch_bounds__(kGetrsThreads) k_getrs(int n, const float *lu_re, const float *lu_im, long long lda,
                                                         long long a_stride, const int *piv, long long piv_stride,
                                                         float *b_re, float *b_im, long long ldb, long long b_stride) {
    extern __shared__ float s_x[];
    __shared__ float t_r[32 * 33], t_i[32 * 33];
    __shared__ int s_pv[1024];
    float *xr = s_x, *xi = s_x + n;
    const int mat = blockIdx.y, rhs = blockIdx.x;
    const float *Ar = lu_re + (size_t)mat * a_stride, *Ai = lu_im + (size_t)mat * a_stride;
    float *br = b_re + (size_t)mat * b_stride + rhs, *bi = b_im + (size_t)mat * b_stride + rhs;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        xr[i] = br[(size_t)i * ldb];
        xi[i] = bi[(size_t)i * ldb];
    }
    const int *pv = piv ? piv + (size_t)mat * piv_stride : nullptr;
    auto permute = [&](bool reverse) {
        const int nchunk = (n + 1023) / 1024;
        for (int qq = 0; qq < nchunk; ++qq) {
            const int base = (reverse ? nchunk - 1 - qq : qq) * 1024;
            const int cnt = min(1024, n - base);
            __syncthreads();
            for (int i = threadIdx.x; i < cnt; i += blockDim.x) s_pv[i] = pv[base + i];
            __syncthreads();
            if (threadIdx.x == 0)
                for (int t = 0; t < cnt; ++t) {
                    const int k = reverse ? cnt - 1 - t : t;
                    const int p = s_pv[k], r = base + k;
                    if (p != r && p >= 0 && p < n) {
                        float tmp = xr[r]; xr[r] = xr[p]; xr[p] = tmp;
                        tmp = xi[r]; xi[r] = xi[p]; xi[p] = tmp;
                    }
                }
        }
    };
    if (TR == 0 && pv) permute(false);
    __syncthreads();
    float *wt_r = TR == 0 ? s_x + 2 * n : nullptr;          // per-warp 32 x 33 tiles (op = A)
    float *wt_i = TR == 0 ? wt_r + (kGetrsThreads / 32) * 32 * 33 : nullptr;
    if (TR == 0) {
        getrs_phase<true, true, 0>(n, Ar, Ai, lda, xr, xi, t_r, t_i, wt_r, wt_i);
        getrs_phase<false, false, 0>(n, Ar, Ai, lda, xr, xi, t_r, t_i, wt_r, wt_i);
    } else {
        getrs_phase<true, false, TR>(n, Ar, Ai, lda, xr, xi, t_r, t_i, nullptr, nullptr);
        getrs_phase<false, true, TR>(n, Ar, Ai, lda, xr, xi, t_r, t_i, nullptr, nullptr);
    }
    if (TR != 0 && pv) permute(true);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        br[(size_t)i * ldb] = xr[i];
        bi[(size_t)i * ldb] = xi[i];
    }
}

// ---------------------------------------------------------------------------
// Blocked solves for many CTAs per right-hand side, op(A) = A, A^T or A^H
// (TR = 0, 1, 2).  With P A = L U:
//   op = A:    x = U^-1 L^-1 P b       (L unit lower, then U upper)
//   op = A^T:  x = P^T L^-T U^-T b     (U^T lower non-unit, then L^T upper unit)
//   op = A^H:  the same with conjugates.
// The rows are cut into kTB-row blocks.  One launch per block step: CTA 0
// of each (rhs, matrix) applies the finished block's x to the next block's
// rows and solves that block's diagonal triangle; the other CTAs apply the
// finished block to all later rows (op = A: warp per row over the row's
// contiguous segment; op = A^T / A^H: thread per row over the block's
// contiguous rows of the factor).  A prologue CTA per (rhs, matrix) applies
// the interchanges (op = A) and solves the first block; an epilogue CTA
// applies the reverse interchanges (op = A^T / A^H).  x lives in b.
// ---------------------------------------------------------------------------
constexpr int kTB = 128;          // rows per block step
constexpr int kTrsvThreads = 256;
constexpr int kTrsvRows = 64;     // rows per update CTA, op = A (8 warps x 8 rows)
constexpr int kTrsvRowsT = 256;   // rows per update CTA, op = A^T / A^H (thread per row)

// element (i, j) of op(A) from the stored factors
template <int TR>
__device__ __forceinline__ void op_elem(const float *Ar, const float *Ai, long long lda, int i, int j, float &re,
                                        float &im) {
    if (TR == 0) {
        re = Ar[(size_t)i * lda + j];
        im = Ai[(size_t)i * lda + j];
    } else {
        re = Ar[(size_t)j * lda + i];
        im = TR == 2 ? -Ai[(size_t)j * lda + i] : Ai[(size_t)j * lda + i];
    }
}

// Solve the diagonal triangle of op-rows [g0, g1) in place (x in global):
// lower (sub-blocks from the top) or upper (from the bottom), unit or
// non-unit diagonal.  All kTrsvThreads threads take part.
template <bool LOWER, bool UNIT, int TR>
__device__ void trsv_diag(const float *Ar, const float *Ai, long long lda, float *xr, float *xi, long long ldb,
                          int g0, int g1, float *s_tr, float *s_ti, float *s_xr, float *s_xi) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const int gb = g1 - g0;
    const int nsub = (gb + 31) / 32;
    for (int q = 0; q < nsub; ++q) {
        const int sb = LOWER ? q : nsub - 1 - q;
        const int s0 = g0 + sb * 32, s1 = min(g1, s0 + 32), sw = s1 - s0;
        // stage the 32 x 32 diagonal tile of op(A) (pitch 33) and the sub-block's x
        for (int e = tid; e < 32 * 32; e += blockDim.x) {
            const int r = e >> 5, c = e & 31;
            float tr = 0.f, ti = 0.f;
            if (r < sw && c < sw) op_elem<TR>(Ar, Ai, lda, s0 + r, s0 + c, tr, ti);
            s_tr[r * 33 + c] = tr;
            s_ti[r * 33 + c] = ti;
        }
        if (tid < 32) {
            s_xr[tid] = tid < sw ? xr[(size_t)(s0 + tid) * ldb] : 0.f;
            s_xi[tid] = tid < sw ? xi[(size_t)(s0 + tid) * ldb] : 0.f;
        }
        __syncthreads();
        if (warp == 0) {
            // column sweep: lane i holds x_i; step j finalises x_j and removes
            // its contribution from the remaining rows
            float vr = s_xr[lane], vi = s_xi[lane];
            for (int t = 0; t < sw; ++t) {
                const int j = LOWER ? t : sw - 1 - t;
                if (!UNIT && lane == j) {
                    const float dr = s_tr[j * 33 + j], di = s_ti[j * 33 + j];
                    const float den = 1.0f / (dr * dr + di * di);
                    const float yr = vr, yi = vi;
                    vr = (yr * dr + yi * di) * den;
                    vi = (yi * dr - yr * di) * den;
                }
                const float jr = __shfl_sync(0xffffffffu, vr, j), ji = __shfl_sync(0xffffffffu, vi, j);
                if (LOWER ? lane > j : lane < j) {
                    const float lr = s_tr[lane * 33 + j], li = s_ti[lane * 33 + j];
                    vr -= lr * jr - li * ji;
                    vi -= lr * ji + li * jr;
                }
            }
            s_xr[lane] = vr;
            s_xi[lane] = vi;
            if (lane < sw) {
                xr[(size_t)(s0 + lane) * ldb] = vr;
                xi[(size_t)(s0 + lane) * ldb] = vi;
            }
        }
        __syncthreads();
        // remaining rows of this diagonal block: below (lower) or above (upper)
        const int u0 = LOWER ? s1 : g0, u1 = LOWER ? g1 : s0;
        for (int i = u0 + warp; i < u1; i += nw) {
            float pr = 0.f, pi = 0.f;
            if (lane < sw) {
                float ar, ai;
                op_elem<TR>(Ar, Ai, lda, i, s0 + lane, ar, ai);
                pr = ar * s_xr[lane] - ai * s_xi[lane];
                pi = ar * s_xi[lane] + ai * s_xr[lane];
            }
            for (int o = 16; o > 0; o >>= 1) {
                pr += __shfl_xor_sync(0xffffffffu, pr, o);
                pi += __shfl_xor_sync(0xffffffffu, pi, o);
            }
            if (lane == 0) {
                xr[(size_t)i * ldb] -= pr;
                xi[(size_t)i * ldb] -= pi;
            }
        }
        __syncthreads();
    }
}

// op-rows [r0, r1): x_i -= op(A)[i, f0:f0+fw] x[f0:f0+fw], x of the block staged in s_x*
template <int TR>
__device__ __forceinline__ void trsv_apply(const float *Ar, const float *Ai, long long lda, float *xr, float *xi,
                                           long long ldb, int f0, int fw, int r0, int r1, const float *s_xr,
                                           const float *s_xi) {
    if (TR == 0) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int i = r0 + warp; i < r1; i += nw) {
            const float *rr = Ar + (size_t)i * lda + f0, *ri = Ai + (size_t)i * lda + f0;
            float pr = 0.f, pi = 0.f;
#pragma unroll
            for (int c0 = 0; c0 < kTB; c0 += 32) {
                const int c = c0 + lane;
                if (c < fw) {
                    const float ar = rr[c], ai = ri[c];
                    pr += ar * s_xr[c] - ai * s_xi[c];
                    pi += ar * s_xi[c] + ai * s_xr[c];
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                pr += __shfl_xor_sync(0xffffffffu, pr, o);
                pi += __shfl_xor_sync(0xffffffffu, pi, o);
            }
            if (lane == 0) {
                xr[(size_t)i * ldb] -= pr;
                xi[(size_t)i * ldb] -= pi;
            }
        }
    } else {
        // op(A)[i, c] = A[c, i] (conjugated for A^H): threads over i read rows c coalesced
        const float cs = TR == 2 ? -1.f : 1.f;
        for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
            float pr = 0.f, pi = 0.f;
#pragma unroll 8
            for (int c = 0; c < fw; ++c) {
                const float ar = Ar[(size_t)(f0 + c) * lda + i], ai = cs * Ai[(size_t)(f0 + c) * lda + i];
                pr += ar * s_xr[c] - ai * s_xi[c];
                pi += ar * s_xi[c] + ai * s_xr[c];
            }
            xr[(size_t)i * ldb] -= pr;
            xi[(size_t)i * ldb] -= pi;
        }
    }
}

// Apply the interchanges to the whole vector in shared memory: forward order
// (P b, op = A) or reverse order (P^T v, op = A^T / A^H).
template <bool REVERSE>
__device__ void trsv_permute(int n, const int *pv, float *xr, float *xi, long long ldb, float *vr, float *vi) {
    __shared__ int s_pv[1024];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        vr[i] = xr[(size_t)i * ldb];
        vi[i] = xi[(size_t)i * ldb];
    }
    const int nchunk = (n + 1023) / 1024;
    for (int q = 0; q < nchunk; ++q) {
        const int base = (REVERSE ? nchunk - 1 - q : q) * 1024;
        const int cnt = min(1024, n - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += blockDim.x) s_pv[i] = pv[base + i];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int t = 0; t < cnt; ++t) {
                const int k = REVERSE ? cnt - 1 - t : t;
                const int p = s_pv[k], r = base + k;
                if (p != r && p >= 0 && p < n) {
                    float tmp = vr[r]; vr[r] = vr[p]; vr[p] = tmp;
                    tmp = vi[r]; vi[r] = vi[p]; vi[p] = tmp;
                }
            }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        xr[(size_t)i * ldb] = vr[i];
        xi[(size_t)i * ldb] = vi[i];
    }
    __syncthreads();
}

// Prologue: one CTA per (rhs, matrix).  First phase (lower operator): the
// interchanges for op = A, then the first block; second phase (upper
// operator): the last block.
template <bool LOWER, bool UNIT, int TR>
__global__ void __launch_bounds__(kTrsvThreads) k_trsv_first(int n, const float *lu_re, const float *lu_im,
                                                             long long lda, long long a_stride, const int *piv,
                                                             long long piv_stride, float *b_re, float *b_im,
                                                             long long ldb, long long b_stride) {
    extern __shared__ float s_x[];
    __shared__ float s_tr[32 * 33], s_ti[32 * 33], s_xr[32], s_xi[32];
    const int mat = blockIdx.y, rhs = blockIdx.x;
    const float *Ar = lu_re + (size_t)mat * a_stride, *Ai = lu_im + (size_t)mat * a_stride;
    float *xr = b_re + (size_t)mat * b_stride + rhs, *xi = b_im + (size_t)mat * b_stride + rhs;
    if (LOWER) {
        if (TR == 0 && piv) trsv_permute<false>(n, piv + (size_t)mat * piv_stride, xr, xi, ldb, s_x, s_x + n);
        trsv_diag<true, UNIT, TR>(Ar, Ai, lda, xr, xi, ldb, 0, min(n, kTB), s_tr, s_ti, s_xr, s_xi);
    } else {
        const int last = (n - 1) / kTB;
        trsv_diag<false, UNIT, TR>(Ar, Ai, lda, xr, xi, ldb, last * kTB, n, s_tr, s_ti, s_xr, s_xi);
    }
}

// Epilogue for op = A^T / A^H: x = P^T v.
__global__ void __launch_bounds__(kTrsvThreads) k_trsv_unpermute(int n, const int *piv, long long piv_stride,
                                                                 float *b_re, float *b_im, long long ldb,
                                                                 long long b_stride) {
    extern __shared__ float s_x[];
    const int mat = blockIdx.y, rhs = blockIdx.x;
    float *xr = b_re + (size_t)mat * b_stride + rhs, *xi = b_im + (size_t)mat * b_stride + rhs;
    trsv_permute<true>(n, piv + (size_t)mat * piv_stride, xr, xi, ldb, s_x, s_x + n);
}

// Block step: x of block `blk` is final.  Lower: CTA 0 updates and solves
// block blk+1, CTAs >= 1 update rows from block blk+2 on.  Upper: CTA 0
// updates and solves block blk-1, CTAs >= 1 update rows before block blk-1.
template <bool LOWER, bool UNIT, int TR>
__global__ void __launch_bounds__(kTrsvThreads) k_trsv_step(int n, const float *lu_re, const float *lu_im,
                                                            long long lda, long long a_stride, float *b_re,
                                                            float *b_im, long long ldb, long long b_stride, int blk) {
    __shared__ float s_fr[kTB], s_fi[kTB];
    __shared__ float s_tr[32 * 33], s_ti[32 * 33], s_xr[32], s_xi[32];
    constexpr int RPC = TR == 0 ? kTrsvRows : kTrsvRowsT;
    const int mat = blockIdx.z, rhs = blockIdx.y;
    const float *Ar = lu_re + (size_t)mat * a_stride, *Ai = lu_im + (size_t)mat * a_stride;
    float *xr = b_re + (size_t)mat * b_stride + rhs, *xi = b_im + (size_t)mat * b_stride + rhs;
    const int f0 = blk * kTB, f1 = min(n, f0 + kTB), fw = f1 - f0;
    for (int c = threadIdx.x; c < kTB; c += blockDim.x) {
        s_fr[c] = c < fw ? xr[(size_t)(f0 + c) * ldb] : 0.f;
        s_fi[c] = c < fw ? xi[(size_t)(f0 + c) * ldb] : 0.f;
    }
    __syncthreads();
    int g0, g1, o0, o1;  // next diagonal block, other rows
    if (LOWER) {
        g0 = f1; g1 = min(n, g0 + kTB); o0 = g1; o1 = n;
    } else {
        g1 = f0; g0 = max(0, g1 - kTB); o0 = 0; o1 = g0;
    }
    if (blockIdx.x == 0) {
        trsv_apply<TR>(Ar, Ai, lda, xr, xi, ldb, f0, fw, g0, g1, s_fr, s_fi);
        __syncthreads();
        trsv_diag<LOWER, UNIT, TR>(Ar, Ai, lda, xr, xi, ldb, g0, g1, s_tr, s_ti, s_xr, s_xi);
    } else {
        const int r0 = o0 + (blockIdx.x - 1) * RPC;
        const int r1 = min(o1, r0 + RPC);
        if (r0 < r1) trsv_apply<TR>(Ar, Ai, lda, xr, xi, ldb, f0, fw, r0, r1, s_fr, s_fi);
    }
}

// One triangular phase: the prologue block and the block steps.
template <bool LOWER, bool UNIT, int TR>
int trsv_phase(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
               const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
               cudaStream_t st) {
    {
        const int rc = func_opt_in((const void *)k_trsv_first<LOWER, UNIT, TR>, 200 * 1024);
        if (rc != HBEM_OK) return rc;
    }
    constexpr int RPC = TR == 0 ? kTrsvRows : kTrsvRowsT;
    const int nblk = (n + kTB - 1) / kTB;
    const size_t smem = (LOWER && TR == 0 && piv) ? (size_t)n * 2 * sizeof(float) : 0;
    k_trsv_first<LOWER, UNIT, TR><<<dim3(nrhs, batch), kTrsvThreads, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv,
                                                                               piv_stride, b_re, b_im, ldb, b_stride);
    HBEM_LAUNCH_CHECK("k_trsv_first");
    if (LOWER) {
        for (int blk = 0; blk + 1 < nblk; ++blk) {
            const int rest = std::max(0, n - (blk + 2) * kTB);
            const int ctas = 1 + (rest + RPC - 1) / RPC;
            k_trsv_step<LOWER, UNIT, TR><<<dim3(ctas, nrhs, batch), kTrsvThreads, 0, st>>>(
                n, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, blk);
            HBEM_LAUNCH_CHECK("k_trsv_step");
        }
    } else {
        for (int blk = nblk - 1; blk > 0; --blk) {
            const int rest = std::max(0, (blk - 1) * kTB);
            const int ctas = 1 + (rest + RPC - 1) / RPC;
            k_trsv_step<LOWER, UNIT, TR><<<dim3(ctas, nrhs, batch), kTrsvThreads, 0, st>>>(
                n, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, blk);
            HBEM_LAUNCH_CHECK("k_trsv_step");
        }
    }
    return HBEM_OK;
}

// piv == nullptr: no interchanges (a solve with the factors L U themselves).
int lu_solve_blocked(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                     long long a_stride, const int *piv, long long piv_stride, float *b_re, float *b_im,
                     long long ldb, long long b_stride, int trans, cudaStream_t st) {
    int rc;
    if (trans == HBEM_TRANS_N) {
        rc = trsv_phase<true, true, 0>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb,
                                       b_stride, st);
        if (rc == HBEM_OK)
            rc = trsv_phase<false, false, 0>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, nullptr, piv_stride, b_re,
                                             b_im, ldb, b_stride, st);
        return rc;
    }
    if (trans == HBEM_TRANS_T) {
        rc = trsv_phase<true, false, 1>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, nullptr, piv_stride, b_re, b_im,
                                        ldb, b_stride, st);
        if (rc == HBEM_OK)
            rc = trsv_phase<false, true, 1>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, nullptr, piv_stride, b_re,
                                            b_im, ldb, b_stride, st);
    } else {
        rc = trsv_phase<true, false, 2>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, nullptr, piv_stride, b_re, b_im,
                                        ldb, b_stride, st);
        if (rc == HBEM_OK)
            rc = trsv_phase<false, true, 2>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, nullptr, piv_stride, b_re,
                                            b_im, ldb, b_stride, st);
    }
    if (rc == HBEM_OK && piv) {
        {
            const int rc = func_opt_in((const void *)k_trsv_unpermute, 200 * 1024);
            if (rc != HBEM_OK) return rc;
        }
        k_trsv_unpermute<<<dim3(nrhs, batch), kTrsvThreads, (size_t)n * 2 * sizeof(float), st>>>(n, piv, piv_stride,
                                                                                                 b_re, b_im, ldb,
                                                                                                 b_stride);
        HBEM_LAUNCH_CHECK("k_trsv_unpermute");
    }
    return rc;
}

// ---------------------------------------------------------------------------
// Wavefront triangular solves: one launch per triangular phase with many
// CTAs per right-hand side.  Each CTA owns one 32-row block of op(A).  It
// takes a ticket t = q * systems + sys from a counter (q: the block's place
// in the phase order), so every block it waits for belongs to a CTA that
// took an earlier ticket and is therefore resident: the wait graph has no
// cycle and no CTA waits on one that cannot run.
// Finished x values travel through a mailbox of 64-bit words (re, im),
// cleared to all-ones before the phase; an x value is never all-ones (NaNs
// are written in canonical form), so a word that is not all-ones is final,
// and one relaxed 64-bit load both announces and delivers it: no fence, no
// flag.  Each warp waits only for the x values it consumes, with the factor
// entries of that block loaded before the wait.  After the last block the
// CTA solves its diagonal triangle (warp 0 column sweep) and posts its x.
// Waits are bounded: past the limit a warp raises the launch's abort word
// (the other CTAs stop waiting), the CTA writes NaN into its block and sets
// the module's fault word, which the synchronising callers report.
// ---------------------------------------------------------------------------
constexpr int kWaveThreads = 256;
constexpr int kWaveSpinLimit = 1 << 22;   // polls of >= 32 ns: seconds before a wait gives up
// (HBEM_TUNE_WAVE_SPIN lowers it, so that a test can make a wait run out)
constexpr unsigned long long kWaveEmpty = ~0ull;

struct WaveCtl {
    int ticket[2];   // per phase
    int abort;
    int pad;
};

static __device__ int g_wave_fault;

// A non-zero status word of a factorisation's tensor-core update raises the
// fault word as well.
__global__ void k_fold_status(const int *status) {
    if (*status) atomicExch(&g_wave_fault, 1);
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long pack_x(float re, float im) {
    if (re != re) re = __int_as_float(0x7fc00000);
    if (im != im) im = __int_as_float(0x7fc00000);
    return (unsigned long long)__float_as_uint(re) | ((unsigned long long)__float_as_uint(im) << 32);
}

__device__ __forceinline__ float x_re(unsigned long long w) { return __uint_as_float((unsigned)w); }
__device__ __forceinline__ float x_im(unsigned long long w) { return __uint_as_float((unsigned)(w >> 32)); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Warp-wide wait until every lane's word (need: the lane reads one) is
// posted; returns false on abort or timeout.
__device__ __forceinline__ bool wave_wait(const unsigned long long *addr, bool need, unsigned long long &w,
                                          WaveCtl *ctl, int spin_limit) {
    w = need ? ld_relaxed_u64(addr) : 0ull;
    if (__all_sync(0xffffffffu, w != kWaveEmpty)) return true;
    unsigned ns = 32;
    for (int spins = 1;; ++spins) {
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
        if (w == kWaveEmpty) w = ld_relaxed_u64(addr);
        if (__all_sync(0xffffffffu, w != kWaveEmpty)) return true;
        if ((spins & 15) == 0 && __any_sync(0xffffffffu, *(volatile int *)&ctl->abort != 0)) return false;
        if (spins > spin_limit) {
            if ((threadIdx.x & 31) == 0) {
                atomicExch(&ctl->abort, 1);
                atomicExch(&g_wave_fault, 1);
            }
            return false;
        }
    }
}

template <bool LOWER, bool UNIT, int TR>
__global__ void __launch_bounds__(kWaveThreads) k_trsv_wave(int n, int nblk, int nrhs, int systems,
                                                            const float *__restrict__ lu_re,
                                                            const float *__restrict__ lu_im, long long lda,
                                                            long long a_stride, float *b_re, float *b_im,
                                                            long long ldb, long long b_stride, WaveCtl *ctl,
                                                            int phase, unsigned long long *mbox,
                                                            const int *active, int spin_limit) {
    __shared__ float s_tr[32 * 33], s_ti[32 * 33];
    __shared__ float s_pr[8][33], s_pi[8][33];
    __shared__ int s_ticket, s_abort;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_ticket = atomicAdd(&ctl->ticket[phase], 1);
        s_abort = 0;
    }
    __syncthreads();
    const int t = s_ticket;
    const int q = t / systems, sys = t - q * systems;
    if (q >= nblk) return;
    if (active && active[sys / nrhs] == 0) return;   // the whole system is skipped; nobody waits on it
    const int mat = sys / nrhs, rhs = sys - mat * nrhs;
    const float *Ar = lu_re + (size_t)mat * a_stride, *Ai = lu_im + (size_t)mat * a_stride;
    float *xr = b_re + (size_t)mat * b_stride + rhs, *xi = b_im + (size_t)mat * b_stride + rhs;
    unsigned long long *mb = mbox + (size_t)sys * n;
    const int b = LOWER ? q : nblk - 1 - q;
    const int j0 = b * 32, jb = min(32, n - j0);

    // this block's right-hand side (no other CTA writes it in this phase)
    float rb_r = 0.f, rb_i = 0.f;
    if (warp == 0 && lane < jb) {
        rb_r = xr[(size_t)(j0 + lane) * ldb];
        rb_i = xi[(size_t)(j0 + lane) * ldb];
    }
    // diagonal triangle of op(A) (lanes along a factor row for every op)
    for (int e = tid; e < 32 * 32; e += kWaveThreads) {
        const int r = TR == 0 ? (e >> 5) : (e & 31), c = TR == 0 ? (e & 31) : (e >> 5);
        float tr = 0.f, ti = 0.f;
        if (r < jb && c < jb && (LOWER ? c <= r : c >= r)) op_at<TR>(Ar, Ai, lda, j0 + r, j0 + c, tr, ti);
        s_tr[r * 33 + c] = tr;
        s_ti[r * 33 + c] = ti;
    }

    // op = A: warp w holds rows w + 8k of the block, lanes over the columns of
    // a finished block; op = A^T / A^H: warp w takes factor rows w + 8k of a
    // finished block, lane i accumulates op-row i of this block
    const float cs = TR == 2 ? -1.f : 1.f;
    auto load_a = [&](int qc, float (&pr)[4], float (&pi)[4]) {
        const int c0 = (LOWER ? qc : nblk - 1 - qc) * 32;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (TR == 0) {
                const int col = c0 + lane, r = warp + 8 * k;
                const bool ok = col < n && r < jb;
                pr[k] = ok ? __ldg(Ar + (size_t)(j0 + r) * lda + col) : 0.f;
                pi[k] = ok ? __ldg(Ai + (size_t)(j0 + r) * lda + col) : 0.f;
            } else {
                const int jr = c0 + warp + 8 * k;
                const bool ok = jr < n && lane < jb;
                pr[k] = ok ? __ldg(Ar + (size_t)jr * lda + j0 + lane) : 0.f;
                pi[k] = ok ? cs * __ldg(Ai + (size_t)jr * lda + j0 + lane) : 0.f;
            }
        }
    };
    float accr[4] = {0.f, 0.f, 0.f, 0.f}, acci[4] = {0.f, 0.f, 0.f, 0.f};
    float nr[4], ni[4];   // factor entries of block qc, loaded before its x is waited for
    bool aborted = false;
    if (q > 0) load_a(0, nr, ni);
    for (int qc = 0; qc < q; ++qc) {
        const int c0 = (LOWER ? qc : nblk - 1 - qc) * 32;
        // op = A: lane l needs x[c0 + l]; op = A^T / A^H: lane k < 4 fetches x[c0 + w + 8k]
        const int xi_idx = TR == 0 ? c0 + lane : c0 + warp + 8 * lane;
        const bool need = TR == 0 ? xi_idx < n : (lane < 4 && xi_idx < n);
        unsigned long long w;
        if (!wave_wait(mb + (need ? xi_idx : 0), need, w, ctl, spin_limit)) {
            aborted = true;
            break;
        }
        float pr[4], pi[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { pr[k] = nr[k]; pi[k] = ni[k]; }
        if (qc + 1 < q) load_a(qc + 1, nr, ni);
        if (TR == 0) {
            const float x_r = x_re(w), x_i = x_im(w);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                accr[k] = fmaf(pr[k], x_r, fmaf(-pi[k], x_i, accr[k]));
                acci[k] = fmaf(pr[k], x_i, fmaf(pi[k], x_r, acci[k]));
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const unsigned long long wk = __shfl_sync(0xffffffffu, w, k);
                const float x_r = x_re(wk), x_i = x_im(wk);
                accr[k] = fmaf(pr[k], x_r, fmaf(-pi[k], x_i, accr[k]));
                acci[k] = fmaf(pr[k], x_i, fmaf(pi[k], x_r, acci[k]));
            }
        }
    }
    if (aborted && lane == 0) s_abort = 1;
    // per-row sums of the finished blocks' contributions
    if (TR == 0) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float vr = warp_sum(accr[k]), vi = warp_sum(acci[k]);
            if (lane == 0) { s_pr[0][warp + 8 * k] = vr; s_pi[0][warp + 8 * k] = vi; }
        }
    } else {
        s_pr[warp][lane] = (accr[0] + accr[1]) + (accr[2] + accr[3]);
        s_pi[warp][lane] = (acci[0] + acci[1]) + (acci[2] + acci[3]);
    }
    __syncthreads();
    if (warp != 0) return;
    float sr, si;
    if (TR == 0) {
        sr = s_pr[0][lane];
        si = s_pi[0][lane];
    } else {
        sr = 0.f;
        si = 0.f;
#pragma unroll
        for (int w = 0; w < 8; ++w) { sr += s_pr[w][lane]; si += s_pi[w][lane]; }
    }
    float vr = rb_r - sr, vi = rb_i - si;
    // the lane's own diagonal entry and 1 / |d|^2, ahead of the sweep
    float dr = 1.f, di = 0.f, den = 1.f;
    if (!UNIT && lane < jb) {
        dr = s_tr[lane * 33 + lane];
        di = s_ti[lane * 33 + lane];
        den = 1.0f / (dr * dr + di * di);
    }
    // column sweep: lane i holds x_i; step j finalises x_j
#pragma unroll
    for (int s = 0; s < 32; ++s) {
        if (s < jb) {
            const int j = LOWER ? s : jb - 1 - s;
            if (!UNIT && lane == j) {
                const float yr = vr, yi = vi;
                vr = (yr * dr + yi * di) * den;
                vi = (yi * dr - yr * di) * den;
            }
            const float jr = __shfl_sync(0xffffffffu, vr, j), ji = __shfl_sync(0xffffffffu, vi, j);
            if (LOWER ? lane > j : lane < j) {
                const float lr = s_tr[lane * 33 + j], li = s_ti[lane * 33 + j];
                vr -= lr * jr - li * ji;
                vi -= lr * ji + li * jr;
            }
        }
    }
    if (s_abort) { vr = __int_as_float(0x7fc00000); vi = vr; }
    if (lane < jb) {
        st_relaxed_u64(mb + j0 + lane, pack_x(vr, vi));
        xr[(size_t)(j0 + lane) * ldb] = vr;
        xi[(size_t)(j0 + lane) * ldb] = vi;
    }
}

template <bool REVERSE>
__global__ void __launch_bounds__(kTrsvThreads) k_trsv_permute(int n, int nrhs, const int *piv, long long piv_stride,
                                                               float *b_re, float *b_im, long long ldb,
                                                               long long b_stride, const int *active) {
    extern __shared__ float s_x[];
    const int mat = blockIdx.y, rhs = blockIdx.x;
    if (active && active[mat] == 0) return;
    float *xr = b_re + (size_t)mat * b_stride + rhs, *xi = b_im + (size_t)mat * b_stride + rhs;
    trsv_permute<REVERSE>(n, piv + (size_t)mat * piv_stride, xr, xi, ldb, s_x, s_x + n);
}

// control block, then one mailbox of n words per system for each phase
size_t wave_scratch_bytes(long long systems, int n) {
    return sizeof(WaveCtl) + 2 * sizeof(unsigned long long) * (size_t)systems * (size_t)n;
}

template <bool LOWER, bool UNIT, int TR>
int launch_wave(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                long long a_stride, float *b_re, float *b_im, long long ldb, long long b_stride, WaveCtl *ctl,
                int phase, unsigned long long *mbox, const int *active, cudaStream_t st) {
    const int nblk = (n + 31) / 32;
    const int systems = nrhs * batch;
    const int spin = tuning(HBEM_TUNE_WAVE_SPIN) > 0 ? tuning(HBEM_TUNE_WAVE_SPIN) : kWaveSpinLimit;
    k_trsv_wave<LOWER, UNIT, TR><<<(unsigned)((long long)nblk * systems), kWaveThreads, 0, st>>>(
        n, nblk, nrhs, systems, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, ctl, phase, mbox, active,
        spin);
    HBEM_LAUNCH_CHECK("k_trsv_wave");
    return HBEM_OK;
}

// Both phases of a solve.  `scratch` (wave_scratch_bytes(nrhs * batch, n),
// 16-byte aligned) may be given by the caller; else it is taken from the
// stream's pool.  `active` (per matrix, optional) skips matrices.
int lu_solve_wave(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                  long long a_stride, const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb,
                  long long b_stride, int trans, const int *active, void *scratch, cudaStream_t st) {
    const long long systems = (long long)nrhs * batch;
    if ((long long)((n + 31) / 32) * systems >= (1LL << 31)) return fail(HBEM_ERR_ARG, "hbem_lu_solve: too many blocks");
    {
        int rc = func_opt_in((const void *)k_trsv_permute<false>, 200 * 1024);
        if (rc == HBEM_OK) rc = func_opt_in((const void *)k_trsv_permute<true>, 200 * 1024);
        if (rc != HBEM_OK) return rc;
    }
    const size_t bytes = wave_scratch_bytes(systems, n);
    void *mem = scratch;
    if (!mem) HBEM_CUDA(cudaMallocAsync(&mem, bytes, st));
    auto done = [&](int rc) {
        if (!scratch) cudaFreeAsync(mem, st);
        return rc;
    };
    WaveCtl *ctl = static_cast<WaveCtl *>(mem);
    unsigned long long *mb0 = reinterpret_cast<unsigned long long *>(ctl + 1), *mb1 = mb0 + systems * n;
    cudaError_t e = cudaMemsetAsync(ctl, 0, sizeof(WaveCtl), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(mb0, 0xff, bytes - sizeof(WaveCtl), st);
    if (e != cudaSuccess) return done(cuda_fail(e, "hbem_lu_solve: scratch"));
    const size_t psmem = (size_t)n * 2 * sizeof(float);
    int rc = HBEM_OK;
    if (trans == HBEM_TRANS_N) {
        if (piv) {
            k_trsv_permute<false><<<dim3(nrhs, batch), kTrsvThreads, psmem, st>>>(n, nrhs, piv, piv_stride, b_re, b_im,
                                                                                 ldb, b_stride, active);
            e = cudaGetLastError();
            if (e != cudaSuccess) return done(cuda_fail(e, "k_trsv_permute"));
            count_launch();
        }
        rc = launch_wave<true, true, 0>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, ctl,
                                        0, mb0, active, st);
        if (rc == HBEM_OK)
            rc = launch_wave<false, false, 0>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride,
                                              ctl, 1, mb1, active, st);
        return done(rc);
    }
    if (trans == HBEM_TRANS_T) {
        rc = launch_wave<true, false, 1>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, ctl,
                                         0, mb0, active, st);
        if (rc == HBEM_OK)
            rc = launch_wave<false, true, 1>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride,
                                             ctl, 1, mb1, active, st);
    } else {
        rc = launch_wave<true, false, 2>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride, ctl,
                                         0, mb0, active, st);
        if (rc == HBEM_OK)
            rc = launch_wave<false, true, 2>(n, nrhs, batch, lu_re, lu_im, lda, a_stride, b_re, b_im, ldb, b_stride,
                                             ctl, 1, mb1, active, st);
    }
    if (rc == HBEM_OK && piv) {
        k_trsv_permute<true><<<dim3(nrhs, batch), kTrsvThreads, psmem, st>>>(n, nrhs, piv, piv_stride, b_re, b_im, ldb,
                                                                            b_stride, active);
        e = cudaGetLastError();
        if (e != cudaSuccess) return done(cuda_fail(e, "k_trsv_permute"));
        count_launch();
    }
    return done(rc);
}

// ---------------------------------------------------------------------------
// 1-norm condition estimate of the factored matrices, as LAPACK cgecon with
// norm '1' (the reference's estimateReciprocalCondition, main.swift:463-503,
// 7898): Hager's method in Higham's formulation (LAPACK CLACN2) on L U
// without the interchanges, then rcond = (1 / est) / ||A||_1.
// Per-matrix state machine (st[f]):
//   0: solve (LU) w = x for the first time        -> est, x = sign(w), go 1
//   1: solve (LU)^H w = x                         -> j = argmax |w|; x = e_j, go 2
//                                                    (or the alternative vector, go 3)
//   2: solve (LU) w = e_j                         -> est; if not larger: go 3,
//                                                    else x = sign(w), go 1
//   3: solve (LU) w = alternative vector          -> est = max(est, 2 ||w||_1 / 3n), done (4)
// ---------------------------------------------------------------------------
struct RcState {
    double est, estold;
    int st, j, iter, pad;
};

// ||A||_1 = max_j sum_i |a_ij| (clange '1').  Block (32, 8): lanes over 32
// consecutive columns (coalesced rows), 8 row groups reduced in shared memory.
__global__ void __launch_bounds__(256) k_norm1(int n, const float *a_re, const float *a_im, long long lda,
                                               long long a_stride, unsigned *out_bits) {
    __shared__ double s_col[8][33];
    const int mat = blockIdx.y;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + tx;
    double sacc = 0.0;
    if (j < n) {
        const float *ar = a_re + (size_t)mat * a_stride + j, *ai = a_im + (size_t)mat * a_stride + j;
        float part = 0.f;
        int cnt = 0;
#pragma unroll 4
        for (int i = ty; i < n; i += 8) {
            const float re = ar[(size_t)i * lda], im = ai[(size_t)i * lda];
            part += sqrtf(fmaf(re, re, im * im));
            if (++cnt == 64) { sacc += part; part = 0.f; cnt = 0; }   // FP32 runs of 64, FP64 total
        }
        sacc += part;
    }
    s_col[ty][tx] = sacc;
    __syncthreads();
    if (ty == 0) {
        double t = 0.0;
#pragma unroll
        for (int g = 0; g < 8; ++g) t += s_col[g][tx];
        float v = (j < n) ? (float)t : 0.f;
        for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (tx == 0) atomicMax(out_bits + mat, __float_as_uint(v));
    }
}

__global__ void k_rc_init(int n, float *x_re, float *x_im, long long stride, RcState *state) {
    const int mat = blockIdx.y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x_re[(size_t)mat * stride + i] = 1.0f / (float)n;
        x_im[(size_t)mat * stride + i] = 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        RcState s0{};
        s0.st = 0;
        state[mat] = s0;
    }
}

// w = x for the matrices in `want` states (w is solved in place next);
// active[mat] marks them for the solve
__global__ void k_rc_copy(int n, const float *x_re, const float *x_im, float *w_re, float *w_im, long long stride,
                          const RcState *state, int want_lo, int want_hi, int *active) {
    const int mat = blockIdx.y;
    const int st = state[mat].st;
    const bool want = st >= want_lo && st <= want_hi;
    if (blockIdx.x == 0 && threadIdx.x == 0) active[mat] = want ? 1 : 0;
    if (!want) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        w_re[(size_t)mat * stride + i] = x_re[(size_t)mat * stride + i];
        w_im[(size_t)mat * stride + i] = x_im[(size_t)mat * stride + i];
    }
}

__device__ void block_sum_max(double &sum, float &mx, int &imx) {
    __shared__ double s_sum[32];
    __shared__ float s_mx[32];
    __shared__ int s_imx[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        const float om = __shfl_xor_sync(0xffffffffu, mx, o);
        const int oi = __shfl_xor_sync(0xffffffffu, imx, o);
        if (om > mx || (om == mx && oi < imx)) { mx = om; imx = oi; }
    }
    if (lane == 0) { s_sum[warp] = sum; s_mx[warp] = mx; s_imx[warp] = imx; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        float m = -1.f;
        int im = 0x7fffffff;
        for (int w = 0; w < nw; ++w) {
            t += s_sum[w];
            if (s_mx[w] > m || (s_mx[w] == m && s_imx[w] < im)) { m = s_mx[w]; im = s_imx[w]; }
        }
        s_sum[0] = t; s_mx[0] = m; s_imx[0] = im;
    }
    __syncthreads();
    sum = s_sum[0]; mx = s_mx[0]; imx = s_imx[0];
    __syncthreads();
}

// After a (LU) w solve (states 0, 2, 3): one CTA per matrix.
__global__ void k_rc_after_a(int n, float *x_re, float *x_im, const float *w_re, const float *w_im, long long stride,
                             RcState *state) {
    const int mat = blockIdx.x;
    RcState sv = state[mat];
    if (sv.st != 0 && sv.st != 2 && sv.st != 3) return;
    const float *wr = w_re + (size_t)mat * stride, *wi = w_im + (size_t)mat * stride;
    float *xr = x_re + (size_t)mat * stride, *xi = x_im + (size_t)mat * stride;
    double sum = 0.0;
    float mx = -1.f;
    int imx = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += blockDim.x) sum += hypot((double)wr[i], (double)wi[i]);
    block_sum_max(sum, mx, imx);
    const float safmin = 1.17549435e-38f;
    bool to_sign = false, to_alt = false;
    if (sv.st == 0) {
        sv.est = sum;
        if (n == 1) { sv.st = 4; }
        else { to_sign = true; sv.st = 1; }
    } else if (sv.st == 2) {
        sv.estold = sv.est;
        sv.est = sum;
        if (sv.est <= sv.estold) { to_alt = true; sv.st = 3; }   // LAPACK keeps the new estimate here
        else { to_sign = true; sv.st = 1; }
    } else {  // alternative estimate
        const double temp = 2.0 * sum / (3.0 * n);
        if (temp > sv.est) sv.est = temp;
        sv.st = 4;
    }
    if (to_sign) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float a = hypotf(wr[i], wi[i]);
            if (a > safmin) { xr[i] = wr[i] / a; xi[i] = wi[i] / a; }
            else { xr[i] = 1.f; xi[i] = 0.f; }
        }
    } else if (to_alt) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float sgn = (i & 1) ? -1.f : 1.f;
            xr[i] = sgn * (1.0f + (float)i / (float)(n - 1));
            xi[i] = 0.f;
        }
    }
    if (threadIdx.x == 0) state[mat] = sv;
}

// After a (LU)^H w solve (state 1): one CTA per matrix.
__global__ void k_rc_after_h(int n, float *x_re, float *x_im, const float *w_re, const float *w_im, long long stride,
                             RcState *state, int itmax) {
    const int mat = blockIdx.x;
    RcState sv = state[mat];
    if (sv.st != 1) return;
    const float *wr = w_re + (size_t)mat * stride, *wi = w_im + (size_t)mat * stride;
    float *xr = x_re + (size_t)mat * stride, *xi = x_im + (size_t)mat * stride;
    double sum = 0.0;
    float mx = -1.f;
    int imx = 0x7fffffff;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float a = hypotf(wr[i], wi[i]);
        if (a > mx || (a == mx && i < imx)) { mx = a; imx = i; }
    }
    block_sum_max(sum, mx, imx);
    if (imx < 0 || imx >= n) imx = 0;
    bool to_ej = false;
    if (sv.iter == 0) {
        // first pass (LAPACK ISAVE(1) = 2): j = argmax, iteration 2
        sv.j = imx;
        sv.iter = 2;
        to_ej = true;
    } else {
        // LAPACK ISAVE(1) = 4: continue while |w_jlast| != |w_j| and iter < itmax
        const int jlast = sv.j;
        sv.j = imx;
        const float a_last = hypotf(wr[jlast], wi[jlast]);
        if (a_last != mx && sv.iter < itmax) { sv.iter += 1; to_ej = true; }
    }
    if (to_ej) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) { xr[i] = (i == sv.j) ? 1.f : 0.f; xi[i] = 0.f; }
        sv.st = 2;
    } else {
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float sgn = (i & 1) ? -1.f : 1.f;
            xr[i] = sgn * (1.0f + (float)i / (float)(n - 1));
            xi[i] = 0.f;
        }
        sv.st = 3;
    }
    if (threadIdx.x == 0) state[mat] = sv;
}

__global__ void k_rc_finish(int batch, const RcState *state, const unsigned *anorm_bits, double *rcond, int *pending) {
    const int mat = blockIdx.x * blockDim.x + threadIdx.x;
    if (mat >= batch) return;
    const RcState sv = state[mat];
    if (sv.st != 4) atomicAdd(pending, 1);
    const double an = (double)__uint_as_float(anorm_bits[mat]);
    rcond[mat] = (sv.est != 0.0 && an != 0.0) ? (1.0 / sv.est) / an : 0.0;
}

// FP64 residual r = b - A x (one warp per row), and per-matrix norms;
// matrices whose `active` flag (optional) is 0 are skipped.
__global__ void __launch_bounds__(256) k_residual(int n, const float *a_re, const float *a_im, long long lda,
                                                  long long a_stride, const float *b_re, const float *b_im,
                                                  long long b_stride, const float *x_re, const float *x_im,
                                                  long long x_stride, float *r_re, float *r_im, double *norms,
                                                  const int *active = nullptr) {
    const int mat = blockIdx.y;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n || (active && !active[mat])) return;
    const float *Ar = a_re + (size_t)mat * a_stride + (size_t)warp * lda;
    const float *Ai = a_im + (size_t)mat * a_stride + (size_t)warp * lda;
    const float *xr = x_re + (size_t)mat * x_stride, *xi = x_im + (size_t)mat * x_stride;
    double sr = 0, si = 0;
    for (int c = lane; c < n; c += 32) {
        const double ar = Ar[c], ai = Ai[c], vr = xr[c], vi = xi[c];
        sr += ar * vr - ai * vi;
        si += ar * vi + ai * vr;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        const double rr = (double)b_re[(size_t)mat * b_stride + warp] - sr;
        const double ri = (double)b_im[(size_t)mat * b_stride + warp] - si;
        r_re[(size_t)mat * x_stride + warp] = (float)rr;
        r_im[(size_t)mat * x_stride + warp] = (float)ri;
        const double bb = (double)b_re[(size_t)mat * b_stride + warp] * b_re[(size_t)mat * b_stride + warp] +
                          (double)b_im[(size_t)mat * b_stride + warp] * b_im[(size_t)mat * b_stride + warp];
        atomicAdd(&norms[2 * mat], rr * rr + ri * ri);
        atomicAdd(&norms[2 * mat + 1], bb);
    }
}

// The stopping rule of refine() on the device, one thread per matrix, for the
// refinement without host synchronisation: pass `it` has just computed the
// residual norms of the matrices still active; a matrix stops at the
// tolerance, after max_iter passes, or once a pass no longer lowered its
// residual.  iters / resid (optional) receive the passes applied and the
// best relative residual.
__global__ void k_refine_decide(int batch, int it, int max_iter, double tol, const double *norms, double *best,
                                int *active, int *count, int *iters, double *resid) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= batch || (it > 0 && !active[m])) return;
    if (it == 0) count[m] = 0;
    const double rel = norms[2 * m + 1] > 0 ? sqrt(norms[2 * m] / norms[2 * m + 1]) : 0.0;
    const bool stalled = it > 0 && !(rel < best[m]);
    const double res = stalled ? best[m] : rel;
    best[m] = res;
    const int act = (!stalled && rel > tol && it < max_iter) ? 1 : 0;
    active[m] = act;
    count[m] += act;
    if (iters) iters[m] = count[m];
    if (resid) resid[m] = res;
}

__global__ void k_axpy_active(int n, float *x_re, float *x_im, long long x_stride, const float *d_re,
                              const float *d_im, const int *active) {
    const int mat = blockIdx.y;
    if (!active[mat]) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x_re[(size_t)mat * x_stride + i] += d_re[(size_t)mat * x_stride + i];
        x_im[(size_t)mat * x_stride + i] += d_im[(size_t)mat * x_stride + i];
    }
}

}  // namespace

template <int CS>
int launch_panel_cluster_t(float *a_re, float *a_im, long long lda, long long a_stride, int n, int c, int w, int *piv,
                           long long piv_stride, int *info, int batch, int R, size_t smem, cudaStream_t st) {
    {
        const int rc = func_opt_in((const void *)k_panel_cluster<CS>, 200 * 1024, CS > 8);
        if (rc != HBEM_OK) return rc;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS, batch);
    cfg.blockDim = dim3(kPanelRowsThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CS;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    HBEM_CUDA(cudaLaunchKernelEx(&cfg, k_panel_cluster<CS>, a_re, a_im, lda, a_stride, n, c, w, R, piv, piv_stride,
                                 info));
    HBEM_LAUNCH_CHECK("k_panel_cluster");
    return HBEM_OK;
}

// Largest cluster the panel kernel uses: 16 CTAs (a non-portable size) where
// the device co-schedules a 16-CTA cluster of full-size panel CTAs, else 8.
int panel_cluster_max(size_t smem_cap) {
    // per device (the query and the attributes are per device); a data race
    // on the cache only repeats the same query
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    if (const int c = cached[dev].load()) return c;
    int cmax = 8;
    if (func_opt_in((const void *)k_panel_cluster<16>, 200 * 1024, true) == HBEM_OK) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(16, 1);
        cfg.blockDim = dim3(kPanelRowsThreads);
        cfg.dynamicSmemBytes = smem_cap;
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = 16;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int clusters = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, k_panel_cluster<16>, &cfg) == cudaSuccess && clusters > 0)
            cmax = 16;
    }
    cudaGetLastError();   // a refused query leaves no sticky error
    cached[dev].store(cmax);
    return cmax;
}

int launch_panel_cluster(float *a_re, float *a_im, long long lda, long long a_stride, int n, int c, int w, int *piv,
                         long long piv_stride, int *info, int batch, size_t smem_cap, int cmax, cudaStream_t st) {
    const int m = n - c;
    const size_t row_bytes = (size_t)(w + 1) * 8;
    const int rows_cap = (int)(smem_cap / row_bytes);
    int cs = 2;
    while (cs < cmax && (long long)cs * rows_cap < m) cs *= 2;
    int R = (m + cs - 1) / cs;
    if (R < 64) R = 64;  // row j (< nb <= 64) always lives in CTA 0
    const size_t smem = (size_t)R * row_bytes;
    if (cs == 2) return launch_panel_cluster_t<2>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info, batch, R, smem, st);
    if (cs == 4) return launch_panel_cluster_t<4>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info, batch, R, smem, st);
    if (cs == 8) return launch_panel_cluster_t<8>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info, batch, R, smem, st);
    return launch_panel_cluster_t<16>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info, batch, R, smem, st);
}

// Look-ahead streams of one caller stream: the factorisation chain runs on a
// high-priority stream, the bulk of each trailing update on a low-priority
// one; both fork from and join back into the caller's stream (so a CUDA
// graph capture of the caller's stream takes them in).  Created on first use
// per (device, caller stream) and kept for the process.
struct LookaheadStreams {
    int device;
    cudaStream_t key, chain, bulk;
    cudaEvent_t fork, join_chain, join_bulk, split[2], bulk_done[2];
};

static std::mutex g_la_mu;
static std::vector<LookaheadStreams *> g_la;

static int lookahead_streams(cudaStream_t key, LookaheadStreams **out) {
    int dev = 0;
    HBEM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_la_mu);
    for (auto *l : g_la)
        if (l->device == dev && l->key == key) {
            *out = l;
            return HBEM_OK;
        }
    int least = 0, greatest = 0;
    HBEM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    auto *l = new LookaheadStreams{};
    l->device = dev;
    l->key = key;
    cudaError_t e = cudaStreamCreateWithPriority(&l->chain, cudaStreamNonBlocking, greatest);
    if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&l->bulk, cudaStreamNonBlocking, least);
    cudaEvent_t *evs[] = {&l->fork, &l->join_chain, &l->join_bulk, &l->split[0], &l->split[1], &l->bulk_done[0],
                          &l->bulk_done[1]};
    for (auto *ev : evs)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        delete l;   // handles created before the failure are left to the process
        return cuda_fail(e, "hbem_lu_factor: look-ahead streams");
    }
    g_la.push_back(l);
    *out = l;
    return HBEM_OK;
}

// The FP32 LU's look-ahead bulk update on the tensor cores (TF32x3): the
// built-in choice of HBEM_PREC_TF32X3, or HBEM_TUNE_LU_UPDATE = 2.  Measured
// on one B200: n = 1043 x 40 factors in 6.5 instead of 7.4 ms, 4096 x 4 in
// 28.2 instead of 29.6 ms and 18 749 x 2 in 701 instead of 1130 ms; but the
// split products keep 22 of FP32's 24 significand bits, and on a BEM matrix
// (the 1952-dof quarter horn) the unrefined solution is 5.5e-5 from LAPACK
// instead of the FP32 LU's < 1e-5.  So HBEM_PREC_PLAIN (cgesv) keeps the
// exact-FP32 CUDA-core update, and the TF32x3 bulk is for callers that refine
// with FP64 residuals, which recover the FP32 LU's solution accuracy.
static bool plain_update_on_tensor_cores(int precision) {
    const int v = tuning(HBEM_TUNE_LU_UPDATE);
    return v == 2 || (v == 0 && precision == HBEM_PREC_TF32X3);
}

int lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
              long long piv_stride, int *info, int precision, cudaStream_t st) {
    // Two-level blocking: 64-column blocks (128 for the mixed LU, so its
    // tensor-core update streams the trailing matrix once per 128 columns)
    // whose (n - b0) x NB panel is factored by inner sub-panels (64, 32 or 16
    // wide) with updates confined to the block's columns; then the row swaps,
    // the NB-row TRSM (in 64-row halves) and a K = NB trailing update per block.
    // Look-ahead: the trailing update of block b is cut into the next block's
    // 64 columns (on the chain, in FP32 on the CUDA cores, so block b+1's
    // panels can start) and the rest (on the bulk stream, on the tensor cores
    // in mixed precision, overlapping block b+1's panels, which touch only
    // block b+1's columns); block b+1's row swaps, which touch every other
    // column, wait for it.  The tensor-core workspace and status word are
    // only used on the bulk stream (and on the chain after it has joined).
    const size_t smem_cap = 200 * 1024;
    // 128-column blocks (one K = 128 update per block, half the C stream of
    // K = 64) pay for large matrices: 18 749 x 2 factors in 417 instead of
    // 498 ms, 18 749 x 8 in 1460 instead of 1867 ms.  Below that the K = 128
    // update, whose 128 KB resident A leaves its B ring one 32-column tile
    // deep, runs at 23 % of HBM where K = 64 reaches 57 % (n = 8192: 2.0 ms
    // per launch against 0.8 ms for half the K), so 8192 x 4 takes 112 vs
    // 85 ms and 10 000 x 2 98 vs 83 ms.
    const int blk_want = tuning(HBEM_TUNE_LU_BLOCK);
    const int NB = (precision == HBEM_PREC_MIXED && n > 256 && (blk_want == 128 || (blk_want == 0 && n > 16000)))
                       ? 128
                       : 64;
    HBEM_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, st));
    // K = 64 block updates on the tensor cores: BF16x3 (mixed precision), or
    // TF32x3 for the plain LU's look-ahead bulk when selected; their barrier
    // waits report through this status word
    int *status = nullptr;
    TcWorkspace *tc = nullptr;
    const bool tf32_bulk = precision != HBEM_PREC_MIXED && n > 2 * NB && tuning(HBEM_TUNE_LU_LOOKAHEAD) != 1 &&
                           plain_update_on_tensor_cores(precision);
    if ((precision == HBEM_PREC_MIXED && n > 64) || tf32_bulk) {
        HBEM_CUDA(cudaMallocAsync((void **)&status, sizeof(int), st));
        HBEM_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
        // TF32x3: below n = 12 000 each 64-column block as two K = 32 passes
        // in the 64 KB-A, 64-column-tile shape (the K = 64 shape's 128 KB A
        // leaves too short a B ring: 15 % tensor-pipe and 17 % HBM activity;
        // 1044 x 40 6.2 -> 6.0 ms, 2976 x 40 71 -> 62 ms, 4096 x 8 43 -> 36 ms,
        // 10 000 x 2 137 -> 116 ms); above, one K = 64 pass, whose single
        // read-modify-write of C wins at 18 749 x 2 (701 ms against 831 ms)
        const int tf32_kc = blk_want == 32 ? 32 : blk_want == 64 ? 64 : (n < 12000 ? 32 : 64);
        int rc = tc_workspace_create(n, batch, tf32_bulk, tf32_bulk ? tf32_kc : NB, &tc, st);
        if (rc != HBEM_OK) {
            cudaFreeAsync(status, st);
            return rc;
        }
    }
    LookaheadStreams *la = nullptr;
    if (n > 2 * NB && tuning(HBEM_TUNE_LU_LOOKAHEAD) != 1) {
        int rc = lookahead_streams(st, &la);
        if (rc != HBEM_OK) return rc;
        HBEM_CUDA(cudaEventRecord(la->fork, st));
        HBEM_CUDA(cudaStreamWaitEvent(la->chain, la->fork, 0));
        HBEM_CUDA(cudaStreamWaitEvent(la->bulk, la->fork, 0));
    }
    cudaStream_t cs = la ? la->chain : st;   // the factorisation chain
    bool bulk_pending = false;
    int parity = 0;
    auto finish = [&](int rc) -> int {
        if (la) {
            // join both streams back into the caller's stream, also on errors
            cudaEventRecord(la->join_chain, la->chain);
            cudaEventRecord(la->join_bulk, la->bulk);
            cudaStreamWaitEvent(st, la->join_chain, 0);
            cudaStreamWaitEvent(st, la->join_bulk, 0);
        }
        tc_workspace_destroy(tc, st);
        if (status) {
            // nothing waits for the host here (the caller's next launches
            // queue behind the factorisation, and a graph capture may be
            // running): a timed-out wait of the tensor-core update is folded
            // into the module fault word, which hbem_solve_status,
            // hbem_refine and hbem_solve_batch report
            k_fold_status<<<1, 1, 0, st>>>(status);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) count_launch();
            else if (rc == HBEM_OK) rc = cuda_fail(e, "k_fold_status");
            cudaFreeAsync(status, st);
        }
        return rc;
    };
    auto launched = [&](const char *what) -> int {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, what);
        count_launch();
        return HBEM_OK;
    };
    auto stream_call = [&](cudaError_t e, const char *what) -> int {
        return e == cudaSuccess ? HBEM_OK : cuda_fail(e, what);
    };
    HBEM_CUDA(cudaFuncSetAttribute(k_panel_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    HBEM_CUDA(cudaFuncSetAttribute(k_panel_reg<64, 1, 384>, cudaFuncAttributeMaxDynamicSharedMemorySize, 384 * 129 * 4));
    HBEM_CUDA(cudaFuncSetAttribute(k_panel_reg<32, 1, 768>, cudaFuncAttributeMaxDynamicSharedMemorySize, 768 * 65 * 4));
    HBEM_CUDA(cudaFuncSetAttribute(k_panel_reg<16, 1, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, 1024 * 33 * 4));
    // sub-panels held in registers, one row per thread (64 columns up to 384
    // rows, 32 up to 768, 16 up to 1024), when asked for; false: use the
    // shared-memory or cluster kernels.  Not the default: on one B200 the
    // n = 1043 x 40 factorisation takes 6.69 ms with them against 6.56 ms
    // (TF32x3 bulk; 7.50 against 7.47 ms with the CUDA-core bulk).  Either
    // kind costs about 2.4 us per column, which is the two CTA barriers and
    // the pivot-row exchange of every column, not the row traffic that the
    // registers remove.
    auto panel_in_registers = [&](int c, int w) -> bool {
        if (tuning(HBEM_TUNE_LU_PANEL_KERNEL) != 1) return false;
        const int m = n - c;
        const size_t ssm = (size_t)m * (2 * w + 1) * sizeof(float);
        if (w == 64 && m <= 384)
            k_panel_reg<64, 1, 384><<<batch, 384, ssm, cs>>>(a_re, a_im, lda, a_stride, n, c, piv, piv_stride, info);
        else if (w == 32 && m <= 768)
            k_panel_reg<32, 1, 768><<<batch, 768, ssm, cs>>>(a_re, a_im, lda, a_stride, n, c, piv, piv_stride, info);
        else if (w == 16 && m <= 1024)
            k_panel_reg<16, 1, 1024><<<batch, 1024, ssm, cs>>>(a_re, a_im, lda, a_stride, n, c, piv, piv_stride, info);
        else
            return false;
        return true;
    };
    HBEM_CUDA(cudaFuncSetAttribute(k_swap_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSwapSmem));
    const int cmax = panel_cluster_max(smem_cap);
    // Row swaps of block [b0, b0 + bw) on the columns [lo, hi) minus
    // [ex, ex + exw), and U12 = L11^-1 A12 on its columns [t_lo, t_hi) (all
    // >= b0 + bw).  A block wider than 64 goes in two 64-row halves: swaps and
    // TRSM of the first half, swaps of the second, the second half's rows of
    // [t_lo, t_hi) updated with the first half's U12 (CUDA cores), then the
    // TRSM of the second half alone.
    auto swap_trsm = [&](int b0, int bw, int lo, int hi, int ex, int exw, int t_lo, int t_hi,
                         cudaStream_t s) -> int {
        if (hi - lo - exw <= 0) return HBEM_OK;
        dim3 grid((hi - lo - exw + kSwapCols - 1) / kSwapCols, batch);
        k_swap_trsm<<<grid, kSwapThreads, kSwapSmem, s>>>(a_re, a_im, lda, a_stride, b0, std::min(bw, 64), lo, hi, ex,
                                                          exw, b0 + bw, piv, piv_stride);
        int rc = launched("k_swap_trsm");
        if (rc != HBEM_OK || bw <= 64) return rc;
        const int b1 = b0 + 64, h2 = bw - 64;
        k_swap_trsm<<<grid, kSwapThreads, kSwapSmem, s>>>(a_re, a_im, lda, a_stride, b1, h2, lo, hi, ex, exw, hi, piv,
                                                          piv_stride);
        rc = launched("k_swap_trsm");
        if (rc != HBEM_OK || t_hi <= t_lo) return rc;
        // rows [b1, b0 + bw) only: the row bound of the update is b0 + bw
        rc = launch_trailing_simt(b0 + bw, batch, b0, 64, b1, t_lo, t_hi, a_re, a_im, lda, a_stride, s);
        if (rc != HBEM_OK) return rc;
        dim3 g2((t_hi - t_lo + kSwapCols - 1) / kSwapCols, batch);
        k_swap_trsm<<<g2, kSwapThreads, kSwapSmem, s>>>(a_re, a_im, lda, a_stride, b1, h2, t_lo, t_hi, t_hi, 0, t_lo,
                                                        nullptr, piv_stride);
        return launched("k_swap_trsm");
    };
    for (int b0 = 0; b0 < n; b0 += NB) {
        const int bw = std::min(NB, n - b0);
        // the whole block as one panel while one CTA holds it; else inner width
        // 32 while one CTA holds the sub-panel, else 16 while one CTA holds
        // that, else 32 while an 8-CTA cluster holds it, else 16 (in a 16-CTA
        // cluster where an 8-CTA one is too small and the device has them)
        const size_t rows = (size_t)(n - b0);
        const int want = tuning(HBEM_TUNE_LU_PANEL);
        int nbi;
        if (want == 16) nbi = 16;
        else if (want == 32) nbi = rows <= 8 * (smem_cap / (33 * 8)) ? 32 : 16;
        else if (rows * 65 * 8 <= smem_cap || (want == 64 && rows <= 8 * (smem_cap / (65 * 8)))) nbi = 64;
        else if (rows * 33 * 8 <= smem_cap) nbi = 32;
        else if (rows * 17 * 8 <= smem_cap) nbi = 16;
        else nbi = rows <= 8 * (smem_cap / (33 * 8)) ? 32 : 16;
        for (int c = b0; c < b0 + bw; c += nbi) {
            const int w = std::min(nbi, b0 + bw - c);
            const size_t psmem = (size_t)(n - c) * (w + 1) * 8;
            int rc = HBEM_OK;
            if (panel_in_registers(c, w)) {
                rc = launched("k_panel_reg");
            } else if (psmem <= smem_cap) {
                k_panel_rows<<<batch, kPanelRowsThreads, psmem, cs>>>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride,
                                                                  info);
                rc = launched("k_panel_rows");
            } else if ((size_t)(n - c) <= (size_t)cmax * (smem_cap / ((size_t)(w + 1) * 8))) {
                rc = launch_panel_cluster(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info, batch, smem_cap,
                                          cmax, cs);
            } else {
                k_panel<<<batch, kPanelThreads, 0, cs>>>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info);
                rc = launched("k_panel");
            }
            if (rc != HBEM_OK) return finish(rc);
            const int other = bw - w;  // block columns outside this sub-panel
            if (other > 0) {
                dim3 grid((other + kSwapCols - 1) / kSwapCols, batch);
                k_swap_trsm<<<grid, kSwapThreads, kSwapSmem, cs>>>(a_re, a_im, lda, a_stride, c, w, b0, b0 + bw, c,
                                                                   w, c + w, piv, piv_stride);
                rc = launched("k_swap_trsm");
                if (rc != HBEM_OK) return finish(rc);
            }
            if (c + w < b0 + bw) {
                rc = launch_trailing_update(n, batch, c, w, c + w, b0 + bw, a_re, a_im, lda, a_stride, nullptr,
                                            nullptr, cs);
                if (rc != HBEM_OK) return finish(rc);
            }
        }
        if (bulk_pending) {
            // the row swaps below touch the columns of the previous bulk update
            int rc = stream_call(cudaStreamWaitEvent(cs, la->bulk_done[parity ^ 1], 0), "look-ahead join");
            if (rc != HBEM_OK) return finish(rc);
            bulk_pending = false;
        }
        const int outside = n - bw;
        const int next_end = std::min(n, b0 + bw + NB);
        // SMs the persistent tensor-core update leaves to the chain (by
        // default none: with the TF32x3 bulk in K = 32 passes, leaving 32 SMs
        // gave n = 1044 x 40 5.98 against 5.87 ms and 1542 x 40 16.4 against
        // 15.3 ms)
        const int tc_reserve = tuning(HBEM_TUNE_LU_RESERVE) > 0 ? tuning(HBEM_TUNE_LU_RESERVE) - 1 : 0;
        const bool split = la && next_end < n;
        if (outside > 0) {
            // with look-ahead the chain swaps (and solves) only the next block's
            // columns; the bulk stream swaps the rest before its update
            const int lo = split ? b0 + bw : 0, hi = split ? next_end : n;
            const int ex = split ? hi : b0, exw = split ? 0 : bw;
            int rc = swap_trsm(b0, bw, lo, hi, ex, exw, b0 + bw, hi, cs);
            if (rc != HBEM_OK) return finish(rc);
        }
        if (b0 + bw < n) {
            int rc;
            if (split) {
                rc = launch_trailing_simt(n, batch, b0, bw, b0 + bw, b0 + bw, next_end, a_re, a_im, lda, a_stride, cs);
                if (rc == HBEM_OK) rc = stream_call(cudaEventRecord(la->split[parity], cs), "look-ahead fork");
                if (rc == HBEM_OK)
                    rc = stream_call(cudaStreamWaitEvent(la->bulk, la->split[parity], 0), "look-ahead fork");
                if (rc == HBEM_OK)   // columns [0, b0) and [next_end, n): swaps, and the TRSM right of the block
                    rc = swap_trsm(b0, bw, 0, n, b0, next_end - b0, next_end, n, la->bulk);
                if (rc == HBEM_OK)
                    rc = tc ? launch_trailing_tc(tc, n, batch, b0, b0 + bw, next_end, n, a_re, a_im, lda, a_stride,
                                                 status, la->bulk, tc_reserve)
                            : launch_trailing_simt(n, batch, b0, bw, b0 + bw, next_end, n, a_re, a_im, lda, a_stride,
                                                   la->bulk);
                if (rc == HBEM_OK)
                    rc = stream_call(cudaEventRecord(la->bulk_done[parity], la->bulk), "look-ahead fork");
                if (rc != HBEM_OK) return finish(rc);
                bulk_pending = true;
                parity ^= 1;
            } else {
                rc = launch_trailing_update(n, batch, b0, bw, b0 + bw, n, a_re, a_im, lda, a_stride, tc, status, cs);
                if (rc != HBEM_OK) return finish(rc);
            }
        }
    }
    return finish(HBEM_OK);
}

int lu_solve_single(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                    long long a_stride, const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb,
                    long long b_stride, int trans, cudaStream_t st);

// piv == nullptr solves with L U itself (no interchanges).  `active` (per
// matrix, optional) lets the wavefront solve skip matrices; `wave_scratch`
// (wave_scratch_bytes(nrhs * batch, n), optional) is its control block and
// mailboxes.
int lu_solve_ex(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
                const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
                int trans, const int *active, void *wave_scratch, cudaStream_t st) {
    const size_t smem = (size_t)n * 2 * sizeof(float);
    if (smem > 200 * 1024) return fail(HBEM_ERR_ARG, "hbem_lu_solve: n too large for the staged solve");
    // one CTA per right-hand side for small n; the wavefront solve otherwise
    // (the blocked block steps remain selectable)
    const int solve_mode = tuning(HBEM_TUNE_LU_SOLVE);
    if (solve_mode == 1 || (solve_mode == 0 && n <= kTB))
        return lu_solve_single(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride,
                               trans, st);
    if (solve_mode == 2)
        return lu_solve_blocked(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride,
                                trans, st);
    return lu_solve_wave(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, trans,
                         active, wave_scratch, st);
}

int lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
             int trans, cudaStream_t st) {
    return lu_solve_ex(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, trans,
                       nullptr, nullptr, st);
}

// Reports (and clears) a timed-out wavefront wait; synchronises the stream.
int wave_fault_check(cudaStream_t st) {
    int h = 0;
    cudaError_t e = cudaMemcpyFromSymbolAsync(&h, g_wave_fault, sizeof(int), 0, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "triangular solve status");
    if (h == 0) return HBEM_OK;
    const int zero = 0;
    cudaMemcpyToSymbolAsync(g_wave_fault, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    return fail(HBEM_ERR_STATE, "a bounded device wait timed out: a triangular solve's wait for an earlier block (its "
                                "results are NaN) or a factorisation's tensor-core update");
}

int lu_solve_single(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                    long long a_stride, const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb,
                    long long b_stride, int trans, cudaStream_t st) {
    const size_t smem = (size_t)n * 2 * sizeof(float);
    {
        int rc = func_opt_in((const void *)k_getrs<0>, 200 * 1024);
        if (rc == HBEM_OK) rc = func_opt_in((const void *)k_getrs<1>, 200 * 1024);
        if (rc == HBEM_OK) rc = func_opt_in((const void *)k_getrs<2>, 200 * 1024);
        if (rc != HBEM_OK) return rc;
    }
    dim3 grid(nrhs, batch);
    const size_t tiles = (size_t)2 * (kGetrsThreads / 32) * 32 * 33 * sizeof(float);
    if (trans == HBEM_TRANS_N && smem + tiles <= 200 * 1024)
        k_getrs<0><<<grid, kGetrsThreads, smem + tiles, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re,
                                                             b_im, ldb, b_stride);
    else if (trans == HBEM_TRANS_N)
        return lu_solve_blocked(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride,
                                trans, st);
    else if (trans == HBEM_TRANS_T)
        k_getrs<1><<<grid, kGetrsThreads, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb,
                                                     b_stride);
    else
        k_getrs<2><<<grid, kGetrsThreads, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb,
                                                     b_stride);
    HBEM_LAUNCH_CHECK("k_getrs");
    return HBEM_OK;
}

int matrix_norm1(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                 float *anorm, cudaStream_t st) {
    unsigned *bits = reinterpret_cast<unsigned *>(anorm);
    HBEM_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned) * batch, st));
    k_norm1<<<dim3((n + 31) / 32, batch), 256, 0, st>>>(n, a_re, a_im, lda, a_stride, bits);
    HBEM_LAUNCH_CHECK("k_norm1");
    return HBEM_OK;
}

int lu_rcond(int n, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const float *anorm, double *rcond, cudaStream_t st) {
    constexpr int kItMax = 5;
    float *x = nullptr, *w = nullptr;
    RcState *state = nullptr;
    int *pending = nullptr, *active = nullptr;
    void *wave = nullptr;
    const long long stride = n;
    HBEM_CUDA(cudaMallocAsync((void **)&x, sizeof(float) * 2 * (size_t)batch * n, st));
    HBEM_CUDA(cudaMallocAsync((void **)&w, sizeof(float) * 2 * (size_t)batch * n, st));
    HBEM_CUDA(cudaMallocAsync((void **)&state, sizeof(RcState) * batch, st));
    HBEM_CUDA(cudaMallocAsync((void **)&pending, sizeof(int), st));
    HBEM_CUDA(cudaMallocAsync((void **)&active, sizeof(int) * batch, st));
    HBEM_CUDA(cudaMallocAsync(&wave, wave_scratch_bytes(batch, n), st));
    float *xr = x, *xi = x + (size_t)batch * n, *wr = w, *wi = w + (size_t)batch * n;
    const dim3 gv((n + 255) / 256 < 64 ? (n + 255) / 256 : 64, batch);
    int rc = HBEM_OK;
    auto launched = [&](const char *what) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, what); return false; }
        count_launch();
        return true;
    };
    // solves for the matrices k_rc_copy marked active
    auto solve = [&](int trans) {
        return lu_solve_ex(n, 1, batch, lu_re, lu_im, lda, a_stride, nullptr, n, wr, wi, 1, stride, trans, active, wave,
                           st);
    };
    k_rc_init<<<gv, 256, 0, st>>>(n, xr, xi, stride, state);
    // first estimator step: (LU) w = x for every matrix
    if (launched("k_rc_init")) {
        k_rc_copy<<<gv, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state, 0, 3, active);
        if (launched("k_rc_copy")) rc = solve(HBEM_TRANS_N);
        if (rc == HBEM_OK) { k_rc_after_a<<<batch, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state); launched("k_rc_after_a"); }
    }
    // A fixed number of rounds, with no host synchronisation: matrices that
    // finish drop out on the device (their solves and state updates are
    // skipped), so the estimate can run on its own stream beside the solves.
    // Five rounds finish every matrix (CLACN2's at most kItMax (LU)^H solves,
    // then the alternating-sign estimate); one spare.
    for (int round = 0; round < kItMax + 1 && rc == HBEM_OK; ++round) {
        // (LU)^H solves for matrices in state 1, then (LU) solves for states 2 and 3
        k_rc_copy<<<gv, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state, 1, 1, active);
        if (!launched("k_rc_copy")) break;
        rc = solve(HBEM_TRANS_C);
        if (rc != HBEM_OK) break;
        k_rc_after_h<<<batch, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state, kItMax);
        if (!launched("k_rc_after_h")) break;
        k_rc_copy<<<gv, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state, 2, 3, active);
        if (!launched("k_rc_copy")) break;
        rc = solve(HBEM_TRANS_N);
        if (rc != HBEM_OK) break;
        k_rc_after_a<<<batch, 256, 0, st>>>(n, xr, xi, wr, wi, stride, state);
        if (!launched("k_rc_after_a")) break;
        // stop once every matrix is done
        cudaError_t e = cudaMemsetAsync(pending, 0, sizeof(int), st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "rcond memset"); break; }
        k_rc_finish<<<(batch + 127) / 128, 128, 0, st>>>(batch, state, reinterpret_cast<const unsigned *>(anorm), rcond,
                                                         pending);
        if (!launched("k_rc_finish")) break;
    }
    cudaFreeAsync(x, st);
    cudaFreeAsync(w, st);
    cudaFreeAsync(state, st);
    cudaFreeAsync(pending, st);
    cudaFreeAsync(active, st);
    cudaFreeAsync(wave, st);
    return rc;
}

int refine(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
           const float *lu_re, const float *lu_im, long long lu_stride, const int *piv, long long piv_stride,
           const float *b_re, const float *b_im, long long b_stride, float *x_re, float *x_im, long long x_stride,
           double tol, int max_iter, int *iters, double *resid, cudaStream_t st) {
    // scratch: correction vectors (batch * x_stride * 2 floats) + norms + active flags
    float *d = nullptr;
    double *norms = nullptr;
    int *active = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&d, sizeof(float) * 2 * (size_t)batch * x_stride, st));
    HBEM_CUDA(cudaMallocAsync((void **)&norms, sizeof(double) * 2 * batch, st));
    HBEM_CUDA(cudaMallocAsync((void **)&active, sizeof(int) * batch, st));
    std::vector<double> h_norms(2 * batch);
    std::vector<int> h_active(batch, 1), h_iters(batch, 0);
    std::vector<double> h_res(batch, 0.0), h_best(batch, 0.0);
    int rc = HBEM_OK;
    float *dr = d, *di = d + (size_t)batch * x_stride;
    for (int it = 0; it <= max_iter && rc == HBEM_OK; ++it) {
        if (cudaMemsetAsync(norms, 0, sizeof(double) * 2 * batch, st) != cudaSuccess) { rc = cuda_fail(cudaGetLastError(), "memset"); break; }
        dim3 g((n * 32 + 255) / 256, batch);
        k_residual<<<g, 256, 0, st>>>(n, a_re, a_im, lda, a_stride, b_re, b_im, b_stride, x_re, x_im, x_stride, dr, di, norms,
                                      it > 0 ? active : nullptr);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_residual"); break; }
        count_launch();
        e = cudaMemcpyAsync(h_norms.data(), norms, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "refine sync"); break; }
        bool any = false;
        for (int m = 0; m < batch; ++m) {
            if (!h_active[m]) continue;
            const double rel = h_norms[2 * m + 1] > 0 ? std::sqrt(h_norms[2 * m] / h_norms[2 * m + 1]) : 0.0;
            // stop at the tolerance, after max_iter passes, or once a pass no
            // longer lowers the residual (the FP32 storage floor of x)
            const bool stalled = it > 0 && !(rel < h_best[m]);
            h_res[m] = stalled ? h_best[m] : rel;
            h_best[m] = h_res[m];
            h_active[m] = (!stalled && rel > tol && it < max_iter) ? 1 : 0;
            if (h_active[m]) { ++h_iters[m]; any = true; }
        }
        if (!any) break;
        e = cudaMemcpyAsync(active, h_active.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "refine copy"); break; }
        rc = lu_solve_ex(n, 1, batch, lu_re, lu_im, lda, lu_stride, piv, piv_stride, dr, di, 1, x_stride, HBEM_TRANS_N,
                         active, nullptr, st);
        if (rc != HBEM_OK) break;
        k_axpy_active<<<dim3((n + 255) / 256, batch), 256, 0, st>>>(n, x_re, x_im, x_stride, dr, di, active);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_axpy_active"); break; }
        count_launch();
    }
    if (rc == HBEM_OK && (iters || resid)) {
        cudaError_t e = cudaSuccess;
        if (iters) e = cudaMemcpyAsync(iters, h_iters.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && resid) e = cudaMemcpyAsync(resid, h_res.data(), sizeof(double) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(e, "refine results");
    }
    if (rc == HBEM_OK) rc = wave_fault_check(st);
    cudaFreeAsync(d, st);
    cudaFreeAsync(norms, st);
    cudaFreeAsync(active, st);
    return rc;
}

// refine() without host synchronisation: max_iter correction passes are
// always issued (a matrix that has stopped skips the residual, the solve's
// wavefront blocks and the update) and the stopping rule runs on the device,
// so the whole call can be captured in a CUDA graph.  A timed-out wavefront
// wait is left for hbem_solve_status.
int refine_async(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                 const float *lu_re, const float *lu_im, long long lu_stride, const int *piv, long long piv_stride,
                 const float *b_re, const float *b_im, long long b_stride, float *x_re, float *x_im,
                 long long x_stride, double tol, int max_iter, int *iters, double *resid, cudaStream_t st) {
    const size_t nd = 2 * (size_t)batch * x_stride;
    const size_t bytes = sizeof(double) * 3 * (size_t)batch + sizeof(float) * nd + sizeof(int) * 2 * (size_t)batch;
    unsigned char *mem = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&mem, bytes, st));
    double *norms = reinterpret_cast<double *>(mem), *best = norms + 2 * batch;
    float *dr = reinterpret_cast<float *>(best + batch), *di = dr + (size_t)batch * x_stride;
    int *active = reinterpret_cast<int *>(dr + nd), *count = active + batch;
    int rc = HBEM_OK;
    for (int it = 0; it <= max_iter && rc == HBEM_OK; ++it) {
        cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * 2 * batch, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "memset"); break; }
        k_residual<<<dim3((n * 32 + 255) / 256, batch), 256, 0, st>>>(n, a_re, a_im, lda, a_stride, b_re, b_im,
                                                                      b_stride, x_re, x_im, x_stride, dr, di, norms,
                                                                      it > 0 ? active : nullptr);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_residual"); break; }
        count_launch();
        k_refine_decide<<<(batch + 127) / 128, 128, 0, st>>>(batch, it, max_iter, tol, norms, best, active, count,
                                                              iters, resid);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_refine_decide"); break; }
        count_launch();
        if (it == max_iter) break;
        rc = lu_solve_ex(n, 1, batch, lu_re, lu_im, lda, lu_stride, piv, piv_stride, dr, di, 1, x_stride, HBEM_TRANS_N,
                         active, nullptr, st);
        if (rc != HBEM_OK) break;
        k_axpy_active<<<dim3((n + 255) / 256, batch), 256, 0, st>>>(n, x_re, x_im, x_stride, dr, di, active);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_axpy_active"); break; }
        count_launch();
    }
    cudaFreeAsync(mem, st);
    return rc;
}

// ---------------------------------------------------------------------------
// Refinement without allocation.  The scratch of hbem_refine (correction
// vectors, FP64 norm accumulators, active flags, the wavefront solve's
// control block and mailboxes) lives in one fixed
// module-scope device array instead of stream-ordered allocations, for
// callers that may not allocate device memory: a process whose memory is
// held by another caching allocator (a cudaMallocAsync from the default pool
// can then fail although the host framework has room cached), or a hot loop
// that must never enter an allocator.  Sizes: batch <= kNoAllocMaxBatch and
// batch * x_stride <= kNoAllocMaxElems complex elements (4 MiB of vectors,
// 8 MiB of mailboxes).
// Every call, on any stream or thread, shares this one array per device, so
// calls must not overlap; the array keeps the last call's contents, and the
// norms are cleared by each pass before they accumulate.
// ---------------------------------------------------------------------------
constexpr long long kNoAllocMaxElems = 1LL << 19;
constexpr int kNoAllocMaxBatch = 256;
constexpr size_t kNoAllocVecBytes = sizeof(float) * (size_t)kNoAllocMaxElems;  // one of re / im
constexpr size_t kNoAllocNormOff = 2 * kNoAllocVecBytes;
constexpr size_t kNoAllocActiveOff = kNoAllocNormOff + sizeof(double) * 2 * kNoAllocMaxBatch;
constexpr size_t kNoAllocWaveOff = kNoAllocActiveOff + sizeof(int) * kNoAllocMaxBatch;   // 16-byte aligned
constexpr size_t kNoAllocBytes = kNoAllocWaveOff + sizeof(WaveCtl) + 2 * sizeof(unsigned long long) * kNoAllocMaxElems;
static_assert(kNoAllocWaveOff % 16 == 0, "wave control block alignment");

static __device__ __align__(256) unsigned char g_refine_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
static std::mutex g_noalloc_mu;
static unsigned char *g_noalloc_ptr[kNoAllocMaxDevices];

// Device address of the scratch array on the current device.  The first call
// on a device looks the symbol up (which may load the module there).
static int noalloc_scratch(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "hbem_refine_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(HBEM_ERR_ARG, "hbem_refine_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_refine_scratch);
        if (e != cudaSuccess || !p) return cuda_fail(e, "hbem_refine_noalloc: cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return HBEM_OK;
}

int refine_noalloc(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                   const float *lu_re, const float *lu_im, long long lu_stride, const int *piv, long long piv_stride,
                   const float *b_re, const float *b_im, long long b_stride, float *x_re, float *x_im,
                   long long x_stride, double tol, int max_iter, int *iters, double *resid, cudaStream_t st) {
    if (batch > kNoAllocMaxBatch)
        return fail(HBEM_ERR_ARG, "hbem_refine_noalloc: batch exceeds the fixed scratch limit of 256 matrices");
    if ((long long)batch * x_stride > kNoAllocMaxElems)
        return fail(HBEM_ERR_ARG,
                    "hbem_refine_noalloc: batch * x_stride exceeds the fixed scratch limit of 524288 complex elements");
    unsigned char *base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc != HBEM_OK) return rc;
    float *dr = reinterpret_cast<float *>(base);
    float *di = reinterpret_cast<float *>(base + kNoAllocVecBytes);
    double *norms = reinterpret_cast<double *>(base + kNoAllocNormOff);
    int *active = reinterpret_cast<int *>(base + kNoAllocActiveOff);
    void *wave = base + kNoAllocWaveOff;
    double h_norms[2 * kNoAllocMaxBatch];
    int h_active[kNoAllocMaxBatch], h_iters[kNoAllocMaxBatch];
    double h_res[kNoAllocMaxBatch], h_best[kNoAllocMaxBatch];
    for (int m = 0; m < batch; ++m) {
        h_active[m] = 1;
        h_iters[m] = 0;
        h_res[m] = 0.0;
        h_best[m] = 0.0;
    }
    for (int it = 0; it <= max_iter && rc == HBEM_OK; ++it) {
        cudaError_t e = cudaMemsetAsync(norms, 0, sizeof(double) * 2 * batch, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "hbem_refine_noalloc: memset"); break; }
        dim3 g((n * 32 + 255) / 256, batch);
        k_residual<<<g, 256, 0, st>>>(n, a_re, a_im, lda, a_stride, b_re, b_im, b_stride, x_re, x_im, x_stride, dr, di, norms,
                                      it > 0 ? active : nullptr);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_residual"); break; }
        count_launch();
        e = cudaMemcpyAsync(h_norms, norms, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "hbem_refine_noalloc: sync"); break; }
        bool any = false;
        for (int m = 0; m < batch; ++m) {
            if (!h_active[m]) continue;
            const double rel = h_norms[2 * m + 1] > 0 ? std::sqrt(h_norms[2 * m] / h_norms[2 * m + 1]) : 0.0;
            const bool stalled = it > 0 && !(rel < h_best[m]);
            h_res[m] = stalled ? h_best[m] : rel;
            h_best[m] = h_res[m];
            h_active[m] = (!stalled && rel > tol && it < max_iter) ? 1 : 0;
            if (h_active[m]) { ++h_iters[m]; any = true; }
        }
        if (!any) break;
        e = cudaMemcpyAsync(active, h_active, sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "hbem_refine_noalloc: copy"); break; }
        rc = lu_solve_ex(n, 1, batch, lu_re, lu_im, lda, lu_stride, piv, piv_stride, dr, di, 1, x_stride, HBEM_TRANS_N,
                         active, wave, st);
        if (rc != HBEM_OK) break;
        k_axpy_active<<<dim3((n + 255) / 256, batch), 256, 0, st>>>(n, x_re, x_im, x_stride, dr, di, active);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_axpy_active"); break; }
        count_launch();
    }
    if (rc == HBEM_OK && (iters || resid)) {
        cudaError_t e = cudaSuccess;
        if (iters) e = cudaMemcpyAsync(iters, h_iters, sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && resid) e = cudaMemcpyAsync(resid, h_res, sizeof(double) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(e, "hbem_refine_noalloc: results");
    }
    if (rc == HBEM_OK) rc = wave_fault_check(st);
    return rc;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
                              long long piv_stride, int *info, int precision, void *stream) {
    keep_pool_memory();
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !piv || !info) return fail(HBEM_ERR_ARG, "hbem_lu_factor: NULL pointer");
    if (lda < n || a_stride < lda * (long long)n || piv_stride < n) return fail(HBEM_ERR_ARG, "hbem_lu_factor: bad strides");
    if (precision != HBEM_PREC_PLAIN && precision != HBEM_PREC_MIXED && precision != HBEM_PREC_TF32X3)
        return fail(HBEM_ERR_ARG, "hbem_lu_factor: precision must be HBEM_PREC_PLAIN, HBEM_PREC_TF32X3 or HBEM_PREC_MIXED");
    return lu_factor(n, batch, a_re, a_im, lda, a_stride, piv, piv_stride, info, precision,
                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                             long long a_stride, const int *piv, long long piv_stride, float *b_re, float *b_im,
                             long long ldb, long long b_stride, int trans, void *stream) {
    if (n <= 0 || batch <= 0 || nrhs <= 0) return HBEM_OK;
    if (!lu_re || !lu_im || !piv || !b_re || !b_im) return fail(HBEM_ERR_ARG, "hbem_lu_solve: NULL pointer");
    if (lda < n || ldb < nrhs || b_stride < ldb * (long long)n - (ldb - nrhs) || piv_stride < n)
        return fail(HBEM_ERR_ARG, "hbem_lu_solve: bad strides");
    if (trans < 0 || trans > 2) return fail(HBEM_ERR_ARG, "hbem_lu_solve: trans must be 0, 1 or 2");
    return lu_solve(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, trans,
                    reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_refine(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                           const float *lu_re, const float *lu_im, long long lu_stride, const int *piv,
                           long long piv_stride, const float *b_re, const float *b_im, long long b_stride,
                           float *x_re, float *x_im, long long x_stride, double tol, int max_iter, int *iters,
                           double *resid, void *stream) {
    keep_pool_memory();
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !lu_re || !lu_im || !piv || !b_re || !b_im || !x_re || !x_im)
        return fail(HBEM_ERR_ARG, "hbem_refine: NULL pointer");
    if (x_stride < n || b_stride < n || max_iter < 0 || !(tol > 0)) return fail(HBEM_ERR_ARG, "hbem_refine: bad arguments");
    if (lda < n || a_stride < lda * (long long)n || lu_stride < lda * (long long)n || piv_stride < n)
        return fail(HBEM_ERR_ARG, "hbem_refine: lda/a_stride/lu_stride/piv_stride too small");
    return refine(n, batch, a_re, a_im, lda, a_stride, lu_re, lu_im, lu_stride, piv, piv_stride, b_re, b_im, b_stride,
                  x_re, x_im, x_stride, tol, max_iter, iters, resid, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_refine_async(int n, int batch, const float *a_re, const float *a_im, long long lda,
                                 long long a_stride, const float *lu_re, const float *lu_im, long long lu_stride,
                                 const int *piv, long long piv_stride, const float *b_re, const float *b_im,
                                 long long b_stride, float *x_re, float *x_im, long long x_stride, double tol,
                                 int max_iter, int *iters, double *resid, void *stream) {
    keep_pool_memory();
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !lu_re || !lu_im || !piv || !b_re || !b_im || !x_re || !x_im)
        return fail(HBEM_ERR_ARG, "hbem_refine_async: NULL pointer");
    if (x_stride < n || b_stride < n || max_iter < 0 || !(tol > 0))
        return fail(HBEM_ERR_ARG, "hbem_refine_async: bad arguments");
    if (lda < n || a_stride < lda * (long long)n || lu_stride < lda * (long long)n || piv_stride < n)
        return fail(HBEM_ERR_ARG, "hbem_refine_async: lda/a_stride/lu_stride/piv_stride too small");
    return refine_async(n, batch, a_re, a_im, lda, a_stride, lu_re, lu_im, lu_stride, piv, piv_stride, b_re, b_im,
                        b_stride, x_re, x_im, x_stride, tol, max_iter, iters, resid,
                        reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_refine_noalloc(int n, int batch, const float *a_re, const float *a_im, long long lda,
                                   long long a_stride, const float *lu_re, const float *lu_im, long long lu_stride,
                                   const int *piv, long long piv_stride, const float *b_re, const float *b_im,
                                   long long b_stride, float *x_re, float *x_im, long long x_stride, double tol,
                                   int max_iter, int *iters, double *resid, void *stream) {
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !lu_re || !lu_im || !piv || !b_re || !b_im || !x_re || !x_im)
        return fail(HBEM_ERR_ARG, "hbem_refine_noalloc: NULL pointer");
    if (x_stride < n || b_stride < n || max_iter < 0 || !(tol > 0))
        return fail(HBEM_ERR_ARG, "hbem_refine_noalloc: bad arguments");
    if (lda < n || a_stride < lda * (long long)n || lu_stride < lda * (long long)n || piv_stride < n)
        return fail(HBEM_ERR_ARG, "hbem_refine_noalloc: lda/a_stride/lu_stride/piv_stride too small");
    return refine_noalloc(n, batch, a_re, a_im, lda, a_stride, lu_re, lu_im, lu_stride, piv, piv_stride, b_re, b_im,
                          b_stride, x_re, x_im, x_stride, tol, max_iter, iters, resid,
                          reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_matrix_norm1(int n, int batch, const float *a_re, const float *a_im, long long lda,
                                 long long a_stride, float *anorm, void *stream) {
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !anorm) return fail(HBEM_ERR_ARG, "hbem_matrix_norm1: NULL pointer");
    if (lda < n || a_stride < lda * (long long)n) return fail(HBEM_ERR_ARG, "hbem_matrix_norm1: bad strides");
    return matrix_norm1(n, batch, a_re, a_im, lda, a_stride, anorm, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_lu_rcond(int n, int batch, const float *lu_re, const float *lu_im, long long lda,
                             long long a_stride, const float *anorm, double *rcond, void *stream) {
    keep_pool_memory();
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!lu_re || !lu_im || !anorm || !rcond) return fail(HBEM_ERR_ARG, "hbem_lu_rcond: NULL pointer");
    if (lda < n || a_stride < lda * (long long)n) return fail(HBEM_ERR_ARG, "hbem_lu_rcond: bad strides");
    if ((size_t)n * 2 * sizeof(float) > 200 * 1024) return fail(HBEM_ERR_ARG, "hbem_lu_rcond: n too large");
    return lu_rcond(n, batch, lu_re, lu_im, lda, a_stride, anorm, rcond, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_solve_status(void *stream) {
    return wave_fault_check(reinterpret_cast<cudaStream_t>(stream));
}
