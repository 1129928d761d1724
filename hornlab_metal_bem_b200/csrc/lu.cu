// Batched complex LU with partial pivoting and triangular solves on sm_100a,
// replacing LAPACK cgesv/cgetrf/cgetrs (reference main.swift:7834-7941,
// 8015-8020).  Matrices are planar (re, im) float32, row-major.
//
// Two-level right-looking blocked factorisation, batched over matrices:
//   for each 64-column block b0:
//     for each inner sub-panel c (32 or 16 columns):
//       k_panel      : factor rows c..n of the sub-panel with partial pivoting
//                      (pivot = first max |re|+|im|, as LAPACK's icamax),
//                      staged in shared memory when it fits, else in L2;
//       k_swap_trsm  : swap + forward-solve the other columns of the block;
//       trailing     : update the block's remaining columns (K = 16/32);
//     k_swap_trsm    : the block's 64 swaps on all other columns and the
//                      64-row TRSM U12 = L11^-1 A12;
//     trailing       : A22 -= L21 U12 with K = 64.
// The solve applies the pivots then runs blocked forward / backward
// substitution (op(A) = A, A^T or A^H).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "hbem_internal.h"

namespace hbem {

// A[start:n, start:col_end] -= A[start:n, k0:k0+kw] * A[k0:k0+kw, start:col_end]
int launch_trailing_update(int n, int batch, int k0, int kw, int start, int col_end, float *a_re, float *a_im,
                           long long lda, long long a_stride, int precision, cudaStream_t st);

namespace {

constexpr int kPanelThreads = 512;

__device__ __forceinline__ float cabs1(float r, float i) { return fabsf(r) + fabsf(i); }

// Block-wide argmax of (value, index), ties to the smallest index.
__device__ void block_argmax(float &v, int &idx, float *s_v, int *s_i) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
    }
    if (lane == 0) { s_v[warp] = v; s_i[warp] = idx; }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        v = lane < nw ? s_v[lane] : -1.f;
        idx = lane < nw ? s_i[lane] : 0x7fffffff;
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, v, o);
            const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
            if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
        }
        if (lane == 0) { s_v[0] = v; s_i[0] = idx; }
    }
    __syncthreads();
    v = s_v[0];
    idx = s_i[0];
    __syncthreads();
}

// Panel factorisation.  SMEM: panel rows k0..n-1 x nb columns staged in
// shared memory (planar), written back at the end.
template <bool SMEM>
__global__ void __launch_bounds__(kPanelThreads) k_panel(float *a_re, float *a_im, long long lda, long long a_stride,
                                                         int n, int k0, int nb, int *piv, long long piv_stride,
                                                         int *info) {
    extern __shared__ float s_panel[];
    __shared__ float s_v[32];
    __shared__ int s_i[32];
    __shared__ float s_prow[2][64];
    const int b = blockIdx.x;
    float *are = a_re + (size_t)b * a_stride, *aim = a_im + (size_t)b * a_stride;
    int *pv = piv + (size_t)b * piv_stride;
    const int m = n - k0;  // panel rows
    float *pre = s_panel, *pim = s_panel + (size_t)m * nb;
    // element (row r in [0,m), col j in [0,nb)) of the panel
    auto RE = [&](int r, int j) -> float & { return SMEM ? pre[(size_t)r * nb + j] : are[(size_t)(k0 + r) * lda + k0 + j]; };
    auto IM = [&](int r, int j) -> float & { return SMEM ? pim[(size_t)r * nb + j] : aim[(size_t)(k0 + r) * lda + k0 + j]; };
    if (SMEM) {
        for (int e = threadIdx.x; e < m * nb; e += blockDim.x) {
            const int r = e / nb, j = e - r * nb;
            pre[e] = are[(size_t)(k0 + r) * lda + k0 + j];
            pim[e] = aim[(size_t)(k0 + r) * lda + k0 + j];
        }
        __syncthreads();
    }
    int first_zero = 0;
    for (int j = 0; j < nb; ++j) {
        float v = -1.f;
        int idx = 0x7fffffff;
        for (int r = j + threadIdx.x; r < m; r += blockDim.x) {
            const float c = cabs1(RE(r, j), IM(r, j));
            if (c > v) { v = c; idx = r; }
        }
        block_argmax(v, idx, s_v, s_i);
        const int p = idx;
        if (threadIdx.x == 0) pv[k0 + j] = k0 + p;
        if (p != j) {
            for (int c = threadIdx.x; c < nb; c += blockDim.x) {
                const float tr = RE(j, c), ti = IM(j, c);
                RE(j, c) = RE(p, c);
                IM(j, c) = IM(p, c);
                RE(p, c) = tr;
                IM(p, c) = ti;
            }
        }
        __syncthreads();
        const float dr = RE(j, j), di = IM(j, j);
        const bool zero = (dr == 0.f && di == 0.f);
        if (zero && first_zero == 0) first_zero = k0 + j + 1;
        for (int c = threadIdx.x; c < nb; c += blockDim.x) {
            s_prow[0][c] = RE(j, c);
            s_prow[1][c] = IM(j, c);
        }
        __syncthreads();
        if (!zero) {
            // 1 / pivot
            const float den = 1.0f / (dr * dr + di * di);
            const float ir = dr * den, ii = -di * den;
            // scale column j below the diagonal and update the panel's trailing columns
            const int cols = nb - j - 1;
            const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
            for (int r = j + 1 + warp; r < m; r += nw) {
                const float xr = RE(r, j), xi = IM(r, j);
                const float lr = xr * ir - xi * ii, li = xr * ii + xi * ir;
                for (int c = lane; c < cols; c += 32) {
                    const int cc = j + 1 + c;
                    const float ur = s_prow[0][cc], ui = s_prow[1][cc];
                    RE(r, cc) -= lr * ur - li * ui;
                    IM(r, cc) -= lr * ui + li * ur;
                }
                __syncwarp();
                if (lane == 0) {
                    RE(r, j) = lr;
                    IM(r, j) = li;
                }
            }
        }
        __syncthreads();
    }
    if (SMEM) {
        for (int e = threadIdx.x; e < m * nb; e += blockDim.x) {
            const int r = e / nb, j = e - r * nb;
            are[(size_t)(k0 + r) * lda + k0 + j] = pre[e];
            aim[(size_t)(k0 + r) * lda + k0 + j] = pim[e];
        }
    }
    if (threadIdx.x == 0 && first_zero && info[b] == 0) info[b] = first_zero;
}

// Row swaps + forward substitution for a column range.  One thread per
// column of [col_lo, col_hi) minus the panel [ex_lo, ex_lo + np): apply the
// pivots of rows k0 .. k0+np-1 in order; columns >= trsm_lo then solve
// L11 x = a with the unit-lower L11 = A[k0:k0+np, k0:k0+np] (np <= 64), in
// 16-row register chunks whose updates of the remaining rows go through L2.
__global__ void __launch_bounds__(128) k_swap_trsm(float *a_re, float *a_im, long long lda, long long a_stride,
                                                   int k0, int np, int col_lo, int col_hi, int ex_lo,
                                                   int trsm_lo, const int *piv, long long piv_stride) {
    __shared__ float Lr[64][65], Li[64][65];
    __shared__ int s_piv[64];
    const int b = blockIdx.y;
    float *are = a_re + (size_t)b * a_stride, *aim = a_im + (size_t)b * a_stride;
    const int *pv = piv + (size_t)b * piv_stride;
    const bool any_trsm = trsm_lo < col_hi;
    if (any_trsm)
        for (int e = threadIdx.x; e < np * np; e += blockDim.x) {
            const int r = e / np, c = e - r * np;
            Lr[r][c] = are[(size_t)(k0 + r) * lda + k0 + c];
            Li[r][c] = aim[(size_t)(k0 + r) * lda + k0 + c];
        }
    for (int e = threadIdx.x; e < np; e += blockDim.x) s_piv[e] = pv[k0 + e];
    __syncthreads();
    int col = col_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ex_lo) col += np;
    if (col >= col_hi) return;
    for (int j = 0; j < np; ++j) {
        const int p = s_piv[j];
        if (p != k0 + j) {
            const size_t o1 = (size_t)(k0 + j) * lda + col, o2 = (size_t)p * lda + col;
            const float tr = are[o1], ti = aim[o1];
            are[o1] = are[o2];
            aim[o1] = aim[o2];
            are[o2] = tr;
            aim[o2] = ti;
        }
    }
    if (col < trsm_lo) return;
    for (int q0 = 0; q0 < np; q0 += 16) {
        const int qn = min(16, np - q0);
        float xr[16], xi[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i < qn) {
                xr[i] = are[(size_t)(k0 + q0 + i) * lda + col];
                xi[i] = aim[(size_t)(k0 + q0 + i) * lda + col];
            }
#pragma unroll
        for (int i = 1; i < 16; ++i)
            if (i < qn) {
                float sr = xr[i], si = xi[i];
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (j < i) {
                        sr -= Lr[q0 + i][q0 + j] * xr[j] - Li[q0 + i][q0 + j] * xi[j];
                        si -= Lr[q0 + i][q0 + j] * xi[j] + Li[q0 + i][q0 + j] * xr[j];
                    }
                xr[i] = sr;
                xi[i] = si;
            }
#pragma unroll
        for (int i = 0; i < 16; ++i)
            if (i < qn) {
                are[(size_t)(k0 + q0 + i) * lda + col] = xr[i];
                aim[(size_t)(k0 + q0 + i) * lda + col] = xi[i];
            }
        // rows below this chunk inside L11's range
        for (int r = q0 + qn; r < np; ++r) {
            float sr = are[(size_t)(k0 + r) * lda + col], si = aim[(size_t)(k0 + r) * lda + col];
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (j < qn) {
                    sr -= Lr[r][q0 + j] * xr[j] - Li[r][q0 + j] * xi[j];
                    si -= Lr[r][q0 + j] * xi[j] + Li[r][q0 + j] * xr[j];
                }
            are[(size_t)(k0 + r) * lda + col] = sr;
            aim[(size_t)(k0 + r) * lda + col] = si;
        }
    }
}

// ---------------------------------------------------------------------------
// Triangular solves.  One CTA per (matrix, right-hand side); x staged in
// shared memory; 32-row diagonal blocks solved by warp 0, off-diagonal
// updates by all warps with coalesced row reads.
// TRANS: 0 = A, 1 = A^T, 2 = A^H.
// ---------------------------------------------------------------------------
template <int TRANS>
__global__ void __launch_bounds__(512) k_getrs(int n, const float *lu_re, const float *lu_im, long long lda,
                                               long long a_stride, const int *piv, long long piv_stride, float *b_re,
                                               float *b_im, long long ldb, long long b_stride, int nrhs) {
    extern __shared__ float s_x[];
    float *xr = s_x, *xi = s_x + n;
    const int mat = blockIdx.y, rhs = blockIdx.x;
    const float *Ar = lu_re + (size_t)mat * a_stride, *Ai = lu_im + (size_t)mat * a_stride;
    const int *pv = piv + (size_t)mat * piv_stride;
    float *br = b_re + (size_t)mat * b_stride, *bi = b_im + (size_t)mat * b_stride;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    const float cs = TRANS == 2 ? -1.f : 1.f;  // conjugation sign on the imaginary part
    for (int i = tid; i < n; i += blockDim.x) {
        xr[i] = br[(size_t)i * ldb + rhs];
        xi[i] = bi[(size_t)i * ldb + rhs];
    }
    __syncthreads();
    // element accessors of op(L) / op(U)
    auto Lr_ = [&](int r, int c) { return TRANS ? Ar[(size_t)c * lda + r] : Ar[(size_t)r * lda + c]; };
    auto Li_ = [&](int r, int c) { return TRANS ? cs * Ai[(size_t)c * lda + r] : Ai[(size_t)r * lda + c]; };
    if (TRANS == 0) {
        if (tid == 0)
            for (int i = 0; i < n; ++i) {
                const int p = pv[i];
                if (p != i) {
                    float t = xr[i]; xr[i] = xr[p]; xr[p] = t;
                    t = xi[i]; xi[i] = xi[p]; xi[p] = t;
                }
            }
        __syncthreads();
        // forward: L unit lower (rows i, cols < i)
        for (int j0 = 0; j0 < n; j0 += 32) {
            const int jb = min(32, n - j0);
            if (warp == 0) {
                for (int i = 1; i < jb; ++i) {
                    float pr = 0, pi = 0;
                    if (lane < i) {
                        const float lr = Ar[(size_t)(j0 + i) * lda + j0 + lane], li = Ai[(size_t)(j0 + i) * lda + j0 + lane];
                        pr = lr * xr[j0 + lane] - li * xi[j0 + lane];
                        pi = lr * xi[j0 + lane] + li * xr[j0 + lane];
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        pr += __shfl_xor_sync(0xffffffffu, pr, o);
                        pi += __shfl_xor_sync(0xffffffffu, pi, o);
                    }
                    if (lane == 0) { xr[j0 + i] -= pr; xi[j0 + i] -= pi; }
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int i = j0 + jb + warp; i < n; i += nw) {
                float pr = 0, pi = 0;
                if (lane < jb) {
                    const float lr = Ar[(size_t)i * lda + j0 + lane], li = Ai[(size_t)i * lda + j0 + lane];
                    pr = lr * xr[j0 + lane] - li * xi[j0 + lane];
                    pi = lr * xi[j0 + lane] + li * xr[j0 + lane];
                }
                for (int o = 16; o > 0; o >>= 1) {
                    pr += __shfl_xor_sync(0xffffffffu, pr, o);
                    pi += __shfl_xor_sync(0xffffffffu, pi, o);
                }
                if (lane == 0) { xr[i] -= pr; xi[i] -= pi; }
            }
            __syncthreads();
        }
        // backward: U upper (non-unit)
        for (int j1 = n; j1 > 0; j1 -= 32) {
            const int j0 = max(0, j1 - 32), jb = j1 - j0;
            if (warp == 0) {
                for (int i = jb - 1; i >= 0; --i) {
                    float pr = 0, pi = 0;
                    if (lane > i && lane < jb) {
                        const float ur = Ar[(size_t)(j0 + i) * lda + j0 + lane], ui = Ai[(size_t)(j0 + i) * lda + j0 + lane];
                        pr = ur * xr[j0 + lane] - ui * xi[j0 + lane];
                        pi = ur * xi[j0 + lane] + ui * xr[j0 + lane];
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        pr += __shfl_xor_sync(0xffffffffu, pr, o);
                        pi += __shfl_xor_sync(0xffffffffu, pi, o);
                    }
                    if (lane == 0) {
                        const float dr = Ar[(size_t)(j0 + i) * lda + j0 + i], di = Ai[(size_t)(j0 + i) * lda + j0 + i];
                        const float yr = xr[j0 + i] - pr, yi = xi[j0 + i] - pi;
                        const float den = 1.0f / (dr * dr + di * di);
                        xr[j0 + i] = (yr * dr + yi * di) * den;
                        xi[j0 + i] = (yi * dr - yr * di) * den;
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int i = warp; i < j0; i += nw) {
                float pr = 0, pi = 0;
                if (lane < jb) {
                    const float ur = Ar[(size_t)i * lda + j0 + lane], ui = Ai[(size_t)i * lda + j0 + lane];
                    pr = ur * xr[j0 + lane] - ui * xi[j0 + lane];
                    pi = ur * xi[j0 + lane] + ui * xr[j0 + lane];
                }
                for (int o = 16; o > 0; o >>= 1) {
                    pr += __shfl_xor_sync(0xffffffffu, pr, o);
                    pi += __shfl_xor_sync(0xffffffffu, pi, o);
                }
                if (lane == 0) { xr[i] -= pr; xi[i] -= pi; }
            }
            __syncthreads();
        }
    } else {
        // op(A) = U^op L^op P ; solve U^op z = b (forward, U^op lower, non-unit),
        // then L^op w = z (backward, unit upper), then x = P^T w.
        for (int j0 = 0; j0 < n; j0 += 32) {
            const int jb = min(32, n - j0);
            if (warp == 0) {
                for (int i = 0; i < jb; ++i) {
                    float pr = 0, pi = 0;
                    if (lane < i) {
                        // (U^op)[r][c] = op(U[c][r]), r = j0+i, c = j0+lane
                        const float ur = Ar[(size_t)(j0 + lane) * lda + j0 + i];
                        const float ui = cs * Ai[(size_t)(j0 + lane) * lda + j0 + i];
                        pr = ur * xr[j0 + lane] - ui * xi[j0 + lane];
                        pi = ur * xi[j0 + lane] + ui * xr[j0 + lane];
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        pr += __shfl_xor_sync(0xffffffffu, pr, o);
                        pi += __shfl_xor_sync(0xffffffffu, pi, o);
                    }
                    if (lane == 0) {
                        const float dr = Ar[(size_t)(j0 + i) * lda + j0 + i], di = cs * Ai[(size_t)(j0 + i) * lda + j0 + i];
                        const float yr = xr[j0 + i] - pr, yi = xi[j0 + i] - pi;
                        const float den = 1.0f / (dr * dr + di * di);
                        xr[j0 + i] = (yr * dr + yi * di) * den;
                        xi[j0 + i] = (yi * dr - yr * di) * den;
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            // rows i >= j0+jb: x_i -= sum_{c in block} op(U[c][i]) x_c.  Column i of
            // U^op is row i of U: read U[c][i] with lanes over i for coalescing.
            for (int i0 = j0 + jb; i0 < n; i0 += blockDim.x) {
                const int i = i0 + tid;
                if (i < n) {
                    float pr = 0, pi = 0;
                    for (int c = 0; c < jb; ++c) {
                        const float ur = Ar[(size_t)(j0 + c) * lda + i], ui = cs * Ai[(size_t)(j0 + c) * lda + i];
                        pr += ur * xr[j0 + c] - ui * xi[j0 + c];
                        pi += ur * xi[j0 + c] + ui * xr[j0 + c];
                    }
                    xr[i] -= pr;
                    xi[i] -= pi;
                }
            }
            __syncthreads();
        }
        for (int j1 = n; j1 > 0; j1 -= 32) {
            const int j0 = max(0, j1 - 32), jb = j1 - j0;
            if (warp == 0) {
                for (int i = jb - 1; i >= 0; --i) {
                    float pr = 0, pi = 0;
                    if (lane > i && lane < jb) {
                        // (L^op)[r][c] = op(L[c][r]), r = j0+i, c = j0+lane > r
                        const float lr = Lr_(j0 + i, j0 + lane), li = Li_(j0 + i, j0 + lane);
                        pr = lr * xr[j0 + lane] - li * xi[j0 + lane];
                        pi = lr * xi[j0 + lane] + li * xr[j0 + lane];
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        pr += __shfl_xor_sync(0xffffffffu, pr, o);
                        pi += __shfl_xor_sync(0xffffffffu, pi, o);
                    }
                    if (lane == 0) { xr[j0 + i] -= pr; xi[j0 + i] -= pi; }
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int i0 = 0; i0 < j0; i0 += blockDim.x) {
                const int i = i0 + tid;
                if (i < j0) {
                    float pr = 0, pi = 0;
                    for (int c = 0; c < jb; ++c) {
                        const float lr = Ar[(size_t)(j0 + c) * lda + i], li = cs * Ai[(size_t)(j0 + c) * lda + i];
                        pr += lr * xr[j0 + c] - li * xi[j0 + c];
                        pi += lr * xi[j0 + c] + li * xr[j0 + c];
                    }
                    xr[i] -= pr;
                    xi[i] -= pi;
                }
            }
            __syncthreads();
        }
        if (tid == 0)
            for (int i = n - 1; i >= 0; --i) {
                const int p = pv[i];
                if (p != i) {
                    float t = xr[i]; xr[i] = xr[p]; xr[p] = t;
                    t = xi[i]; xi[i] = xi[p]; xi[p] = t;
                }
            }
        __syncthreads();
    }
    for (int i = tid; i < n; i += blockDim.x) {
        br[(size_t)i * ldb + rhs] = xr[i];
        bi[(size_t)i * ldb + rhs] = xi[i];
    }
}

// FP64 residual r = b - A x (one warp per row), and per-matrix norms.
__global__ void __launch_bounds__(256) k_residual(int n, const float *a_re, const float *a_im, long long lda,
                                                  long long a_stride, const float *b_re, const float *b_im,
                                                  long long b_stride, const float *x_re, const float *x_im,
                                                  long long x_stride, float *r_re, float *r_im, double *norms) {
    const int mat = blockIdx.y;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
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

int lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
              long long piv_stride, int *info, int precision, cudaStream_t st) {
    // Two-level blocking: 64-column blocks whose (n - b0) x 64 panel is
    // factored by inner sub-panels (32 wide when the sub-panel fits shared
    // memory, else 16) with updates confined to the block's columns; then one
    // row-swap pass, a 64-row TRSM and a K = 64 trailing update per block.
    const size_t smem_cap = 200 * 1024;
    constexpr int NB = 64;
    HBEM_CUDA(cudaMemsetAsync(info, 0, sizeof(int) * batch, st));
    HBEM_CUDA(cudaFuncSetAttribute(k_panel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    for (int b0 = 0; b0 < n; b0 += NB) {
        const int bw = std::min(NB, n - b0);
        const int nbi = ((size_t)(n - b0) * 32 * 8 <= smem_cap) ? 32 : 16;
        for (int c = b0; c < b0 + bw; c += nbi) {
            const int w = std::min(nbi, b0 + bw - c);
            const size_t psmem = (size_t)(n - c) * w * 8;
            if (psmem <= smem_cap)
                k_panel<true><<<batch, kPanelThreads, psmem, st>>>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info);
            else
                k_panel<false><<<batch, kPanelThreads, 0, st>>>(a_re, a_im, lda, a_stride, n, c, w, piv, piv_stride, info);
            HBEM_LAUNCH_CHECK("k_panel");
            const int other = bw - w;  // block columns outside this sub-panel
            if (other > 0) {
                dim3 grid((other + 127) / 128, batch);
                k_swap_trsm<<<grid, 128, 0, st>>>(a_re, a_im, lda, a_stride, c, w, b0, b0 + bw, c, c + w, piv, piv_stride);
                HBEM_LAUNCH_CHECK("k_swap_trsm");
            }
            if (c + w < b0 + bw) {
                int rc = launch_trailing_update(n, batch, c, w, c + w, b0 + bw, a_re, a_im, lda, a_stride, precision, st);
                if (rc != HBEM_OK) return rc;
            }
        }
        const int outside = n - bw;
        if (outside > 0) {
            dim3 grid((outside + 127) / 128, batch);
            k_swap_trsm<<<grid, 128, 0, st>>>(a_re, a_im, lda, a_stride, b0, bw, 0, n, b0, b0 + bw, piv, piv_stride);
            HBEM_LAUNCH_CHECK("k_swap_trsm");
        }
        if (b0 + bw < n) {
            int rc = launch_trailing_update(n, batch, b0, bw, b0 + bw, n, a_re, a_im, lda, a_stride, precision, st);
            if (rc != HBEM_OK) return rc;
        }
    }
    return HBEM_OK;
}

int lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
             int trans, cudaStream_t st) {
    const size_t smem = (size_t)n * 2 * sizeof(float);
    if (smem > 200 * 1024) return fail(HBEM_ERR_ARG, "hbem_lu_solve: n too large for the staged solve");
    dim3 grid(nrhs, batch);
    if (trans == HBEM_TRANS_N) {
        HBEM_CUDA(cudaFuncSetAttribute(k_getrs<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_getrs<0><<<grid, 512, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, nrhs);
    } else if (trans == HBEM_TRANS_T) {
        HBEM_CUDA(cudaFuncSetAttribute(k_getrs<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_getrs<1><<<grid, 512, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, nrhs);
    } else {
        HBEM_CUDA(cudaFuncSetAttribute(k_getrs<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_getrs<2><<<grid, 512, smem, st>>>(n, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride, nrhs);
    }
    HBEM_LAUNCH_CHECK("k_getrs");
    return HBEM_OK;
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
    std::vector<double> h_res(batch, 0.0);
    int rc = HBEM_OK;
    float *dr = d, *di = d + (size_t)batch * x_stride;
    for (int it = 0; it <= max_iter && rc == HBEM_OK; ++it) {
        if (cudaMemsetAsync(norms, 0, sizeof(double) * 2 * batch, st) != cudaSuccess) { rc = cuda_fail(cudaGetLastError(), "memset"); break; }
        dim3 g((n * 32 + 255) / 256, batch);
        k_residual<<<g, 256, 0, st>>>(n, a_re, a_im, lda, a_stride, b_re, b_im, b_stride, x_re, x_im, x_stride, dr, di, norms);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_residual"); break; }
        count_launch();
        e = cudaMemcpyAsync(h_norms.data(), norms, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "refine sync"); break; }
        bool any = false;
        for (int m = 0; m < batch; ++m) {
            const double rel = h_norms[2 * m + 1] > 0 ? std::sqrt(h_norms[2 * m] / h_norms[2 * m + 1]) : 0.0;
            h_res[m] = rel;
            h_active[m] = (h_active[m] && rel > tol && it < max_iter) ? 1 : 0;
            if (h_active[m]) { ++h_iters[m]; any = true; }
        }
        if (!any) break;
        e = cudaMemcpyAsync(active, h_active.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) { rc = cuda_fail(e, "refine copy"); break; }
        rc = lu_solve(n, 1, batch, lu_re, lu_im, lda, lu_stride, piv, piv_stride, dr, di, 1, x_stride, HBEM_TRANS_N, st);
        if (rc != HBEM_OK) break;
        k_axpy_active<<<dim3((n + 255) / 256, batch), 256, 0, st>>>(n, x_re, x_im, x_stride, dr, di, active);
        e = cudaGetLastError();
        if (e != cudaSuccess) { rc = cuda_fail(e, "k_axpy_active"); break; }
        count_launch();
    }
    if (rc == HBEM_OK && iters) {
        cudaError_t e = cudaMemcpyAsync(iters, h_iters.data(), sizeof(int) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && resid) e = cudaMemcpyAsync(resid, h_res.data(), sizeof(double) * batch, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = cuda_fail(e, "refine results");
    }
    cudaFreeAsync(d, st);
    cudaFreeAsync(norms, st);
    cudaFreeAsync(active, st);
    return rc;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
                              long long piv_stride, int *info, int precision, void *stream) {
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !piv || !info) return fail(HBEM_ERR_ARG, "hbem_lu_factor: NULL pointer");
    if (lda < n || a_stride < lda * (long long)n || piv_stride < n) return fail(HBEM_ERR_ARG, "hbem_lu_factor: bad strides");
    if (precision != HBEM_PREC_PLAIN && precision != HBEM_PREC_MIXED)
        return fail(HBEM_ERR_ARG, "hbem_lu_factor: precision must be HBEM_PREC_PLAIN or HBEM_PREC_MIXED");
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
    if (n <= 0 || batch <= 0) return HBEM_OK;
    if (!a_re || !a_im || !lu_re || !lu_im || !piv || !b_re || !b_im || !x_re || !x_im)
        return fail(HBEM_ERR_ARG, "hbem_refine: NULL pointer");
    if (x_stride < n || b_stride < n || max_iter < 0 || !(tol > 0)) return fail(HBEM_ERR_ARG, "hbem_refine: bad arguments");
    return refine(n, batch, a_re, a_im, lda, a_stride, lu_re, lu_im, lu_stride, piv, piv_stride, b_re, b_im, b_stride,
                  x_re, x_im, x_stride, tol, max_iter, iters, resid, reinterpret_cast<cudaStream_t>(stream));
}
