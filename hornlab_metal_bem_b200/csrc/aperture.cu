// Coupled infinite baffle: interior BIE on the cavity surface coupled to the
// Rayleigh half-space through the aperture faces at z = 0.
//
// Reference (main.swift): aperture geometry 915-964, S_ia / S_aa projections
// 1178-1290 (+ Duffy 1011-1087), Schur solve 7597-7789, Rayleigh field
// 1397-1444.  The reference forms T = (2 S_aa)^-1 P_avg and A - S_ia T
// (an n x n x m product).  Here P_avg is applied as a sparse scatter instead:
// X = S_ia (2 S_aa)^-1 (n x m x m), then A[:, d] -= X[:, r] / 3 for the three
// dofs d of every aperture face r -- the same matrix with n/m times fewer
// flops.  For large apertures (m comparable to n, where forming (2 S_aa)^-1
// costs more than the solve) the reference's augmented twin
// (main.swift:7504-7595) is used instead: one (m + n) system
//   [[-2 S_aa, P_avg], [-S_ia, A]] [q_a; p] = [0; b]
// built by k_ib_augment and factored by the batched LU.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "hbem_internal.h"

namespace hbem {
int lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
              long long piv_stride, int *info, int precision, cudaStream_t st);
int lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
             int trans, cudaStream_t st);

namespace {

__device__ __forceinline__ float aqx(int q) {
    return q == 0 ? HBEM_QX0 : q == 1 ? HBEM_QX1 : q == 2 ? HBEM_QX2 : q == 3 ? HBEM_QX3 : q == 4 ? HBEM_QX4 : HBEM_QX5;
}
__device__ __forceinline__ float aqy(int q) {
    return q == 0 ? HBEM_QY0 : q == 1 ? HBEM_QY1 : q == 2 ? HBEM_QY2 : q == 3 ? HBEM_QY3 : q == 4 ? HBEM_QY4 : HBEM_QY5;
}
__device__ __forceinline__ float aqw(int q) { return (q == 0 || q == 2 || q == 3) ? HBEM_QWA : HBEM_QWB; }

// G / (1/(4 pi)) for one sample, complex k
__device__ __forceinline__ void green(float dx, float dy, float dz, float k, float kt, float ki, float &gr, float &gi) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float u = rsqrtf(r2);
    u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    float t = r * kt;
    t -= rintf(t);
    float s, c;
    sincospif(2.0f * t, &s, &c);
    if (ki != 0.f) u *= __expf(-ki * r);
    gr = u * c;
    gi = u * s;
}

struct ApArgs {
    const float4 *qp;   // (T, 6) original order
    const float4 *nrm;  // (T) normal + 2 area
    const int *l2g;
    const int *ap;      // (m) aperture triangles
    const float *areas;
    float *out_re, *out_im;
    long long stride;
    int T, m, sym;
    float rw;
    float k[64], kt[64], ki[64];
};

__device__ __forceinline__ void image_sum(int sym, float4 y, float4 x, float k, float kt, float ki, float &gr, float &gi) {
    float r, i;
    green(y.x - x.x, y.y - x.y, y.z - x.z, k, kt, ki, r, i);
    gr += r; gi += i;
    if (sym == 1 || sym == 3) { green(-y.x - x.x, y.y - x.y, y.z - x.z, k, kt, ki, r, i); gr += r; gi += i; }
    if (sym == 2 || sym == 3) { green(y.x - x.x, -y.y - x.y, y.z - x.z, k, kt, ki, r, i); gr += r; gi += i; }
    if (sym == 3) { green(-y.x - x.x, -y.y - x.y, y.z - x.z, k, kt, ki, r, i); gr += r; gi += i; }
    if (sym == 4) { green(y.x - x.x, y.y - x.y, -y.z - x.z, k, kt, ki, r, i); gr += r; gi += i; }
}

// S_ia regular part: one thread per (test triangle, aperture triangle).
// The coincident self-point is the r^2 <= 1e-14 sample (identical points).
__global__ void __launch_bounds__(128) k_ap_slp(const __grid_constant__ ApArgs a) {
    const int test = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = blockIdx.y, f = blockIdx.z;
    if (test >= a.T) return;
    const int trial = a.ap[t];
    const float k = a.k[f], kt = a.kt[f], ki = a.ki[f];
    float sr[3] = {0, 0, 0}, si[3] = {0, 0, 0};
    for (int qa = 0; qa < 6; ++qa) {
        const float4 x = a.qp[(size_t)test * 6 + qa];
        float hr = 0, hi = 0;
#pragma unroll
        for (int qb = 0; qb < 6; ++qb) {
            const float4 y = a.qp[(size_t)trial * 6 + qb];
            float gr = 0, gi = 0;
            image_sum(a.sym, y, x, k, kt, ki, gr, gi);
            hr = fmaf(gr, aqw(qb), hr);
            hi = fmaf(gi, aqw(qb), hi);
        }
        const float b[3] = {1.f - aqx(qa) - aqy(qa), aqx(qa), aqy(qa)};
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            sr[i] = fmaf(aqw(qa) * b[i], hr, sr[i]);
            si[i] = fmaf(aqw(qa) * b[i], hi, si[i]);
        }
    }
    const float scale = HBEM_INV4PI * a.nrm[test].w * a.nrm[trial].w * a.rw;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const size_t o = (size_t)f * a.stride + (size_t)a.l2g[test * 3 + i] * a.m + t;
        atomicAdd(a.out_re + o, sr[i] * scale);
        atomicAdd(a.out_im + o, si[i] * scale);
    }
}

// S_aa regular part: one thread per (test, trial) aperture pair.
__global__ void __launch_bounds__(128) k_ap_avg(const __grid_constant__ ApArgs a) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y, f = blockIdx.z;
    if (c >= a.m) return;
    const int test = a.ap[r], trial = a.ap[c];
    const float k = a.k[f], kt = a.kt[f];
    float sr = 0, si = 0;
    for (int qa = 0; qa < 6; ++qa) {
        const float4 x = a.qp[(size_t)test * 6 + qa];
        float hr = 0, hi = 0;
#pragma unroll
        for (int qb = 0; qb < 6; ++qb) {
            const float4 y = a.qp[(size_t)trial * 6 + qb];
            float gr = 0, gi = 0;
            image_sum(a.sym, y, x, k, kt, 0.f, gr, gi);
            hr = fmaf(gr, aqw(qb), hr);
            hi = fmaf(gi, aqw(qb), hi);
        }
        // sum over the three test basis functions is 1
        sr = fmaf(aqw(qa), hr, sr);
        si = fmaf(aqw(qa), hi, si);
    }
    const float scale = HBEM_INV4PI * a.nrm[test].w * a.nrm[trial].w / fmaxf(a.areas[test], 1e-38f);
    const size_t o = (size_t)f * a.stride + (size_t)r * a.m + c;
    a.out_re[o] += sr * scale;
    a.out_im[o] += si * scale;
}

__global__ void k_scale_identity(float *saa_re, float *saa_im, float *id_re, float *id_im, int m, long long stride) {
    const int f = blockIdx.y;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < m * m; e += gridDim.x * blockDim.x) {
        saa_re[(size_t)f * stride + e] *= 2.f;
        saa_im[(size_t)f * stride + e] *= 2.f;
        const int r = e / m, c = e - r * m;
        id_re[(size_t)f * stride + e] = r == c ? 1.f : 0.f;
        id_im[(size_t)f * stride + e] = 0.f;
    }
}

// C (M x N) = A (M x K) * B (K x N), complex planar, row-major, batched.
__global__ void __launch_bounds__(256) k_cgemm(const float *a_re, const float *a_im, long long lda, long long sa,
                                               const float *b_re, const float *b_im, long long ldb, long long sb,
                                               float *c_re, float *c_im, long long ldc, long long sc, int M, int N,
                                               int K) {
    constexpr int KC = 16;
    __shared__ __align__(16) float Lr[KC][64], Li[KC][64];
    __shared__ __align__(16) float Ur[KC][64], Ui[KC][64];
    const int mat = blockIdx.z;
    const float *A_r = a_re + (size_t)mat * sa, *A_i = a_im + (size_t)mat * sa;
    const float *B_r = b_re + (size_t)mat * sb, *B_i = b_im + (size_t)mat * sb;
    const int row0 = blockIdx.y * 64, col0 = blockIdx.x * 64;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    float cr[4][4] = {}, ci[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += KC) {
        for (int e = tid; e < 64 * KC; e += 256) {
            const int r = e / KC, kk = e - r * KC;
            const bool ok = row0 + r < M && k0 + kk < K;
            Lr[kk][r] = ok ? A_r[(size_t)(row0 + r) * lda + k0 + kk] : 0.f;
            Li[kk][r] = ok ? A_i[(size_t)(row0 + r) * lda + k0 + kk] : 0.f;
        }
        for (int e = tid; e < 64 * KC; e += 256) {
            const int kk = e / 64, c = e - kk * 64;
            const bool ok = col0 + c < N && k0 + kk < K;
            Ur[kk][c] = ok ? B_r[(size_t)(k0 + kk) * ldb + col0 + c] : 0.f;
            Ui[kk][c] = ok ? B_i[(size_t)(k0 + kk) * ldb + col0 + c] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            float ar[4], ai[4], br[4], bi[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ar[i] = Lr[kk][ty * 4 + i]; ai[i] = Li[kk][ty * 4 + i];
                br[i] = Ur[kk][tx * 4 + i]; bi[i] = Ui[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    cr[i][j] = fmaf(ar[i], br[j], fmaf(-ai[i], bi[j], cr[i][j]));
                    ci[i][j] = fmaf(ar[i], bi[j], fmaf(ai[i], br[j], ci[i][j]));
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = row0 + ty * 4 + i;
        if (r >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = col0 + tx * 4 + j;
            if (c >= N) continue;
            c_re[(size_t)mat * sc + (size_t)r * ldc + c] = cr[i][j];
            c_im[(size_t)mat * sc + (size_t)r * ldc + c] = ci[i][j];
        }
    }
}

// A[i][d] -= X[i][r] / 3 for the dofs d of aperture face r.
__global__ void k_ib_scatter(float *a_re, float *a_im, long long a_stride, const float *x_re, const float *x_im,
                             long long x_stride, const int *ap, const int *l2g, int n, int m) {
    const int f = blockIdx.z, r = blockIdx.y;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float vr = x_re[(size_t)f * x_stride + (size_t)i * m + r] * (1.0f / 3.0f);
    const float vi = x_im[(size_t)f * x_stride + (size_t)i * m + r] * (1.0f / 3.0f);
    const int t = ap[r];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const size_t o = (size_t)f * a_stride + (size_t)i * n + l2g[t * 3 + l];
        atomicAdd(a_re + o, -vr);
        atomicAdd(a_im + o, -vi);
    }
}

// Per-frequency max |re|, |im| of the three blocks that set the scaling of the
// augmented system: mx[3 f + 0] = A block of K, + 1 = S_ia, + 2 = S_aa
// (non-negative floats order like their bit patterns, so atomicMax on the
// bits is exact).
__global__ void k_ib_block_max(const float *k_re, const float *k_im, long long ldk, long long k_stride,
                               const float *sia_re, const float *sia_im, const float *saa_re, const float *saa_im,
                               int n, int m, unsigned *mx) {
    const int f = blockIdx.z, which = blockIdx.y;
    float v = 0.f;
    if (which == 0) {
        const long long tot = (long long)n * n;
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
            const long long r = e / n, c = e - r * n;
            const size_t o = (size_t)f * k_stride + (size_t)(m + r) * ldk + (m + c);
            v = fmaxf(v, fmaxf(fabsf(k_re[o]), fabsf(k_im[o])));
        }
    } else {
        const long long tot = which == 1 ? (long long)n * m : (long long)m * m;
        const float *xr = which == 1 ? sia_re + (size_t)f * tot : saa_re + (size_t)f * tot;
        const float *xi = which == 1 ? sia_im + (size_t)f * tot : saa_im + (size_t)f * tot;
        for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x)
            v = fmaxf(v, fmaxf(fabsf(xr[e]), fabsf(xi[e])));
    }
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(mx + 3 * f + which, __float_as_uint(v));
}

// Block scaling of the augmented system: q_a = alpha q~ (columns < m times
// alpha) and the aperture rows times beta, with alpha = max|A| / max|S_ia|,
// beta = max|A| / (alpha max|2 S_aa|): the unscaled system mixes entries
// ~1e-4 (S_aa), 1/3 (P_avg), ~1e-6 (A) and ~1e-8 (S_ia), which inflates its
// condition number by orders of magnitude over the Schur complement's.
__device__ __forceinline__ void ib_scales(const unsigned *mx, int f, float &alpha, float &beta) {
    const float a = __uint_as_float(mx[3 * f]), sia = __uint_as_float(mx[3 * f + 1]), saa = __uint_as_float(mx[3 * f + 2]);
    alpha = (a > 0.f && sia > 0.f) ? a / sia : 1.f;
    beta = (a > 0.f && saa > 0.f) ? a / (2.f * alpha * saa) : 1.f;
}

// Augmented coupled matrix K (N = m + n, row-major, ldk): rows r < m are
// beta [-2 alpha S_aa[r, :] | P_avg[r, :]] (P_avg: 1/3 on the three dofs of
// aperture face r), rows m + i take -alpha S_ia[i, :] in columns < m; the A
// block (columns >= m) is assembled in place by hbem_assemble.
__global__ void k_ib_augment(const float *sia_re, const float *sia_im, const float *saa_re, const float *saa_im,
                             float *k_re, float *k_im, long long ldk, long long k_stride, const int *ap,
                             const int *l2g, int n, int m, const unsigned *mx, float *alpha_out) {
    const int f = blockIdx.z, row = blockIdx.y;
    const long long N = (long long)n + m;
    float alpha, beta;
    ib_scales(mx, f, alpha, beta);
    if (row == 0 && blockIdx.x == 0 && threadIdx.x == 0) alpha_out[f] = alpha;
    float *kr = k_re + (size_t)f * k_stride + (size_t)row * ldk, *ki = k_im + (size_t)f * k_stride + (size_t)row * ldk;
    if (row < m) {
        const float *sr = saa_re + (size_t)f * m * m + (size_t)row * m, *si = saa_im + (size_t)f * m * m + (size_t)row * m;
        const int t = ap[row];
        const int d0 = l2g[3 * t], d1 = l2g[3 * t + 1], d2 = l2g[3 * t + 2];
        const float s_aa = -2.f * alpha * beta, s_p = beta * (1.0f / 3.0f);
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < N; c += (long long)gridDim.x * blockDim.x) {
            float vr, vi = 0.f;
            if (c < m) {
                vr = s_aa * sr[c];
                vi = s_aa * si[c];
            } else {
                const int d = (int)(c - m);
                vr = (d == d0 || d == d1 || d == d2) ? s_p : 0.f;
            }
            kr[c] = vr;
            ki[c] = vi;
        }
    } else {
        const int i = row - m;
        const float *sr = sia_re + (size_t)f * n * m + (size_t)i * m, *si = sia_im + (size_t)f * n * m + (size_t)i * m;
        for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < m; c += gridDim.x * blockDim.x) {
            kr[c] = -alpha * sr[c];
            ki[c] = -alpha * si[c];
        }
    }
}

// q_a = M (P_avg p): one warp per aperture row
__global__ void k_ib_qa(const float *p_re, const float *p_im, int n, const float *m_re, const float *m_im, int m,
                        const int *ap, const int *l2g, float *qa_re, float *qa_im) {
    const int f = blockIdx.y;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= m) return;
    const float *pr = p_re + (size_t)f * n, *pi = p_im + (size_t)f * n;
    double sr = 0, si = 0;
    for (int c = lane; c < m; c += 32) {
        const int t = ap[c];
        const int d0 = l2g[3 * t], d1 = l2g[3 * t + 1], d2 = l2g[3 * t + 2];
        const float ar = (pr[d0] + pr[d1] + pr[d2]) * (1.0f / 3.0f), ai = (pi[d0] + pi[d1] + pi[d2]) * (1.0f / 3.0f);
        const float mr = m_re[(size_t)f * m * m + (size_t)r * m + c], mi = m_im[(size_t)f * m * m + (size_t)r * m + c];
        sr += (double)mr * ar - (double)mi * ai;
        si += (double)mr * ai + (double)mi * ar;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
    }
    if (lane == 0) {
        qa_re[(size_t)f * m + r] = (float)sr;
        qa_im[(size_t)f * m + r] = (float)si;
    }
}

// Rayleigh field: one CTA per (frequency, observation point), threads over
// aperture quadrature points.
__global__ void __launch_bounds__(256) k_rayleigh(const __grid_constant__ ApArgs a, const float *qa_re,
                                                  const float *qa_im, const float *obs, int n_obs, float *out_re,
                                                  float *out_im) {
    const int o = blockIdx.x, f = blockIdx.y;
    const float ox = obs[o], oy = obs[n_obs + o], oz = obs[2 * n_obs + o];
    float *dr = out_re + (size_t)f * n_obs + o, *di = out_im + (size_t)f * n_obs + o;
    if (oz < -1.0e-5f) {
        if (threadIdx.x == 0) { *dr = 0.f; *di = 0.f; }
        return;
    }
    const float ez = oz < 0.f ? 0.f : oz;
    const float4 x = make_float4(ox, oy, ez, 0.f);
    const float k = a.k[f], kt = a.kt[f];
    float ar = 0, ai = 0;
    for (int e = threadIdx.x; e < a.m * 6; e += blockDim.x) {
        const int t = e / 6, q = e - 6 * t;
        const int tri = a.ap[t];
        const float qr = qa_re[(size_t)f * a.m + t], qi = qa_im[(size_t)f * a.m + t];
        const float4 y = a.qp[(size_t)tri * 6 + q];
        float gr = 0, gi = 0;
        image_sum(a.sym == 4 ? 0 : a.sym, y, x, k, kt, 0.f, gr, gi);
        const float w = aqw(q) * a.nrm[tri].w;
        ar += (gr * qr - gi * qi) * w;
        ai += (gr * qi + gi * qr) * w;
    }
    __shared__ float s[2][32];
    for (int off = 16; off > 0; off >>= 1) {
        ar += __shfl_xor_sync(0xffffffffu, ar, off);
        ai += __shfl_xor_sync(0xffffffffu, ai, off);
    }
    if ((threadIdx.x & 31) == 0) { s[0][threadIdx.x >> 5] = ar; s[1][threadIdx.x >> 5] = ai; }
    __syncthreads();
    if (threadIdx.x == 0) {
        float tr = 0, ti = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tr += s[0][w]; ti += s[1][w]; }
        *dr = -2.0f * HBEM_INV4PI * tr;
        *di = -2.0f * HBEM_INV4PI * ti;
    }
}

void fill_ap_args(ApArgs &a, const Session &s, const float *k_re, const float *k_im, int f0, int nf) {
    a.qp = s.d_fqp; a.nrm = s.d_fnrm; a.l2g = s.d_l2g; a.ap = s.d_ap_tris; a.areas = s.d_areas;
    a.T = s.n_triangles; a.m = s.m_ap; a.sym = s.sym;
    a.rw = (float)(1 << ((s.sym & 1) + ((s.sym >> 1) & 1) + ((s.sym >> 2) & 1)));
    for (int f = 0; f < nf; ++f) {
        a.k[f] = k_re[f0 + f];
        a.kt[f] = (float)((double)k_re[f0 + f] / (2.0 * 3.14159265358979323846));
        a.ki[f] = k_im ? k_im[f0 + f] : 0.f;
    }
}

}  // namespace
}  // namespace hbem

using namespace hbem;

extern "C" int hbem_session_set_aperture(hbem_session *h, int aperture_tag) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_session_set_aperture: NULL session");
    if (aperture_tag <= 0) return fail(HBEM_ERR_ARG, "aperture_tag must be positive");
    if (s->sym == 4) return fail(HBEM_ERR_ARG, "coupled infinite baffle does not compose with the xy symmetry plane");
    std::vector<int> ap, loc(s->n_triangles, -1);
    for (int t = 0; t < s->n_triangles; ++t)
        if (s->tags[t] == aperture_tag) {
            loc[t] = (int)ap.size();
            ap.push_back(t);
        }
    if (ap.empty()) return fail(HBEM_ERR_ARG, "aperture_tag " + std::to_string(aperture_tag) + " selects no triangles");
    HBEM_CUDA(cudaSetDevice(s->device));
    if (s->d_ap_tris) cudaFree(s->d_ap_tris);
    if (s->d_ap_local) cudaFree(s->d_ap_local);
    s->d_ap_tris = s->d_ap_local = nullptr;
    HBEM_CUDA(cudaMalloc((void **)&s->d_ap_tris, sizeof(int) * ap.size()));
    HBEM_CUDA(cudaMalloc((void **)&s->d_ap_local, sizeof(int) * loc.size()));
    HBEM_CUDA(cudaMemcpy(s->d_ap_tris, ap.data(), sizeof(int) * ap.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_ap_local, loc.data(), sizeof(int) * loc.size(), cudaMemcpyHostToDevice));
    s->aperture_tag = aperture_tag;
    s->m_ap = (int)ap.size();
    s->ap_tris = ap;
    return HBEM_OK;
}

extern "C" int hbem_aperture_assemble(hbem_session *h, int n_freq, const float *k_re, const float *k_im,
                                      const float *kf_re, float *sia_re, float *sia_im, float *saa_re, float *saa_im,
                                      void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_aperture_assemble: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_aperture_assemble: no aperture set");
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !kf_re || !sia_re || !sia_im || !saa_re || !saa_im) return fail(HBEM_ERR_ARG, "hbem_aperture_assemble: NULL pointer");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long n = s->n_dof, m = s->m_ap;
    HBEM_CUDA(cudaMemsetAsync(sia_re, 0, sizeof(float) * n * m * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(sia_im, 0, sizeof(float) * n * m * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(saa_re, 0, sizeof(float) * m * m * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(saa_im, 0, sizeof(float) * m * m * n_freq, st));
    for (int f0 = 0; f0 < n_freq; f0 += 64) {
        const int nf = std::min(64, n_freq - f0);
        ApArgs a{};
        fill_ap_args(a, *s, k_re, k_im, f0, nf);
        a.out_re = sia_re + (size_t)f0 * n * m; a.out_im = sia_im + (size_t)f0 * n * m; a.stride = n * m;
        k_ap_slp<<<dim3((s->n_triangles + 127) / 128, (unsigned)m, nf), 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k_ap_slp");
        ApArgs b{};
        fill_ap_args(b, *s, kf_re, nullptr, f0, nf);
        b.out_re = saa_re + (size_t)f0 * m * m; b.out_im = saa_im + (size_t)f0 * m * m; b.stride = m * m;
        k_ap_avg<<<dim3((unsigned)((m + 127) / 128), (unsigned)m, nf), 128, 0, st>>>(b);
        HBEM_LAUNCH_CHECK("k_ap_avg");
    }
    ApertureOut o0{0, sia_re, sia_im, nullptr, nullptr, n * m, m * m};
    int rc = launch_duffy(*s, n_freq, k_re, k_im, nullptr, nullptr, 0, nullptr, nullptr, nullptr, nullptr, n, n * n,
                          nullptr, nullptr, n, st, &o0);
    if (rc != HBEM_OK) return rc;
    ApertureOut o1{1, nullptr, nullptr, saa_re, saa_im, n * m, m * m};
    return launch_duffy(*s, n_freq, kf_re, nullptr, nullptr, nullptr, 0, nullptr, nullptr, nullptr, nullptr, n, n * n,
                        nullptr, nullptr, n, st, &o1);
}

extern "C" int hbem_coupled_ib_schur(hbem_session *h, int n_freq, float *a_re, float *a_im, const float *sia_re,
                                     const float *sia_im, float *saa_re, float *saa_im, float *minv_re,
                                     float *minv_im, int *info, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_schur: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_coupled_ib_schur: no aperture set");
    if (n_freq <= 0) return HBEM_OK;
    if (!a_re || !a_im || !sia_re || !sia_im || !saa_re || !saa_im || !minv_re || !minv_im || !info)
        return fail(HBEM_ERR_ARG, "hbem_coupled_ib_schur: NULL pointer");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const long long n = s->n_dof, m = s->m_ap;
    // M = (2 S_aa)^-1 by LU and m identity right-hand sides
    k_scale_identity<<<dim3((unsigned)((m * m + 255) / 256 < 1024 ? (m * m + 255) / 256 : 1024), n_freq), 256, 0, st>>>(
        saa_re, saa_im, minv_re, minv_im, (int)m, m * m);
    HBEM_LAUNCH_CHECK("k_scale_identity");
    int *piv = nullptr;
    float *x = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&piv, sizeof(int) * m * n_freq, st));
    HBEM_CUDA(cudaMallocAsync((void **)&x, sizeof(float) * 2 * n * m * n_freq, st));
    int rc = lu_factor((int)m, n_freq, saa_re, saa_im, m, m * m, piv, m, info, HBEM_PREC_PLAIN, st);
    if (rc == HBEM_OK)
        rc = lu_solve((int)m, (int)m, n_freq, saa_re, saa_im, m, m * m, piv, m, minv_re, minv_im, m, m * m,
                      HBEM_TRANS_N, st);
    if (rc == HBEM_OK) {
        float *xr = x, *xi = x + (size_t)n * m * n_freq;
        dim3 g((unsigned)((m + 63) / 64), (unsigned)((n + 63) / 64), n_freq);
        k_cgemm<<<g, 256, 0, st>>>(sia_re, sia_im, m, n * m, minv_re, minv_im, m, m * m, xr, xi, m, n * m, (int)n,
                                   (int)m, (int)m);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "k_cgemm");
        else {
            count_launch();
            k_ib_scatter<<<dim3((unsigned)((n + 255) / 256), (unsigned)m, n_freq), 256, 0, st>>>(
                a_re, a_im, n * n, xr, xi, n * m, s->d_ap_tris, s->d_l2g, (int)n, (int)m);
            e = cudaGetLastError();
            if (e != cudaSuccess) rc = cuda_fail(e, "k_ib_scatter");
            else count_launch();
        }
    }
    cudaFreeAsync(piv, st);
    cudaFreeAsync(x, st);
    return rc;
}

extern "C" int hbem_coupled_ib_field(hbem_session *h, int n_freq, const float *kf_re, const float *p_re,
                                     const float *p_im, const float *minv_re, const float *minv_im,
                                     const float *obs_3xn, int n_obs, float *qa_re, float *qa_im, float *out_re,
                                     float *out_im, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_coupled_ib_field: no aperture set");
    if (n_freq <= 0) return HBEM_OK;
    const bool qa_given = !minv_re && !minv_im;
    if (!kf_re || !qa_re || !qa_im || (!qa_given && (!p_re || !p_im || !minv_re || !minv_im)) ||
        (n_obs > 0 && (!obs_3xn || !out_re || !out_im)))
        return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field: NULL pointer");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int m = s->m_ap;
    if (!qa_given) {
        k_ib_qa<<<dim3((m + 7) / 8, n_freq), 256, 0, st>>>(p_re, p_im, s->n_dof, minv_re, minv_im, m, s->d_ap_tris,
                                                           s->d_l2g, qa_re, qa_im);
        HBEM_LAUNCH_CHECK("k_ib_qa");
    }
    if (n_obs <= 0) return HBEM_OK;
    for (int f0 = 0; f0 < n_freq; f0 += 64) {
        const int nf = std::min(64, n_freq - f0);
        ApArgs a{};
        fill_ap_args(a, *s, kf_re, nullptr, f0, nf);
        k_rayleigh<<<dim3(n_obs, nf), 256, 0, st>>>(a, qa_re + (size_t)f0 * m, qa_im + (size_t)f0 * m, obs_3xn, n_obs,
                                                    out_re + (size_t)f0 * n_obs, out_im + (size_t)f0 * n_obs);
        HBEM_LAUNCH_CHECK("k_rayleigh");
    }
    return HBEM_OK;
}

extern "C" int hbem_coupled_ib_augment(hbem_session *h, int n_freq, const float *sia_re, const float *sia_im,
                                       const float *saa_re, const float *saa_im, float *k_re, float *k_im,
                                       long long ldk, long long k_stride, float *alpha, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_augment: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_coupled_ib_augment: no aperture set");
    if (n_freq <= 0) return HBEM_OK;
    if (!sia_re || !sia_im || !saa_re || !saa_im || !k_re || !k_im || !alpha)
        return fail(HBEM_ERR_ARG, "hbem_coupled_ib_augment: NULL pointer");
    const long long n = s->n_dof, m = s->m_ap, N = n + m;
    if (ldk < N || k_stride < ldk * N) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_augment: bad strides");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned *mx = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&mx, sizeof(unsigned) * 3 * n_freq, st));
    int rc = HBEM_OK;
    cudaError_t e = cudaMemsetAsync(mx, 0, sizeof(unsigned) * 3 * n_freq, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "hbem_coupled_ib_augment: memset");
    if (rc == HBEM_OK) {
        k_ib_block_max<<<dim3(256, 3, n_freq), 256, 0, st>>>(k_re, k_im, ldk, k_stride, sia_re, sia_im, saa_re, saa_im,
                                                            (int)n, (int)m, mx);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "k_ib_block_max");
        else count_launch();
    }
    if (rc == HBEM_OK) {
        const unsigned gx = (unsigned)std::min<long long>(16, (N + 255) / 256);
        k_ib_augment<<<dim3(gx, (unsigned)N, n_freq), 256, 0, st>>>(sia_re, sia_im, saa_re, saa_im, k_re, k_im, ldk,
                                                                   k_stride, s->d_ap_tris, s->d_l2g, (int)n, (int)m,
                                                                   mx, alpha);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(e, "k_ib_augment");
        else count_launch();
    }
    cudaFreeAsync(mx, st);
    return rc;
}
