// Exterior field and surface-pressure reductions, batched over frequencies.
//
//   p(x_o) = sum_tri sum_q w_q 2|tau| sum_images [dG/dn_y(x_o, y_q) p(y_q) - G(x_o, y_q) q_tri]
//   (reference evaluate_field_regular, main.swift:4135-4203; real k only, as there)
//
// One CTA per (frequency, tile of 8 observation points); threads stride over
// triangles, interpolate the P1 pressure to the 6 quadrature points once per
// triangle, and accumulate the 8 observation sums in registers before a block
// reduction.  Tag averages (main.swift:807-841) use FP64 block sums.
//
// Phase accuracy: at 2 m and 20 kHz, k r is ~730 rad, so an FP32 distance
// (relative error ~6e-8) alone puts ~4e-5 rad into the phase, which the sum
// over the surface turns into a field error of the same size and up to
// 0.01 dB of directivity near the pattern's nulls.  The distance is therefore
// carried in FP64 from the exact difference of the float coordinates (an FP32
// root refined by one FP64 Newton step) and the phase is reduced in turns in
// FP64; sine and cosine of the reduced phase, the amplitudes and the sums
// stay FP32.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "hbem_internal.h"

namespace hbem {
namespace {

constexpr int kObsTile = 8;
constexpr int kFieldThreads = 256;

struct FieldArgs {
    const float4 *qp;    // (T, 6) original order
    const float4 *nrm;   // (T) normal + 2 area
    const int *l2g;
    const float *p_re, *p_im, *q_re, *q_im, *obs;
    float *out_re, *out_im;
    long long p_stride, q_stride, out_stride;
    int T, n_obs, sym;
    float k[64];
    double kt[64];   // k / (2 pi): turns per metre
};

__device__ __forceinline__ float fqw(int q) { return (q == 0 || q == 2 || q == 3) ? HBEM_QWA : HBEM_QWB; }
__device__ __forceinline__ float fqx(int q) {
    return q == 0 ? HBEM_QX0 : q == 1 ? HBEM_QX1 : q == 2 ? HBEM_QX2 : q == 3 ? HBEM_QX3 : q == 4 ? HBEM_QX4 : HBEM_QX5;
}
__device__ __forceinline__ float fqy(int q) {
    return q == 0 ? HBEM_QY0 : q == 1 ? HBEM_QY1 : q == 2 ? HBEM_QY2 : q == 3 ? HBEM_QY3 : q == 4 ? HBEM_QY4 : HBEM_QY5;
}

// adds (D p - G q) for one source point y seen from the observation point o:
// the distance for the phase from the exact double differences of the float
// inputs (yx .. oz), the amplitude and the projection from the FP32
// differences (fy - fo) — no double-to-float conversions on the hot path, whose
// conversion / MUFU pipe bounds this kernel
__device__ __forceinline__ void fsample(double yx, double yy, double yz, double ox, double oy, double oz, float fyx,
                                        float fyy, float fyz, float fox, float foy, float foz, float nx, float ny,
                                        float nz, float k, double kt, float pr, float pi, float qr, float qi,
                                        float &ar, float &ai) {
    const double dxd = yx - ox, dyd = yy - oy, dzd = yz - oz;
    const double r2d = fma(dxd, dxd, fma(dyd, dyd, dzd * dzd));
    const float dx = fyx - fox, dy = fyy - foy, dz = fyz - foz;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float rinv = rsqrtf(r2);
    rinv = r2 > 1.0e-14f ? rinv : 0.0f;
    const float rf = r2 * rinv;
    // one Newton step in FP64: r = rf + (r2 - rf^2) / (2 rf)
    const double rfd = (double)rf;
    const double r = fma(fma(-rfd, rfd, r2d), (double)(0.5f * rinv), rfd);
    double td = r * kt;
    td -= rint(td);
    float s, c;
    sincospif(2.0f * (float)td, &s, &c);
    const float gc = rinv * c, gs = rinv * s;
    const float proj = fmaf(dx, nx, fmaf(dy, ny, dz * nz)) * rinv;
    const float dre = fmaf(gc, -rinv, -gs * k) * proj;
    const float dim = fmaf(gc, k, -gs * rinv) * proj;
    ar += dre * pr - dim * pi - (gc * qr - gs * qi);
    ai += dre * pi + dim * pr - (gc * qi + gs * qr);
}

template <int SYM>
__global__ void __launch_bounds__(kFieldThreads, 2) k_field(const __grid_constant__ FieldArgs a) {
    __shared__ double s_obs[kObsTile][3];
    __shared__ float s_obsf[kObsTile][3];
    __shared__ float s_red[kFieldThreads / 32][kObsTile][2];
    const int f = blockIdx.y;
    const int o0 = blockIdx.x * kObsTile;
    const int nob = min(kObsTile, a.n_obs - o0);
    if (threadIdx.x < kObsTile * 3) {
        const int o = threadIdx.x / 3, c = threadIdx.x % 3;
        const float v = o < nob ? a.obs[(size_t)c * a.n_obs + o0 + o] : 0.f;
        s_obs[o][c] = v;
        s_obsf[o][c] = v;
    }
    __syncthreads();
    const float k = a.k[f];
    const double kt = a.kt[f];
    const float *pre = a.p_re + (size_t)f * a.p_stride, *pim = a.p_im + (size_t)f * a.p_stride;
    const float *qre = a.q_re + (size_t)f * a.q_stride, *qim = a.q_im + (size_t)f * a.q_stride;
    float accr[kObsTile], acci[kObsTile];
#pragma unroll
    for (int o = 0; o < kObsTile; ++o) accr[o] = acci[o] = 0.f;
    for (int t = threadIdx.x; t < a.T; t += kFieldThreads) {
        const float4 nj = a.nrm[t];
        const int d0 = a.l2g[3 * t], d1 = a.l2g[3 * t + 1], d2 = a.l2g[3 * t + 2];
        const float p0r = pre[d0], p1r = pre[d1], p2r = pre[d2];
        const float p0i = pim[d0], p1i = pim[d1], p2i = pim[d2];
        const float qr = qre[t], qi = qim[t];
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            const float4 yf = a.qp[(size_t)t * 6 + q];
            const double yx = yf.x, yy = yf.y, yz = yf.z;
            const float b1 = fqx(q), b2 = fqy(q), b0 = 1.f - b1 - b2;
            const float w = fqw(q) * nj.w;
            const float pr = (b0 * p0r + b1 * p1r + b2 * p2r) * w, pi = (b0 * p0i + b1 * p1i + b2 * p2i) * w;
            const float wqr = qr * w, wqi = qi * w;
#pragma unroll
            for (int o = 0; o < kObsTile; ++o) {
                // the observation point re-read per use (volatile): kept in registers for
                // all eight points the copies would push the kernel past 128 registers
                const volatile double *vd = s_obs[o];
                const double ox = vd[0], oy = vd[1], oz = vd[2];
                const volatile float *vo = s_obsf[o];
                const float fx = vo[0], fy = vo[1], fz = vo[2];
                fsample(yx, yy, yz, ox, oy, oz, yf.x, yf.y, yf.z, fx, fy, fz, nj.x, nj.y, nj.z, k, kt, pr, pi, wqr, wqi,
                        accr[o], acci[o]);
                if (SYM == 1 || SYM == 3)
                    fsample(-yx, yy, yz, ox, oy, oz, -yf.x, yf.y, yf.z, fx, fy, fz, -nj.x, nj.y, nj.z, k, kt, pr, pi, wqr,
                            wqi, accr[o], acci[o]);
                if (SYM == 2 || SYM == 3)
                    fsample(yx, -yy, yz, ox, oy, oz, yf.x, -yf.y, yf.z, fx, fy, fz, nj.x, -nj.y, nj.z, k, kt, pr, pi, wqr,
                            wqi, accr[o], acci[o]);
                if (SYM == 3)
                    fsample(-yx, -yy, yz, ox, oy, oz, -yf.x, -yf.y, yf.z, fx, fy, fz, -nj.x, -nj.y, nj.z, k, kt, pr, pi,
                            wqr, wqi, accr[o], acci[o]);
                if (SYM == 4)
                    fsample(yx, yy, -yz, ox, oy, oz, yf.x, yf.y, -yf.z, fx, fy, fz, nj.x, nj.y, -nj.z, k, kt, pr, pi, wqr,
                            wqi, accr[o], acci[o]);
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 0; o < kObsTile; ++o) {
#pragma unroll
        for (int s = 16; s > 0; s >>= 1) {
            accr[o] += __shfl_xor_sync(0xffffffffu, accr[o], s);
            acci[o] += __shfl_xor_sync(0xffffffffu, acci[o], s);
        }
        if (lane == 0) {
            s_red[warp][o][0] = accr[o];
            s_red[warp][o][1] = acci[o];
        }
    }
    __syncthreads();
    if (threadIdx.x < nob * 2) {
        const int o = threadIdx.x >> 1, c = threadIdx.x & 1;
        float v = 0.f;
        for (int w = 0; w < kFieldThreads / 32; ++w) v += s_red[w][o][c];
        v *= HBEM_INV4PI;
        float *dst = c ? a.out_im : a.out_re;
        dst[(size_t)f * a.out_stride + o0 + o] = v;
    }
}

__global__ void k_tag_avg(const int *__restrict__ tags, const float *__restrict__ areas, const int *__restrict__ l2g,
                          const float *p_re, const float *p_im, long long p_stride, int T, const int *__restrict__ want,
                          double *out, int n_tags) {
    const int f = blockIdx.y, ti = blockIdx.x;
    const int tag = want[ti];
    const float *pr = p_re + (size_t)f * p_stride, *pi = p_im + (size_t)f * p_stride;
    double sr = 0, si = 0, sa = 0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        if (tags[t] != tag) continue;
        const double ar = areas[t];
        if (!(ar > 0.0)) continue;
        const int d0 = l2g[3 * t], d1 = l2g[3 * t + 1], d2 = l2g[3 * t + 2];
        sr += ((double)pr[d0] + (double)pr[d1] + (double)pr[d2]) / 3.0 * ar;
        si += ((double)pi[d0] + (double)pi[d1] + (double)pi[d2]) / 3.0 * ar;
        sa += ar;
    }
    __shared__ double s[3][32];
    for (int o = 16; o > 0; o >>= 1) {
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
        si += __shfl_xor_sync(0xffffffffu, si, o);
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s[0][warp] = sr; s[1][warp] = si; s[2][warp] = sa; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0, a1 = 0, a2 = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) { a0 += s[0][w]; a1 += s[1][w]; a2 += s[2][w]; }
        double *o = out + ((size_t)f * n_tags + ti) * 2;
        if (a2 < 1e-30) { o[0] = 0; o[1] = 0; }
        else { o[0] = a0 / a2; o[1] = a1 / a2; }
    }
}

}  // namespace

int launch_field(Session &s, int n_freq, const float *k_re, const float *p_re, const float *p_im, long long p_stride,
                 const float *q_re, const float *q_im, long long q_stride, const float *obs, int n_obs, float *out_re,
                 float *out_im, long long out_stride, cudaStream_t st) {
    for (int f0 = 0; f0 < n_freq; f0 += 64) {
        const int nf = std::min(64, n_freq - f0);
        FieldArgs a{};
        a.qp = s.d_fqp; a.nrm = s.d_fnrm; a.l2g = s.d_l2g;
        a.p_re = p_re + (size_t)f0 * p_stride; a.p_im = p_im + (size_t)f0 * p_stride;
        a.q_re = q_re + (size_t)f0 * q_stride; a.q_im = q_im + (size_t)f0 * q_stride;
        a.obs = obs;
        a.out_re = out_re + (size_t)f0 * out_stride; a.out_im = out_im + (size_t)f0 * out_stride;
        a.p_stride = p_stride; a.q_stride = q_stride; a.out_stride = out_stride;
        a.T = s.n_triangles; a.n_obs = n_obs; a.sym = s.sym;
        for (int f = 0; f < nf; ++f) {
            a.k[f] = k_re[f0 + f];
            a.kt[f] = (double)k_re[f0 + f] / (2.0 * 3.14159265358979323846);
        }
        dim3 grid((n_obs + kObsTile - 1) / kObsTile, nf);
        switch (s.sym) {
            case 0: k_field<0><<<grid, kFieldThreads, 0, st>>>(a); break;
            case 1: k_field<1><<<grid, kFieldThreads, 0, st>>>(a); break;
            case 2: k_field<2><<<grid, kFieldThreads, 0, st>>>(a); break;
            case 3: k_field<3><<<grid, kFieldThreads, 0, st>>>(a); break;
            default: k_field<4><<<grid, kFieldThreads, 0, st>>>(a); break;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "k_field launch");
        count_launch();
        ++s.launches;
    }
    return HBEM_OK;
}

int launch_tag_avg(Session &s, int n_freq, const float *p_re, const float *p_im, long long p_stride,
                   const int *d_want, int n_tags, double *out, cudaStream_t st) {
    if (n_tags <= 0) return HBEM_OK;
    dim3 grid(n_tags, n_freq);
    k_tag_avg<<<grid, 256, 0, st>>>(s.d_tags, s.d_areas, s.d_l2g, p_re, p_im, p_stride, s.n_triangles, d_want, out, n_tags);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_tag_avg launch");
    count_launch();
    ++s.launches;
    return HBEM_OK;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_field(hbem_session *h, int n_freq, const float *k_re, const float *p_re, const float *p_im,
                          long long p_stride, const float *q_re, const float *q_im, long long q_stride,
                          const float *obs_3xn, int n_obs, float *out_re, float *out_im, long long out_stride,
                          void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_field: NULL session");
    if (n_freq <= 0 || n_obs <= 0) return HBEM_OK;
    if (!k_re || !p_re || !p_im || !q_re || !q_im || !obs_3xn || !out_re || !out_im)
        return fail(HBEM_ERR_ARG, "hbem_field: NULL pointer");
    if (p_stride < s->n_dof || q_stride < s->n_triangles || out_stride < n_obs)
        return fail(HBEM_ERR_ARG, "hbem_field: stride too small");
    HBEM_CUDA(cudaSetDevice(s->device));
    return launch_field(*s, n_freq, k_re, p_re, p_im, p_stride, q_re, q_im, q_stride, obs_3xn, n_obs, out_re, out_im,
                        out_stride, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_reduce_tag_avg(hbem_session *h, int n_freq, const float *p_re, const float *p_im,
                                   long long p_stride, const int *tags_host, int n_tags, double *out, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg: NULL session");
    if (n_freq <= 0 || n_tags <= 0) return HBEM_OK;
    if (!p_re || !p_im || !tags_host || !out) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg: NULL pointer");
    if (n_tags > 64) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg: at most 64 tags per call");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // the tag list rides in the session's status page (4 ints) when short, else a scratch copy
    int *d_want = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&d_want, sizeof(int) * n_tags, st));
    HBEM_CUDA(cudaMemcpyAsync(d_want, tags_host, sizeof(int) * n_tags, cudaMemcpyHostToDevice, st));
    int rc = launch_tag_avg(*s, n_freq, p_re, p_im, p_stride, d_want, n_tags, out, st);
    cudaFreeAsync(d_want, st);
    return rc;
}

extern "C" int hbem_reduce_tag_avg_device(hbem_session *h, int n_freq, const float *p_re, const float *p_im,
                                          long long p_stride, const int *tags_device, int n_tags, double *out,
                                          void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg_device: NULL session");
    if (n_freq <= 0 || n_tags <= 0) return HBEM_OK;
    if (!p_re || !p_im || !tags_device || !out) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg_device: NULL pointer");
    if (n_tags > 64) return fail(HBEM_ERR_ARG, "hbem_reduce_tag_avg_device: at most 64 tags per call");
    HBEM_CUDA(cudaSetDevice(s->device));
    return launch_tag_avg(*s, n_freq, p_re, p_im, p_stride, tags_device, n_tags, out, reinterpret_cast<cudaStream_t>(stream));
}
