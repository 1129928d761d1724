// Trailing update of the blocked LU: A22 -= L21 * U12 (complex, planar),
// batched over matrices.  K = 16/32 inside a block column, 64 for the
// block's trailing matrix.
//
// CUDA-core path: 64 x 64 complex output tile per 256-thread CTA, 4 x 4
// complex outputs per thread, L and U tiles staged in shared memory with
// 128-bit broadcast reads; FP32 FMA gives the exact-FP32 products of
// LAPACK cgemm-based cgetrf.
#include <cuda_runtime.h>

#include <algorithm>

#include "hbem_internal.h"

namespace hbem {
namespace {

// C[start:n, start:col_end] -= L[start:n, k0:k0+kw] * U[k0:k0+kw, start:col_end]
// with kw a multiple of 16; K is consumed in 16-wide shared-memory chunks.
__global__ void __launch_bounds__(256) k_trailing_simt(float *a_re, float *a_im, long long lda, long long a_stride,
                                                       int n, int k0, int kw, int start, int col_end) {
    constexpr int KC = 16;
    __shared__ __align__(16) float Lr[KC][64], Li[KC][64];
    __shared__ __align__(16) float Ur[KC][64], Ui[KC][64];
    const int mat = blockIdx.z;
    float *are = a_re + (size_t)mat * a_stride, *aim = a_im + (size_t)mat * a_stride;
    const int row0 = start + blockIdx.y * 64, col0 = start + blockIdx.x * 64;
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    float cr[4][4], ci[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cr[i][j] = ci[i][j] = 0.f;
    for (int kc = 0; kc < kw; kc += KC) {
        for (int e = tid; e < 64 * KC; e += 256) {
            const int r = e / KC, kk = e - r * KC;
            const int gr = row0 + r;
            float vr = 0.f, vi = 0.f;
            if (gr < n) {
                vr = are[(size_t)gr * lda + k0 + kc + kk];
                vi = aim[(size_t)gr * lda + k0 + kc + kk];
            }
            Lr[kk][r] = vr;
            Li[kk][r] = vi;
        }
        for (int e = tid; e < 64 * KC; e += 256) {
            const int kk = e / 64, c = e - kk * 64;
            const int gc = col0 + c;
            float vr = 0.f, vi = 0.f;
            if (gc < col_end) {
                vr = are[(size_t)(k0 + kc + kk) * lda + gc];
                vi = aim[(size_t)(k0 + kc + kk) * lda + gc];
            }
            Ur[kk][c] = vr;
            Ui[kk][c] = vi;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            const float4 lr = *reinterpret_cast<const float4 *>(&Lr[kk][ty * 4]);
            const float4 li = *reinterpret_cast<const float4 *>(&Li[kk][ty * 4]);
            const float4 ur = *reinterpret_cast<const float4 *>(&Ur[kk][tx * 4]);
            const float4 ui = *reinterpret_cast<const float4 *>(&Ui[kk][tx * 4]);
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

int launch_trailing_update(int n, int batch, int k0, int kw, int start, int col_end, float *a_re, float *a_im,
                           long long lda, long long a_stride, int precision, cudaStream_t st) {
    (void)precision;
    const int m = n - start, w = col_end - start;
    if (m <= 0 || w <= 0) return HBEM_OK;
    if (kw % 16) return fail(HBEM_ERR_ARG, "trailing update: K must be a multiple of 16");
    dim3 grid((w + 63) / 64, (m + 63) / 64, batch);
    k_trailing_simt<<<grid, 256, 0, st>>>(a_re, a_im, lda, a_stride, n, k0, kw, start, col_end);
    HBEM_LAUNCH_CHECK("k_trailing_simt");
    return HBEM_OK;
}

}  // namespace hbem
