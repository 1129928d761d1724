// One-call batched sweep over host buffers (hbem_solve_batch): the drop-in
// for the reference's assemble_solve_evaluate_standard_neumann_batch
// (hornlab_metal_bem/metal/native.py:737-1203, helper main.swift:8869-9878).
//
// Frequencies are processed in chunks whose dense matrices fit the device
// memory budget; within a chunk every stage is one batched launch set on one
// stream: corrected assembly -> LU -> solve (-> FP64-residual refinement) ->
// field -> tag reductions.  Nothing round-trips to the host between stages.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hbem_internal.h"

namespace hbem {
int lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride, int *piv,
              long long piv_stride, int *info, int precision, cudaStream_t st);
int lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const int *piv, long long piv_stride, float *b_re, float *b_im, long long ldb, long long b_stride,
             int trans, cudaStream_t st);
int matrix_norm1(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                 float *anorm, cudaStream_t st);
int lu_rcond(int n, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
             const float *anorm, double *rcond, cudaStream_t st);
int refine(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
           const float *lu_re, const float *lu_im, long long lu_stride, const int *piv, long long piv_stride,
           const float *b_re, const float *b_im, long long b_stride, float *x_re, float *x_im, long long x_stride,
           double tol, int max_iter, int *iters, double *resid, cudaStream_t st);
int wave_fault_check(cudaStream_t st);
int launch_field(Session &s, int n_freq, const float *k_re, const float *p_re, const float *p_im, long long p_stride,
                 const float *q_re, const float *q_im, long long q_stride, const float *obs, int n_obs, float *out_re,
                 float *out_im, long long out_stride, cudaStream_t st);
int launch_tag_avg(Session &s, int n_freq, const float *p_re, const float *p_im, long long p_stride,
                   const int *d_want, int n_tags, double *out, cudaStream_t st);
int lu_factor_f64(int n, int batch, double *a_re, double *a_im, long long lda, long long a_stride, int *piv,
                  long long piv_stride, int *info, cudaStream_t st);
int lu_solve_f64(int n, int nrhs, int batch, const double *lu_re, const double *lu_im, long long lda,
                 long long a_stride, const int *piv, long long piv_stride, double *b_re, double *b_im, long long ldb,
                 long long b_stride, cudaStream_t st);
int widen_f64(int rows, int cols, int batch, const float *sr, const float *si, long long sld, long long sstride,
              double *dr, double *di, long long dld, long long dstride, cudaStream_t st);
int narrow_f64(int rows, int cols, int batch, const double *sr, const double *si, long long sld, long long sstride,
               float *dr, float *di, long long dld, long long dstride, cudaStream_t st);

namespace {

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

struct Layout {
    size_t q, a, a0, a64, x64, x, b, piv, info, obs, fld, tag, want, iters, resid, anorm, rcond, total;
};

// Leading dimension of the dense FP32 matrices: n rounded up to a multiple of
// 4 floats, so every row starts on a 16-byte boundary and the trailing
// updates read and write C as float4 (an odd n = 1043 made three rows in four
// take the scalar path: the 1043 x 40 LU 7.4 -> 6.5 ms with the exact-FP32
// update, 6.5 -> 6.2 ms with the TF32x3 one, measured at n = 1044).
size_t matrix_ld(size_t n) { return (n + 3) & ~(size_t)3; }

Layout layout(const Session &s, int nf, int n_src, int n_obs, int n_tags, bool keep_a, bool fp64) {
    const size_t n = s.n_dof, T = s.n_triangles, ns = (size_t)n_src, ld = matrix_ld(n);
    Layout L{};
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes); return o; };
    L.q = take(2 * sizeof(float) * ns * nf * T);
    L.a = take(2 * sizeof(float) * nf * n * ld);
    L.a0 = keep_a ? take(2 * sizeof(float) * nf * n * ld) : 0;
    L.a64 = fp64 ? take(2 * sizeof(double) * nf * n * n) : 0;
    L.x64 = fp64 ? take(2 * sizeof(double) * ns * nf * n) : 0;
    L.x = take(2 * sizeof(float) * ns * nf * n);
    L.b = take(2 * sizeof(float) * ns * nf * n);
    L.piv = take(sizeof(int) * nf * n);
    L.info = take(sizeof(int) * nf);
    L.obs = take(3 * sizeof(float) * std::max(1, n_obs));
    L.fld = take(2 * sizeof(float) * ns * nf * std::max(1, n_obs));
    L.tag = take(2 * sizeof(double) * ns * nf * std::max(1, n_tags));
    L.want = take(sizeof(int) * std::max(1, n_tags));
    L.iters = take(sizeof(int) * ns * nf);
    L.resid = take(sizeof(double) * ns * nf);
    L.anorm = take(sizeof(float) * nf);
    L.rcond = take(sizeof(double) * nf);
    L.total = off;
    return L;
}

int ensure_ws(Session &s, size_t bytes) {
    if (s.ws_bytes >= bytes) return HBEM_OK;
    if (s.ws) cudaFree(s.ws);
    s.ws = nullptr;
    s.ws_bytes = 0;
    HBEM_CUDA(cudaMalloc(&s.ws, bytes));
    s.ws_bytes = bytes;
    return HBEM_OK;
}

}  // namespace
}  // namespace hbem

using namespace hbem;

// The sweep for n_src right-hand sides (velocity sources) sharing each
// frequency's matrix: one assembly pass fills A and every source's b, one LU,
// then one solve (and refinement) per source, field and tag averages for all
// (source, frequency) cases in one launch each.  Host arrays per source are
// source-major: q (n_src, n_freq, T), field (n_src, n_freq, n_obs), tag_avg
// (n_src, n_freq, n_tags, 2), surface (n_src, n_freq, n), refine_iters /
// refine_resid (n_src, n_freq); info and rcond are per frequency.
static int solve_batch_impl(hbem_session *h, int n_freq, int n_src, const float *k_re, const float *k_im,
                            const float *q_re, const float *q_im, const float *obs_3xn, int n_obs, const int *tags,
                            int n_tags, int precision, double refine_tol, int refine_max_iter, float *field_re,
                            float *field_im, double *tag_avg, float *surface_re, float *surface_im, int *info,
                            int *refine_iters, double *refine_resid, double *rcond, float *timings_ms, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_solve_batch: NULL session");
    if (n_freq <= 0) return HBEM_OK;
    if (n_src < 1 || n_src > 8) return fail(HBEM_ERR_ARG, "hbem_solve_batch_multi: n_src must be 1 .. 8");
    if (!k_re || !q_re || !q_im || !info) return fail(HBEM_ERR_ARG, "hbem_solve_batch: NULL input");
    if (n_obs > 0 && (!obs_3xn || !field_re || !field_im)) return fail(HBEM_ERR_ARG, "hbem_solve_batch: NULL field buffers");
    if (n_tags > 0 && (!tags || !tag_avg)) return fail(HBEM_ERR_ARG, "hbem_solve_batch: NULL tag buffers");
    if (n_tags > 64) return fail(HBEM_ERR_ARG, "hbem_solve_batch: at most 64 tags");
    if ((surface_re == nullptr) != (surface_im == nullptr)) return fail(HBEM_ERR_ARG, "hbem_solve_batch: surface pointers");
    if (precision != HBEM_PREC_PLAIN && precision != HBEM_PREC_MIXED && precision != HBEM_PREC_FP64)
        return fail(HBEM_ERR_ARG, "hbem_solve_batch: bad precision");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f]) || (k_im && !std::isfinite(k_im[f])))
            return fail(HBEM_ERR_ARG, "hbem_solve_batch: non-finite wavenumber");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const bool fp64 = precision == HBEM_PREC_FP64;
    const bool do_refine = !fp64 && ((precision == HBEM_PREC_MIXED) || refine_max_iter > 0);
    const int max_iter = precision == HBEM_PREC_MIXED ? std::max(1, refine_max_iter) : refine_max_iter;
    const double tol = refine_tol > 0 ? refine_tol : 1e-6;
    const size_t n = s->n_dof, T = s->n_triangles, ns = (size_t)n_src, ld = matrix_ld(n);

    // chunk size: the whole sweep when the session's workspace already holds
    // it (no device query on repeated calls), else dense matrices within
    // ~60 % of free memory
    int chunk = n_freq;
    if (layout(*s, chunk, n_src, n_obs, n_tags, do_refine, fp64).total > s->ws_bytes) {
        size_t free_b = 0, total_b = 0;
        HBEM_CUDA(cudaMemGetInfo(&free_b, &total_b));
        free_b += s->ws_bytes;
        while (chunk > 1 && layout(*s, chunk, n_src, n_obs, n_tags, do_refine, fp64).total > free_b * 6 / 10)
            chunk = (chunk + 1) / 2;
    }
    const Layout L = layout(*s, chunk, n_src, n_obs, n_tags, do_refine, fp64);
    int rc = ensure_ws(*s, L.total);
    if (rc != HBEM_OK) return rc;
    if (rcond && !s->aux) {
        // the condition estimate runs on a second stream beside the solves,
        // refinement and field (it only reads the factors)
        int lo = 0, hi = 0;
        HBEM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        HBEM_CUDA(cudaStreamCreateWithPriority(&s->aux, cudaStreamNonBlocking, lo));
        HBEM_CUDA(cudaEventCreateWithFlags(&s->aux_fork, cudaEventDisableTiming));
        HBEM_CUDA(cudaEventCreateWithFlags(&s->aux_join, cudaEventDisableTiming));
    }
    char *ws = static_cast<char *>(s->ws);
    float *dq = reinterpret_cast<float *>(ws + L.q);
    float *da = reinterpret_cast<float *>(ws + L.a);
    float *da0 = do_refine ? reinterpret_cast<float *>(ws + L.a0) : nullptr;
    float *dx = reinterpret_cast<float *>(ws + L.x);
    float *db = reinterpret_cast<float *>(ws + L.b);
    int *dpiv = reinterpret_cast<int *>(ws + L.piv);
    int *dinfo = reinterpret_cast<int *>(ws + L.info);
    float *dobs = reinterpret_cast<float *>(ws + L.obs);
    float *dfld = reinterpret_cast<float *>(ws + L.fld);
    double *dtag = reinterpret_cast<double *>(ws + L.tag);
    int *dwant = reinterpret_cast<int *>(ws + L.want);
    int *diters = reinterpret_cast<int *>(ws + L.iters);
    double *dres = reinterpret_cast<double *>(ws + L.resid);
    float *danorm = reinterpret_cast<float *>(ws + L.anorm);
    double *drcond = reinterpret_cast<double *>(ws + L.rcond);
    double *da64 = fp64 ? reinterpret_cast<double *>(ws + L.a64) : nullptr;
    double *dx64 = fp64 ? reinterpret_cast<double *>(ws + L.x64) : nullptr;

    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (auto &e : ev) {
        if (rc == HBEM_OK) {
            const cudaError_t err = cudaEventCreate(&e);
            if (err != cudaSuccess) rc = cuda_fail(err, "cudaEventCreate");
        }
    }
    auto ok = [&](cudaError_t e, const char *what) {
        if (rc == HBEM_OK && e != cudaSuccess) rc = cuda_fail(e, what);
        return rc == HBEM_OK;
    };
    float t_asm = 0, t_solve = 0, t_field = 0, t_total = 0;
    if (rc == HBEM_OK) ok(cudaEventRecord(ev[4], st), "cudaEventRecord");
    if (n_obs > 0) ok(cudaMemcpyAsync(dobs, obs_3xn, 3 * sizeof(float) * n_obs, cudaMemcpyHostToDevice, st), "obs");
    if (n_tags > 0) ok(cudaMemcpyAsync(dwant, tags, sizeof(int) * n_tags, cudaMemcpyHostToDevice, st), "tags");
    std::vector<float> k_rep;

    for (int f0 = 0; f0 < n_freq && rc == HBEM_OK; f0 += chunk) {
        const int nf = std::min(chunk, n_freq - f0);
        const size_t qs = (size_t)nf * T, xs = (size_t)nf * n;   // per-source strides on the device
        float *qr = dq, *qi = dq + ns * qs;
        for (int sv = 0; sv < n_src; ++sv) {
            const size_t ho = ((size_t)sv * n_freq + f0) * T;
            ok(cudaMemcpyAsync(qr + sv * qs, q_re + ho, sizeof(float) * qs, cudaMemcpyHostToDevice, st), "q");
            ok(cudaMemcpyAsync(qi + sv * qs, q_im + ho, sizeof(float) * qs, cudaMemcpyHostToDevice, st), "q");
        }
        float *ar = da, *ai = da + (size_t)nf * n * ld;
        float *br = db, *bi = db + ns * xs;
        float *xr = dx, *xi = dx + ns * xs;
        ok(cudaEventRecord(ev[0], st), "cudaEventRecord");
        if (rc != HBEM_OK) break;
        rc = hbem_assemble_multi(h, nf, k_re + f0, k_im ? k_im + f0 : nullptr, n_src, qr, qi, (long long)T,
                                 (long long)qs, nullptr, nullptr, ar, ai, (long long)ld, (long long)(n * ld), br, bi,
                                 (long long)n, (long long)xs, HBEM_ASM_CORRECTED, st);
        if (rc != HBEM_OK) break;
        ok(cudaEventRecord(ev[1], st), "cudaEventRecord");
        ok(cudaMemcpyAsync(xr, br, sizeof(float) * ns * xs, cudaMemcpyDeviceToDevice, st), "x");
        ok(cudaMemcpyAsync(xi, bi, sizeof(float) * ns * xs, cudaMemcpyDeviceToDevice, st), "x");
        float *a0r = nullptr, *a0i = nullptr;
        if (do_refine) {
            a0r = da0;
            a0i = da0 + (size_t)nf * n * ld;
            ok(cudaMemcpyAsync(a0r, ar, sizeof(float) * nf * n * ld, cudaMemcpyDeviceToDevice, st), "A copy");
            ok(cudaMemcpyAsync(a0i, ai, sizeof(float) * nf * n * ld, cudaMemcpyDeviceToDevice, st), "A copy");
        }
        if (rc != HBEM_OK) break;
        if (rcond) {
            rc = matrix_norm1((int)n, nf, ar, ai, (long long)ld, (long long)(n * ld), danorm, st);
            if (rc != HBEM_OK) break;
        }
        const long long nn = (long long)(n * n), na = (long long)(n * ld), lda = (long long)ld;
        if (fp64) {
            // the reference's float64 dense solve: widen the FP32 system to
            // complex128, factor and solve in FP64, narrow the solution
            double *a64r = da64, *a64i = da64 + (size_t)nf * n * n;
            double *x64r = dx64, *x64i = dx64 + ns * xs;
            rc = widen_f64((int)n, (int)n, nf, ar, ai, lda, na, a64r, a64i, (long long)n, nn, st);
            if (rc == HBEM_OK)
                rc = widen_f64(1, (int)n, n_src * nf, br, bi, (long long)n, (long long)n, x64r, x64i, (long long)n,
                               (long long)n, st);
            if (rc == HBEM_OK)
                rc = lu_factor_f64((int)n, nf, a64r, a64i, (long long)n, nn, dpiv, (long long)n, dinfo, st);
            for (int sv = 0; sv < n_src && rc == HBEM_OK; ++sv)
                rc = lu_solve_f64((int)n, 1, nf, a64r, a64i, (long long)n, nn, dpiv, (long long)n, x64r + sv * xs,
                                  x64i + sv * xs, 1, (long long)n, st);
            if (rc == HBEM_OK)
                rc = narrow_f64(1, (int)n, n_src * nf, x64r, x64i, (long long)n, (long long)n, xr, xi, (long long)n,
                                (long long)n, st);
            if (rc == HBEM_OK && rcond) {
                // condition estimate from the FP64 factors narrowed to FP32, on the second stream
                rc = narrow_f64((int)n, (int)n, nf, a64r, a64i, (long long)n, nn, ar, ai, lda, na, st);
                if (rc == HBEM_OK && ok(cudaEventRecord(s->aux_fork, st), "fork") &&
                    ok(cudaStreamWaitEvent(s->aux, s->aux_fork, 0), "fork"))
                    rc = lu_rcond((int)n, nf, ar, ai, lda, na, danorm, drcond, s->aux);
                if (rc == HBEM_OK) ok(cudaEventRecord(s->aux_join, s->aux), "join");
            }
            if (rc != HBEM_OK) break;
        } else {
            // with refinement on, the FP32 LU's bulk update runs on the tensor
            // cores (TF32x3): the FP64-residual passes recover the accuracy
            // its 22-bit split products give away
            const int lu_prec = (precision == HBEM_PREC_PLAIN && do_refine) ? HBEM_PREC_TF32X3 : precision;
            rc = lu_factor((int)n, nf, ar, ai, lda, na, dpiv, (long long)n, dinfo, lu_prec, st);
            if (rc != HBEM_OK) break;
            if (rcond) {
                // condition estimate on the second stream, beside the solves (both only read the factors)
                if (ok(cudaEventRecord(s->aux_fork, st), "fork") && ok(cudaStreamWaitEvent(s->aux, s->aux_fork, 0), "fork"))
                    rc = lu_rcond((int)n, nf, ar, ai, lda, na, danorm, drcond, s->aux);
                if (rc == HBEM_OK) ok(cudaEventRecord(s->aux_join, s->aux), "join");
                if (rc != HBEM_OK) break;
            }
            for (int sv = 0; sv < n_src && rc == HBEM_OK; ++sv)
                rc = lu_solve((int)n, 1, nf, ar, ai, lda, na, dpiv, (long long)n, xr + sv * xs, xi + sv * xs,
                              1, (long long)n, HBEM_TRANS_N, st);
            if (rc != HBEM_OK) break;
        }
        if (do_refine) {
            for (int sv = 0; sv < n_src && rc == HBEM_OK; ++sv)
                rc = refine((int)n, nf, a0r, a0i, lda, na, ar, ai, na, dpiv, (long long)n, br + sv * xs,
                            bi + sv * xs, (long long)n, xr + sv * xs, xi + sv * xs, (long long)n, tol, max_iter,
                            diters + (size_t)sv * nf, dres + (size_t)sv * nf, st);
            if (rc != HBEM_OK) break;
        }
        ok(cudaEventRecord(ev[2], st), "cudaEventRecord");
        // field and tag averages for every (source, frequency) case at once
        k_rep.resize(ns * nf);
        for (int sv = 0; sv < n_src; ++sv)
            for (int f = 0; f < nf; ++f) k_rep[(size_t)sv * nf + f] = k_re[f0 + f];
        const size_t fs = (size_t)nf * std::max(1, n_obs);
        float *fr = dfld, *fi = dfld + ns * fs;
        if (rc == HBEM_OK && n_obs > 0)
            rc = launch_field(*s, n_src * nf, k_rep.data(), xr, xi, (long long)n, qr, qi, (long long)T, dobs, n_obs, fr,
                              fi, (long long)n_obs, st);
        if (rc == HBEM_OK && n_tags > 0) rc = launch_tag_avg(*s, n_src * nf, xr, xi, (long long)n, dwant, n_tags, dtag, st);
        if (rc != HBEM_OK) break;
        // join the condition estimate before the next chunk reuses the factors' buffer
        if (rcond) ok(cudaStreamWaitEvent(st, s->aux_join, 0), "join");
        ok(cudaEventRecord(ev[3], st), "cudaEventRecord");
        for (int sv = 0; sv < n_src; ++sv) {
            const size_t hf = (size_t)sv * n_freq + f0;   // first host case of this source in the chunk
            if (n_obs > 0) {
                ok(cudaMemcpyAsync(field_re + hf * n_obs, fr + sv * fs, sizeof(float) * nf * n_obs,
                                   cudaMemcpyDeviceToHost, st), "field");
                ok(cudaMemcpyAsync(field_im + hf * n_obs, fi + sv * fs, sizeof(float) * nf * n_obs,
                                   cudaMemcpyDeviceToHost, st), "field");
            }
            if (n_tags > 0)
                ok(cudaMemcpyAsync(tag_avg + hf * n_tags * 2, dtag + (size_t)sv * nf * n_tags * 2,
                                   2 * sizeof(double) * nf * n_tags, cudaMemcpyDeviceToHost, st), "tag averages");
            if (surface_re) {
                ok(cudaMemcpyAsync(surface_re + hf * n, xr + sv * xs, sizeof(float) * xs, cudaMemcpyDeviceToHost, st),
                   "surface");
                ok(cudaMemcpyAsync(surface_im + hf * n, xi + sv * xs, sizeof(float) * xs, cudaMemcpyDeviceToHost, st),
                   "surface");
            }
            if (do_refine && refine_iters)
                ok(cudaMemcpyAsync(refine_iters + hf, diters + (size_t)sv * nf, sizeof(int) * nf,
                                   cudaMemcpyDeviceToHost, st), "iters");
            if (do_refine && refine_resid)
                ok(cudaMemcpyAsync(refine_resid + hf, dres + (size_t)sv * nf, sizeof(double) * nf,
                                   cudaMemcpyDeviceToHost, st), "resid");
        }
        ok(cudaMemcpyAsync(info + f0, dinfo, sizeof(int) * nf, cudaMemcpyDeviceToHost, st), "info");
        if (rcond) ok(cudaMemcpyAsync(rcond + f0, drcond, sizeof(double) * nf, cudaMemcpyDeviceToHost, st), "rcond");
        ok(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        if (rc != HBEM_OK) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[0], ev[1]); t_asm += ms;
        cudaEventElapsedTime(&ms, ev[1], ev[2]); t_solve += ms;
        cudaEventElapsedTime(&ms, ev[2], ev[3]); t_field += ms;
    }
    if (rc == HBEM_OK) {
        cudaEventRecord(ev[0], st);
        cudaStreamSynchronize(st);
        cudaEventElapsedTime(&t_total, ev[4], ev[0]);
        rc = wave_fault_check(st);
    }
    if (rc == HBEM_OK) {
        if (!do_refine) {
            if (refine_iters) std::memset(refine_iters, 0, sizeof(int) * ns * n_freq);
            if (refine_resid) std::memset(refine_resid, 0, sizeof(double) * ns * n_freq);
        }
        if (timings_ms) {
            timings_ms[0] = t_asm;
            timings_ms[1] = t_solve;
            timings_ms[2] = t_field;
            timings_ms[3] = t_total;
        }
    } else {
        cudaStreamSynchronize(st);
        if (s->aux) cudaStreamSynchronize(s->aux);
    }
    for (auto &e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

extern "C" int hbem_solve_batch(hbem_session *h, int n_freq, const float *k_re, const float *k_im, const float *q_re,
                                const float *q_im, const float *obs_3xn, int n_obs, const int *tags, int n_tags,
                                int precision, double refine_tol, int refine_max_iter, float *field_re,
                                float *field_im, double *tag_avg, float *surface_re, float *surface_im, int *info,
                                int *refine_iters, double *refine_resid, double *rcond, float *timings_ms,
                                void *stream) {
    return solve_batch_impl(h, n_freq, 1, k_re, k_im, q_re, q_im, obs_3xn, n_obs, tags, n_tags, precision, refine_tol,
                            refine_max_iter, field_re, field_im, tag_avg, surface_re, surface_im, info, refine_iters,
                            refine_resid, rcond, timings_ms, stream);
}

extern "C" int hbem_solve_batch_multi(hbem_session *h, int n_freq, int n_src, const float *k_re, const float *k_im,
                                      const float *q_re, const float *q_im, const float *obs_3xn, int n_obs,
                                      const int *tags, int n_tags, int precision, double refine_tol,
                                      int refine_max_iter, float *field_re, float *field_im, double *tag_avg,
                                      float *surface_re, float *surface_im, int *info, int *refine_iters,
                                      double *refine_resid, double *rcond, float *timings_ms, void *stream) {
    return solve_batch_impl(h, n_freq, n_src, k_re, k_im, q_re, q_im, obs_3xn, n_obs, tags, n_tags, precision,
                            refine_tol, refine_max_iter, field_re, field_im, tag_avg, surface_re, surface_im, info,
                            refine_iters, refine_resid, rcond, timings_ms, stream);
}
