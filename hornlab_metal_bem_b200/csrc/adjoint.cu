// Adjoint (reverse-mode) of the discrete forward map
//   vertices -> (A, b) -> p = A^-1 b -> exterior field F = Fp p + Fq q
// for the shape gradient of a real objective L(F).  With g = dL/dRe F +
// i dL/dIm F per observation point (torch's convention for complex outputs):
//   g_p    = Fp^H g                         (hbem_field_adjoint)
//   lambda = A^-H g_p                       (hbem_lu_solve, HBEM_TRANS_C, reusing the factors)
//   dL/dX  = Re g^H dF/dX |_p               (hbem_field_backward)
//          - Re lambda^H (dA/dX) p + Re lambda^H (db/dX)   (hbem_assemble_backward)
// Nothing of size dA/dX is stored: every kernel recomputes its quadrature
// samples and contracts them on the fly with the adjoint weights.
//
// Every term of the forward has the form, per quadrature sample (x, y) with
// weight w (reference-coordinate weight, geometry independent),
//   w J_tau [ u_p s(r) (d . N) + u_q J_sigma G(r) ],   d = y - x,
// where N = (Y1 - Y0) x (Y2 - Y0) is the trial triangle's area normal
// (|N| = J_sigma = 2 area), J_tau the test Jacobian (1 for an observation
// point), G = e^{ikr} / r, s = G' / r, and u_p, u_q complex adjoint weights:
//   assembly: u_p = -Lambda(x) P(y), u_q = Lambda(x) q_sigma with
//             Lambda(x) = sum_i conj(lambda_i) phi_i(x), P(y) = sum_j p_j phi_j(y)
//   field:    u_p = conj(g_o) P(y),  u_q = -conj(g_o) q_sigma.
// Its derivatives (real parts summed over frequencies):
//   dF/dd = [u_p s' (d.N) / r + u_q J s] d + [u_p s] N,   dF/dN = [u_p s] d,
//   dF/dJ_sigma = u_q G,   s' = e^{ikr} (3/r - k^2 r - 3ik) / r^3,
// then x, y move with the barycentric weights of their sample and N, J with
// the edge cross products.  The quadrature (6-point Dunavant for far pairs,
// the Duffy rules for touching pairs, the mass term -1/2 M) is exactly the
// forward's, so the result is the exact derivative of the discrete forward
// (main.swift:3443-3480 kernels, 4090-4120 pair assembly, 4246-4431 Duffy).
// Real wavenumbers and sessions without symmetry planes only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "hbem_internal.h"

namespace hbem {
namespace {

constexpr int kBwdTest = 32;
constexpr int kBwdTrial = 64;
constexpr int kBwdThreads = 256;
constexpr int kBwdMaxF = 16;        // frequencies staged per launch
constexpr float kTwoPi = 6.28318530717958647692f;

__device__ __forceinline__ float bqx(int q) {
    return q == 0 ? HBEM_QX0 : q == 1 ? HBEM_QX1 : q == 2 ? HBEM_QX2 : q == 3 ? HBEM_QX3 : q == 4 ? HBEM_QX4 : HBEM_QX5;
}
__device__ __forceinline__ float bqy(int q) {
    return q == 0 ? HBEM_QY0 : q == 1 ? HBEM_QY1 : q == 2 ? HBEM_QY2 : q == 3 ? HBEM_QY3 : q == 4 ? HBEM_QY4 : HBEM_QY5;
}
__device__ __forceinline__ float bqw(int q) { return (q == 0 || q == 2 || q == 3) ? HBEM_QWA : HBEM_QWB; }

__device__ __forceinline__ float rnd(float t) {
    const float big = 12582912.0f;
    return __fsub_rn(__fadd_rn(t, big), big);
}

struct Freqs {
    float k[kBwdMaxF];
    float kt[kBwdMaxF];   // k / (2 pi)
};

// Running sums of one (test, trial) pair or one sample set.
struct PairAcc {
    float gx[3][3];   // d/dX of the test triangle's vertices (or unused for observation points)
    float gy[3][3];   // d/dY of the trial triangle's vertices through y
    float gn[3];      // d/dN
    float gjs;        // d/dJ_sigma
    float gjt;        // d/dJ_tau
};

__device__ __forceinline__ void acc_zero(PairAcc &a) {
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) a.gx[l][c] = a.gy[l][c] = 0.f;
    a.gn[0] = a.gn[1] = a.gn[2] = 0.f;
    a.gjs = a.gjt = 0.f;
}

// One geometric sample: d = y - x, trial area normal N (|N| = js), test
// barycentrics tb, trial barycentrics sb, weight w (includes J_tau's
// reference weight but not J_tau), jt = J_tau.  up/uq: per-frequency complex
// adjoint weights, provided by a functor uw(f, up_re, up_im, uq_re, uq_im).
template <typename UW>
__device__ __forceinline__ void bwd_sample(PairAcc &acc, float dx, float dy, float dz, const float (&N)[3], float js,
                                           const float (&tb)[3], const float (&sb)[3], float w, float jt,
                                           const Freqs &fq, int nf, UW uw) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if (!(r2 > 1.0e-14f)) return;
    const float u1 = rsqrtf(r2);
    const float r = r2 * u1;
    const float u3 = u1 * u1 * u1;
    const float dn = fmaf(dx, N[0], fmaf(dy, N[1], dz * N[2]));
    float Ad = 0.f, An = 0.f, Aj = 0.f, Af = 0.f;
    for (int f = 0; f < nf; ++f) {
        const float k = fq.k[f];
        float t = r * fq.kt[f];
        t -= rnd(t);
        float sn, cs;
        __sincosf(t * kTwoPi, &sn, &cs);
        const float kr = k * r;
        // s = E (-1 + i k r) / r^3, s' = E (3/r - k^2 r - 3ik) / r^3, G = E / r
        const float s_re = u3 * (-cs - sn * kr), s_im = u3 * (-sn + cs * kr);
        const float a = 3.f * u1 - k * kr, bb = 3.f * k;
        const float sp_re = u3 * (cs * a + sn * bb), sp_im = u3 * (sn * a - cs * bb);
        const float g_re = u1 * cs, g_im = u1 * sn;
        float up_re, up_im, uq_re, uq_im;
        uw(f, up_re, up_im, uq_re, uq_im);
        const float ups = up_re * s_re - up_im * s_im;        // Re(u_p s)
        const float upsp = up_re * sp_re - up_im * sp_im;     // Re(u_p s')
        const float uqs = uq_re * s_re - uq_im * s_im;        // Re(u_q s)
        const float uqg = uq_re * g_re - uq_im * g_im;        // Re(u_q G)
        An += ups;
        Ad = fmaf(upsp, dn * u1, fmaf(js, uqs, Ad));
        Aj += uqg;
        Af = fmaf(ups, dn, fmaf(js, uqg, Af));
    }
    const float W = w * jt;
    const float gd[3] = {W * fmaf(Ad, dx, An * N[0]), W * fmaf(Ad, dy, An * N[1]), W * fmaf(Ad, dz, An * N[2])};
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            acc.gx[l][c] = fmaf(-tb[l], gd[c], acc.gx[l][c]);
            acc.gy[l][c] = fmaf(sb[l], gd[c], acc.gy[l][c]);
        }
    const float wn = W * An;
    acc.gn[0] = fmaf(wn, dx, acc.gn[0]);
    acc.gn[1] = fmaf(wn, dy, acc.gn[1]);
    acc.gn[2] = fmaf(wn, dz, acc.gn[2]);
    acc.gjs = fmaf(W, Aj, acc.gjs);
    acc.gjt = fmaf(w, Af, acc.gjt);
}

// d/dV of a scalar through N = (V1 - V0) x (V2 - V0) given g = d/dN:
// dV1 = e2 x g, dV2 = g x e1, dV0 = -(dV1 + dV2).
__device__ __forceinline__ void normal_to_vertices(const float (&V)[3][3], const float (&g)[3], float (&out)[3][3]) {
    const float e1[3] = {V[1][0] - V[0][0], V[1][1] - V[0][1], V[1][2] - V[0][2]};
    const float e2[3] = {V[2][0] - V[0][0], V[2][1] - V[0][1], V[2][2] - V[0][2]};
    out[1][0] = e2[1] * g[2] - e2[2] * g[1];
    out[1][1] = e2[2] * g[0] - e2[0] * g[2];
    out[1][2] = e2[0] * g[1] - e2[1] * g[0];
    out[2][0] = g[1] * e1[2] - g[2] * e1[1];
    out[2][1] = g[2] * e1[0] - g[0] * e1[2];
    out[2][2] = g[0] * e1[1] - g[1] * e1[0];
#pragma unroll
    for (int c = 0; c < 3; ++c) out[0][c] = -(out[1][c] + out[2][c]);
}

__device__ __forceinline__ void area_normal(const float (&V)[3][3], float (&N)[3], float &J) {
    const float e1[3] = {V[1][0] - V[0][0], V[1][1] - V[0][1], V[1][2] - V[0][2]};
    const float e2[3] = {V[2][0] - V[0][0], V[2][1] - V[0][1], V[2][2] - V[0][2]};
    N[0] = e1[1] * e2[2] - e1[2] * e2[1];
    N[1] = e1[2] * e2[0] - e1[0] * e2[2];
    N[2] = e1[0] * e2[1] - e1[1] * e2[0];
    J = sqrtf(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
}

// Fold N / J_sigma / J_tau sums into per-vertex gradients.
__device__ __forceinline__ void finish_pair(const PairAcc &acc, const float (&TV)[3][3], const float (&SV)[3][3],
                                            const float (&N)[3], float js, float (&gt)[3][3], float (&gs)[3][3],
                                            bool with_test) {
    const float ijs = js > 0.f ? 1.f / js : 0.f;
    const float gN[3] = {fmaf(acc.gjs * ijs, N[0], acc.gn[0]), fmaf(acc.gjs * ijs, N[1], acc.gn[1]),
                         fmaf(acc.gjs * ijs, N[2], acc.gn[2])};
    float dS[3][3];
    normal_to_vertices(SV, gN, dS);
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) gs[l][c] = acc.gy[l][c] + dS[l][c];
    if (with_test) {
        float Nt[3], jt;
        area_normal(TV, Nt, jt);
        const float s = jt > 0.f ? acc.gjt / jt : 0.f;
        const float g[3] = {s * Nt[0], s * Nt[1], s * Nt[2]};
        float dT[3][3];
        normal_to_vertices(TV, g, dT);
#pragma unroll
        for (int l = 0; l < 3; ++l)
#pragma unroll
            for (int c = 0; c < 3; ++c) gt[l][c] = acc.gx[l][c] + dT[l][c];
    }
}

struct BwdArgs {
    const float *verts;   // (3, V)
    const int *tris;      // (3, T)
    const int *l2g;       // (T, 3)
    const float *lam_re, *lam_im;   // (F, n) adjoint
    const float *p_re, *p_im;       // (F, n) surface pressure
    const float *q_re, *q_im;       // (F, T) Neumann data
    long long lam_stride, p_stride, q_stride;
    const unsigned *sing;           // T x T bitmap of Duffy (touching) pairs
    double *grad;                   // (3, V), accumulated
    int V, T, nf;
    Freqs fq;
};

// ---------------------------------------------------------------------------
// Regular pairs: 32 test x 64 trial triangles per CTA, thread (lane, warp)
// takes test lane and trial warp + 8 j, all staged frequencies per sample.
// Touching pairs are skipped (their Duffy rule replaces the regular rule).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kBwdThreads) k_asm_bwd(const __grid_constant__ BwdArgs a) {
    extern __shared__ float sh[];
    const int nf = a.nf;
    float *sL = sh;                                        // [f][q][test][2]
    float *sP = sL + (size_t)nf * 6 * kBwdTest * 2;        // [f][q][trial][2]
    float *sQ = sP + (size_t)nf * 6 * kBwdTrial * 2;       // [f][trial][2]
    __shared__ float sTV[kBwdTest][9], sSV[kBwdTrial][9];
    __shared__ float gT[kBwdTest][9], gS[kBwdTrial][9];
    const int T = a.T, V = a.V;
    const int t0 = blockIdx.y * kBwdTest, s0 = blockIdx.x * kBwdTrial;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int e = tid; e < kBwdTest * 9; e += kBwdThreads) {
        const int i = e / 9, lc = e - 9 * i, l = lc / 3, c = lc - 3 * l;
        const int t = t0 + i;
        sTV[i][lc] = t < T ? a.verts[(size_t)c * V + a.tris[(size_t)l * T + t]] : 0.f;
        gT[i][lc] = 0.f;
    }
    for (int e = tid; e < kBwdTrial * 9; e += kBwdThreads) {
        const int i = e / 9, lc = e - 9 * i, l = lc / 3, c = lc - 3 * l;
        const int t = s0 + i;
        sSV[i][lc] = t < T ? a.verts[(size_t)c * V + a.tris[(size_t)l * T + t]] : 0.f;
        gS[i][lc] = 0.f;
    }
    for (int e = tid; e < nf * 6 * kBwdTest; e += kBwdThreads) {
        const int f = e / (6 * kBwdTest), rem = e - f * 6 * kBwdTest, q = rem / kBwdTest, i = rem - q * kBwdTest;
        const int t = t0 + i;
        float lr = 0.f, li = 0.f;
        if (t < T) {
            const float b[3] = {1.f - bqx(q) - bqy(q), bqx(q), bqy(q)};
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const int d = a.l2g[(size_t)t * 3 + l];
                lr = fmaf(b[l], a.lam_re[(size_t)f * a.lam_stride + d], lr);
                li = fmaf(-b[l], a.lam_im[(size_t)f * a.lam_stride + d], li);   // conj(lambda)
            }
        }
        sL[2 * e] = lr;
        sL[2 * e + 1] = li;
    }
    for (int e = tid; e < nf * 6 * kBwdTrial; e += kBwdThreads) {
        const int f = e / (6 * kBwdTrial), rem = e - f * 6 * kBwdTrial, q = rem / kBwdTrial, i = rem - q * kBwdTrial;
        const int t = s0 + i;
        float pr = 0.f, pi = 0.f;
        if (t < T) {
            const float b[3] = {1.f - bqx(q) - bqy(q), bqx(q), bqy(q)};
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                const int d = a.l2g[(size_t)t * 3 + l];
                pr = fmaf(b[l], a.p_re[(size_t)f * a.p_stride + d], pr);
                pi = fmaf(b[l], a.p_im[(size_t)f * a.p_stride + d], pi);
            }
        }
        sP[2 * e] = pr;
        sP[2 * e + 1] = pi;
    }
    for (int e = tid; e < nf * kBwdTrial; e += kBwdThreads) {
        const int f = e / kBwdTrial, i = e - f * kBwdTrial;
        const int t = s0 + i;
        sQ[2 * e] = t < T && a.q_re ? a.q_re[(size_t)f * a.q_stride + t] : 0.f;
        sQ[2 * e + 1] = t < T && a.q_im ? a.q_im[(size_t)f * a.q_stride + t] : 0.f;
    }
    __syncthreads();
    const int ti = lane;
    const int tt = t0 + ti;
    if (tt < T) {
        float TV[3][3];
#pragma unroll
        for (int l = 0; l < 3; ++l)
#pragma unroll
            for (int c = 0; c < 3; ++c) TV[l][c] = sTV[ti][3 * l + c];
        float Nt[3], jt;
        area_normal(TV, Nt, jt);
        for (int si = warp; si < kBwdTrial; si += kBwdThreads / 32) {
            const int st = s0 + si;
            if (st >= T) break;
            const size_t bit = (size_t)tt * T + st;
            if ((a.sing[bit >> 5] >> (bit & 31)) & 1u) continue;
            float SV[3][3];
#pragma unroll
            for (int l = 0; l < 3; ++l)
#pragma unroll
                for (int c = 0; c < 3; ++c) SV[l][c] = sSV[si][3 * l + c];
            float N[3], js;
            area_normal(SV, N, js);
            PairAcc acc;
            acc_zero(acc);
            for (int qa = 0; qa < 6; ++qa) {
                const float tb[3] = {1.f - bqx(qa) - bqy(qa), bqx(qa), bqy(qa)};
                float x[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) x[c] = tb[0] * TV[0][c] + tb[1] * TV[1][c] + tb[2] * TV[2][c];
                const float wa = bqw(qa);
#pragma unroll 1
                for (int qb = 0; qb < 6; ++qb) {
                    const float sb[3] = {1.f - bqx(qb) - bqy(qb), bqx(qb), bqy(qb)};
                    float y[3];
#pragma unroll
                    for (int c = 0; c < 3; ++c) y[c] = sb[0] * SV[0][c] + sb[1] * SV[1][c] + sb[2] * SV[2][c];
                    auto uw = [&](int f, float &upr, float &upi, float &uqr, float &uqi) {
                        const float lr = sL[2 * ((f * 6 + qa) * kBwdTest + ti)];
                        const float li = sL[2 * ((f * 6 + qa) * kBwdTest + ti) + 1];
                        const float pr = sP[2 * ((f * 6 + qb) * kBwdTrial + si)];
                        const float pi = sP[2 * ((f * 6 + qb) * kBwdTrial + si) + 1];
                        const float qr = sQ[2 * (f * kBwdTrial + si)], qi = sQ[2 * (f * kBwdTrial + si) + 1];
                        upr = -(lr * pr - li * pi);
                        upi = -(lr * pi + li * pr);
                        uqr = lr * qr - li * qi;
                        uqi = lr * qi + li * qr;
                    };
                    bwd_sample(acc, y[0] - x[0], y[1] - x[1], y[2] - x[2], N, js, tb, sb, wa * bqw(qb), jt, a.fq, nf, uw);
                }
            }
            float gt[3][3], gs[3][3];
            finish_pair(acc, TV, SV, N, js, gt, gs, true);
#pragma unroll
            for (int l = 0; l < 3; ++l)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    atomicAdd(&gT[ti][3 * l + c], gt[l][c]);
                    atomicAdd(&gS[si][3 * l + c], gs[l][c]);
                }
        }
    }
    __syncthreads();
    for (int e = tid; e < kBwdTest * 9; e += kBwdThreads) {
        const int i = e / 9, lc = e - 9 * i, l = lc / 3, c = lc - 3 * l;
        const int t = t0 + i;
        if (t < T && gT[i][lc] != 0.f)
            atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + t], (double)gT[i][lc] * HBEM_INV4PI);
    }
    for (int e = tid; e < kBwdTrial * 9; e += kBwdThreads) {
        const int i = e / 9, lc = e - 9 * i, l = lc / 3, c = lc - 3 * l;
        const int t = s0 + i;
        if (t < T && gS[i][lc] != 0.f)
            atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + t], (double)gS[i][lc] * HBEM_INV4PI);
    }
}

// ---------------------------------------------------------------------------
// Touching pairs: one warp per Duffy pair, lanes over the rule's points (the
// forward's remapped Sauter-Schwab points and weights).
// ---------------------------------------------------------------------------
struct DuffyBwdArgs {
    BwdArgs b;
    const DuffyPair *pairs;
    const float4 *rule;
    const float *rule_w;
    int n_pairs;
    int rule_off[3], rule_cnt[3];
};

__device__ __forceinline__ float drefx(int l) { return l == 1 ? 1.f : 0.f; }
__device__ __forceinline__ float drefy(int l) { return l == 2 ? 1.f : 0.f; }
__device__ __forceinline__ void dremap(float x, float y, int kind, int l1, int l2, float &ox, float &oy) {
    if (kind == 2) {
        const int vc = 3 - l1 - l2;
        const float ax = drefx(l1), ay = drefy(l1);
        ox = ax + x * (drefx(l2) - ax) + y * (drefx(vc) - ax);
        oy = ay + x * (drefy(l2) - ay) + y * (drefy(vc) - ay);
    } else if (kind == 3 && l1 == 1) {
        ox = 1.f - x - y;
        oy = y;
    } else if (kind == 3 && l1 == 2) {
        ox = x;
        oy = 1.f - x - y;
    } else {
        ox = x;
        oy = y;
    }
}

__global__ void __launch_bounds__(256) k_duffy_bwd(const __grid_constant__ DuffyBwdArgs d) {
    const BwdArgs &a = d.b;
    const int lane = threadIdx.x & 31;
    const int pi = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (pi >= d.n_pairs) return;
    const DuffyPair pr = d.pairs[pi];
    const int T = a.T, V = a.V, nf = a.nf;
    float TV[3][3], SV[3][3];
    int td[3], sd[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int vt = a.tris[(size_t)l * T + pr.test], vs = a.tris[(size_t)l * T + pr.trial];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            TV[l][c] = a.verts[(size_t)c * V + vt];
            SV[l][c] = a.verts[(size_t)c * V + vs];
        }
        td[l] = a.l2g[(size_t)pr.test * 3 + l];
        sd[l] = a.l2g[(size_t)pr.trial * 3 + l];
    }
    float N[3], js, Nt[3], jt;
    area_normal(SV, N, js);
    area_normal(TV, Nt, jt);
    PairAcc acc;
    acc_zero(acc);
    const int ri = pr.kind - 1;
    const int off = d.rule_off[ri], cnt = d.rule_cnt[ri];
    for (int q = lane; q < cnt; q += 32) {
        const float4 r = __ldg(&d.rule[off + q]);
        const float w = __ldg(&d.rule_w[off + q]);
        float tx, ty, sx, sy;
        dremap(r.x, r.y, pr.kind, pr.tl1, pr.tl2, tx, ty);
        dremap(r.z, r.w, pr.kind, pr.sl1, pr.sl2, sx, sy);
        const float tb[3] = {1.f - tx - ty, tx, ty};
        const float sb[3] = {1.f - sx - sy, sx, sy};
        float x[3], y[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[c] = tb[0] * TV[0][c] + tb[1] * TV[1][c] + tb[2] * TV[2][c];
            y[c] = sb[0] * SV[0][c] + sb[1] * SV[1][c] + sb[2] * SV[2][c];
        }
        auto uw = [&](int f, float &upr, float &upi, float &uqr, float &uqi) {
            float lr = 0.f, li = 0.f, pr_ = 0.f, pi_ = 0.f;
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                lr = fmaf(tb[l], a.lam_re[(size_t)f * a.lam_stride + td[l]], lr);
                li = fmaf(-tb[l], a.lam_im[(size_t)f * a.lam_stride + td[l]], li);
                pr_ = fmaf(sb[l], a.p_re[(size_t)f * a.p_stride + sd[l]], pr_);
                pi_ = fmaf(sb[l], a.p_im[(size_t)f * a.p_stride + sd[l]], pi_);
            }
            const float qr = a.q_re ? a.q_re[(size_t)f * a.q_stride + pr.trial] : 0.f;
            const float qi = a.q_im ? a.q_im[(size_t)f * a.q_stride + pr.trial] : 0.f;
            upr = -(lr * pr_ - li * pi_);
            upi = -(lr * pi_ + li * pr_);
            uqr = lr * qr - li * qi;
            uqi = lr * qi + li * qr;
        };
        bwd_sample(acc, y[0] - x[0], y[1] - x[1], y[2] - x[2], N, js, tb, sb, w, jt, a.fq, nf, uw);
    }
    // warp reduction of the 23 sums (FP32 lanes, reduced in FP64)
    float *flat = &acc.gx[0][0];
    double red[23];
#pragma unroll
    for (int e = 0; e < 23; ++e) {
        double v = (double)flat[e];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        red[e] = v;
    }
    if (lane == 0) {
#pragma unroll
        for (int e = 0; e < 23; ++e) flat[e] = (float)red[e];
        float gt[3][3], gs[3][3];
        finish_pair(acc, TV, SV, N, js, gt, gs, true);
        const double sc = (double)HBEM_INV4PI * (double)pr.weight;
#pragma unroll
        for (int l = 0; l < 3; ++l)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + pr.test], sc * gt[l][c]);
                atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + pr.trial], sc * gs[l][c]);
            }
    }
}

// Mass term -1/2 M of A: dL/dX += 1/2 Re sum_ij conj(lambda_i) p_j c_ij d|tau|/dX,
// c_ii = 1/6, c_ij = 1/12 (main.swift:4112-4120).  One thread per triangle.
__global__ void k_mass_bwd(const __grid_constant__ BwdArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.T) return;
    const int T = a.T, V = a.V;
    float TV[3][3];
    int td[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int v = a.tris[(size_t)l * T + t];
#pragma unroll
        for (int c = 0; c < 3; ++c) TV[l][c] = a.verts[(size_t)c * V + v];
        td[l] = a.l2g[(size_t)t * 3 + l];
    }
    double S = 0.0;
    for (int f = 0; f < a.nf; ++f)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double lr = a.lam_re[(size_t)f * a.lam_stride + td[i]], li = a.lam_im[(size_t)f * a.lam_stride + td[i]];
                const double pr = a.p_re[(size_t)f * a.p_stride + td[j]], pi = a.p_im[(size_t)f * a.p_stride + td[j]];
                S += (lr * pr + li * pi) * (i == j ? 1.0 / 6.0 : 1.0 / 12.0);   // Re(conj(lambda) p)
            }
    // d|tau|/dX = 1/2 dJ/dX, dJ/dN = N / J
    float N[3], J;
    area_normal(TV, N, J);
    const float s = J > 0.f ? (float)(0.25 * S) / J : 0.f;
    const float g[3] = {s * N[0], s * N[1], s * N[2]};
    float dT[3][3];
    normal_to_vertices(TV, g, dT);
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + t], (double)dT[l][c]);
}

// T x T bitmap of touching pairs from the Duffy pair list (no symmetry: masks 0).
__global__ void k_sing_bits(const DuffyPair *pairs, int n_pairs, int T, unsigned *bits) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    const DuffyPair p = pairs[i];
    const size_t b = (size_t)p.test * T + p.trial;
    atomicOr(bits + (b >> 5), 1u << (b & 31));
}

// ---------------------------------------------------------------------------
// Field adjoint and field backward.  Observation point o, trial triangle sigma.
// ---------------------------------------------------------------------------
struct FieldBwdArgs {
    const float *verts;
    const int *tris, *l2g;
    const float *obs;            // (3, n_obs)
    const float *g_re, *g_im;    // (F, n_obs) dL/dRe F + i dL/dIm F
    const float *p_re, *p_im;    // (F, n)
    const float *q_re, *q_im;    // (F, T)
    float *gp_re, *gp_im;        // (F, n) output of the adjoint
    double *grad;                // (3, V)
    long long g_stride, p_stride, q_stride;
    int V, T, n_obs, nf;
    Freqs fq;
};

// g_p = Fp^H g: thread per (triangle, frequency), loop over observation points.
__global__ void k_field_adj(const __grid_constant__ FieldBwdArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.y;
    if (t >= a.T) return;
    const int T = a.T, V = a.V;
    float SV[3][3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int v = a.tris[(size_t)l * T + t];
#pragma unroll
        for (int c = 0; c < 3; ++c) SV[l][c] = a.verts[(size_t)c * V + v];
    }
    float N[3], js;
    area_normal(SV, N, js);
    const float k = a.fq.k[f], kt = a.fq.kt[f];
    float accr[3] = {0.f, 0.f, 0.f}, acci[3] = {0.f, 0.f, 0.f};
    for (int o = 0; o < a.n_obs; ++o) {
        const float ox = a.obs[o], oy = a.obs[a.n_obs + o], oz = a.obs[2 * a.n_obs + o];
        const float gr = a.g_re[(size_t)f * a.g_stride + o], gi = a.g_im[(size_t)f * a.g_stride + o];
        for (int qb = 0; qb < 6; ++qb) {
            const float sb[3] = {1.f - bqx(qb) - bqy(qb), bqx(qb), bqy(qb)};
            const float dx = sb[0] * SV[0][0] + sb[1] * SV[1][0] + sb[2] * SV[2][0] - ox;
            const float dy = sb[0] * SV[0][1] + sb[1] * SV[1][1] + sb[2] * SV[2][1] - oy;
            const float dz = sb[0] * SV[0][2] + sb[1] * SV[1][2] + sb[2] * SV[2][2] - oz;
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (!(r2 > 1.0e-14f)) continue;
            const float u1 = rsqrtf(r2), r = r2 * u1, u3 = u1 * u1 * u1;
            float tt = r * kt;
            tt -= rnd(tt);
            float sn, cs;
            __sincosf(tt * kTwoPi, &sn, &cs);
            const float kr = k * r;
            const float dn = fmaf(dx, N[0], fmaf(dy, N[1], dz * N[2])) * bqw(qb);
            // Fp value (times 1/4 pi): w s (d.N); conj(value) * g
            const float vr = u3 * (-cs - sn * kr) * dn, vi = u3 * (-sn + cs * kr) * dn;
            const float cr = vr * gr + vi * gi, ci = vr * gi - vi * gr;
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                accr[l] = fmaf(sb[l], cr, accr[l]);
                acci[l] = fmaf(sb[l], ci, acci[l]);
            }
        }
    }
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int d = a.l2g[(size_t)t * 3 + l];
        atomicAdd(a.gp_re + (size_t)f * a.p_stride + d, accr[l] * HBEM_INV4PI);
        atomicAdd(a.gp_im + (size_t)f * a.p_stride + d, acci[l] * HBEM_INV4PI);
    }
}

// dL/dX of Re g^H F at fixed p: thread per triangle, all frequencies and points.
__global__ void k_field_bwd(const __grid_constant__ FieldBwdArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.T) return;
    const int T = a.T, V = a.V, nf = a.nf;
    float SV[3][3];
    int sd[3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int v = a.tris[(size_t)l * T + t];
#pragma unroll
        for (int c = 0; c < 3; ++c) SV[l][c] = a.verts[(size_t)c * V + v];
        sd[l] = a.l2g[(size_t)t * 3 + l];
    }
    float N[3], js;
    area_normal(SV, N, js);
    PairAcc acc;
    acc_zero(acc);
    const float tb[3] = {0.f, 0.f, 0.f};
    for (int o = 0; o < a.n_obs; ++o) {
        const float ox = a.obs[o], oy = a.obs[a.n_obs + o], oz = a.obs[2 * a.n_obs + o];
        for (int qb = 0; qb < 6; ++qb) {
            const float sb[3] = {1.f - bqx(qb) - bqy(qb), bqx(qb), bqy(qb)};
            float y[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) y[c] = sb[0] * SV[0][c] + sb[1] * SV[1][c] + sb[2] * SV[2][c];
            auto uw = [&](int f, float &upr, float &upi, float &uqr, float &uqi) {
                const float gr = a.g_re[(size_t)f * a.g_stride + o], gi = -a.g_im[(size_t)f * a.g_stride + o];  // conj(g)
                float pr = 0.f, pi = 0.f;
#pragma unroll
                for (int l = 0; l < 3; ++l) {
                    pr = fmaf(sb[l], a.p_re[(size_t)f * a.p_stride + sd[l]], pr);
                    pi = fmaf(sb[l], a.p_im[(size_t)f * a.p_stride + sd[l]], pi);
                }
                const float qr = a.q_re ? a.q_re[(size_t)f * a.q_stride + t] : 0.f;
                const float qi = a.q_im ? a.q_im[(size_t)f * a.q_stride + t] : 0.f;
                upr = gr * pr - gi * pi;
                upi = gr * pi + gi * pr;
                uqr = -(gr * qr - gi * qi);
                uqi = -(gr * qi + gi * qr);
            };
            bwd_sample(acc, y[0] - ox, y[1] - oy, y[2] - oz, N, js, tb, sb, bqw(qb), 1.f, a.fq, nf, uw);
        }
    }
    float TV[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    float gt[3][3], gs[3][3];
    finish_pair(acc, TV, SV, N, js, gt, gs, false);
#pragma unroll
    for (int l = 0; l < 3; ++l)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            atomicAdd(a.grad + (size_t)c * V + a.tris[(size_t)l * T + t], (double)gs[l][c] * HBEM_INV4PI);
}

void fill_freqs(Freqs &fq, const float *k_re, int f0, int nf) {
    for (int f = 0; f < nf; ++f) {
        fq.k[f] = k_re[f0 + f];
        fq.kt[f] = (float)((double)k_re[f0 + f] / (2.0 * 3.14159265358979323846));
    }
}

int check_adjoint_session(const Session *s, const char *who) {
    if (!s) return fail(HBEM_ERR_ARG, std::string(who) + ": NULL session");
    if (s->sym != 0) return fail(HBEM_ERR_ARG, std::string(who) + ": shape gradients need a session without symmetry planes");
    if (s->n_near > 0)
        return fail(HBEM_ERR_STATE, std::string(who) + ": shape gradients do not include the near-field subdivision; "
                                                       "turn it off (level 0)");
    return HBEM_OK;
}

}  // namespace
}  // namespace hbem

using namespace hbem;

extern "C" int hbem_session_set_vertices(hbem_session *h, const float *vertices_3xv, const float *areas,
                                         const float *normals_3xt) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_session_set_vertices: NULL session");
    if (!vertices_3xv || !areas || !normals_3xt) return fail(HBEM_ERR_ARG, "hbem_session_set_vertices: NULL pointer");
    const int T = s->n_triangles, V = s->n_vertices;
    for (int t = 0; t < T; ++t)
        if (!(areas[t] > 0.0f) || !std::isfinite(areas[t]))
            return fail(HBEM_ERR_ARG, "hbem_session_set_vertices: triangle " + std::to_string(t) + " has non-positive area");
    HBEM_CUDA(cudaSetDevice(s->device));
    s->verts.assign(vertices_3xv, vertices_3xv + 3LL * V);
    s->areas.assign(areas, areas + T);
    s->normals.assign(normals_3xt, normals_3xt + 3LL * T);
    // quadrature points and normal + jacobian, original and spatial order
    // (the same construction as at session creation; topology, tiles and
    // Duffy pairs are kept)
    static const double QX[6] = {HBEM_QX0, HBEM_QX1, HBEM_QX2, HBEM_QX3, HBEM_QX4, HBEM_QX5};
    static const double QY[6] = {HBEM_QY0, HBEM_QY1, HBEM_QY2, HBEM_QY3, HBEM_QY4, HBEM_QY5};
    std::vector<float4> qp((size_t)T * 6), nrm(T), sqp((size_t)T * 6), snrm(T);
    for (int t = 0; t < T; ++t) {
        double P[3][3];
        for (int l = 0; l < 3; ++l) {
            const int v = s->tris[(size_t)l * T + t];
            for (int c = 0; c < 3; ++c) P[l][c] = s->verts[(size_t)c * V + v];
        }
        for (int q = 0; q < 6; ++q) {
            const double b1 = 1.0 - QX[q] - QY[q], b2 = QX[q], b3 = QY[q];
            double x[3];
            for (int c = 0; c < 3; ++c) x[c] = b1 * P[0][c] + b2 * P[1][c] + b3 * P[2][c];
            qp[(size_t)t * 6 + q] = make_float4((float)x[0], (float)x[1], (float)x[2], 0.f);
        }
        nrm[t] = make_float4(s->normals[t], s->normals[T + t], s->normals[2 * T + t], 2.0f * s->areas[t]);
    }
    for (int i = 0; i < T; ++i) {
        const int t = s->order[i];
        for (int q = 0; q < 6; ++q) sqp[(size_t)i * 6 + q] = qp[(size_t)t * 6 + q];
        snrm[i] = nrm[t];
    }
    HBEM_CUDA(cudaMemcpy(s->d_qp, sqp.data(), sizeof(float4) * sqp.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_nrm, snrm.data(), sizeof(float4) * snrm.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_fqp, qp.data(), sizeof(float4) * qp.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_fnrm, nrm.data(), sizeof(float4) * nrm.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_verts, s->verts.data(), sizeof(float) * s->verts.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_areas, s->areas.data(), sizeof(float) * T, cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s->d_normals, s->normals.data(), sizeof(float) * s->normals.size(), cudaMemcpyHostToDevice));
    return HBEM_OK;
}

extern "C" int hbem_field_adjoint(hbem_session *h, int n_freq, const float *k_re, const float *obs_3xn, int n_obs,
                                  const float *g_re, const float *g_im, long long g_stride, float *gp_re, float *gp_im,
                                  long long gp_stride, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    int rc = check_adjoint_session(s, "hbem_field_adjoint");
    if (rc != HBEM_OK) return rc;
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !obs_3xn || !g_re || !g_im || !gp_re || !gp_im || n_obs <= 0)
        return fail(HBEM_ERR_ARG, "hbem_field_adjoint: NULL pointer or no observation points");
    if (g_stride < n_obs || gp_stride < s->n_dof) return fail(HBEM_ERR_ARG, "hbem_field_adjoint: bad strides");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    HBEM_CUDA(cudaMemset2DAsync(gp_re, gp_stride * sizeof(float), 0, s->n_dof * sizeof(float), n_freq, st));
    HBEM_CUDA(cudaMemset2DAsync(gp_im, gp_stride * sizeof(float), 0, s->n_dof * sizeof(float), n_freq, st));
    for (int f0 = 0; f0 < n_freq; f0 += kBwdMaxF) {
        const int nf = std::min(kBwdMaxF, n_freq - f0);
        FieldBwdArgs a{};
        a.verts = s->d_verts; a.tris = s->d_tris; a.l2g = s->d_l2g; a.obs = obs_3xn;
        a.g_re = g_re + (size_t)f0 * g_stride; a.g_im = g_im + (size_t)f0 * g_stride;
        a.gp_re = gp_re + (size_t)f0 * gp_stride; a.gp_im = gp_im + (size_t)f0 * gp_stride;
        a.g_stride = g_stride; a.p_stride = gp_stride;
        a.V = s->n_vertices; a.T = s->n_triangles; a.n_obs = n_obs; a.nf = nf;
        fill_freqs(a.fq, k_re, f0, nf);
        k_field_adj<<<dim3((s->n_triangles + 127) / 128, nf), 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k_field_adj");
    }
    return HBEM_OK;
}

extern "C" int hbem_field_backward(hbem_session *h, int n_freq, const float *k_re, const float *obs_3xn, int n_obs,
                                   const float *g_re, const float *g_im, long long g_stride, const float *p_re,
                                   const float *p_im, long long p_stride, const float *q_re, const float *q_im,
                                   long long q_stride, double *grad_3xv, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    int rc = check_adjoint_session(s, "hbem_field_backward");
    if (rc != HBEM_OK) return rc;
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !obs_3xn || !g_re || !g_im || !p_re || !p_im || !grad_3xv || n_obs <= 0)
        return fail(HBEM_ERR_ARG, "hbem_field_backward: NULL pointer or no observation points");
    if (g_stride < n_obs || p_stride < s->n_dof || ((q_re || q_im) && q_stride < s->n_triangles))
        return fail(HBEM_ERR_ARG, "hbem_field_backward: bad strides");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (int f0 = 0; f0 < n_freq; f0 += kBwdMaxF) {
        const int nf = std::min(kBwdMaxF, n_freq - f0);
        FieldBwdArgs a{};
        a.verts = s->d_verts; a.tris = s->d_tris; a.l2g = s->d_l2g; a.obs = obs_3xn;
        a.g_re = g_re + (size_t)f0 * g_stride; a.g_im = g_im + (size_t)f0 * g_stride;
        a.p_re = p_re + (size_t)f0 * p_stride; a.p_im = p_im + (size_t)f0 * p_stride;
        a.q_re = q_re ? q_re + (size_t)f0 * q_stride : nullptr; a.q_im = q_im ? q_im + (size_t)f0 * q_stride : nullptr;
        a.grad = grad_3xv; a.g_stride = g_stride; a.p_stride = p_stride; a.q_stride = q_stride;
        a.V = s->n_vertices; a.T = s->n_triangles; a.n_obs = n_obs; a.nf = nf;
        fill_freqs(a.fq, k_re, f0, nf);
        k_field_bwd<<<(s->n_triangles + 127) / 128, 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k_field_bwd");
    }
    return HBEM_OK;
}

extern "C" int hbem_assemble_backward(hbem_session *h, int n_freq, const float *k_re, const float *k_im,
                                      const float *lam_re, const float *lam_im, long long lam_stride,
                                      const float *p_re, const float *p_im, long long p_stride, const float *q_re,
                                      const float *q_im, long long q_stride, double *grad_3xv, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    int rc = check_adjoint_session(s, "hbem_assemble_backward");
    if (rc != HBEM_OK) return rc;
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !lam_re || !lam_im || !p_re || !p_im || !grad_3xv)
        return fail(HBEM_ERR_ARG, "hbem_assemble_backward: NULL pointer");
    if (k_im)
        for (int f = 0; f < n_freq; ++f)
            if (k_im[f] != 0.f) return fail(HBEM_ERR_ARG, "hbem_assemble_backward: complex wavenumbers are not supported");
    const int T = s->n_triangles, V = s->n_vertices, n = s->n_dof;
    if (lam_stride < n || p_stride < n || ((q_re || q_im) && q_stride < T))
        return fail(HBEM_ERR_ARG, "hbem_assemble_backward: bad strides");
    HBEM_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // touching-pair bitmap, built once per session
    if (!s->d_sing_bits) {
        const size_t words = ((size_t)T * T + 31) / 32;
        HBEM_CUDA(cudaMalloc((void **)&s->d_sing_bits, words * sizeof(unsigned)));
        HBEM_CUDA(cudaMemsetAsync(s->d_sing_bits, 0, words * sizeof(unsigned), st));
        if (s->n_pairs > 0) {
            k_sing_bits<<<(s->n_pairs + 255) / 256, 256, 0, st>>>(s->d_pairs, s->n_pairs, T, s->d_sing_bits);
            HBEM_LAUNCH_CHECK("k_sing_bits");
        }
    }
    {
        const int rc = func_opt_in((const void *)k_asm_bwd, 200 * 1024);
        if (rc != HBEM_OK) return rc;
    }
    for (int f0 = 0; f0 < n_freq; f0 += kBwdMaxF) {
        const int nf = std::min(kBwdMaxF, n_freq - f0);
        BwdArgs a{};
        a.verts = s->d_verts; a.tris = s->d_tris; a.l2g = s->d_l2g;
        a.lam_re = lam_re + (size_t)f0 * lam_stride; a.lam_im = lam_im + (size_t)f0 * lam_stride;
        a.p_re = p_re + (size_t)f0 * p_stride; a.p_im = p_im + (size_t)f0 * p_stride;
        a.q_re = q_re ? q_re + (size_t)f0 * q_stride : nullptr; a.q_im = q_im ? q_im + (size_t)f0 * q_stride : nullptr;
        a.lam_stride = lam_stride; a.p_stride = p_stride; a.q_stride = q_stride;
        a.sing = s->d_sing_bits; a.grad = grad_3xv; a.V = V; a.T = T; a.nf = nf;
        fill_freqs(a.fq, k_re, f0, nf);
        const size_t smem = sizeof(float) * (size_t)nf * (6 * kBwdTest * 2 + 6 * kBwdTrial * 2 + kBwdTrial * 2);
        dim3 grid((T + kBwdTrial - 1) / kBwdTrial, (T + kBwdTest - 1) / kBwdTest);
        k_asm_bwd<<<grid, kBwdThreads, smem, st>>>(a);
        HBEM_LAUNCH_CHECK("k_asm_bwd");
        if (s->n_pairs > 0) {
            DuffyBwdArgs d{};
            d.b = a; d.pairs = s->d_pairs; d.rule = s->d_rule; d.rule_w = s->d_rule_w; d.n_pairs = s->n_pairs;
            for (int i = 0; i < 3; ++i) { d.rule_off[i] = s->rule_off[i]; d.rule_cnt[i] = s->rule_cnt[i]; }
            k_duffy_bwd<<<(s->n_pairs + 7) / 8, 256, 0, st>>>(d);
            HBEM_LAUNCH_CHECK("k_duffy_bwd");
        }
        k_mass_bwd<<<(T + 127) / 128, 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k_mass_bwd");
    }
    return HBEM_OK;
}
