// Near-field subdivision of the regular quadrature (the reference's optional
// near quadrature: HORNLAB_METAL_BEM_NATIVE_NEAR_QUADRATURE, main.swift:
// 2410-2560 pair list, 2840-2912 subdivided blocks, 3072-3202 correction).
//
// Triangle pairs that are close but share no vertex (centroid distance under
// threshold x the longer of their longest edges) are poorly served by the
// 6 x 6 Dunavant rule.  For every such (test image, trial image) pair the
// correction (subdivided block - regular block) is added to A and the
// right-hand sides at weight 1 (the enumeration over image masks carries the
// symmetry factor), with the Robin coupling, as the Duffy corrections are.
//
// Device side: one warp per (near pair, wavenumber).  Lanes stride over the
// (6 4^L)^2 point pairs of the subdivided rule and the 36 regular point pairs
// (negated weights), each lane keeping FP32 sums of the 3 SLP rows and 9 DLP
// entries; the warp totals are formed in FP64 before the single rounding into
// A and b.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <unordered_map>
#include <vector>

#include "hbem_internal.h"

namespace hbem {
namespace {

constexpr int kNearMaxFreq = 64;
constexpr int kNearMaxSources = 8;

struct NearArgs {
    const int4 *pairs;
    const float4 *rule;      // subdivided rule: (xi, eta, w, 0)
    const float *verts;
    const int *tris;
    const int *l2g;
    const float *areas;
    const float *normals;
    const float *q_re, *q_im, *beta_re, *beta_im;
    float *a_re, *a_im, *b_re, *b_im;
    long long q_stride, q_src_stride, lda, a_stride, b_stride, b_src_stride;
    int V, T, n_pairs, n_sub, n_src;
    float k[kNearMaxFreq], kt[kNearMaxFreq], ki[kNearMaxFreq];
};

__device__ __forceinline__ float nqx(int q) {
    return q == 0 ? HBEM_QX0 : q == 1 ? HBEM_QX1 : q == 2 ? HBEM_QX2 : q == 3 ? HBEM_QX3 : q == 4 ? HBEM_QX4 : HBEM_QX5;
}
__device__ __forceinline__ float nqy(int q) {
    return q == 0 ? HBEM_QY0 : q == 1 ? HBEM_QY1 : q == 2 ? HBEM_QY2 : q == 3 ? HBEM_QY3 : q == 4 ? HBEM_QY4 : HBEM_QY5;
}
__device__ __forceinline__ float nqw(int q) { return (q == 0 || q == 2 || q == 3) ? HBEM_QWA : HBEM_QWB; }
__device__ __forceinline__ float round_turn(float t) {
    const float big = 12582912.0f;   // 1.5 * 2^23: adding and removing it rounds |t| < 2^22
    return __fsub_rn(__fadd_rn(t, big), big);
}

// G and dG/dn_y without the 1/(4 pi) factor (applied once per block), k = k + i ki:
// G = e^{i k r} e^{-ki r} / r, D = G (i k - ki - 1/r) ((y - x) . n) / r; r^2 <= 1e-14 adds nothing.
__device__ __forceinline__ void near_sample(float dx, float dy, float dz, float nx, float ny, float nz, float k,
                                            float kt, float ki, float &gre, float &gim, float &dre, float &dim) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float u = rsqrtf(r2);
    u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    float t = r * kt;
    t -= round_turn(t);
    float sn, cs;
    __sincosf(t * 6.28318530717958647692f, &sn, &cs);
    float g = u, fre = -u;
    if (ki != 0.f) {
        g *= __expf(-ki * r);
        fre -= ki;
    }
    gre = g * cs;
    gim = g * sn;
    const float proj = fmaf(dx, nx, fmaf(dy, ny, dz * nz)) * u;
    dre = (gre * fre - gim * k) * proj;
    dim = (gre * k + gim * fre) * proj;
}

__global__ void __launch_bounds__(256) k_near(const __grid_constant__ NearArgs p) {
    const int lane = threadIdx.x & 31;
    const int pi = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (pi >= p.n_pairs) return;
    const int f = blockIdx.y;
    const int4 pr = p.pairs[pi];
    const int test = pr.x, trial = pr.y, tm = pr.z, sm = pr.w;
    const int V = p.V, T = p.T;
    float P[3][3], S[3][3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int vt = p.tris[l * T + test], vs = p.tris[l * T + trial];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P[l][c] = p.verts[c * V + vt];
            S[l][c] = p.verts[c * V + vs];
        }
    }
    const float ts[3] = {(tm & 1) ? -1.f : 1.f, (tm & 2) ? -1.f : 1.f, (tm & 4) ? -1.f : 1.f};
    const float ss[3] = {(sm & 1) ? -1.f : 1.f, (sm & 2) ? -1.f : 1.f, (sm & 4) ? -1.f : 1.f};
    const bool tswap = __popc(tm) & 1, sswap = __popc(sm) & 1;
    const float nx = ss[0] * p.normals[trial], ny = ss[1] * p.normals[T + trial], nz = ss[2] * p.normals[2 * T + trial];
    const float k = p.k[f], kt = p.kt[f], ki = p.ki[f];
    float acc[24];
#pragma unroll
    for (int e = 0; e < 24; ++e) acc[e] = 0.f;
    const int s2 = p.n_sub * p.n_sub;
    for (int idx = lane; idx < s2 + 36; idx += 32) {
        float txi, teta, sxi, seta, w;
        if (idx < s2) {
            const int a = idx / p.n_sub, b = idx - a * p.n_sub;
            const float4 ra = __ldg(&p.rule[a]), rb = __ldg(&p.rule[b]);
            txi = ra.x; teta = ra.y; sxi = rb.x; seta = rb.y;
            w = ra.z * rb.z;
        } else {
            const int rq = idx - s2, a = rq / 6, b = rq - 6 * (rq / 6);
            txi = nqx(a); teta = nqy(a); sxi = nqx(b); seta = nqy(b);
            w = -(nqw(a) * nqw(b));
        }
        // image reference coordinates -> the original triangle's (an odd mirror reverses local order)
        if (tswap) { const float t = txi; txi = teta; teta = t; }
        if (sswap) { const float t = sxi; sxi = seta; seta = t; }
        const float tb[3] = {1.f - txi - teta, txi, teta}, sb[3] = {1.f - sxi - seta, sxi, seta};
        float d[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float x = ts[c] * (tb[0] * P[0][c] + tb[1] * P[1][c] + tb[2] * P[2][c]);
            const float y = ss[c] * (sb[0] * S[0][c] + sb[1] * S[1][c] + sb[2] * S[2][c]);
            d[c] = y - x;
        }
        float gre, gim, dre, dim;
        near_sample(d[0], d[1], d[2], nx, ny, nz, k, kt, ki, gre, gim, dre, dim);
        gre *= w; gim *= w; dre *= w; dim *= w;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            acc[2 * i] = fmaf(gre, tb[i], acc[2 * i]);
            acc[2 * i + 1] = fmaf(gim, tb[i], acc[2 * i + 1]);
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const float er = dre * sb[j], ei = dim * sb[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                acc[6 + 2 * (3 * i + j)] = fmaf(er, tb[i], acc[6 + 2 * (3 * i + j)]);
                acc[7 + 2 * (3 * i + j)] = fmaf(ei, tb[i], acc[7 + 2 * (3 * i + j)]);
            }
        }
    }
    // warp totals in FP64; every lane ends with all of them
    double v[24];
#pragma unroll
    for (int e = 0; e < 24; ++e) {
        v[e] = acc[e];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[e] += __shfl_xor_sync(0xffffffffu, v[e], o);
    }
    if (lane >= 12) return;
    const double scale = (double)HBEM_INV4PI * (2.0 * (double)p.areas[test]) * (2.0 * (double)p.areas[trial]);
    const int i_row = lane < 9 ? lane / 3 : lane - 9;
    double sr = 0.0, si = 0.0;   // SLP delta of this lane's row
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (i == i_row) { sr = v[2 * i] * scale; si = v[2 * i + 1] * scale; }
    const int row = p.l2g[test * 3 + i_row];
    if (lane < 9) {
        const int j = lane - 3 * (lane / 3);
        double dr = 0.0, di = 0.0;
#pragma unroll
        for (int e = 0; e < 9; ++e)
            if (e == lane) { dr = v[6 + 2 * e] * scale; di = v[7 + 2 * e] * scale; }
        const float br = p.beta_re ? p.beta_re[trial] : 0.f, bi = p.beta_im ? p.beta_im[trial] : 0.f;
        if (br != 0.f || bi != 0.f) {   // - (1/3) (i k beta) delta_SLP, k = k + i ki
            const double ikb_re = -(double)ki * br - (double)k * bi, ikb_im = -(double)ki * bi + (double)k * br;
            dr -= (sr * ikb_re - si * ikb_im) / 3.0;
            di -= (sr * ikb_im + si * ikb_re) / 3.0;
        }
        const size_t o = (size_t)f * p.a_stride + (size_t)row * p.lda + p.l2g[trial * 3 + j];
        atomicAdd(p.a_re + o, (float)dr);
        atomicAdd(p.a_im + o, (float)di);
    } else if (p.q_re && p.b_re) {
        for (int sv = 0; sv < p.n_src; ++sv) {
            const size_t oq = (size_t)sv * p.q_src_stride + (size_t)f * p.q_stride + trial;
            const float qr = p.q_re[oq], qi = p.q_im[oq];
            if (qr == 0.f && qi == 0.f) continue;
            const size_t o = (size_t)sv * p.b_src_stride + (size_t)f * p.b_stride + row;
            atomicAdd(p.b_re + o, (float)(sr * qr - si * qi));
            atomicAdd(p.b_im + o, (float)(sr * qi + si * qr));
        }
    }
}

// Bounding box, centroid and longest edge of a triangle image.
struct NearMetric {
    double c[3], lo[3], hi[3], edge;
};

NearMetric near_metric(const Session &s, int t, int mask) {
    const int V = s.n_vertices, T = s.n_triangles;
    double p[3][3];
    for (int l = 0; l < 3; ++l) {
        const int v = s.tris[(size_t)l * T + t];
        for (int c = 0; c < 3; ++c) {
            const double sg = (mask >> c) & 1 ? -1.0 : 1.0;
            p[l][c] = sg * (double)s.verts[(size_t)c * V + v];
        }
    }
    NearMetric m{};
    double e2 = 0.0;
    for (int c = 0; c < 3; ++c) {
        m.c[c] = (p[0][c] + p[1][c] + p[2][c]) / 3.0;
        m.lo[c] = std::min(p[0][c], std::min(p[1][c], p[2][c]));
        m.hi[c] = std::max(p[0][c], std::max(p[1][c], p[2][c]));
    }
    for (int a = 0; a < 3; ++a) {
        const int b = (a + 1) % 3;
        double d2 = 0.0;
        for (int c = 0; c < 3; ++c) d2 += (p[a][c] - p[b][c]) * (p[a][c] - p[b][c]);
        e2 = std::max(e2, d2);
    }
    m.edge = std::sqrt(e2);
    return m;
}

double gap(double alo, double ahi, double blo, double bhi) {
    if (ahi < blo) return blo - ahi;
    if (bhi < alo) return alo - bhi;
    return 0.0;
}

// Near, non-touching image pairs (test, trial, test mask, trial mask), sorted
// by trial, trial mask, test mask, test (main.swift:2471-2556).  Candidates
// come from a uniform grid of test-image centroids whose cell is the largest
// possible cutoff, so only the 27 neighbouring cells are searched.
std::vector<int4> build_near_pairs(const Session &s, double threshold) {
    const int T = s.n_triangles;
    std::vector<int> masks{0};
    if (s.sym == 1) masks.push_back(1);
    else if (s.sym == 2) masks.push_back(2);
    else if (s.sym == 4) masks.push_back(4);
    else if (s.sym == 3) { masks.push_back(1); masks.push_back(2); masks.push_back(3); }
    const int nm = (int)masks.size();
    std::vector<NearMetric> mt((size_t)nm * T);
    double emax = 0.0;
    for (int mi = 0; mi < nm; ++mi)
        for (int t = 0; t < T; ++t) {
            mt[(size_t)mi * T + t] = near_metric(s, t, masks[mi]);
            emax = std::max(emax, mt[(size_t)mi * T + t].edge);
        }
    const double h = std::max(threshold * emax, 1e-30);
    auto cell = [&](const double *c, int dx, int dy, int dz) {
        const long long ix = (long long)std::floor(c[0] / h) + dx, iy = (long long)std::floor(c[1] / h) + dy,
                        iz = (long long)std::floor(c[2] / h) + dz;
        return (unsigned long long)((ix & 0x1FFFFF) | ((iy & 0x1FFFFF) << 21) | ((iz & 0x1FFFFF) << 42));
    };
    std::vector<std::unordered_map<unsigned long long, std::vector<int>>> grid(nm);
    for (int mi = 0; mi < nm; ++mi)
        for (int t = 0; t < T; ++t) grid[mi][cell(mt[(size_t)mi * T + t].c, 0, 0, 0)].push_back(t);
    std::vector<int4> out;
    std::vector<int> cand;
    for (int trial = 0; trial < T; ++trial)
        for (int si = 0; si < nm; ++si) {
            const NearMetric &sm = mt[(size_t)si * T + trial];
            for (int ti = 0; ti < nm; ++ti) {
                cand.clear();
                for (int dx = -1; dx <= 1; ++dx)
                    for (int dy = -1; dy <= 1; ++dy)
                        for (int dz = -1; dz <= 1; ++dz) {
                            auto it = grid[ti].find(cell(sm.c, dx, dy, dz));
                            if (it != grid[ti].end()) cand.insert(cand.end(), it->second.begin(), it->second.end());
                        }
                std::sort(cand.begin(), cand.end());
                for (int test : cand) {
                    const NearMetric &tm = mt[(size_t)ti * T + test];
                    const double cut = threshold * std::max(tm.edge, sm.edge), cut2 = cut * cut;
                    const double gx = gap(tm.lo[0], tm.hi[0], sm.lo[0], sm.hi[0]);
                    const double gy = gap(tm.lo[1], tm.hi[1], sm.lo[1], sm.hi[1]);
                    const double gz = gap(tm.lo[2], tm.hi[2], sm.lo[2], sm.hi[2]);
                    if (gx * gx + gy * gy + gz * gz > cut2) continue;
                    const double dx = tm.c[0] - sm.c[0], dy = tm.c[1] - sm.c[1], dz = tm.c[2] - sm.c[2];
                    if (dx * dx + dy * dy + dz * dz >= cut2) continue;
                    if (image_shared_vertices(s, test, trial, masks[ti], masks[si]) > 0) continue;
                    out.push_back(make_int4(test, trial, masks[ti], masks[si]));
                }
            }
        }
    return out;
}

// The 6-point Dunavant rule on each sub-triangle of `level` midpoint
// subdivisions (4^level sub-triangles, the reference's order), weights
// scaled by the sub-triangle's area ratio.
std::vector<float4> subdivided_rule(int level) {
    static const double QX[6] = {0.4459484909159651, 0.0915762135097710, 0.1081030181680700,
                                 0.4459484909159651, 0.8168475729804590, 0.0915762135097710};
    static const double QY[6] = {0.4459484909159651, 0.0915762135097700, 0.4459484909159651,
                                 0.1081030181680700, 0.0915762135097700, 0.8168475729804580};
    static const double QW[6] = {0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.2233815896780110,
                                 0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.1099517436553220};
    std::vector<std::array<double, 6>> subs{{0.0, 0.0, 1.0, 0.0, 0.0, 1.0}};
    for (int l = 0; l < level; ++l) {
        std::vector<std::array<double, 6>> next;
        for (const auto &t : subs) {
            const double ab[2] = {0.5 * (t[0] + t[2]), 0.5 * (t[1] + t[3])};
            const double bc[2] = {0.5 * (t[2] + t[4]), 0.5 * (t[3] + t[5])};
            const double ca[2] = {0.5 * (t[4] + t[0]), 0.5 * (t[5] + t[1])};
            next.push_back({t[0], t[1], ab[0], ab[1], ca[0], ca[1]});
            next.push_back({ab[0], ab[1], t[2], t[3], bc[0], bc[1]});
            next.push_back({ca[0], ca[1], bc[0], bc[1], t[4], t[5]});
            next.push_back({ab[0], ab[1], bc[0], bc[1], ca[0], ca[1]});
        }
        subs.swap(next);
    }
    std::vector<float4> rule;
    for (const auto &t : subs) {
        const double det = std::fabs((t[2] - t[0]) * (t[5] - t[1]) - (t[3] - t[1]) * (t[4] - t[0]));
        for (int q = 0; q < 6; ++q)
            rule.push_back(make_float4((float)(t[0] + QX[q] * (t[2] - t[0]) + QY[q] * (t[4] - t[0])),
                                       (float)(t[1] + QX[q] * (t[3] - t[1]) + QY[q] * (t[5] - t[1])),
                                       (float)(QW[q] * det), 0.f));
    }
    return rule;
}

}  // namespace

int launch_near(Session &s, int n_freq, const float *k_re, const float *k_im, int n_src, const float *q_re,
                const float *q_im, long long q_stride, long long q_src_stride, const float *beta_re,
                const float *beta_im, float *a_re, float *a_im, long long lda, long long a_stride, float *b_re,
                float *b_im, long long b_stride, long long b_src_stride, cudaStream_t st) {
    if (s.n_near <= 0) return HBEM_OK;
    if (n_src < 1 || n_src > kNearMaxSources) return fail(HBEM_ERR_ARG, "near-field correction: 1 .. 8 sources");
    for (int f0 = 0; f0 < n_freq; f0 += kNearMaxFreq) {
        const int nf = std::min(kNearMaxFreq, n_freq - f0);
        NearArgs a{};
        a.pairs = s.d_near;
        a.rule = s.d_subrule;
        a.verts = s.d_verts; a.tris = s.d_tris; a.l2g = s.d_l2g; a.areas = s.d_areas; a.normals = s.d_normals;
        a.q_re = (q_re && b_re) ? q_re + (size_t)f0 * q_stride : nullptr;
        a.q_im = (q_im && b_re) ? q_im + (size_t)f0 * q_stride : nullptr;
        a.beta_re = beta_re; a.beta_im = beta_im;
        a.a_re = a_re + (size_t)f0 * a_stride; a.a_im = a_im + (size_t)f0 * a_stride;
        a.b_re = b_re ? b_re + (size_t)f0 * b_stride : nullptr;
        a.b_im = b_im ? b_im + (size_t)f0 * b_stride : nullptr;
        a.q_stride = q_stride; a.q_src_stride = q_src_stride; a.lda = lda; a.a_stride = a_stride;
        a.b_stride = b_stride; a.b_src_stride = b_src_stride;
        a.V = s.n_vertices; a.T = s.n_triangles; a.n_pairs = s.n_near; a.n_sub = s.n_sub; a.n_src = n_src;
        for (int f = 0; f < nf; ++f) {
            a.k[f] = k_re[f0 + f];
            a.kt[f] = (float)((double)k_re[f0 + f] / (2.0 * 3.14159265358979323846));
            a.ki[f] = k_im ? k_im[f0 + f] : 0.f;
        }
        k_near<<<dim3((s.n_near + 7) / 8, nf), 256, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k_near");
        ++s.launches;
    }
    return HBEM_OK;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_session_set_near_quadrature(hbem_session *h, int level, double threshold) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_session_set_near_quadrature: NULL session");
    if (level < 0 || level > 2)
        return fail(HBEM_ERR_ARG, "hbem_session_set_near_quadrature: level must be 0 (off), 1 or 2");
    if (level > 0 && !(threshold > 0.0 && std::isfinite(threshold)))
        return fail(HBEM_ERR_ARG, "hbem_session_set_near_quadrature: threshold must be finite and positive");
    HBEM_CUDA(cudaSetDevice(s->device));
    if (s->d_near) cudaFree(s->d_near);
    if (s->d_subrule) cudaFree(s->d_subrule);
    s->d_near = nullptr;
    s->d_subrule = nullptr;
    s->n_near = s->n_sub = 0;
    s->near_level = 0;
    s->near_threshold = 0.0;
    if (level == 0) return HBEM_OK;
    const std::vector<int4> pairs = build_near_pairs(*s, threshold);
    const std::vector<float4> rule = subdivided_rule(level);
    if (!pairs.empty()) {
        HBEM_CUDA(cudaMalloc((void **)&s->d_near, sizeof(int4) * pairs.size()));
        HBEM_CUDA(cudaMemcpy(s->d_near, pairs.data(), sizeof(int4) * pairs.size(), cudaMemcpyHostToDevice));
        HBEM_CUDA(cudaMalloc((void **)&s->d_subrule, sizeof(float4) * rule.size()));
        HBEM_CUDA(cudaMemcpy(s->d_subrule, rule.data(), sizeof(float4) * rule.size(), cudaMemcpyHostToDevice));
    }
    s->n_near = (int)pairs.size();
    s->n_sub = (int)rule.size();
    s->near_level = level;
    s->near_threshold = threshold;
    return HBEM_OK;
}
