// FP64 path on the GPU: double-precision corrected assembly, exterior field and
// a complex128 LU with its solve.
//
// Two uses:
//  * the accuracy statement of every FP32 result: the same discretisation
//    (6-point Dunavant rule on far pairs, the 4^4-point Duffy rules on touching
//    pairs, images, row weight, mass and Robin terms: main.swift:1726-1841,
//    2974-3070, 1843-1895) evaluated in double precision from the session's
//    float32 geometry, so the difference to the FP32 path is arithmetic error
//    only;
//  * dense_solve_dtype = "float64": the reference widens the FP32-assembled
//    system to complex128 and calls zgesv (main.swift:7101-7185); here the
//    widened system is factored by hbem_lu_factor_f64 and solved by
//    hbem_lu_solve_f64.
//
// Assembly is written for clarity over speed (it states errors, it is not the
// hot path): one thread per (test triangle, trial triangle) pair with its
// images, one thread per Duffy pair, double atomics into A and b.
//
// LU: blocked right-looking, 32-column panels, partial pivoting with the first
// maximum of |re| + |im| (LAPACK izamax).  Per panel column two launches over
// many CTAs (pivot search with a last-block reduction, then scale and rank-1
// update of the panel's remaining columns; no CTA waits on another), then the
// row interchanges outside the panel, the unit-lower triangular solve for the
// block row of U, and the trailing update on the CUDA cores' FP64 pipe.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "hbem_internal.h"

namespace hbem {
namespace {

__constant__ double c64_qx[6] = {0.4459484909159651, 0.0915762135097710, 0.1081030181680700,
                                 0.4459484909159651, 0.8168475729804590, 0.0915762135097710};
__constant__ double c64_qy[6] = {0.4459484909159651, 0.0915762135097700, 0.4459484909159651,
                                 0.1081030181680700, 0.0915762135097700, 0.8168475729804580};
__constant__ double c64_qw[6] = {0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.2233815896780110,
                                 0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.1099517436553220};
constexpr double kInv4Pi = 0.07957747154594767;
constexpr int kMaxF64 = 32;    // wavenumbers per assembly / field launch

// G = e^{ikr} / (4 pi r) and dG/dn_y = G (ik - 1/r) ((y - x) . n) / r for
// k = kr + i ki, added to the running sums; r = 0 adds nothing.
__device__ __forceinline__ void green_dlp(double dx, double dy, double dz, double nx, double ny, double nz, double kr,
                                          double ki, double &gre, double &gim, double &dre, double &dim) {
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= 0.0) return;
    const double r = sqrt(r2);
    double s = kInv4Pi / r;
    if (ki != 0.0) s *= exp(-ki * r);
    double sn, cs;
    sincos(kr * r, &sn, &cs);
    const double g_re = cs * s, g_im = sn * s;
    const double proj = (dx * nx + dy * ny + dz * nz) / r;
    const double fre = -1.0 / r - ki, fim = kr;
    gre += g_re;
    gim += g_im;
    dre += (g_re * fre - g_im * fim) * proj;
    dim += (g_re * fim + g_im * fre) * proj;
}

__device__ __forceinline__ void mirror3(double &x, double &y, double &z, int mask) {
    if (mask & 1) x = -x;
    if (mask & 2) y = -y;
    if (mask & 4) z = -z;
}

// point on triangle t at reference coordinates (xi, eta): (1 - xi - eta) P0 + xi P1 + eta P2
__device__ __forceinline__ void point_on(const double *__restrict__ tv, int t, double xi, double eta, double &x,
                                         double &y, double &z) {
    const double *P = tv + (size_t)t * 9;
    const double b1 = 1.0 - xi - eta;
    x = b1 * P[0] + xi * P[3] + eta * P[6];
    y = b1 * P[1] + xi * P[4] + eta * P[7];
    z = b1 * P[2] + xi * P[5] + eta * P[8];
}

struct Geo64 {
    const double *tv;    // (T, 3 vertices, xyz)
    const double *nrm;   // (T, 4): normal, area
    const int *l2g;      // (T, 3)
    int T, sym;
    int masks[3], n_masks;
    double rw;           // 2^planes row weight
};

struct Asm64Args {
    Geo64 g;
    const double *q_re, *q_im, *beta_re, *beta_im;
    long long q_stride;
    double *a_re, *a_im, *b_re, *b_im;
    long long lda, a_stride, b_stride;
    int nf;
    double kr[kMaxF64], ki[kMaxF64];
};

// Regular 6 x 6 quadrature of every (test, trial) pair with the trial's images
// (main.swift:1726-1841).  Grid: x = trial chunks of 128, y = test triangles
// (strided), z = wavenumber.
__global__ void __launch_bounds__(128) k64_regular(const __grid_constant__ Asm64Args p) {
    const Geo64 &g = p.g;
    const int f = blockIdx.z;
    const double kr = p.kr[f], ki = p.ki[f];
    __shared__ double s_tp[6][3];
    for (int test = blockIdx.y; test < g.T; test += gridDim.y) {
        __syncthreads();
        if (threadIdx.x < 6) {
            const int a = threadIdx.x;
            point_on(g.tv, test, c64_qx[a], c64_qy[a], s_tp[a][0], s_tp[a][1], s_tp[a][2]);
        }
        __syncthreads();
        const int trial = blockIdx.x * blockDim.x + threadIdx.x;
        if (trial >= g.T) continue;
        const double nx = g.nrm[4 * trial], ny = g.nrm[4 * trial + 1], nz = g.nrm[4 * trial + 2];
        const double jac = (2.0 * g.nrm[4 * test + 3]) * (2.0 * g.nrm[4 * trial + 3]);
        double blk_re[9], blk_im[9], slp_re[3], slp_im[3];
#pragma unroll
        for (int i = 0; i < 9; ++i) blk_re[i] = blk_im[i] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i) slp_re[i] = slp_im[i] = 0.0;
        for (int a = 0; a < 6; ++a) {
            const double tb[3] = {1.0 - c64_qx[a] - c64_qy[a], c64_qx[a], c64_qy[a]};
            const double tx = s_tp[a][0], ty = s_tp[a][1], tz = s_tp[a][2];
            for (int b = 0; b < 6; ++b) {
                double sx, sy, sz;
                point_on(g.tv, trial, c64_qx[b], c64_qy[b], sx, sy, sz);
                const double sb[3] = {1.0 - c64_qx[b] - c64_qy[b], c64_qx[b], c64_qy[b]};
                const double w = c64_qw[a] * c64_qw[b] * jac;
                double gre = 0, gim = 0, dre = 0, dim = 0;
                green_dlp(sx - tx, sy - ty, sz - tz, nx, ny, nz, kr, ki, gre, gim, dre, dim);
                for (int m = 0; m < g.n_masks; ++m) {
                    double ix = sx, iy = sy, iz = sz, jx = nx, jy = ny, jz = nz;
                    mirror3(ix, iy, iz, g.masks[m]);
                    mirror3(jx, jy, jz, g.masks[m]);
                    green_dlp(ix - tx, iy - ty, iz - tz, jx, jy, jz, kr, ki, gre, gim, dre, dim);
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    slp_re[i] += gre * (tb[i] * w);
                    slp_im[i] += gim * (tb[i] * w);
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        blk_re[i * 3 + j] += dre * (tb[i] * sb[j] * w);
                        blk_im[i * 3 + j] += dim * (tb[i] * sb[j] * w);
                    }
                }
            }
        }
        const double q_re = p.q_re ? p.q_re[(size_t)f * p.q_stride + trial] : 0.0;
        const double q_im = p.q_im ? p.q_im[(size_t)f * p.q_stride + trial] : 0.0;
        const double be_re = p.beta_re ? p.beta_re[trial] : 0.0, be_im = p.beta_im ? p.beta_im[trial] : 0.0;
        const bool robin = be_re != 0.0 || be_im != 0.0;
        // i k beta with k = kr + i ki: (-ki + i kr)(be_re + i be_im)
        const double rc_re = -ki * be_re - kr * be_im, rc_im = -ki * be_im + kr * be_re;
        double *are = p.a_re + (size_t)f * p.a_stride, *aim = p.a_im + (size_t)f * p.a_stride;
        for (int i = 0; i < 3; ++i) {
            const int row = g.l2g[test * 3 + i];
            if (p.b_re && (q_re != 0.0 || q_im != 0.0)) {
                atomicAdd(p.b_re + (size_t)f * p.b_stride + row, (slp_re[i] * q_re - slp_im[i] * q_im) * g.rw);
                atomicAdd(p.b_im + (size_t)f * p.b_stride + row, (slp_re[i] * q_im + slp_im[i] * q_re) * g.rw);
            }
            for (int j = 0; j < 3; ++j) {
                const int col = g.l2g[trial * 3 + j];
                double t_re = blk_re[i * 3 + j], t_im = blk_im[i * 3 + j];
                if (robin) {
                    t_re -= (slp_re[i] * rc_re - slp_im[i] * rc_im) * (1.0 / 3.0);
                    t_im -= (slp_re[i] * rc_im + slp_im[i] * rc_re) * (1.0 / 3.0);
                }
                if (test == trial) t_re -= 0.5 * g.nrm[4 * test + 3] * (i == j ? 1.0 / 6.0 : 1.0 / 12.0);
                atomicAdd(are + (size_t)row * p.lda + col, t_re * g.rw);
                atomicAdd(aim + (size_t)row * p.lda + col, t_im * g.rw);
            }
        }
    }
}

struct Duffy64Args {
    Asm64Args a;
    const DuffyPair *pairs;
    int n_pairs;
    const double *rule;   // 5 doubles per point: test (xi, eta), trial (xi, eta), weight
    int rule_off[3], rule_cnt[3];
};

__device__ __forceinline__ double refx(int l) { return l == 1 ? 1.0 : 0.0; }
__device__ __forceinline__ double refy(int l) { return l == 2 ? 1.0 : 0.0; }

// Place a rule point of a touching pair on the shared edge / vertex
// (main.swift:2701-2725): l1, l2 are the image-local ids of the shared vertices.
__device__ __forceinline__ void remap(double x, double y, int kind, int l1, int l2, double &ox, double &oy) {
    if (kind == 1) {
        ox = x;
        oy = y;
    } else if (kind == 2) {
        const int vc = 3 - l1 - l2;
        const double ax = refx(l1), ay = refy(l1), bx = refx(l2), by = refy(l2), cx = refx(vc), cy = refy(vc);
        ox = ax + x * (bx - ax) + y * (cx - ax);
        oy = ay + x * (by - ay) + y * (cy - ay);
    } else if (l1 == 0) {
        ox = x;
        oy = y;
    } else if (l1 == 1) {
        ox = 1.0 - x - y;
        oy = y;
    } else {
        ox = x;
        oy = 1.0 - x - y;
    }
}

// One point pair of a (test image, trial image) block, given in image
// reference coordinates: an odd mirror reverses local order, so the original
// triangle's coordinates swap (main.swift:2131-2136).
__device__ __forceinline__ void pair_point(const Geo64 &g, int test, int trial, int tm, int sm, double txi, double teta,
                                           double sxi, double seta, double w, double nx, double ny, double nz,
                                           double kr, double ki, double (&s_re)[3], double (&s_im)[3],
                                           double (&d_re)[9], double (&d_im)[9]) {
    if (__popc(tm) & 1) { const double t = txi; txi = teta; teta = t; }
    if (__popc(sm) & 1) { const double t = sxi; sxi = seta; seta = t; }
    double tx, ty, tz, sx, sy, sz;
    point_on(g.tv, test, txi, teta, tx, ty, tz);
    mirror3(tx, ty, tz, tm);
    point_on(g.tv, trial, sxi, seta, sx, sy, sz);
    mirror3(sx, sy, sz, sm);
    double gre = 0, gim = 0, dre = 0, dim = 0;
    green_dlp(sx - tx, sy - ty, sz - tz, nx, ny, nz, kr, ki, gre, gim, dre, dim);
    gre *= w; gim *= w; dre *= w; dim *= w;
    const double tb[3] = {1.0 - txi - teta, txi, teta}, sb[3] = {1.0 - sxi - seta, sxi, seta};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        s_re[i] += gre * tb[i];
        s_im[i] += gim * tb[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            d_re[i * 3 + j] += dre * (tb[i] * sb[j]);
            d_im[i * 3 + j] += dim * (tb[i] * sb[j]);
        }
    }
}

// Duffy correction (singular rule minus regular 6 x 6) of every touching pair
// (main.swift:2974-3070), weight 2 on folded exact image twins.
// Grid: x = pair chunks of 128, y = wavenumber.
__global__ void __launch_bounds__(128) k64_duffy(const __grid_constant__ Duffy64Args p) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= p.n_pairs) return;
    const Geo64 &g = p.a.g;
    const int f = blockIdx.y;
    const double kr = p.a.kr[f], ki = p.a.ki[f];
    const DuffyPair pr = p.pairs[pi];
    double nx = g.nrm[4 * pr.trial], ny = g.nrm[4 * pr.trial + 1], nz = g.nrm[4 * pr.trial + 2];
    mirror3(nx, ny, nz, pr.trial_mask);
    const double jac = (2.0 * g.nrm[4 * pr.test + 3]) * (2.0 * g.nrm[4 * pr.trial + 3]);
    double rs_re[3] = {0, 0, 0}, rs_im[3] = {0, 0, 0}, rd_re[9], rd_im[9];
    double ss_re[3] = {0, 0, 0}, ss_im[3] = {0, 0, 0}, sd_re[9], sd_im[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) rd_re[i] = rd_im[i] = sd_re[i] = sd_im[i] = 0.0;
    for (int a = 0; a < 6; ++a)
        for (int b = 0; b < 6; ++b)
            pair_point(g, pr.test, pr.trial, pr.test_mask, pr.trial_mask, c64_qx[a], c64_qy[a], c64_qx[b], c64_qy[b],
                       c64_qw[a] * c64_qw[b] * jac, nx, ny, nz, kr, ki, rs_re, rs_im, rd_re, rd_im);
    const int kind = pr.kind;
    const double *rule = p.rule + 5 * (size_t)p.rule_off[kind - 1];
    const int cnt = p.rule_cnt[kind - 1];
    for (int q = 0; q < cnt; ++q) {
        const double *r = rule + 5 * q;
        double tx, ty, sx, sy;
        remap(r[0], r[1], kind, pr.tl1, pr.tl2, tx, ty);
        remap(r[2], r[3], kind, pr.sl1, pr.sl2, sx, sy);
        pair_point(g, pr.test, pr.trial, pr.test_mask, pr.trial_mask, tx, ty, sx, sy, r[4] * jac, nx, ny, nz, kr, ki,
                   ss_re, ss_im, sd_re, sd_im);
    }
    const double wgt = (double)pr.weight;
    const double q_re = p.a.q_re ? p.a.q_re[(size_t)f * p.a.q_stride + pr.trial] : 0.0;
    const double q_im = p.a.q_im ? p.a.q_im[(size_t)f * p.a.q_stride + pr.trial] : 0.0;
    const double be_re = p.a.beta_re ? p.a.beta_re[pr.trial] : 0.0;
    const double be_im = p.a.beta_im ? p.a.beta_im[pr.trial] : 0.0;
    const bool robin = be_re != 0.0 || be_im != 0.0;
    const double rc_re = -ki * be_re - kr * be_im, rc_im = -ki * be_im + kr * be_re;
    double *are = p.a.a_re + (size_t)f * p.a.a_stride, *aim = p.a.a_im + (size_t)f * p.a.a_stride;
    for (int i = 0; i < 3; ++i) {
        const int row = g.l2g[pr.test * 3 + i];
        const double ds_re = ss_re[i] - rs_re[i], ds_im = ss_im[i] - rs_im[i];
        if (p.a.b_re && (q_re != 0.0 || q_im != 0.0)) {
            atomicAdd(p.a.b_re + (size_t)f * p.a.b_stride + row, (ds_re * q_re - ds_im * q_im) * wgt);
            atomicAdd(p.a.b_im + (size_t)f * p.a.b_stride + row, (ds_re * q_im + ds_im * q_re) * wgt);
        }
        for (int j = 0; j < 3; ++j) {
            const int col = g.l2g[pr.trial * 3 + j];
            double d_re = sd_re[i * 3 + j] - rd_re[i * 3 + j], d_im = sd_im[i * 3 + j] - rd_im[i * 3 + j];
            if (robin) {
                d_re -= (ds_re * rc_re - ds_im * rc_im) * (1.0 / 3.0);
                d_im -= (ds_re * rc_im + ds_im * rc_re) * (1.0 / 3.0);
            }
            atomicAdd(are + (size_t)row * p.a.lda + col, d_re * wgt);
            atomicAdd(aim + (size_t)row * p.a.lda + col, d_im * wgt);
        }
    }
}

struct Field64Args {
    Geo64 g;
    const double *p_re, *p_im, *q_re, *q_im;
    long long p_stride, q_stride;
    const float *obs;
    int n_obs;
    double *out_re, *out_im;
    long long out_stride;
    double kr[kMaxF64];
};

// Exterior field p(x) = sum_tri sum_a w [dG/dn_y p(y_a) - G q_tri] with images,
// real wavenumber (main.swift:1843-1895).  One CTA per (observation point,
// wavenumber), threads over triangles, FP64 block reduction.
__global__ void __launch_bounds__(256) k64_field(const __grid_constant__ Field64Args p) {
    const Geo64 &g = p.g;
    const int o = blockIdx.x, f = blockIdx.y;
    const double kr = p.kr[f];
    const double ox = p.obs[o], oy = p.obs[p.n_obs + o], oz = p.obs[2 * p.n_obs + o];
    const double *pr = p.p_re + (size_t)f * p.p_stride, *pim = p.p_im + (size_t)f * p.p_stride;
    double acc_re = 0.0, acc_im = 0.0;
    for (int tri = threadIdx.x; tri < g.T; tri += blockDim.x) {
        const double nx = g.nrm[4 * tri], ny = g.nrm[4 * tri + 1], nz = g.nrm[4 * tri + 2];
        const double jac = 2.0 * g.nrm[4 * tri + 3];
        const double qv_re = p.q_re[(size_t)f * p.q_stride + tri], qv_im = p.q_im[(size_t)f * p.q_stride + tri];
        double pv_re[3], pv_im[3];
        for (int l = 0; l < 3; ++l) {
            const int d = g.l2g[tri * 3 + l];
            pv_re[l] = pr[d];
            pv_im[l] = pim[d];
        }
        for (int a = 0; a < 6; ++a) {
            double sx, sy, sz;
            point_on(g.tv, tri, c64_qx[a], c64_qy[a], sx, sy, sz);
            const double b[3] = {1.0 - c64_qx[a] - c64_qy[a], c64_qx[a], c64_qy[a]};
            const double ps_re = pv_re[0] * b[0] + pv_re[1] * b[1] + pv_re[2] * b[2];
            const double ps_im = pv_im[0] * b[0] + pv_im[1] * b[1] + pv_im[2] * b[2];
            const double w = c64_qw[a] * jac;
            for (int m = -1; m < g.n_masks; ++m) {
                double ix = sx, iy = sy, iz = sz, jx = nx, jy = ny, jz = nz;
                if (m >= 0) {
                    mirror3(ix, iy, iz, g.masks[m]);
                    mirror3(jx, jy, jz, g.masks[m]);
                }
                double gre = 0, gim = 0, dre = 0, dim = 0;
                green_dlp(ix - ox, iy - oy, iz - oz, jx, jy, jz, kr, 0.0, gre, gim, dre, dim);
                acc_re += ((dre * ps_re - dim * ps_im) - (gre * qv_re - gim * qv_im)) * w;
                acc_im += ((dre * ps_im + dim * ps_re) - (gre * qv_im + gim * qv_re)) * w;
            }
        }
    }
    __shared__ double s_re[8], s_im[8];
    for (int off = 16; off > 0; off >>= 1) {
        acc_re += __shfl_xor_sync(0xffffffffu, acc_re, off);
        acc_im += __shfl_xor_sync(0xffffffffu, acc_im, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_re[warp] = acc_re;
        s_im[warp] = acc_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0, i = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            r += s_re[w];
            i += s_im[w];
        }
        p.out_re[(size_t)f * p.out_stride + o] = r;
        p.out_im[(size_t)f * p.out_stride + o] = i;
    }
}

// ---------------------------------------------------------------------------
// Coupled infinite baffle in FP64 (main.swift:1178-1290 projections, their
// Duffy deltas 1011-1087, Rayleigh field 1397-1444)
// ---------------------------------------------------------------------------
struct Ap64Args {
    Geo64 g;
    const int *ap;        // (m) aperture triangles, ascending ids
    const int *ap_local;  // (T) aperture index or -1
    int m;
    double *out_re, *out_im;
    long long stride;
    double kr[kMaxF64], ki[kMaxF64];
};

// G summed over the images of y (the 1 / (4 pi) included), seen from x
__device__ __forceinline__ void green_images(const Geo64 &g, double yx, double yy, double yz, double x0, double x1,
                                             double x2, double kr, double ki, double &gre, double &gim) {
    double dre = 0, dim = 0;
    green_dlp(yx - x0, yy - x1, yz - x2, 0.0, 0.0, 0.0, kr, ki, gre, gim, dre, dim);
    for (int m = 0; m < g.n_masks; ++m) {
        double ix = yx, iy = yy, iz = yz;
        mirror3(ix, iy, iz, g.masks[m]);
        green_dlp(ix - x0, iy - x1, iz - x2, 0.0, 0.0, 0.0, kr, ki, gre, gim, dre, dim);
    }
}

// S_ia regular part: thread per (test triangle, aperture face); SLP rows of
// the test's three dofs against the face (with images), 2^planes row weight.
__global__ void __launch_bounds__(128) k64_ap_slp(const __grid_constant__ Ap64Args a) {
    const Geo64 &g = a.g;
    const int test = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = blockIdx.y, f = blockIdx.z;
    if (test >= g.T) return;
    const int trial = a.ap[t];
    const double kr = a.kr[f], ki = a.ki[f];
    const double jac = (2.0 * g.nrm[4 * test + 3]) * (2.0 * g.nrm[4 * trial + 3]);
    double sr[3] = {0, 0, 0}, si[3] = {0, 0, 0};
    for (int qa = 0; qa < 6; ++qa) {
        double x0, x1, x2;
        point_on(g.tv, test, c64_qx[qa], c64_qy[qa], x0, x1, x2);
        const double tb[3] = {1.0 - c64_qx[qa] - c64_qy[qa], c64_qx[qa], c64_qy[qa]};
        for (int qb = 0; qb < 6; ++qb) {
            double yx, yy, yz;
            point_on(g.tv, trial, c64_qx[qb], c64_qy[qb], yx, yy, yz);
            double gre = 0, gim = 0;
            green_images(g, yx, yy, yz, x0, x1, x2, kr, ki, gre, gim);
            const double w = c64_qw[qa] * c64_qw[qb] * jac;
            for (int i = 0; i < 3; ++i) {
                sr[i] += gre * (tb[i] * w);
                si[i] += gim * (tb[i] * w);
            }
        }
    }
    for (int i = 0; i < 3; ++i) {
        const size_t o = (size_t)f * a.stride + (size_t)g.l2g[test * 3 + i] * a.m + t;
        atomicAdd(a.out_re + o, sr[i] * g.rw);
        atomicAdd(a.out_im + o, si[i] * g.rw);
    }
}

// S_aa regular part: thread per (test face r, trial face c) of the aperture,
// the SLP summed over the test's basis functions, divided by its area, at the
// real field wavenumber.
__global__ void __launch_bounds__(128) k64_ap_avg(const __grid_constant__ Ap64Args a) {
    const Geo64 &g = a.g;
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y, f = blockIdx.z;
    if (c >= a.m) return;
    const int test = a.ap[r], trial = a.ap[c];
    const double kr = a.kr[f];
    const double jac = (2.0 * g.nrm[4 * test + 3]) * (2.0 * g.nrm[4 * trial + 3]);
    double sr = 0, si = 0;
    for (int qa = 0; qa < 6; ++qa) {
        double x0, x1, x2;
        point_on(g.tv, test, c64_qx[qa], c64_qy[qa], x0, x1, x2);
        for (int qb = 0; qb < 6; ++qb) {
            double yx, yy, yz;
            point_on(g.tv, trial, c64_qx[qb], c64_qy[qb], yx, yy, yz);
            double gre = 0, gim = 0;
            green_images(g, yx, yy, yz, x0, x1, x2, kr, 0.0, gre, gim);
            const double w = c64_qw[qa] * c64_qw[qb] * jac;
            sr += gre * w;
            si += gim * w;
        }
    }
    const double inv = 1.0 / fmax(g.nrm[4 * test + 3], 1e-300);
    const size_t o = (size_t)f * a.stride + (size_t)r * a.m + c;
    a.out_re[o] += sr * inv;
    a.out_im[o] += si * inv;
}

// Duffy SLP deltas of the projections.  mode 1: S_ia gets the delta of every
// pair whose trial is an aperture face (at the pair's weight); mode 2: S_aa
// gets the delta summed over the test basis, divided by the test area, for
// pairs of two aperture faces with an unmirrored test (once each).
__global__ void __launch_bounds__(128) k64_ap_duffy(const __grid_constant__ Ap64Args a, const DuffyPair *pairs,
                                                    int n_pairs, const double *rule_all, int mode, int off1, int cnt1,
                                                    int off2, int cnt2, int off3, int cnt3) {
    const int pi = blockIdx.x * blockDim.x + threadIdx.x;
    if (pi >= n_pairs) return;
    const Geo64 &g = a.g;
    const int f = blockIdx.y;
    const DuffyPair pr = pairs[pi];
    const int ls = a.ap_local[pr.trial];
    if (ls < 0) return;
    if (mode == 2 && (pr.test_mask != 0 || a.ap_local[pr.test] < 0)) return;
    const double kr = a.kr[f], ki = mode == 2 ? 0.0 : a.ki[f];
    double nx = 0, ny = 0, nz = 0;   // the SLP needs no normal
    const double jac = (2.0 * g.nrm[4 * pr.test + 3]) * (2.0 * g.nrm[4 * pr.trial + 3]);
    double rs_re[3] = {0, 0, 0}, rs_im[3] = {0, 0, 0}, ss_re[3] = {0, 0, 0}, ss_im[3] = {0, 0, 0};
    double d_re[9], d_im[9];
    for (int a6 = 0; a6 < 6; ++a6)
        for (int b6 = 0; b6 < 6; ++b6)
            pair_point(g, pr.test, pr.trial, pr.test_mask, pr.trial_mask, c64_qx[a6], c64_qy[a6], c64_qx[b6],
                       c64_qy[b6], c64_qw[a6] * c64_qw[b6] * jac, nx, ny, nz, kr, ki, rs_re, rs_im, d_re, d_im);
    const int kind = pr.kind;
    const int off = kind == 1 ? off1 : (kind == 2 ? off2 : off3), cnt = kind == 1 ? cnt1 : (kind == 2 ? cnt2 : cnt3);
    const double *rule = rule_all + 5 * (size_t)off;
    for (int q = 0; q < cnt; ++q) {
        const double *r = rule + 5 * q;
        double tx, ty, sx, sy;
        remap(r[0], r[1], kind, pr.tl1, pr.tl2, tx, ty);
        remap(r[2], r[3], kind, pr.sl1, pr.sl2, sx, sy);
        pair_point(g, pr.test, pr.trial, pr.test_mask, pr.trial_mask, tx, ty, sx, sy, r[4] * jac, nx, ny, nz, kr, ki,
                   ss_re, ss_im, d_re, d_im);
    }
    if (mode == 1) {
        const double wgt = (double)pr.weight;
        for (int i = 0; i < 3; ++i) {
            const size_t o = (size_t)f * a.stride + (size_t)g.l2g[pr.test * 3 + i] * a.m + ls;
            atomicAdd(a.out_re + o, (ss_re[i] - rs_re[i]) * wgt);
            atomicAdd(a.out_im + o, (ss_im[i] - rs_im[i]) * wgt);
        }
    } else {
        double dr = 0, di = 0;
        for (int i = 0; i < 3; ++i) {
            dr += ss_re[i] - rs_re[i];
            di += ss_im[i] - rs_im[i];
        }
        const double inv = 1.0 / fmax(g.nrm[4 * pr.test + 3], 1e-300);
        const size_t o = (size_t)f * a.stride + (size_t)a.ap_local[pr.test] * a.m + ls;
        atomicAdd(a.out_re + o, dr * inv);
        atomicAdd(a.out_im + o, di * inv);
    }
}

// Rayleigh field p(x) = -2 sum_t q_t sum_a w 2|t| sum_images G(y, x') with
// x' = (x, y, max(z, 0)) for z >= -1e-5, zero below.  CTA per (point, wavenumber).
__global__ void __launch_bounds__(256) k64_rayleigh(const __grid_constant__ Ap64Args a, const double *qa_re,
                                                    const double *qa_im, long long qa_stride, const float *obs,
                                                    int n_obs, long long out_stride) {
    const Geo64 &g = a.g;
    const int o = blockIdx.x, f = blockIdx.y;
    const double kr = a.kr[f];
    const double ox = obs[o], oy = obs[n_obs + o], oz = obs[2 * n_obs + o];
    double acc_re = 0.0, acc_im = 0.0;
    if (oz >= -1e-5) {
        const double ez = oz < 0.0 ? 0.0 : oz;
        for (int t = threadIdx.x; t < a.m; t += blockDim.x) {
            const double q_re = qa_re[(size_t)f * qa_stride + t], q_im = qa_im[(size_t)f * qa_stride + t];
            if (q_re == 0.0 && q_im == 0.0) continue;
            const int tri = a.ap[t];
            const double jac = 2.0 * g.nrm[4 * tri + 3];
            for (int qa = 0; qa < 6; ++qa) {
                double yx, yy, yz;
                point_on(g.tv, tri, c64_qx[qa], c64_qy[qa], yx, yy, yz);
                double gre = 0, gim = 0;
                green_images(g, yx, yy, yz, ox, oy, ez, kr, 0.0, gre, gim);
                const double w = c64_qw[qa] * jac;
                acc_re += (gre * q_re - gim * q_im) * w;
                acc_im += (gre * q_im + gim * q_re) * w;
            }
        }
    }
    __shared__ double s_re[8], s_im[8];
    for (int off = 16; off > 0; off >>= 1) {
        acc_re += __shfl_xor_sync(0xffffffffu, acc_re, off);
        acc_im += __shfl_xor_sync(0xffffffffu, acc_im, off);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_re[warp] = acc_re;
        s_im[warp] = acc_im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0, i = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            r += s_re[w];
            i += s_im[w];
        }
        a.out_re[(size_t)f * out_stride + o] = -2.0 * r;
        a.out_im[(size_t)f * out_stride + o] = -2.0 * i;
    }
}

// ---------------------------------------------------------------------------
// complex128 LU (planar, row-major, lda) and solve
// ---------------------------------------------------------------------------
constexpr int kNB64 = 32;            // panel width
constexpr int kPivRows = 2048;       // rows per pivot-search CTA (256 threads x 8)
constexpr int kMaxPivBlocks = 64;    // pivot-search CTAs per matrix (n <= 131072)

struct Lu64 {
    double *re, *im;
    long long lda, stride;
    int n;
};

__device__ __forceinline__ bool better(double v, int i, double bv, int bi) {
    return v > bv || (v == bv && i < bi);
}

// Pivot of column j: the first row r >= j with the largest |re| + |im|.  Each
// CTA reduces kPivRows rows to a candidate; the last CTA of the matrix to
// finish (ticket counter) reduces the candidates, records piv[j] and info,
// resets the counter and swaps rows j and piv[j] across the panel's columns.
__global__ void __launch_bounds__(256) k64_pivot(Lu64 m, int j, int k0, int kw, double *cand_v, int *cand_i,
                                                 unsigned *ticket, int *piv, long long piv_stride, int *info) {
    const int mat = blockIdx.y, nblk = gridDim.x;
    double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    double bv = -1.0;
    int bi = 0x7fffffff;
    const int r0 = j + blockIdx.x * kPivRows;
    for (int t = threadIdx.x; t < kPivRows; t += 256) {
        const int r = r0 + t;
        if (r >= m.n) break;
        const double v = fabs(are[(size_t)r * m.lda + j]) + fabs(aim[(size_t)r * m.lda + j]);
        if (better(v, r, bv, bi)) { bv = v; bi = r; }
    }
    __shared__ double s_v[8];
    __shared__ int s_i[8];
    __shared__ bool s_last;
    for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
        if (better(ov, oi, bv, bi)) { bv = ov; bi = oi; }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s_v[warp] = bv; s_i[warp] = bi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w)
            if (better(s_v[w], s_i[w], s_v[0], s_i[0])) { s_v[0] = s_v[w]; s_i[0] = s_i[w]; }
        cand_v[mat * kMaxPivBlocks + blockIdx.x] = s_v[0];
        cand_i[mat * kMaxPivBlocks + blockIdx.x] = s_i[0];
        __threadfence();
        const unsigned t = atomicAdd(ticket + mat, 1u);
        s_last = (t == (unsigned)nblk - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __shared__ int s_piv;
    if (threadIdx.x == 0) {
        __threadfence();
        double v = -1.0;
        int i = 0x7fffffff;
        for (int b = 0; b < nblk; ++b) {
            const double cv = __ldcg(cand_v + mat * kMaxPivBlocks + b);
            const int ci = __ldcg(cand_i + mat * kMaxPivBlocks + b);
            if (better(cv, ci, v, i)) { v = cv; i = ci; }
        }
        piv[(size_t)mat * piv_stride + j] = i;
        if (v == 0.0 && info[mat] == 0) info[mat] = j + 1;
        ticket[mat] = 0u;
        s_piv = i;
    }
    __syncthreads();
    const int pr = s_piv;
    if (pr != j && threadIdx.x < kw) {
        const int c = k0 + threadIdx.x;
        double *a1 = are + (size_t)j * m.lda + c, *a2 = are + (size_t)pr * m.lda + c;
        double *b1 = aim + (size_t)j * m.lda + c, *b2 = aim + (size_t)pr * m.lda + c;
        const double t1 = *a1, t2 = *b1;
        *a1 = *a2; *b1 = *b2;
        *a2 = t1; *b2 = t2;
    }
}

// Rows i > j: l = a_ij / a_jj (when the pivot is non-zero), then
// a_ic -= l a_jc for the panel's columns c in (j, k0 + kw).  A warp per row,
// a lane per panel column.
__global__ void __launch_bounds__(256) k64_panel_update(Lu64 m, int j, int k0, int kw) {
    const int mat = blockIdx.y;
    double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double p_re = are[(size_t)j * m.lda + j], p_im = aim[(size_t)j * m.lda + j];
    const bool ok = p_re != 0.0 || p_im != 0.0;
    double r_re = 0.0, r_im = 0.0;
    if (ok) {  // 1 / p, scaled to avoid overflow of |p|^2
        const double s = fmax(fabs(p_re), fabs(p_im));
        const double a = p_re / s, b = p_im / s, d = (a * a + b * b) * s;
        r_re = a / d;
        r_im = -b / d;
    }
    const int c = k0 + lane;
    const bool col = lane < kw && c > j;
    const double u_re = col ? are[(size_t)j * m.lda + c] : 0.0, u_im = col ? aim[(size_t)j * m.lda + c] : 0.0;
    for (int i = j + 1 + blockIdx.x * 8 + warp; i < m.n; i += gridDim.x * 8) {
        double *ar = are + (size_t)i * m.lda, *ai = aim + (size_t)i * m.lda;
        double l_re = ar[j], l_im = ai[j];
        if (ok) {
            const double t = l_re * r_re - l_im * r_im;
            l_im = l_re * r_im + l_im * r_re;
            l_re = t;
        }
        __syncwarp();
        if (lane == 0 && ok) { ar[j] = l_re; ai[j] = l_im; }
        if (col && ok) {
            ar[c] -= l_re * u_re - l_im * u_im;
            ai[c] -= l_re * u_im + l_im * u_re;
        }
    }
}

// Row interchanges of the panel (rows k0 .. k0+kw-1) applied to the columns
// outside it, in order (LAPACK laswp).  A thread per column.
__global__ void __launch_bounds__(256) k64_laswp(Lu64 m, int k0, int kw, const int *piv, long long piv_stride) {
    const int mat = blockIdx.y;
    int c = blockIdx.x * 256 + threadIdx.x;
    const int outside = m.n - kw;
    if (c >= outside) return;
    if (c >= k0) c += kw;
    double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    const int *pv = piv + (size_t)mat * piv_stride;
    for (int j = k0; j < k0 + kw; ++j) {
        const int p = pv[j];
        if (p == j) continue;
        double *a1 = are + (size_t)j * m.lda + c, *a2 = are + (size_t)p * m.lda + c;
        double *b1 = aim + (size_t)j * m.lda + c, *b2 = aim + (size_t)p * m.lda + c;
        const double t1 = *a1, t2 = *b1;
        *a1 = *a2; *b1 = *b2;
        *a2 = t1; *b2 = t2;
    }
}

// U12 = L11^-1 A12 (unit lower L11 of the panel, kw x kw) for the columns
// right of the panel.  A thread per column, L11 in shared memory.
__global__ void __launch_bounds__(128) k64_trsm(Lu64 m, int k0, int kw) {
    const int mat = blockIdx.y;
    double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    __shared__ double L_re[kNB64][kNB64], L_im[kNB64][kNB64];
    for (int e = threadIdx.x; e < kw * kw; e += 128) {
        const int r = e / kw, t = e - r * kw;
        L_re[r][t] = are[(size_t)(k0 + r) * m.lda + k0 + t];
        L_im[r][t] = aim[(size_t)(k0 + r) * m.lda + k0 + t];
    }
    __syncthreads();
    const int c = k0 + kw + blockIdx.x * 128 + threadIdx.x;
    if (c >= m.n) return;
    double x_re[kNB64], x_im[kNB64];
#pragma unroll
    for (int r = 0; r < kNB64; ++r) {
        if (r < kw) {
            x_re[r] = are[(size_t)(k0 + r) * m.lda + c];
            x_im[r] = aim[(size_t)(k0 + r) * m.lda + c];
        }
    }
#pragma unroll
    for (int r = 1; r < kNB64; ++r) {
        if (r < kw) {
            double sr = x_re[r], si = x_im[r];
#pragma unroll
            for (int t = 0; t < r; ++t) {
                sr -= L_re[r][t] * x_re[t] - L_im[r][t] * x_im[t];
                si -= L_re[r][t] * x_im[t] + L_im[r][t] * x_re[t];
            }
            x_re[r] = sr;
            x_im[r] = si;
        }
    }
#pragma unroll
    for (int r = 1; r < kNB64; ++r) {
        if (r < kw) {
            are[(size_t)(k0 + r) * m.lda + c] = x_re[r];
            aim[(size_t)(k0 + r) * m.lda + c] = x_im[r];
        }
    }
}

// A22 -= L21 U12 over rows and columns >= s = k0 + kw, K = kw (<= 32) in two
// chunks of 16.  64 x 64 complex tile per 256-thread CTA, 4 x 4 per thread.
__global__ void __launch_bounds__(256) k64_gemm(Lu64 m, int k0, int kw) {
    constexpr int KC = 16;
    __shared__ double Lr[KC][64], Li[KC][64], Ur[KC][64], Ui[KC][64];
    const int mat = blockIdx.z;
    double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    const int s = k0 + kw;
    const int row0 = s + blockIdx.y * 64, col0 = s + blockIdx.x * 64;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    double cr[4][4], ci[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cr[i][j] = ci[i][j] = 0.0;
    for (int kc = 0; kc < kw; kc += KC) {
        for (int e = tid; e < 64 * KC; e += 256) {
            const int r = e / KC, kk = e - r * KC;
            const int gr = row0 + r, gk = k0 + kc + kk;
            const bool ok = gr < m.n && kc + kk < kw;
            Lr[kk][r] = ok ? are[(size_t)gr * m.lda + gk] : 0.0;
            Li[kk][r] = ok ? aim[(size_t)gr * m.lda + gk] : 0.0;
        }
        for (int e = tid; e < 64 * KC; e += 256) {
            const int kk = e / 64, c = e - kk * 64;
            const int gc = col0 + c, gk = k0 + kc + kk;
            const bool ok = gc < m.n && kc + kk < kw;
            Ur[kk][c] = ok ? are[(size_t)gk * m.lda + gc] : 0.0;
            Ui[kk][c] = ok ? aim[(size_t)gk * m.lda + gc] : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            double a_r[4], a_i[4], b_r[4], b_i[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a_r[i] = Lr[kk][ty * 4 + i];
                a_i[i] = Li[kk][ty * 4 + i];
                b_r[i] = Ur[kk][tx * 4 + i];
                b_i[i] = Ui[kk][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    cr[i][j] = fma(a_r[i], b_r[j], cr[i][j]);
                    cr[i][j] = fma(-a_i[i], b_i[j], cr[i][j]);
                    ci[i][j] = fma(a_r[i], b_i[j], ci[i][j]);
                    ci[i][j] = fma(a_i[i], b_r[j], ci[i][j]);
                }
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int gr = row0 + ty * 4 + i;
        if (gr >= m.n) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gc = col0 + tx * 4 + j;
            if (gc >= m.n) continue;
            are[(size_t)gr * m.lda + gc] -= cr[i][j];
            aim[(size_t)gr * m.lda + gc] -= ci[i][j];
        }
    }
}

struct Rhs64 {
    double *re, *im;
    long long ldb, stride;
    int nrhs;
};

// Apply the row interchanges to each right-hand side, in order.
__global__ void k64_rhs_swap(Lu64 m, const int *piv, long long piv_stride, Rhs64 b, int batch) {
    const int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= batch * b.nrhs) return;
    const int mat = z / b.nrhs, r = z - mat * b.nrhs;
    double *xr = b.re + (size_t)mat * b.stride + r, *xi = b.im + (size_t)mat * b.stride + r;
    const int *pv = piv + (size_t)mat * piv_stride;
    for (int j = 0; j < m.n; ++j) {
        const int p = pv[j];
        if (p == j) continue;
        const double t1 = xr[(size_t)j * b.ldb], t2 = xi[(size_t)j * b.ldb];
        xr[(size_t)j * b.ldb] = xr[(size_t)p * b.ldb];
        xi[(size_t)j * b.ldb] = xi[(size_t)p * b.ldb];
        xr[(size_t)p * b.ldb] = t1;
        xi[(size_t)p * b.ldb] = t2;
    }
}

// Diagonal 32-row block [r0, r0 + 32) of L (unit, LOWER) or U: one warp per
// (matrix, right-hand side), lane = row.
template <bool LOWER>
__global__ void __launch_bounds__(32) k64_trsv_diag(Lu64 m, Rhs64 b, int r0) {
    const int z = blockIdx.x, mat = z / b.nrhs, r = z - mat * b.nrhs;
    const double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    double *xr = b.re + (size_t)mat * b.stride + r, *xi = b.im + (size_t)mat * b.stride + r;
    const int lane = threadIdx.x, row = r0 + lane;
    const int h = min(32, m.n - r0);
    double x_re = lane < h ? xr[(size_t)row * b.ldb] : 0.0, x_im = lane < h ? xi[(size_t)row * b.ldb] : 0.0;
    if (LOWER) {
        for (int t = 0; t < h; ++t) {
            const double vr = __shfl_sync(0xffffffffu, x_re, t), vi = __shfl_sync(0xffffffffu, x_im, t);
            if (lane > t && lane < h) {
                const double lr = are[(size_t)row * m.lda + r0 + t], li = aim[(size_t)row * m.lda + r0 + t];
                x_re -= lr * vr - li * vi;
                x_im -= lr * vi + li * vr;
            }
        }
    } else {
        for (int t = h - 1; t >= 0; --t) {
            if (lane == t) {
                const double ur = are[(size_t)row * m.lda + row], ui = aim[(size_t)row * m.lda + row];
                const double s = fmax(fabs(ur), fabs(ui));
                if (s > 0.0) {
                    const double a = ur / s, c = ui / s, d = (a * a + c * c) * s;
                    const double ir = a / d, ii = -c / d;
                    const double nr = x_re * ir - x_im * ii;
                    x_im = x_re * ii + x_im * ir;
                    x_re = nr;
                } else {
                    x_re = x_im = nan("");
                }
            }
            const double vr = __shfl_sync(0xffffffffu, x_re, t), vi = __shfl_sync(0xffffffffu, x_im, t);
            if (lane < t) {
                const double ur = are[(size_t)row * m.lda + r0 + t], ui = aim[(size_t)row * m.lda + r0 + t];
                x_re -= ur * vr - ui * vi;
                x_im -= ur * vi + ui * vr;
            }
        }
    }
    if (lane < h) {
        xr[(size_t)row * b.ldb] = x_re;
        xi[(size_t)row * b.ldb] = x_im;
    }
}

// x_i -= sum_t A[i][r0 + t] x[r0 + t] for rows i in [i0, i1): a warp per row.
__global__ void __launch_bounds__(256) k64_trsv_update(Lu64 m, Rhs64 b, int r0, int i0, int i1) {
    const int z = blockIdx.y, mat = z / b.nrhs, r = z - mat * b.nrhs;
    const double *are = m.re + (size_t)mat * m.stride, *aim = m.im + (size_t)mat * m.stride;
    double *xr = b.re + (size_t)mat * b.stride + r, *xi = b.im + (size_t)mat * b.stride + r;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int h = min(32, m.n - r0);
    const double v_re = lane < h ? xr[(size_t)(r0 + lane) * b.ldb] : 0.0;
    const double v_im = lane < h ? xi[(size_t)(r0 + lane) * b.ldb] : 0.0;
    for (int i = i0 + blockIdx.x * 8 + warp; i < i1; i += gridDim.x * 8) {
        double sr = 0.0, si = 0.0;
        if (lane < h) {
            const double lr = are[(size_t)i * m.lda + r0 + lane], li = aim[(size_t)i * m.lda + r0 + lane];
            sr = lr * v_re - li * v_im;
            si = lr * v_im + li * v_re;
        }
        for (int off = 16; off > 0; off >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, off);
            si += __shfl_xor_sync(0xffffffffu, si, off);
        }
        if (lane == 0) {
            xr[(size_t)i * b.ldb] -= sr;
            xi[(size_t)i * b.ldb] -= si;
        }
    }
}

__global__ void k64_widen(const float *sr, const float *si, long long sld, long long sstride, double *dr, double *di,
                          long long dld, long long dstride, int rows, int cols) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int mat = blockIdx.y;
    if (e >= (long long)rows * cols) return;
    const int r = (int)(e / cols), c = (int)(e - (long long)r * cols);
    dr[(size_t)mat * dstride + (size_t)r * dld + c] = (double)sr[(size_t)mat * sstride + (size_t)r * sld + c];
    di[(size_t)mat * dstride + (size_t)r * dld + c] = (double)si[(size_t)mat * sstride + (size_t)r * sld + c];
}

__global__ void k64_narrow(const double *sr, const double *si, long long sld, long long sstride, float *dr, float *di,
                           long long dld, long long dstride, int rows, int cols) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int mat = blockIdx.y;
    if (e >= (long long)rows * cols) return;
    const int r = (int)(e / cols), c = (int)(e - (long long)r * cols);
    dr[(size_t)mat * dstride + (size_t)r * dld + c] = (float)sr[(size_t)mat * sstride + (size_t)r * sld + c];
    di[(size_t)mat * dstride + (size_t)r * dld + c] = (float)si[(size_t)mat * sstride + (size_t)r * sld + c];
}

// Session geometry in double (vertices per triangle, normal + area) and the
// Duffy rules built in double, uploaded on first use.
int ensure_geo64(Session &s) {
    if (s.d_geo64) return HBEM_OK;
    const int T = s.n_triangles, V = s.n_vertices;
    std::vector<double> h((size_t)T * 13);
    for (int t = 0; t < T; ++t) {
        for (int l = 0; l < 3; ++l) {
            const int v = s.tris[(size_t)l * T + t];
            for (int c = 0; c < 3; ++c) h[(size_t)t * 9 + l * 3 + c] = (double)s.verts[(size_t)c * V + v];
        }
        double *nr = h.data() + (size_t)T * 9 + 4 * (size_t)t;
        nr[0] = s.normals[t];
        nr[1] = s.normals[T + t];
        nr[2] = s.normals[2 * T + t];
        nr[3] = s.areas[t];
    }
    std::vector<double> rule;
    for (int kind = 1; kind <= 3; ++kind) {
        std::vector<double> rec;
        duffy_rule_table64(kind, rec);
        if ((int)(rec.size() / 5) != s.rule_cnt[kind - 1] || (int)(rule.size() / 5) != s.rule_off[kind - 1])
            return fail(HBEM_ERR_STATE, "FP64 Duffy rule layout differs from the session's");
        rule.insert(rule.end(), rec.begin(), rec.end());
    }
    const size_t bytes = sizeof(double) * (h.size() + rule.size());
    HBEM_CUDA(cudaMalloc((void **)&s.d_geo64, bytes));
    HBEM_CUDA(cudaMemcpy(s.d_geo64, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice));
    HBEM_CUDA(cudaMemcpy(s.d_geo64 + h.size(), rule.data(), sizeof(double) * rule.size(), cudaMemcpyHostToDevice));
    return HBEM_OK;
}

Geo64 geo64(const Session &s) {
    Geo64 g{};
    g.tv = s.d_geo64;
    g.nrm = s.d_geo64 + (size_t)s.n_triangles * 9;
    g.l2g = s.d_l2g;
    g.T = s.n_triangles;
    g.sym = s.sym;
    g.n_masks = 0;
    if (s.sym == 1) { g.masks[0] = 1; g.n_masks = 1; }
    else if (s.sym == 2) { g.masks[0] = 2; g.n_masks = 1; }
    else if (s.sym == 4) { g.masks[0] = 4; g.n_masks = 1; }
    else if (s.sym == 3) { g.masks[0] = 1; g.masks[1] = 2; g.masks[2] = 3; g.n_masks = 3; }
    g.rw = s.sym == 3 ? 4.0 : (s.sym ? 2.0 : 1.0);
    return g;
}

// ---------------------------------------------------------------------------
// CHIEF least squares (reference main.swift:1897-2036, 7186-7409).
//
// Interior point x_c gives one collocation row of the exterior representation,
// which vanishes inside the body: C p = d with
//   C[c][dof] = sum_tri sum_images int D(x_c, y) phi_dof - (int G) (i k beta) / 3,
//   d[c]      = sum_tri (int G) g_tri,
// D and G at the real wavenumber (the field kernels), i k of the Robin fold at
// the complex one; no jump term, no row weight.  The system [A; s C] p =
// [b; s d], s = weight ||A||_inf / ||C||_inf, is solved in the least-squares
// sense in complex128 by Householder QR (LAPACK zgeqrf / zunmqr / ztrtrs, the
// reference's zgels): per column one reflector H = I - tau v v^H (zlarfg), then
// H^H applied to the remaining columns, the right-hand sides included as extra
// columns; then back substitution with R.
// ---------------------------------------------------------------------------
constexpr int kMaxChiefSrc = 8;

struct ChiefArgs {
    Geo64 g;
    const float *pts;                 // (3, m)
    const float *q_re, *q_im;         // (S, F, T) Neumann data
    long long q_stride, q_src_stride;
    const float *beta_re, *beta_im;   // (T) admittances or NULL
    double *c_re, *c_im;              // (F, m, n)
    double *d_re, *d_im;              // (S, F, m)
    int m, n, n_src, nf;
    double kr[kMaxF64], ki[kMaxF64];
};

// Grid: x = triangle blocks of 256, y = CHIEF point, z = wavenumber.
__global__ void __launch_bounds__(256) k64_chief_rows(const __grid_constant__ ChiefArgs p) {
    const Geo64 &g = p.g;
    const int ci = blockIdx.y, f = blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const double ox = p.pts[ci], oy = p.pts[p.m + ci], oz = p.pts[2 * p.m + ci];
    const double kr = p.kr[f], ki = p.ki[f];
    double gs_re = 0.0, gs_im = 0.0;
    if (t < g.T) {
        const double nx = g.nrm[4 * t], ny = g.nrm[4 * t + 1], nz = g.nrm[4 * t + 2];
        const double jac = 2.0 * g.nrm[4 * t + 3];
        double dc_re[3] = {0.0, 0.0, 0.0}, dc_im[3] = {0.0, 0.0, 0.0};
        for (int a = 0; a < 6; ++a) {
            double yx, yy, yz;
            point_on(g.tv, t, c64_qx[a], c64_qy[a], yx, yy, yz);
            const double w = c64_qw[a] * jac;
            const double b[3] = {1.0 - c64_qx[a] - c64_qy[a], c64_qx[a], c64_qy[a]};
            for (int im = -1; im < g.n_masks; ++im) {
                double px = yx, py = yy, pz = yz, mx = nx, my = ny, mz = nz;
                if (im >= 0) {
                    mirror3(px, py, pz, g.masks[im]);
                    mirror3(mx, my, mz, g.masks[im]);
                }
                double gre = 0.0, gim = 0.0, dre = 0.0, dim = 0.0;
                green_dlp(px - ox, py - oy, pz - oz, mx, my, mz, kr, 0.0, gre, gim, dre, dim);
#pragma unroll
                for (int l = 0; l < 3; ++l) {
                    dc_re[l] += dre * b[l] * w;
                    dc_im[l] += dim * b[l] * w;
                }
                gs_re += gre * w;
                gs_im += gim * w;
            }
        }
        double rob_re = 0.0, rob_im = 0.0;
        if (p.beta_re && (p.beta_re[t] != 0.f || p.beta_im[t] != 0.f)) {
            // (int G) (i k beta) / 3 with i k = -ki + i kr
            const double br = p.beta_re[t], bi = p.beta_im[t];
            const double ikb_re = -ki * br - kr * bi, ikb_im = -ki * bi + kr * br;
            rob_re = (gs_re * ikb_re - gs_im * ikb_im) / 3.0;
            rob_im = (gs_re * ikb_im + gs_im * ikb_re) / 3.0;
        }
        double *cr = p.c_re + ((size_t)f * p.m + ci) * p.n, *cim = p.c_im + ((size_t)f * p.m + ci) * p.n;
#pragma unroll
        for (int l = 0; l < 3; ++l) {
            const int d = g.l2g[3 * t + l];
            atomicAdd(cr + d, dc_re[l] - rob_re);
            atomicAdd(cim + d, dc_im[l] - rob_im);
        }
    }
    // d[s][f][ci] += sum over this block's triangles of (int G) g_tri
    __shared__ double s_part[8][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int sv = 0; sv < p.n_src; ++sv) {
        double vr = 0.0, vi = 0.0;
        if (t < g.T && p.q_re) {
            const size_t o = (size_t)sv * p.q_src_stride + (size_t)f * p.q_stride + t;
            const double qr = p.q_re[o], qi = p.q_im[o];
            vr = gs_re * qr - gs_im * qi;
            vi = gs_re * qi + gs_im * qr;
        }
        for (int o = 16; o > 0; o >>= 1) {
            vr += __shfl_xor_sync(0xffffffffu, vr, o);
            vi += __shfl_xor_sync(0xffffffffu, vi, o);
        }
        __syncthreads();
        if (lane == 0) { s_part[warp][0] = vr; s_part[warp][1] = vi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double ar = 0.0, ai = 0.0;
            for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) { ar += s_part[w2][0]; ai += s_part[w2][1]; }
            const size_t o = ((size_t)sv * p.nf + f) * p.m + ci;
            atomicAdd(p.d_re + o, ar);
            atomicAdd(p.d_im + o, ai);
        }
    }
}

// ||X_f||_inf = max_i sum_j |x_ij| of row-major (rows, cols) matrices, one warp
// per row; out[f] (as the bits of a non-negative double) by atomicMax.
template <typename T>
__global__ void k64_inf_norm(int rows, int cols, const T *xr, const T *xi, long long ld, long long stride,
                             unsigned long long *out) {
    const int f = blockIdx.y;
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= rows) return;
    const T *r = xr + (size_t)f * stride + (size_t)row * ld, *i = xi + (size_t)f * stride + (size_t)row * ld;
    double sum = 0.0;
    for (int c = lane; c < cols; c += 32) sum += hypot((double)r[c], (double)i[c]);
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) atomicMax(out + f, (unsigned long long)__double_as_longlong(sum));
}

// M_f = [A_f | B_f; s C_f | s D_f] (rows n + m, ldm >= n + S; B_f, D_f hold the
// S right-hand sides as columns), s_f = weight ||A_f|| / ||C_f|| (weight when
// ||C_f|| = 0).  Grid: x over the elements of one matrix, y = wavenumber.
struct ChiefBuildArgs {
    const float *a_re, *a_im;
    long long lda, a_stride;
    const float *b_re, *b_im;
    long long b_stride, b_src_stride;
    const double *c_re, *c_im, *d_re, *d_im;
    const unsigned long long *anorm, *cnorm;
    double *m_re, *m_im;
    long long ldm, m_stride;
    double *scale;
    double weight;
    int n, m, n_src, nf;
};

__global__ void k64_chief_build(const __grid_constant__ ChiefBuildArgs p) {
    const int f = blockIdx.y;
    const double an = __longlong_as_double((long long)p.anorm[f]), cn = __longlong_as_double((long long)p.cnorm[f]);
    const double sc = p.weight * (cn > 0.0 ? an / cn : 1.0);
    if (blockIdx.x == 0 && threadIdx.x == 0 && p.scale) p.scale[f] = sc;
    const int cols = p.n + p.n_src, rows = p.n + p.m;
    double *mr = p.m_re + (size_t)f * p.m_stride, *mi = p.m_im + (size_t)f * p.m_stride;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)rows * cols;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e / cols), c = (int)(e - (long long)r * cols);
        double vr, vi;
        if (r < p.n) {
            if (c < p.n) {
                const size_t o = (size_t)f * p.a_stride + (size_t)r * p.lda + c;
                vr = p.a_re[o];
                vi = p.a_im[o];
            } else {
                const size_t o = (size_t)(c - p.n) * p.b_src_stride + (size_t)f * p.b_stride + r;
                vr = p.b_re[o];
                vi = p.b_im[o];
            }
        } else {
            const int ci = r - p.n;
            if (c < p.n) {
                const size_t o = ((size_t)f * p.m + ci) * p.n + c;
                vr = sc * p.c_re[o];
                vi = sc * p.c_im[o];
            } else {
                const size_t o = ((size_t)(c - p.n) * p.nf + f) * p.m + ci;
                vr = sc * p.d_re[o];
                vi = sc * p.d_im[o];
            }
        }
        mr[(size_t)r * p.ldm + c] = vr;
        mi[(size_t)r * p.ldm + c] = vi;
    }
}

// Block sum of a double (all threads get it); blockDim.x a multiple of 32, <= 1024.
__device__ __forceinline__ double block_sum(double v, double *s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) s_w[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < nw; ++w) t += s_w[w];
    return t;
}

// Householder reflector of column j (LAPACK zlarfg): alpha = M[j][j],
// x = M[j+1:rows][j]; beta = -sign(Re alpha) |(alpha, x)|, tau =
// ((beta - Re alpha) / beta, -Im alpha / beta), v = x / (alpha - beta) stored
// over x, M[j][j] = beta; tau = 0 when x = 0 and alpha is real.  Also clears u,
// the accumulator of v^H M for the columns after j.  One CTA per matrix.
__global__ void __launch_bounds__(256) k64_hh_reflector(int rows, int cols, int j, double *m_re, double *m_im,
                                                        long long ldm, long long m_stride, double *tau, double *u) {
    __shared__ double s_w[8];
    __shared__ double s_scale[2];
    const int f = blockIdx.x;
    double *mr = m_re + (size_t)f * m_stride, *mi = m_im + (size_t)f * m_stride;
    double acc = 0.0;
    for (int r = j + 1 + threadIdx.x; r < rows; r += blockDim.x) {
        const double a = mr[(size_t)r * ldm + j], b = mi[(size_t)r * ldm + j];
        acc += a * a + b * b;
    }
    const double xn2 = block_sum(acc, s_w);
    double *tf = tau + (size_t)f * 2 * cols + 2 * j;
    if (threadIdx.x == 0) {
        const double ar = mr[(size_t)j * ldm + j], ai = mi[(size_t)j * ldm + j];
        if (xn2 == 0.0 && ai == 0.0) {
            tf[0] = 0.0;
            tf[1] = 0.0;
            s_scale[0] = 1.0;
            s_scale[1] = 0.0;
        } else {
            const double beta = -copysign(sqrt(ar * ar + ai * ai + xn2), ar);
            tf[0] = (beta - ar) / beta;
            tf[1] = -ai / beta;
            // 1 / (alpha - beta)
            const double dr = ar - beta, di = ai, den = dr * dr + di * di;
            s_scale[0] = dr / den;
            s_scale[1] = -di / den;
            mr[(size_t)j * ldm + j] = beta;
            mi[(size_t)j * ldm + j] = 0.0;
        }
    }
    __syncthreads();
    const double sr = s_scale[0], si = s_scale[1];
    for (int r = j + 1 + threadIdx.x; r < rows; r += blockDim.x) {
        const double a = mr[(size_t)r * ldm + j], b = mi[(size_t)r * ldm + j];
        mr[(size_t)r * ldm + j] = a * sr - b * si;
        mi[(size_t)r * ldm + j] = a * si + b * sr;
    }
    for (int c = threadIdx.x; c < 2 * cols; c += blockDim.x) u[(size_t)f * 2 * cols + c] = 0.0;
}

constexpr int kHhRows = 64;   // rows per CTA of the reflector application

// u[c] += sum_r conj(v_r) M[r][c] over this CTA's rows (v_j = 1), c > j.
// Grid: x = column blocks of 256, y = row blocks of kHhRows from j, z = matrix.
__global__ void __launch_bounds__(256) k64_hh_dot(int rows, int cols, int j, const double *m_re, const double *m_im,
                                                  long long ldm, long long m_stride, double *u) {
    const int f = blockIdx.z;
    const int c = j + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const double *mr = m_re + (size_t)f * m_stride, *mi = m_im + (size_t)f * m_stride;
    const int r0 = j + blockIdx.y * kHhRows, r1 = min(rows, r0 + kHhRows);
    double ar = 0.0, ai = 0.0;
    for (int r = r0; r < r1; ++r) {
        const double vr = r == j ? 1.0 : mr[(size_t)r * ldm + j], vi = r == j ? 0.0 : mi[(size_t)r * ldm + j];
        const double xr = mr[(size_t)r * ldm + c], xi = mi[(size_t)r * ldm + c];
        ar += vr * xr + vi * xi;   // conj(v) x
        ai += vr * xi - vi * xr;
    }
    atomicAdd(u + (size_t)f * 2 * cols + 2 * c, ar);
    atomicAdd(u + (size_t)f * 2 * cols + 2 * c + 1, ai);
}

// M[r][c] -= conj(tau) v_r u_c (H^H applied from the left), same grid.
__global__ void __launch_bounds__(256) k64_hh_update(int rows, int cols, int j, double *m_re, double *m_im,
                                                     long long ldm, long long m_stride, const double *tau,
                                                     const double *u) {
    const int f = blockIdx.z;
    const int c = j + 1 + blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    double *mr = m_re + (size_t)f * m_stride, *mi = m_im + (size_t)f * m_stride;
    const double tr = tau[(size_t)f * 2 * cols + 2 * j], ti = -tau[(size_t)f * 2 * cols + 2 * j + 1];
    if (tr == 0.0 && ti == 0.0) return;
    const double ur = u[(size_t)f * 2 * cols + 2 * c], ui = u[(size_t)f * 2 * cols + 2 * c + 1];
    const double wr = tr * ur - ti * ui, wi = tr * ui + ti * ur;   // conj(tau) u_c
    const int r0 = j + blockIdx.y * kHhRows, r1 = min(rows, r0 + kHhRows);
    for (int r = r0; r < r1; ++r) {
        const double vr = r == j ? 1.0 : mr[(size_t)r * ldm + j], vi = r == j ? 0.0 : mi[(size_t)r * ldm + j];
        mr[(size_t)r * ldm + c] -= vr * wr - vi * wi;
        mi[(size_t)r * ldm + c] -= vr * wi + vi * wr;
    }
}

// R p = y by back substitution, R = the upper triangle of M[0:n][0:n], y =
// M[0:n][n + s]; p_i = (y_i - sum_{j > i} R_ij p_j) / R_ii.  One CTA per
// (right-hand side s, matrix); p (F, S, n) complex in global memory.
__global__ void __launch_bounds__(256) k64_upper_solve(int n, int n_src, const double *m_re, const double *m_im,
                                                       long long ldm, long long m_stride, double *p) {
    __shared__ double s_w[8], s_w2[8];
    const int sv = blockIdx.x, f = blockIdx.y;
    const double *mr = m_re + (size_t)f * m_stride, *mi = m_im + (size_t)f * m_stride;
    double *pv = p + ((size_t)f * n_src + sv) * 2 * n;
    for (int i = n - 1; i >= 0; --i) {
        const double *rr = mr + (size_t)i * ldm, *ri = mi + (size_t)i * ldm;
        double ar = 0.0, ai = 0.0;
        for (int c = i + 1 + threadIdx.x; c < n; c += blockDim.x) {
            const double xr = pv[2 * c], xi = pv[2 * c + 1];
            ar += rr[c] * xr - ri[c] * xi;
            ai += rr[c] * xi + ri[c] * xr;
        }
        const double sr = block_sum(ar, s_w), si = block_sum(ai, s_w2);
        if (threadIdx.x == 0) {
            const double yr = rr[n + sv] - sr, yi = ri[n + sv] - si;
            const double dr = rr[i], di = ri[i], den = dr * dr + di * di;
            pv[2 * i] = den > 0.0 ? (yr * dr + yi * di) / den : 0.0;
            pv[2 * i + 1] = den > 0.0 ? (yi * dr - yr * di) / den : 0.0;
        }
        __syncthreads();
    }
}

// x = (float) p; resid = ||s (C p - d)|| / ||b|| per (source, matrix).  One CTA
// per (source, matrix).
__global__ void __launch_bounds__(256) k64_chief_finish(int n, int m, int n_src, int nf, const double *p,
                                                        const double *c_re, const double *c_im, const double *d_re,
                                                        const double *d_im, const double *scale, const float *b_re,
                                                        const float *b_im, long long b_stride, long long b_src_stride,
                                                        float *x_re, float *x_im, long long x_stride,
                                                        long long x_src_stride, double *resid, long long r_stride) {
    __shared__ double s_w[8], s_w2[8];
    const int sv = blockIdx.x, f = blockIdx.y;
    const double *pv = p + ((size_t)f * n_src + sv) * 2 * n;
    double bb = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const size_t o = (size_t)sv * x_src_stride + (size_t)f * x_stride + i;
        x_re[o] = (float)pv[2 * i];
        x_im[o] = (float)pv[2 * i + 1];
        const size_t ob = (size_t)sv * b_src_stride + (size_t)f * b_stride + i;
        bb += (double)b_re[ob] * b_re[ob] + (double)b_im[ob] * b_im[ob];
    }
    const double bn2 = block_sum(bb, s_w);
    double rs = 0.0;
    for (int ci = 0; ci < m; ++ci) {
        const double *cr = c_re + ((size_t)f * m + ci) * n, *cim = c_im + ((size_t)f * m + ci) * n;
        double ar = 0.0, ai = 0.0;
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            ar += cr[c] * pv[2 * c] - cim[c] * pv[2 * c + 1];
            ai += cr[c] * pv[2 * c + 1] + cim[c] * pv[2 * c];
        }
        const double sr = block_sum(ar, s_w), si = block_sum(ai, s_w2);
        const size_t od = ((size_t)sv * nf + f) * m + ci;
        const double er = scale[f] * (sr - d_re[od]), ei = scale[f] * (si - d_im[od]);
        rs += er * er + ei * ei;
    }
    if (threadIdx.x == 0 && resid) resid[(size_t)sv * r_stride + f] = bn2 > 0.0 ? sqrt(rs / bn2) : sqrt(rs);
}

}  // namespace


// Duffy rule records (test xi, eta, trial xi, eta, weight) in double: the same
// Gauss-Legendre 4-point nodes per Duffy coordinate and the same sub-region maps
// as the session's float table (Sauter & Schwab, Boundary Element Methods,
// 2011, ch. 5; the reference's point order, main.swift:2652-2699).
void duffy_rule_table64(int kind, std::vector<double> &rec) {
    const double a1 = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
    const double a2 = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
    const double w1 = (18.0 + std::sqrt(30.0)) / 72.0, w2 = (18.0 - std::sqrt(30.0)) / 72.0;
    const double xs[4] = {0.5 - a2, 0.5 - a1, 0.5 + a1, 0.5 + a2};
    const double ws[4] = {w2, w1, w1, w2};
    rec.clear();
    auto put = [&](double tx, double ty, double sx, double sy, double w) {
        rec.push_back(tx - ty);
        rec.push_back(ty);
        rec.push_back(sx - sy);
        rec.push_back(sy);
        rec.push_back(w);
    };
    for (int a = 0; a < 4; ++a)
        for (int b = 0; b < 4; ++b)
            for (int c = 0; c < 4; ++c)
                for (int d = 0; d < 4; ++d) {
                    const double xi = xs[b], e1 = xs[a], e2 = xs[c], e3 = xs[d];
                    const double e12 = e1 * e2, e123 = e12 * e3;
                    const double base = ws[a] * ws[b] * ws[c] * ws[d];
                    if (kind == 1) {
                        const double w = base * xi * xi * xi * e1 * e1 * e2;
                        put(xi, xi * (1 - e1 + e12), xi * (1 - e123), xi * (1 - e1), w);
                        put(xi * (1 - e123), xi * (1 - e1), xi, xi * (1 - e1 + e12), w);
                        put(xi, xi * (e1 - e12 + e123), xi * (1 - e12), xi * (e1 - e12), w);
                        put(xi * (1 - e12), xi * (e1 - e12), xi, xi * (e1 - e12 + e123), w);
                        put(xi * (1 - e123), xi * (e1 - e123), xi, xi * (e1 - e12), w);
                        put(xi, xi * (e1 - e12), xi * (1 - e123), xi * (e1 - e123), w);
                    } else if (kind == 2) {
                        const double w = base * xi * xi * xi * e1 * e1;
                        put(xi, xi * e1 * e3, xi * (1 - e12), xi * e1 * (1 - e2), w);
                        put(xi, xi * e1, xi * (1 - e123), xi * e1 * e2 * (1 - e3), w * e2);
                        put(xi * (1 - e12), xi * e1 * (1 - e2), xi, xi * e123, w * e2);
                        put(xi * (1 - e123), xi * e12 * (1 - e3), xi, xi * e1, w * e2);
                        put(xi * (1 - e123), xi * e1 * (1 - e2 * e3), xi, xi * e12, w * e2);
                    } else {
                        const double w = base * xi * xi * xi * e2;
                        put(xi, xi * e1, xi * e2, xi * e2 * e3, w);
                        put(xi * e2, xi * e2 * e3, xi, xi * e1, w);
                    }
                }
}

// ---- FP64 LU entry points (internal, also used by hbem_solve_batch) --------
int lu_factor_f64(int n, int batch, double *a_re, double *a_im, long long lda, long long a_stride, int *piv,
                  long long piv_stride, int *info, cudaStream_t st) {
    if (n <= 0 || batch <= 0) return HBEM_OK;
    const int nblk_max = (n + kPivRows - 1) / kPivRows;
    if (nblk_max > kMaxPivBlocks) return fail(HBEM_ERR_ARG, "hbem_lu_factor_f64: n > 131072");
    char *scratch = nullptr;
    const size_t cand_bytes = (size_t)batch * kMaxPivBlocks * (sizeof(double) + sizeof(int));
    const size_t bytes = cand_bytes + (size_t)batch * sizeof(unsigned);
    HBEM_CUDA(cudaMallocAsync((void **)&scratch, bytes, st));
    double *cand_v = reinterpret_cast<double *>(scratch);
    int *cand_i = reinterpret_cast<int *>(scratch + (size_t)batch * kMaxPivBlocks * sizeof(double));
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + cand_bytes);
    int rc = HBEM_OK;
    auto step = [&](cudaError_t e, const char *what) {
        if (rc == HBEM_OK && e != cudaSuccess) rc = cuda_fail(e, what);
    };
    step(cudaMemsetAsync(ticket, 0, (size_t)batch * sizeof(unsigned), st), "cudaMemsetAsync(ticket)");
    step(cudaMemsetAsync(info, 0, (size_t)batch * sizeof(int), st), "cudaMemsetAsync(info)");
    Lu64 m{a_re, a_im, lda, a_stride, n};
    for (int k0 = 0; k0 < n && rc == HBEM_OK; k0 += kNB64) {
        const int kw = std::min(kNB64, n - k0);
        for (int j = k0; j < k0 + kw && rc == HBEM_OK; ++j) {
            const int nblk = (n - j + kPivRows - 1) / kPivRows;
            k64_pivot<<<dim3(nblk, batch), 256, 0, st>>>(m, j, k0, kw, cand_v, cand_i, ticket, piv, piv_stride, info);
            step(cudaGetLastError(), "k64_pivot");
            count_launch();
            const int rows = n - j - 1;
            if (rows > 0) {
                const int gx = std::min((rows + 7) / 8, std::max(1, 1184 / batch));
                k64_panel_update<<<dim3(gx, batch), 256, 0, st>>>(m, j, k0, kw);
                step(cudaGetLastError(), "k64_panel_update");
                count_launch();
            }
        }
        if (n > kw) {
            k64_laswp<<<dim3((n - kw + 255) / 256, batch), 256, 0, st>>>(m, k0, kw, piv, piv_stride);
            step(cudaGetLastError(), "k64_laswp");
            count_launch();
        }
        const int rest = n - k0 - kw;
        if (rest > 0) {
            k64_trsm<<<dim3((rest + 127) / 128, batch), 128, 0, st>>>(m, k0, kw);
            step(cudaGetLastError(), "k64_trsm");
            count_launch();
            k64_gemm<<<dim3((rest + 63) / 64, (rest + 63) / 64, batch), 256, 0, st>>>(m, k0, kw);
            step(cudaGetLastError(), "k64_gemm");
            count_launch();
        }
    }
    cudaFreeAsync(scratch, st);
    return rc;
}

int lu_solve_f64(int n, int nrhs, int batch, const double *lu_re, const double *lu_im, long long lda,
                 long long a_stride, const int *piv, long long piv_stride, double *b_re, double *b_im, long long ldb,
                 long long b_stride, cudaStream_t st) {
    if (n <= 0 || batch <= 0 || nrhs <= 0) return HBEM_OK;
    Lu64 m{const_cast<double *>(lu_re), const_cast<double *>(lu_im), lda, a_stride, n};
    Rhs64 b{b_re, b_im, ldb, b_stride, nrhs};
    const int z = batch * nrhs;
    if (z > 65535) return fail(HBEM_ERR_ARG, "hbem_lu_solve_f64: batch * nrhs > 65535");
    k64_rhs_swap<<<(z + 127) / 128, 128, 0, st>>>(m, piv, piv_stride, b, batch);
    HBEM_LAUNCH_CHECK("k64_rhs_swap");
    for (int r0 = 0; r0 < n; r0 += 32) {
        k64_trsv_diag<true><<<z, 32, 0, st>>>(m, b, r0);
        HBEM_LAUNCH_CHECK("k64_trsv_diag<L>");
        const int i0 = r0 + 32;
        if (i0 < n) {
            const int gx = std::min((n - i0 + 7) / 8, std::max(1, 1184 / z));
            k64_trsv_update<<<dim3(gx, z), 256, 0, st>>>(m, b, r0, i0, n);
            HBEM_LAUNCH_CHECK("k64_trsv_update<L>");
        }
    }
    for (int r0 = ((n - 1) / 32) * 32; r0 >= 0; r0 -= 32) {
        k64_trsv_diag<false><<<z, 32, 0, st>>>(m, b, r0);
        HBEM_LAUNCH_CHECK("k64_trsv_diag<U>");
        if (r0 > 0) {
            const int gx = std::min((r0 + 7) / 8, std::max(1, 1184 / z));
            k64_trsv_update<<<dim3(gx, z), 256, 0, st>>>(m, b, r0, 0, r0);
            HBEM_LAUNCH_CHECK("k64_trsv_update<U>");
        }
    }
    return HBEM_OK;
}

int widen_f64(int rows, int cols, int batch, const float *sr, const float *si, long long sld, long long sstride,
              double *dr, double *di, long long dld, long long dstride, cudaStream_t st) {
    const long long e = (long long)rows * cols;
    if (e <= 0 || batch <= 0) return HBEM_OK;
    k64_widen<<<dim3((unsigned)((e + 255) / 256), batch), 256, 0, st>>>(sr, si, sld, sstride, dr, di, dld, dstride,
                                                                        rows, cols);
    HBEM_LAUNCH_CHECK("k64_widen");
    return HBEM_OK;
}

int narrow_f64(int rows, int cols, int batch, const double *sr, const double *si, long long sld, long long sstride,
               float *dr, float *di, long long dld, long long dstride, cudaStream_t st) {
    const long long e = (long long)rows * cols;
    if (e <= 0 || batch <= 0) return HBEM_OK;
    k64_narrow<<<dim3((unsigned)((e + 255) / 256), batch), 256, 0, st>>>(sr, si, sld, sstride, dr, di, dld, dstride,
                                                                         rows, cols);
    HBEM_LAUNCH_CHECK("k64_narrow");
    return HBEM_OK;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_assemble_f64(hbem_session *h, int n_freq, const double *k_re, const double *k_im,
                                 const double *q_re, const double *q_im, long long q_stride, const double *beta_re,
                                 const double *beta_im, double *a_re, double *a_im, long long lda, long long a_stride,
                                 double *b_re, double *b_im, long long b_stride, int flags, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_assemble_f64: NULL session");
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !a_re || !a_im) return fail(HBEM_ERR_ARG, "hbem_assemble_f64: NULL k or A pointer");
    if (lda < s->n_dof || a_stride < lda * s->n_dof)
        return fail(HBEM_ERR_ARG, "hbem_assemble_f64: lda/a_stride too small");
    if ((q_re == nullptr) != (q_im == nullptr) || (b_re == nullptr) != (b_im == nullptr) ||
        (beta_re == nullptr) != (beta_im == nullptr))
        return fail(HBEM_ERR_ARG, "hbem_assemble_f64: real/imag pointers must be given together");
    if (q_re && q_stride < s->n_triangles) return fail(HBEM_ERR_ARG, "hbem_assemble_f64: q_stride < n_triangles");
    if (b_re && b_stride < s->n_dof) return fail(HBEM_ERR_ARG, "hbem_assemble_f64: b_stride < n_dof");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f]) || (k_im && !std::isfinite(k_im[f])))
            return fail(HBEM_ERR_ARG, "hbem_assemble_f64: non-finite wavenumber");
    HBEM_CUDA(cudaSetDevice(s->device));
    int rc = ensure_geo64(*s);
    if (rc != HBEM_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int n = s->n_dof, T = s->n_triangles;
    if (flags & HBEM_ASM_ZERO) {
        for (int f = 0; f < n_freq; ++f) {
            HBEM_CUDA(cudaMemset2DAsync(a_re + (size_t)f * a_stride, lda * sizeof(double), 0, n * sizeof(double), n, st));
            HBEM_CUDA(cudaMemset2DAsync(a_im + (size_t)f * a_stride, lda * sizeof(double), 0, n * sizeof(double), n, st));
        }
        if (b_re) {
            HBEM_CUDA(cudaMemset2DAsync(b_re, b_stride * sizeof(double), 0, n * sizeof(double), n_freq, st));
            HBEM_CUDA(cudaMemset2DAsync(b_im, b_stride * sizeof(double), 0, n * sizeof(double), n_freq, st));
        }
    }
    for (int f0 = 0; f0 < n_freq; f0 += kMaxF64) {
        const int nf = std::min(kMaxF64, n_freq - f0);
        Asm64Args a{};
        a.g = geo64(*s);
        a.q_re = q_re ? q_re + (size_t)f0 * q_stride : nullptr;
        a.q_im = q_im ? q_im + (size_t)f0 * q_stride : nullptr;
        a.q_stride = q_stride;
        a.beta_re = beta_re;
        a.beta_im = beta_im;
        a.a_re = a_re + (size_t)f0 * a_stride;
        a.a_im = a_im + (size_t)f0 * a_stride;
        a.b_re = b_re ? b_re + (size_t)f0 * b_stride : nullptr;
        a.b_im = b_im ? b_im + (size_t)f0 * b_stride : nullptr;
        a.lda = lda;
        a.a_stride = a_stride;
        a.b_stride = b_stride;
        a.nf = nf;
        for (int f = 0; f < nf; ++f) {
            a.kr[f] = k_re[f0 + f];
            a.ki[f] = k_im ? k_im[f0 + f] : 0.0;
        }
        if (flags & HBEM_ASM_REGULAR) {
            dim3 grid((T + 127) / 128, std::min(T, 65535), nf);
            k64_regular<<<grid, 128, 0, st>>>(a);
            HBEM_LAUNCH_CHECK("k64_regular");
        }
        if ((flags & HBEM_ASM_DUFFY) && s->n_pairs > 0) {
            Duffy64Args d{};
            d.a = a;
            d.pairs = s->d_pairs;
            d.n_pairs = s->n_pairs;
            d.rule = s->d_geo64 + (size_t)T * 13;
            for (int r = 0; r < 3; ++r) {
                d.rule_off[r] = s->rule_off[r];
                d.rule_cnt[r] = s->rule_cnt[r];
            }
            k64_duffy<<<dim3((s->n_pairs + 127) / 128, nf), 128, 0, st>>>(d);
            HBEM_LAUNCH_CHECK("k64_duffy");
        }
    }
    return HBEM_OK;
}

extern "C" int hbem_field_f64(hbem_session *h, int n_freq, const double *k_re, const double *p_re,
                              const double *p_im, long long p_stride, const double *q_re, const double *q_im,
                              long long q_stride, const float *obs_3xn, int n_obs, double *out_re, double *out_im,
                              long long out_stride, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_field_f64: NULL session");
    if (n_freq <= 0 || n_obs <= 0) return HBEM_OK;
    if (!k_re || !p_re || !p_im || !q_re || !q_im || !obs_3xn || !out_re || !out_im)
        return fail(HBEM_ERR_ARG, "hbem_field_f64: NULL pointer");
    if (p_stride < s->n_dof || q_stride < s->n_triangles || out_stride < n_obs)
        return fail(HBEM_ERR_ARG, "hbem_field_f64: stride too small");
    if (n_obs > 2147483647 / 3) return fail(HBEM_ERR_ARG, "hbem_field_f64: too many observation points");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f])) return fail(HBEM_ERR_ARG, "hbem_field_f64: non-finite wavenumber");
    HBEM_CUDA(cudaSetDevice(s->device));
    int rc = ensure_geo64(*s);
    if (rc != HBEM_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (int f0 = 0; f0 < n_freq; f0 += kMaxF64) {
        const int nf = std::min(kMaxF64, n_freq - f0);
        Field64Args a{};
        a.g = geo64(*s);
        a.p_re = p_re + (size_t)f0 * p_stride;
        a.p_im = p_im + (size_t)f0 * p_stride;
        a.q_re = q_re + (size_t)f0 * q_stride;
        a.q_im = q_im + (size_t)f0 * q_stride;
        a.p_stride = p_stride;
        a.q_stride = q_stride;
        a.obs = obs_3xn;
        a.n_obs = n_obs;
        a.out_re = out_re + (size_t)f0 * out_stride;
        a.out_im = out_im + (size_t)f0 * out_stride;
        a.out_stride = out_stride;
        for (int f = 0; f < nf; ++f) a.kr[f] = k_re[f0 + f];
        for (int o0 = 0; o0 < n_obs; o0 += 65535) {
            // grid.x is the observation point: split very long point lists
            Field64Args b = a;
            const int no = std::min(65535, n_obs - o0);
            b.obs = obs_3xn + o0;   // x, y, z rows keep their stride n_obs
            b.out_re = a.out_re + o0;
            b.out_im = a.out_im + o0;
            b.n_obs = n_obs;
            k64_field<<<dim3(no, nf), 256, 0, st>>>(b);
            HBEM_LAUNCH_CHECK("k64_field");
        }
    }
    return HBEM_OK;
}

extern "C" int hbem_lu_factor_f64(int n, int batch, double *a_re, double *a_im, long long lda, long long a_stride,
                                  int *piv, long long piv_stride, int *info, void *stream) {
    if (n < 0 || batch < 0) return fail(HBEM_ERR_ARG, "hbem_lu_factor_f64: negative size");
    if (n == 0 || batch == 0) return HBEM_OK;
    if (!a_re || !a_im || !piv || !info) return fail(HBEM_ERR_ARG, "hbem_lu_factor_f64: NULL pointer");
    if (lda < n || a_stride < lda * n || piv_stride < n)
        return fail(HBEM_ERR_ARG, "hbem_lu_factor_f64: lda/a_stride/piv_stride too small");
    if (batch > 65535) return fail(HBEM_ERR_ARG, "hbem_lu_factor_f64: batch > 65535");
    return lu_factor_f64(n, batch, a_re, a_im, lda, a_stride, piv, piv_stride, info,
                         reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_lu_solve_f64(int n, int nrhs, int batch, const double *lu_re, const double *lu_im, long long lda,
                                 long long a_stride, const int *piv, long long piv_stride, double *b_re,
                                 double *b_im, long long ldb, long long b_stride, int trans, void *stream) {
    if (n < 0 || nrhs < 0 || batch < 0) return fail(HBEM_ERR_ARG, "hbem_lu_solve_f64: negative size");
    if (n == 0 || nrhs == 0 || batch == 0) return HBEM_OK;
    if (trans != HBEM_TRANS_N) return fail(HBEM_ERR_ARG, "hbem_lu_solve_f64: only HBEM_TRANS_N");
    if (!lu_re || !lu_im || !piv || !b_re || !b_im) return fail(HBEM_ERR_ARG, "hbem_lu_solve_f64: NULL pointer");
    if (lda < n || a_stride < lda * n || piv_stride < n || ldb < nrhs || b_stride < ldb * n)
        return fail(HBEM_ERR_ARG, "hbem_lu_solve_f64: lda/a_stride/piv_stride/ldb/b_stride too small");
    return lu_solve_f64(n, nrhs, batch, lu_re, lu_im, lda, a_stride, piv, piv_stride, b_re, b_im, ldb, b_stride,
                        reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int hbem_aperture_assemble_f64(hbem_session *h, int n_freq, const double *k_re, const double *k_im,
                                          const double *kf_re, double *sia_re, double *sia_im, double *saa_re,
                                          double *saa_im, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_aperture_assemble_f64: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_aperture_assemble_f64: no aperture set on the session");
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !kf_re || !sia_re || !sia_im || !saa_re || !saa_im)
        return fail(HBEM_ERR_ARG, "hbem_aperture_assemble_f64: NULL pointer");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f]) || !std::isfinite(kf_re[f]) || (k_im && !std::isfinite(k_im[f])))
            return fail(HBEM_ERR_ARG, "hbem_aperture_assemble_f64: non-finite wavenumber");
    HBEM_CUDA(cudaSetDevice(s->device));
    int rc = ensure_geo64(*s);
    if (rc != HBEM_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int n = s->n_dof, m = s->m_ap, T = s->n_triangles;
    const size_t sia_stride = (size_t)n * m, saa_stride = (size_t)m * m;
    HBEM_CUDA(cudaMemsetAsync(sia_re, 0, sizeof(double) * sia_stride * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(sia_im, 0, sizeof(double) * sia_stride * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(saa_re, 0, sizeof(double) * saa_stride * n_freq, st));
    HBEM_CUDA(cudaMemsetAsync(saa_im, 0, sizeof(double) * saa_stride * n_freq, st));
    const double *rule = s->d_geo64 + (size_t)T * 13;
    for (int f0 = 0; f0 < n_freq; f0 += kMaxF64) {
        const int nf = std::min(kMaxF64, n_freq - f0);
        Ap64Args a{};
        a.g = geo64(*s);
        a.ap = s->d_ap_tris;
        a.ap_local = s->d_ap_local;
        a.m = m;
        // S_ia at the (possibly complex) assembly wavenumber
        for (int f = 0; f < nf; ++f) {
            a.kr[f] = k_re[f0 + f];
            a.ki[f] = k_im ? k_im[f0 + f] : 0.0;
        }
        a.out_re = sia_re + (size_t)f0 * sia_stride;
        a.out_im = sia_im + (size_t)f0 * sia_stride;
        a.stride = (long long)sia_stride;
        k64_ap_slp<<<dim3((T + 127) / 128, m, nf), 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k64_ap_slp");
        if (s->n_pairs > 0) {
            k64_ap_duffy<<<dim3((s->n_pairs + 127) / 128, nf), 128, 0, st>>>(
                a, s->d_pairs, s->n_pairs, rule, 1, s->rule_off[0], s->rule_cnt[0], s->rule_off[1], s->rule_cnt[1],
                s->rule_off[2], s->rule_cnt[2]);
            HBEM_LAUNCH_CHECK("k64_ap_duffy");
        }
        // S_aa at the real field wavenumber
        for (int f = 0; f < nf; ++f) {
            a.kr[f] = kf_re[f0 + f];
            a.ki[f] = 0.0;
        }
        a.out_re = saa_re + (size_t)f0 * saa_stride;
        a.out_im = saa_im + (size_t)f0 * saa_stride;
        a.stride = (long long)saa_stride;
        k64_ap_avg<<<dim3((m + 127) / 128, m, nf), 128, 0, st>>>(a);
        HBEM_LAUNCH_CHECK("k64_ap_avg");
        if (s->n_pairs > 0) {
            k64_ap_duffy<<<dim3((s->n_pairs + 127) / 128, nf), 128, 0, st>>>(
                a, s->d_pairs, s->n_pairs, rule, 2, s->rule_off[0], s->rule_cnt[0], s->rule_off[1], s->rule_cnt[1],
                s->rule_off[2], s->rule_cnt[2]);
            HBEM_LAUNCH_CHECK("k64_ap_duffy");
        }
    }
    return HBEM_OK;
}

extern "C" int hbem_coupled_ib_field_f64(hbem_session *h, int n_freq, const double *kf_re, const double *qa_re,
                                         const double *qa_im, const float *obs_3xn, int n_obs, double *out_re,
                                         double *out_im, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field_f64: NULL session");
    if (s->m_ap <= 0) return fail(HBEM_ERR_STATE, "hbem_coupled_ib_field_f64: no aperture set on the session");
    if (n_freq <= 0 || n_obs <= 0) return HBEM_OK;
    if (!kf_re || !qa_re || !qa_im || !obs_3xn || !out_re || !out_im)
        return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field_f64: NULL pointer");
    if (n_obs > 65535) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field_f64: at most 65535 points per call");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(kf_re[f])) return fail(HBEM_ERR_ARG, "hbem_coupled_ib_field_f64: non-finite wavenumber");
    HBEM_CUDA(cudaSetDevice(s->device));
    int rc = ensure_geo64(*s);
    if (rc != HBEM_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    for (int f0 = 0; f0 < n_freq; f0 += kMaxF64) {
        const int nf = std::min(kMaxF64, n_freq - f0);
        Ap64Args a{};
        a.g = geo64(*s);
        a.ap = s->d_ap_tris;
        a.ap_local = s->d_ap_local;
        a.m = s->m_ap;
        for (int f = 0; f < nf; ++f) a.kr[f] = kf_re[f0 + f];
        a.out_re = out_re + (size_t)f0 * n_obs;
        a.out_im = out_im + (size_t)f0 * n_obs;
        k64_rayleigh<<<dim3(n_obs, nf), 256, 0, st>>>(a, qa_re + (size_t)f0 * s->m_ap, qa_im + (size_t)f0 * s->m_ap,
                                                      s->m_ap, obs_3xn, n_obs, n_obs);
        HBEM_LAUNCH_CHECK("k64_rayleigh");
    }
    return HBEM_OK;
}

// CHIEF least squares for n_freq assembled systems and n_src right-hand sides
// (see k64_chief_rows): frequencies in chunks of at most 32 whose complex128
// working copies fit a quarter of the free device memory.
extern "C" int hbem_chief_lstsq(hbem_session *h, int n_freq, int n_src, const float *k_re, const float *k_im,
                                const float *q_re, const float *q_im, long long q_stride, long long q_src_stride,
                                const float *beta_re, const float *beta_im, const float *a_re, const float *a_im,
                                long long lda, long long a_stride, const float *b_re, const float *b_im,
                                long long b_stride, long long b_src_stride, const float *chief_3xm, int m,
                                double weight, float *x_re, float *x_im, long long x_stride, long long x_src_stride,
                                double *resid, double *scale_out, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: NULL session");
    if (n_freq <= 0) return HBEM_OK;
    if (n_src < 1 || n_src > kMaxChiefSrc) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: 1 .. 8 sources");
    if (!k_re || !a_re || !a_im || !b_re || !b_im || !x_re || !x_im || !chief_3xm || !q_re || !q_im)
        return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: NULL pointer");
    if ((beta_re == nullptr) != (beta_im == nullptr)) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: beta_re/beta_im");
    const int n = s->n_dof, T = s->n_triangles;
    if (m < 1) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: at least one CHIEF point");
    if (!(weight > 0.0) || !std::isfinite(weight)) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: weight must be finite and positive");
    if (lda < n || a_stride < lda * (long long)n || b_stride < n || x_stride < n || q_stride < T ||
        (n_src > 1 && (b_src_stride < b_stride * n_freq || x_src_stride < x_stride * n_freq ||
                       q_src_stride < q_stride * n_freq)))
        return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: strides too small");
    for (int i = 0; i < 3 * m; ++i)
        if (!std::isfinite(chief_3xm[i])) return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: CHIEF points must be finite");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f]) || (k_im && !std::isfinite(k_im[f])))
            return fail(HBEM_ERR_ARG, "hbem_chief_lstsq: wavenumbers must be finite");
    HBEM_CUDA(cudaSetDevice(s->device));
    int rc = ensure_geo64(*s);
    if (rc != HBEM_OK) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const int rows = n + m, cols = n + n_src;
    const long long ldm = cols, m_stride = (long long)rows * ldm;
    size_t free_b = 0, total_b = 0;
    HBEM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_f = (size_t)m_stride * 16 + (size_t)m * n * 16 + (size_t)n_src * (m + 2 * n) * 16 + 64 * (size_t)cols;
    int chunk = (int)std::min<size_t>((size_t)kMaxF64, std::max<size_t>(1, free_b / 4 / per_f));
    const int fc_max = std::min(chunk, n_freq);
    // scratch of one chunk
    const size_t nC = (size_t)fc_max * m * n, nD = (size_t)n_src * fc_max * m, nM = (size_t)fc_max * m_stride;
    const size_t nT = (size_t)fc_max * 2 * cols, nP = (size_t)fc_max * n_src * 2 * n;
    const size_t bytes = sizeof(double) * (2 * nC + 2 * nD + 2 * nM + 2 * nT + nP + fc_max) +
                         sizeof(unsigned long long) * 2 * fc_max + sizeof(float) * 3 * m + 256;
    unsigned char *mem = nullptr;
    HBEM_CUDA(cudaMallocAsync((void **)&mem, bytes, st));
    double *c_re = reinterpret_cast<double *>(mem), *c_im = c_re + nC;
    double *d_re = c_im + nC, *d_im = d_re + nD;
    double *m_re = d_im + nD, *m_im = m_re + nM;
    double *tau = m_im + nM, *u = tau + nT, *pv = u + nT, *sc = pv + nP;
    unsigned long long *anorm = reinterpret_cast<unsigned long long *>(sc + fc_max), *cnorm = anorm + fc_max;
    float *pts = reinterpret_cast<float *>(cnorm + fc_max);
    auto done = [&](int r) {
        cudaFreeAsync(mem, st);
        return r;
    };
    auto launched = [&](const char *what) -> int {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, what);
        count_launch();
        ++s->launches;
        return HBEM_OK;
    };
    if (cudaMemcpyAsync(pts, chief_3xm, sizeof(float) * 3 * m, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return done(cuda_fail(cudaGetLastError(), "hbem_chief_lstsq: points"));
    for (int f0 = 0; f0 < n_freq; f0 += fc_max) {
        const int fc = std::min(fc_max, n_freq - f0);
        cudaError_t e = cudaMemsetAsync(c_re, 0, sizeof(double) * (2 * nC + 2 * nD), st);
        if (e == cudaSuccess) e = cudaMemsetAsync(anorm, 0, sizeof(unsigned long long) * 2 * fc_max, st);
        if (e != cudaSuccess) return done(cuda_fail(e, "hbem_chief_lstsq: memset"));
        ChiefArgs ca{};
        ca.g = geo64(*s);
        ca.pts = pts;
        ca.q_re = q_re + (size_t)f0 * q_stride;
        ca.q_im = q_im + (size_t)f0 * q_stride;
        ca.q_stride = q_stride;
        ca.q_src_stride = q_src_stride;
        ca.beta_re = beta_re;
        ca.beta_im = beta_im;
        ca.c_re = c_re; ca.c_im = c_im; ca.d_re = d_re; ca.d_im = d_im;
        ca.m = m; ca.n = n; ca.n_src = n_src; ca.nf = fc;
        for (int f = 0; f < fc; ++f) {
            ca.kr[f] = k_re[f0 + f];
            ca.ki[f] = k_im ? k_im[f0 + f] : 0.0;
        }
        k64_chief_rows<<<dim3((T + 255) / 256, m, fc), 256, 0, st>>>(ca);
        if ((rc = launched("k64_chief_rows")) != HBEM_OK) return done(rc);
        k64_inf_norm<float><<<dim3((n + 7) / 8, fc), 256, 0, st>>>(n, n, a_re + (size_t)f0 * a_stride,
                                                                  a_im + (size_t)f0 * a_stride, lda, a_stride, anorm);
        if ((rc = launched("k64_inf_norm")) != HBEM_OK) return done(rc);
        k64_inf_norm<double><<<dim3((m + 7) / 8, fc), 256, 0, st>>>(m, n, c_re, c_im, n, (long long)m * n, cnorm);
        if ((rc = launched("k64_inf_norm")) != HBEM_OK) return done(rc);
        ChiefBuildArgs ba{};
        ba.a_re = a_re + (size_t)f0 * a_stride; ba.a_im = a_im + (size_t)f0 * a_stride;
        ba.lda = lda; ba.a_stride = a_stride;
        ba.b_re = b_re + (size_t)f0 * b_stride; ba.b_im = b_im + (size_t)f0 * b_stride;
        ba.b_stride = b_stride; ba.b_src_stride = b_src_stride;
        ba.c_re = c_re; ba.c_im = c_im; ba.d_re = d_re; ba.d_im = d_im;
        ba.anorm = anorm; ba.cnorm = cnorm;
        ba.m_re = m_re; ba.m_im = m_im; ba.ldm = ldm; ba.m_stride = m_stride;
        ba.scale = sc; ba.weight = weight;
        ba.n = n; ba.m = m; ba.n_src = n_src; ba.nf = fc;
        const long long elems = (long long)rows * cols;
        k64_chief_build<<<dim3((unsigned)std::min<long long>((elems + 255) / 256, 4096), fc), 256, 0, st>>>(ba);
        if ((rc = launched("k64_chief_build")) != HBEM_OK) return done(rc);
        for (int j = 0; j < n; ++j) {
            k64_hh_reflector<<<fc, 256, 0, st>>>(rows, cols, j, m_re, m_im, ldm, m_stride, tau, u);
            if ((rc = launched("k64_hh_reflector")) != HBEM_OK) return done(rc);
            const dim3 g((cols - j - 1 + 255) / 256, (rows - j + kHhRows - 1) / kHhRows, fc);
            k64_hh_dot<<<g, 256, 0, st>>>(rows, cols, j, m_re, m_im, ldm, m_stride, u);
            if ((rc = launched("k64_hh_dot")) != HBEM_OK) return done(rc);
            k64_hh_update<<<g, 256, 0, st>>>(rows, cols, j, m_re, m_im, ldm, m_stride, tau, u);
            if ((rc = launched("k64_hh_update")) != HBEM_OK) return done(rc);
        }
        k64_upper_solve<<<dim3(n_src, fc), 256, 0, st>>>(n, n_src, m_re, m_im, ldm, m_stride, pv);
        if ((rc = launched("k64_upper_solve")) != HBEM_OK) return done(rc);
        k64_chief_finish<<<dim3(n_src, fc), 256, 0, st>>>(
            n, m, n_src, fc, pv, c_re, c_im, d_re, d_im, sc, b_re + (size_t)f0 * b_stride, b_im + (size_t)f0 * b_stride,
            b_stride, b_src_stride, x_re + (size_t)f0 * x_stride, x_im + (size_t)f0 * x_stride, x_stride,
            x_src_stride, resid ? resid + f0 : nullptr, n_freq);
        if ((rc = launched("k64_chief_finish")) != HBEM_OK) return done(rc);
        if (scale_out && cudaMemcpyAsync(scale_out + f0, sc, sizeof(double) * fc, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            return done(cuda_fail(cudaGetLastError(), "hbem_chief_lstsq: scale"));
    }
    return done(HBEM_OK);
}
