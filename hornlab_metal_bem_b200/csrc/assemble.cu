// Dense P1 Galerkin assembly of the Helmholtz double-layer system and the
// single-layer right-hand side on sm_100a.
//
//   A_ij = w_sym * sum_{tau ∋ i, sigma ∋ j} sum_images  ∫∫ phi_i phi_j dG/dn_y
//          - 1/2 w_sym * M_ij                      (reference main.swift:3993-4133)
//   b_i  = w_sym * sum_{tau ∋ i} sum_sigma ∫∫ phi_i G  q_sigma   (main.swift:3698-3736)
//   + Robin coupling -1/3 (i k beta_sigma) ∫∫ phi_i G on every (i, j)  (main.swift:4103-4110)
//   + Duffy corrections (singular - regular) on touching pairs (main.swift:4246-4431),
//     folded into A and b on the device (the reference folds them on the CPU,
//     main.swift:6498-6561).
//
// Kernel design (regular part).  A CTA owns a tile of 32 test triangles
// (one per lane) x 64 trial triangles (eight per warp, warp-uniform).  The
// trial tile's quadrature points are staged once in shared memory and read
// as broadcasts; the test points live in registers.  Each lane evaluates
// 36 x (1 + images) kernel samples per pair with one rsqrt and one fast
// sincos of k r (the hardware reduces the argument in turns itself, as
// accurately as the FP32 product k r is; the rounding of that product is the
// phase error either way), factorises the 3x3
// basis products (inner sum over trial points first) and adds the pair block
// into a shared-memory accumulator indexed by the tile's distinct dofs.  The
// tile is flushed once with red.global.add, which cuts global atomics by the
// ~25x dof sharing inside a spatially compact (Morton ordered) tile.  Values
// that come in pairs (the two orders of an unordered pair, the Duffy kernel's
// two wavenumbers) are accumulated as packed FP32 pairs (FFMA2 / FMUL2 /
// FADD2: half the instructions, the same rounding per element).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>

#include "hbem_internal.h"

namespace hbem {

namespace {

constexpr int kMaxFreqPerLaunch = 64;
constexpr int kAsmFreqs = 2;  // wavenumbers per geometric sample in the pair kernel
constexpr int kMaxSources = 8;   // right-hand sides (velocity sources) one assembly pass fills

struct AsmArgs {
    const float4 *qp;
    const float4 *nrm;
    const int4 *tri;
    const uchar4 *test_slot;
    const uchar4 *trial_slot;
    const int *row_off;
    const int *rows;
    const int *col_off;
    const int *cols;
    const float *q_re;
    const float *q_im;
    const float *beta_re;
    const float *beta_im;
    float *a_re;
    float *a_im;
    float *b_re;
    float *b_im;
    long long q_stride, lda, a_stride, b_stride;
    long long q_src_stride, b_src_stride;   // between sources' Neumann rows / right-hand sides
    int T, nf, n_src;
    float rw;
    float k[kMaxFreqPerLaunch];
    float ki[kMaxFreqPerLaunch];
};

__device__ __forceinline__ float qx(int q) {
    return q == 0 ? HBEM_QX0 : q == 1 ? HBEM_QX1 : q == 2 ? HBEM_QX2 : q == 3 ? HBEM_QX3 : q == 4 ? HBEM_QX4 : HBEM_QX5;
}
__device__ __forceinline__ float qy(int q) {
    return q == 0 ? HBEM_QY0 : q == 1 ? HBEM_QY1 : q == 2 ? HBEM_QY2 : q == 3 ? HBEM_QY3 : q == 4 ? HBEM_QY4 : HBEM_QY5;
}
__device__ __forceinline__ float qw(int q) { return (q == 0 || q == 2 || q == 3) ? HBEM_QWA : HBEM_QWB; }
__device__ __forceinline__ float bas(int q, int i) {
    return i == 0 ? 1.0f - qx(q) - qy(q) : (i == 1 ? qx(q) : qy(q));
}

// Per test quadrature point a: wa[a][i] = w_a * phi_i(x_a) (uniform across the
// warp, served from the constant cache).
__constant__ float c_wa[6][3];
__constant__ float c_wb[6][3];   // w_b * phi_j(y_b)
__constant__ float c_w[6];       // w_b
__constant__ float2 c_wa2[6][3]; // (c_wa, c_wa): packed-pair operands

// One geometric sample y - x shared by NF wavenumbers.  Frequency-independent
// part once (distance, 1/r, (y-x).n / r^3); per wavenumber the phase in turns
// reduced to [-1/2, 1/2], one sincos, and the dG/dn_y update
//   D = (c + i s)(-1/r + i k) (y-x).n / r^2     (times 1/(4 pi) later)
// and, when NEED_G, G = (c + i s) / r.
template <int NF, bool CK, bool NEED_G>
__device__ __forceinline__ void sample_nf(float dx, float dy, float dz, float nx, float ny, float nz,
                                          const float (&k)[NF], const float (&ki)[NF],
                                          float (&dre)[NF], float (&dim)[NF], float (&gre)[NF], float (&gim)[NF]) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float u = rsqrtf(r2);
    u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    const float dn = fmaf(dx, nx, fmaf(dy, ny, dz * nz));
    const float h = dn * (u * u);
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        float sn, cs;
        __sincosf(r * k[f], &sn, &cs);
        float hh = h, uu = u, fre = u;
        if (CK) {
            const float damp = __expf(-ki[f] * r);
            hh *= damp;
            uu *= damp;
            fre += ki[f];
        }
        // D = hh (c + i s)(-fre + i k)
        dre[f] = fmaf(-hh, fmaf(cs, fre, sn * k[f]), dre[f]);
        dim[f] = fmaf(hh, fmaf(cs, k[f], -sn * fre), dim[f]);
        if (NEED_G) {
            gre[f] = fmaf(uu, cs, gre[f]);
            gim[f] = fmaf(uu, sn, gim[f]);
        }
    }
}

// sample_nf with the quadrature weight folded into the geometric factors
// (D and G come out multiplied by wgt; the phase and 1/r of E are unscaled).
template <int NF, bool CK>
__device__ __forceinline__ void sample_nf_w(float dx, float dy, float dz, float nx, float ny, float nz,
                                            const float (&k)[NF], const float (&ki)[NF],
                                            float wgt, float (&dre)[NF], float (&dim)[NF], float (&gre)[NF],
                                            float (&gim)[NF]) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float u = rsqrtf(r2);
    u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    const float dn = fmaf(dx, nx, fmaf(dy, ny, dz * nz));
    const float h = dn * (u * u) * wgt, uw = u * wgt;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        float sn, cs;
        __sincosf(r * k[f], &sn, &cs);
        float hh = h, uu = uw, fre = u;
        if (CK) {
            const float damp = __expf(-ki[f] * r);
            hh *= damp;
            uu *= damp;
            fre += ki[f];
        }
        // D = hh (c + i s)(-fre + i k)
        dre[f] = -hh * fmaf(cs, fre, sn * k[f]);
        dim[f] = hh * fmaf(cs, k[f], -sn * fre);
        gre[f] = uu * cs;
        gim[f] = uu * sn;
    }
}

// sample_nf_w for two wavenumbers held in the two halves of packed FP32
// pairs (k2 = (k0, k1)): sm_100 issues two FP32 multiplies / adds / FMAs of a
// pair as one instruction (FMUL2 / FADD2 / FFMA2), each with the rounding of
// its scalar twin.  nk2 = -k2.
template <bool CK>
__device__ __forceinline__ void sample2_w(float dx, float dy, float dz, float nx, float ny, float nz, float2 k2,
                                          float2 nk2, float2 ki2, float wgt, float2 &dre, float2 &dim, float2 &gre,
                                          float2 &gim) {
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float u = rsqrtf(r2);
    u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    const float dn = fmaf(dx, nx, fmaf(dy, ny, dz * nz));
    const float h = dn * (u * u) * wgt, uw = u * wgt;
    const float2 ph = __fmul2_rn(make_float2(r, r), k2);
    float2 sn, cs;
    __sincosf(ph.x, &sn.x, &cs.x);
    __sincosf(ph.y, &sn.y, &cs.y);
    float2 nh = make_float2(-h, -h), uu = make_float2(uw, uw), fre = make_float2(u, u);
    if (CK) {
        const float2 damp = make_float2(__expf(-ki2.x * r), __expf(-ki2.y * r));
        nh = __fmul2_rn(nh, damp);
        uu = __fmul2_rn(uu, damp);
        fre = __fadd2_rn(fre, ki2);
    }
    // D = hh (c + i s)(-fre + i k): re = -hh (c fre + s k), im = -hh (s fre - c k)
    dre = __fmul2_rn(nh, __ffma2_rn(cs, fre, __fmul2_rn(sn, k2)));
    dim = __fmul2_rn(nh, __ffma2_rn(sn, fre, __fmul2_rn(cs, nk2)));
    gre = __fmul2_rn(uu, cs);
    gim = __fmul2_rn(uu, sn);
}

template <int SYM, int NF, bool CK, bool NEED_G>
__device__ __forceinline__ void pair_block(const float4 *__restrict__ tq, const float4 *__restrict__ sp, float nx,
                                           float ny, float nz, bool self, const float (&k)[NF],
                                           const float (&ki)[NF], float (&are)[NF][9],
                                           float (&aim)[NF][9], float (&sre)[NF][3], float (&sim)[NF][3]) {
#pragma unroll
    for (int f = 0; f < NF; ++f) {
#pragma unroll
        for (int i = 0; i < 9; ++i) are[f][i] = aim[f][i] = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i) sre[f][i] = sim[f][i] = 0.0f;
    }
    // The test-point loop stays rolled (test point from shared memory, weights
    // from constant memory) so the kernel body fits the instruction cache;
    // the trial-point loop is unrolled with the image samples.
#pragma unroll 1
    for (int a = 0; a < 6; ++a) {
        const float4 x = tq[a * kTestTile];
        float ere[NF][3], eim[NF][3], hre[NF], him[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            hre[f] = him[f] = 0.f;
#pragma unroll
            for (int j = 0; j < 3; ++j) ere[f][j] = eim[f][j] = 0.f;
        }
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            const float4 y = sp[b];
            float dre[NF], dim[NF], gre[NF], gim[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) dre[f] = dim[f] = gre[f] = gim[f] = 0.f;
            if (!(self && a == b))
                sample_nf<NF, CK, NEED_G>(y.x - x.x, y.y - x.y, y.z - x.z, nx, ny, nz, k, ki, dre, dim, gre, gim);
            if (SYM == 1 || SYM == 3)
                sample_nf<NF, CK, NEED_G>(-y.x - x.x, y.y - x.y, y.z - x.z, -nx, ny, nz, k, ki, dre, dim, gre, gim);
            if (SYM == 2 || SYM == 3)
                sample_nf<NF, CK, NEED_G>(y.x - x.x, -y.y - x.y, y.z - x.z, nx, -ny, nz, k, ki, dre, dim, gre, gim);
            if (SYM == 3)
                sample_nf<NF, CK, NEED_G>(-y.x - x.x, -y.y - x.y, y.z - x.z, -nx, -ny, nz, k, ki, dre, dim, gre,
                                          gim);
            if (SYM == 4)
                sample_nf<NF, CK, NEED_G>(y.x - x.x, y.y - x.y, -y.z - x.z, nx, ny, -nz, k, ki, dre, dim, gre, gim);
#pragma unroll
            for (int f = 0; f < NF; ++f) {
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float wb = qw(b) * bas(b, j);
                    ere[f][j] = fmaf(dre[f], wb, ere[f][j]);
                    eim[f][j] = fmaf(dim[f], wb, eim[f][j]);
                }
                if (NEED_G) {
                    hre[f] = fmaf(gre[f], qw(b), hre[f]);
                    him[f] = fmaf(gim[f], qw(b), him[f]);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float wa = c_wa[a][i];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    are[f][i * 3 + j] = fmaf(wa, ere[f][j], are[f][i * 3 + j]);
                    aim[f][i * 3 + j] = fmaf(wa, eim[f][j], aim[f][i * 3 + j]);
                }
                if (NEED_G) {
                    sre[f][i] = fmaf(wa, hre[f], sre[f][i]);
                    sim[f][i] = fmaf(wa, him[f], sim[f][i]);
                }
            }
        }
    }
}

// blockIdx.z selects a group of NF consecutive frequencies; a missing last
// member (odd count) is computed on a repeated wavenumber and not flushed.
template <int SYM, bool CK, int MINB>
__global__ void __launch_bounds__(kAsmThreads, MINB) k_regular(const __grid_constant__ AsmArgs p) {
    constexpr int NF = kAsmFreqs;
    extern __shared__ float2 s_acc[];
    __shared__ float4 s_qp[kTrialTile * 6];
    __shared__ float4 s_tq[6 * kTestTile];   // test points, [a][lane]
    __shared__ float4 s_nrm[kTrialTile];
    __shared__ uchar4 s_cs[kTrialTile];
    __shared__ float4 s_qb[NF][kTrialTile];
    __shared__ int s_flag[kTrialTile];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int f0 = blockIdx.z * NF;
    const int nfv = min(NF, p.nf - f0);
    const int test_tile = blockIdx.y, trial_tile = blockIdx.x;
    const int T = p.T;
    const int r0 = p.row_off[test_tile], nrows = p.row_off[test_tile + 1] - r0;
    const int c0 = p.col_off[trial_tile], ncols = p.col_off[trial_tile + 1] - c0;
    const int ldc = ncols | 1;  // odd row pitch spreads same-column rows over banks
    const int plane = nrows * ldc + nrows;
    const int tbase = trial_tile * kTrialTile;
    const int ntrial = min(kTrialTile, T - tbase);
    const int test0 = test_tile * kTestTile;
    const int ntest = min(kTestTile, T - test0);

    for (int i = tid; i < NF * plane; i += kAsmThreads) s_acc[i] = make_float2(0.f, 0.f);
    for (int i = tid; i < ntrial * 6; i += kAsmThreads) s_qp[i] = p.qp[(size_t)tbase * 6 + i];
    for (int i = tid; i < ntest * 6; i += kAsmThreads) {
        const int t = i / 6, a = i - 6 * t;
        s_tq[a * kTestTile + t] = p.qp[(size_t)(test0 + t) * 6 + a];
    }
    for (int i = tid; i < ntrial; i += kAsmThreads) {
        s_nrm[i] = p.nrm[tbase + i];
        s_cs[i] = p.trial_slot[tbase + i];
        const int orig = p.tri[tbase + i].w;
        int flag = 0;
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            float4 qb = make_float4(0.f, 0.f, 0.f, 0.f);
            if (p.q_re && f < nfv) {
                qb.x = p.q_re[(size_t)(f0 + f) * p.q_stride + orig];
                qb.y = p.q_im[(size_t)(f0 + f) * p.q_stride + orig];
            }
            if (p.beta_re) {
                qb.z = p.beta_re[orig];
                qb.w = p.beta_im[orig];
            }
            s_qb[f][i] = qb;
            flag |= (qb.x != 0.f || qb.y != 0.f || qb.z != 0.f || qb.w != 0.f) ? 1 : 0;
        }
        s_flag[i] = flag;
    }
    __syncthreads();

    float k[NF], ki[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const int ff = f0 + min(f, nfv - 1);
        k[f] = p.k[ff];
        ki[f] = p.ki[ff];
    }
    const int test = test0 + lane;
    if (lane < ntest) {
        const float tjac = p.nrm[test].w;
        const uchar4 rs = p.test_slot[test];
        const int rslot[3] = {rs.x, rs.y, rs.z};
        const float4 *tq = &s_tq[lane];
        for (int jj = warp; jj < ntrial; jj += kAsmThreads / 32) {
            const float4 nj = s_nrm[jj];
            const bool self = (tbase + jj) == test;
            float are[NF][9], aim[NF][9], sre[NF][3], sim[NF][3];
            if (s_flag[jj])
                pair_block<SYM, NF, CK, true>(tq, &s_qp[jj * 6], nj.x, nj.y, nj.z, self, k, ki, are, aim, sre, sim);
            else
                pair_block<SYM, NF, CK, false>(tq, &s_qp[jj * 6], nj.x, nj.y, nj.z, self, k, ki, are, aim, sre,
                                               sim);
            const float scale = HBEM_INV4PI * tjac * nj.w;
            const uchar4 cs = s_cs[jj];
            const int cslot[3] = {cs.x, cs.y, cs.z};
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const float4 qb = s_qb[f][jj];
                float2 *acc = s_acc + f * plane;
                float2 *rhs = acc + nrows * ldc;
                float rob_re = 0.f, rob_im = 0.f;  // -(1/3) i k beta
                if (qb.z != 0.f || qb.w != 0.f) {
                    // i k beta with k = k + i ki: (-ki + i k)(br + i bi)
                    const float ikb_re = -ki[f] * qb.z - k[f] * qb.w;
                    const float ikb_im = -ki[f] * qb.w + k[f] * qb.z;
                    rob_re = -ikb_re * (1.0f / 3.0f);
                    rob_im = -ikb_im * (1.0f / 3.0f);
                }
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const float s_re = sre[f][i] * scale, s_im = sim[f][i] * scale;
                    const float radd_re = rob_re * s_re - rob_im * s_im;
                    const float radd_im = rob_re * s_im + rob_im * s_re;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        float vre = are[f][i * 3 + j] * scale + radd_re;
                        float vim = aim[f][i * 3 + j] * scale + radd_im;
                        if (self) vre -= 0.25f * tjac * (i == j ? (1.0f / 6.0f) : (1.0f / 12.0f));
                        float2 *dst = &acc[rslot[i] * ldc + cslot[j]];
                        atomicAdd(&dst->x, vre * p.rw);
                        atomicAdd(&dst->y, vim * p.rw);
                    }
                    if (qb.x != 0.f || qb.y != 0.f) {
                        atomicAdd(&rhs[rslot[i]].x, (s_re * qb.x - s_im * qb.y) * p.rw);
                        atomicAdd(&rhs[rslot[i]].y, (s_re * qb.y + s_im * qb.x) * p.rw);
                    }
                }
            }
        }
    }
    __syncthreads();

    for (int f = 0; f < nfv; ++f) {
        const float2 *acc = s_acc + f * plane;
        float *are_g = p.a_re + (size_t)(f0 + f) * p.a_stride;
        float *aim_g = p.a_im + (size_t)(f0 + f) * p.a_stride;
        for (int e = tid; e < nrows * ncols; e += kAsmThreads) {
            const int r = e / ncols, c = e - r * ncols;
            const size_t off = (size_t)p.rows[r0 + r] * p.lda + p.cols[c0 + c];
            const float2 v = acc[r * ldc + c];
            atomicAdd(are_g + off, v.x);
            atomicAdd(aim_g + off, v.y);
        }
        if (p.q_re) {
            const float2 *rhs = acc + nrows * ldc;
            for (int r = tid; r < nrows; r += kAsmThreads) {
                const float2 v = rhs[r];
                if (v.x != 0.f || v.y != 0.f) {
                    const size_t off = (size_t)(f0 + f) * p.b_stride + p.rows[r0 + r];
                    atomicAdd(p.b_re + off, v.x);
                    atomicAdd(p.b_im + off, v.y);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Regular assembly over unordered triangle pairs.  For a sample pair (x on
// the test triangle tau, y on an image M sigma of the trial triangle) the
// double-layer kernel in both orders shares everything but a dot product:
//   dG/dn_y(x, My) = F(r) (d . M n_sigma),   dG/dn_x(y, Mx) = F(r) (-d . n_tau),
//   F = e^{ikr} (ik - 1/r) / r^2,  d = My - x,  r = |d| = |Mx - y|
// (M is an involution and an isometry), and G(r) is the same.  So each
// unordered pair {tau, sigma} (sorted index tau <= sigma) is evaluated once
// (the coincident self-point of tau = sigma has r^2 = 0 exactly and drops out
// through the singular-point guard, as the reference excludes it)
// and adds A[tau dofs][sigma dofs], A[sigma dofs][tau dofs] and both RHS
// rows: one rsqrt / sincos per sample instead of two.  Tiles and the shared
// accumulation are those of k_regular with a second, transposed plane.
// ---------------------------------------------------------------------------
// Without G (NEED_G false) the singular-point guard costs two instructions
// a sample: there r^2 gets 1e-30 added instead, which leaves r^2 of every
// distinct point pair unchanged in FP32 and makes the coincident point
// (d = 0 exactly) contribute exactly 0: its dG/dn terms carry the factor
// d.n = 0 times a finite 1/r^2 = 1e30.
// The two orders ride in the two halves of packed FP32 pairs: dr = (dre,
// tre), di = (dim, tim), one FFMA2 (sm_100: two FP32 FMAs as one
// instruction, each rounded as its scalar twin) for both orders' D or T.
template <bool CK, bool NEED_G>
__device__ __forceinline__ void sample_sym(float dx, float dy, float dz, float nsx, float nsy, float nsz, float ntx,
                                            float nty, float ntz, float k, float ki, float2 &dr, float2 &di,
                                            float &gre, float &gim) {
    const float r2 = NEED_G ? fmaf(dx, dx, fmaf(dy, dy, dz * dz)) : fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, 1.0e-30f)));
    float u = rsqrtf(r2);
    if (NEED_G) u = r2 > 1.0e-14f ? u : 0.0f;
    const float r = r2 * u;
    const float u2 = u * u;
    float hs = fmaf(dx, nsx, fmaf(dy, nsy, dz * nsz)) * u2;
    float ht = -fmaf(dx, ntx, fmaf(dy, nty, dz * ntz)) * u2;
    float sn, cs;
    __sincosf(r * k, &sn, &cs);
    float uu = u, fre = u;
    if (CK) {
        const float damp = __expf(-ki * r);
        hs *= damp;
        ht *= damp;
        uu *= damp;
        fre += ki;
    }
    const float e_re = -fmaf(cs, fre, sn * k), e_im = fmaf(cs, k, -sn * fre);
    const float2 h2 = make_float2(hs, ht);
    dr = __ffma2_rn(h2, make_float2(e_re, e_re), dr);
    di = __ffma2_rn(h2, make_float2(e_im, e_im), di);
    if (NEED_G) {
        gre = fmaf(uu, cs, gre);
        gim = fmaf(uu, sn, gim);
    }
}

// One unordered pair, one wavenumber.  Outputs (times 1/(4 pi) and the
// Jacobians later): fwd[i*3+j] test dof i x trial dof j, trn[j*3+i] trial dof j
// x test dof i; SLP rows sfw[i] (test) and str[j] (trial, summed with the
// test-point weights only).
template <int SYM, bool CK, bool NEED_G>
__device__ __forceinline__ void pair_block_sym(const float4 *__restrict__ tq, const float4 *__restrict__ sp, float nx,
                                               float ny, float nz, float tnx, float tny, float tnz, float k, float ki,
                                               float (&fwr)[9], float (&fwi)[9], float (&tnr)[9],
                                               float (&tni)[9], float (&sfr)[3], float (&sfi)[3], float (&str_)[3],
                                               float (&sti)[3]) {
    float2 Fr[9], Fi[9];   // (fwd[i*3+j], trn[j*3+i])
#pragma unroll
    for (int i = 0; i < 9; ++i) Fr[i] = Fi[i] = make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < 3; ++i) sfr[i] = sfi[i] = str_[i] = sti[i] = 0.0f;
#pragma unroll 1
    for (int a = 0; a < 6; ++a) {
        const float4 x = tq[a * kTestTile];
        float2 er[3], ei[3];
        float hre = 0.f, him = 0.f, g2r[3], g2i[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) { er[j] = ei[j] = make_float2(0.f, 0.f); g2r[j] = g2i[j] = 0.f; }
#pragma unroll
        for (int b = 0; b < 6; ++b) {
            const float4 y = sp[b];
            float2 dr = make_float2(0.f, 0.f), di = make_float2(0.f, 0.f);
            float gre = 0.f, gim = 0.f;
            sample_sym<CK, NEED_G>(y.x - x.x, y.y - x.y, y.z - x.z, nx, ny, nz, tnx, tny, tnz, k, ki, dr, di, gre, gim);
            if (SYM == 1 || SYM == 3)
                sample_sym<CK, NEED_G>(-y.x - x.x, y.y - x.y, y.z - x.z, -nx, ny, nz, tnx, tny, tnz, k, ki,
                                       dr, di, gre, gim);
            if (SYM == 2 || SYM == 3)
                sample_sym<CK, NEED_G>(y.x - x.x, -y.y - x.y, y.z - x.z, nx, -ny, nz, tnx, tny, tnz, k, ki,
                                       dr, di, gre, gim);
            if (SYM == 3)
                sample_sym<CK, NEED_G>(-y.x - x.x, -y.y - x.y, y.z - x.z, -nx, -ny, nz, tnx, tny, tnz, k, ki,
                                       dr, di, gre,
                                        gim);
            if (SYM == 4)
                sample_sym<CK, NEED_G>(y.x - x.x, y.y - x.y, -y.z - x.z, nx, ny, -nz, tnx, tny, tnz, k, ki,
                                       dr, di, gre, gim);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float wb = qw(b) * bas(b, j);
                er[j] = __ffma2_rn(dr, make_float2(wb, wb), er[j]);
                ei[j] = __ffma2_rn(di, make_float2(wb, wb), ei[j]);
                if (NEED_G) {
                    g2r[j] = fmaf(gre, wb, g2r[j]);
                    g2i[j] = fmaf(gim, wb, g2i[j]);
                }
            }
            if (NEED_G) {
                hre = fmaf(gre, qw(b), hre);
                him = fmaf(gim, qw(b), him);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float2 wa = c_wa2[a][i];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                Fr[i * 3 + j] = __ffma2_rn(wa, er[j], Fr[i * 3 + j]);
                Fi[i * 3 + j] = __ffma2_rn(wa, ei[j], Fi[i * 3 + j]);
            }
            if (NEED_G) {
                sfr[i] = fmaf(wa.x, hre, sfr[i]);
                sfi[i] = fmaf(wa.x, him, sfi[i]);
            }
        }
        if (NEED_G) {
            const float wq = c_w[a];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                str_[j] = fmaf(wq, g2r[j], str_[j]);
                sti[j] = fmaf(wq, g2i[j], sti[j]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            fwr[i * 3 + j] = Fr[i * 3 + j].x;
            tnr[j * 3 + i] = Fr[i * 3 + j].y;
            fwi[i * 3 + j] = Fi[i * 3 + j].x;
            tni[j * 3 + i] = Fi[i * 3 + j].y;
        }
}

// blockIdx.z = frequency.  CTAs whose test triangles all follow their trial
// triangles in the sorted order have no unordered pair of their own and exit.
template <int SYM, bool CK, int MINB>
__global__ void __launch_bounds__(kAsmThreads, MINB) k_regular_sym(const __grid_constant__ AsmArgs p) {
    extern __shared__ float2 s_acc[];
    __shared__ float4 s_qp[kTrialTile * 6];
    __shared__ float4 s_tq[kTestTile * 6];
    __shared__ float4 s_nrm[kTrialTile];
    __shared__ uchar4 s_cs[kTrialTile];
    __shared__ float2 s_q[kMaxSources][kTrialTile];    // Neumann data of the trial triangles per source
    __shared__ float2 s_tqq[kMaxSources][kTestTile];   // ... and of the test triangles
    __shared__ float2 s_beta[kTrialTile];
    __shared__ int s_flag[kTrialTile];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int f = blockIdx.z;
    const int test_tile = blockIdx.y, trial_tile = blockIdx.x;
    const int T = p.T;
    const int tbase = trial_tile * kTrialTile;
    const int ntrial = min(kTrialTile, T - tbase);
    const int test0 = test_tile * kTestTile;
    const int ntest = min(kTestTile, T - test0);
    if (test0 > tbase + ntrial - 1) return;   // every test triangle follows every trial triangle
    const int r0 = p.row_off[test_tile], nrows = p.row_off[test_tile + 1] - r0;
    const int c0 = p.col_off[trial_tile], ncols = p.col_off[trial_tile + 1] - c0;
    const int ldc = ncols | 1, ldr = nrows | 1;
    const int nsrc = p.n_src;
    float2 *acc = s_acc;                       // nrows x ldc   (test rows, trial columns)
    float2 *rhs = acc + nrows * ldc;           // nsrc x nrows
    float2 *acc2 = rhs + nsrc * nrows;         // ncols x ldr   (trial rows, test columns)
    float2 *rhs2 = acc2 + ncols * ldr;         // nsrc x ncols
    const int plane = nrows * ldc + nsrc * nrows + ncols * ldr + nsrc * ncols;

    for (int i = tid; i < plane; i += kAsmThreads) s_acc[i] = make_float2(0.f, 0.f);
    for (int i = tid; i < ntrial * 6; i += kAsmThreads) s_qp[i] = p.qp[(size_t)tbase * 6 + i];
    for (int i = tid; i < ntest * 6; i += kAsmThreads) {
        const int t = i / 6, a = i - 6 * t;
        s_tq[a * kTestTile + t] = p.qp[(size_t)(test0 + t) * 6 + a];
    }
    for (int i = tid; i < ntrial; i += kAsmThreads) {
        s_nrm[i] = p.nrm[tbase + i];
        s_cs[i] = p.trial_slot[tbase + i];
        const int orig = p.tri[tbase + i].w;
        int flag = 0;
        for (int sv = 0; sv < nsrc; ++sv) {
            float2 qv = make_float2(0.f, 0.f);
            if (p.q_re) {
                const size_t o = (size_t)sv * p.q_src_stride + (size_t)f * p.q_stride + orig;
                qv = make_float2(p.q_re[o], p.q_im[o]);
            }
            s_q[sv][i] = qv;
            flag |= (qv.x != 0.f || qv.y != 0.f) ? 1 : 0;
        }
        const float2 be = p.beta_re ? make_float2(p.beta_re[orig], p.beta_im[orig]) : make_float2(0.f, 0.f);
        s_beta[i] = be;
        s_flag[i] = flag | ((be.x != 0.f || be.y != 0.f) ? 1 : 0);
    }
    for (int i = tid; i < nsrc * ntest; i += kAsmThreads) {
        const int sv = i / ntest, t = i - sv * ntest;
        float2 qv = make_float2(0.f, 0.f);
        if (p.q_re) {
            const size_t o = (size_t)sv * p.q_src_stride + (size_t)f * p.q_stride + p.tri[test0 + t].w;
            qv = make_float2(p.q_re[o], p.q_im[o]);
        }
        s_tqq[sv][t] = qv;
    }
    __syncthreads();

    const float k = p.k[f], ki = p.ki[f];
    const int test = test0 + lane;
    if (lane < ntest) {
        const float4 tn = p.nrm[test];
        const float tjac = tn.w;
        const uchar4 rs = p.test_slot[test];
        const int rslot[3] = {rs.x, rs.y, rs.z};
        const int torig = p.tri[test].w;
        const float2 tbe = p.beta_re ? make_float2(p.beta_re[torig], p.beta_im[torig]) : make_float2(0.f, 0.f);
        bool tflag = tbe.x != 0.f || tbe.y != 0.f;
        for (int sv = 0; sv < nsrc; ++sv) tflag |= s_tqq[sv][lane].x != 0.f || s_tqq[sv][lane].y != 0.f;
        const float4 *tq = &s_tq[lane];
        // i k beta / 3 terms: Robin rows of the trial (forward) and test (transposed) triangles
        auto robin = [&](float br, float bi, float &rr, float &ri) {
            rr = 0.f;
            ri = 0.f;
            if (br != 0.f || bi != 0.f) {
                const float ikb_re = -ki * br - k * bi;
                const float ikb_im = -ki * bi + k * br;
                rr = -ikb_re * (1.0f / 3.0f);
                ri = -ikb_im * (1.0f / 3.0f);
            }
        };
        float rob2_re, rob2_im;
        robin(tbe.x, tbe.y, rob2_re, rob2_im);
        for (int jj = warp; jj < ntrial; jj += kAsmThreads / 32) {
            const int sigma = tbase + jj;
            if (sigma < test) continue;
            const float4 nj = s_nrm[jj];
            const bool self = sigma == test;
            float fwr[9], fwi[9], tnr[9], tni[9], sfr[3], sfi[3], str_[3], sti[3];
            if (s_flag[jj] || tflag)
                pair_block_sym<SYM, CK, true>(tq, &s_qp[jj * 6], nj.x, nj.y, nj.z, tn.x, tn.y, tn.z, k, ki,
                                              fwr, fwi, tnr, tni, sfr, sfi, str_, sti);
            else
                pair_block_sym<SYM, CK, false>(tq, &s_qp[jj * 6], nj.x, nj.y, nj.z, tn.x, tn.y, tn.z, k, ki,
                                               fwr, fwi, tnr, tni, sfr, sfi, str_, sti);
            const float scale = HBEM_INV4PI * tjac * nj.w;
            const uchar4 cs = s_cs[jj];
            const int cslot[3] = {cs.x, cs.y, cs.z};
            const float2 be = s_beta[jj];
            float rob_re, rob_im;
            robin(be.x, be.y, rob_re, rob_im);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float s_re = sfr[i] * scale, s_im = sfi[i] * scale;
                const float radd_re = rob_re * s_re - rob_im * s_im;
                const float radd_im = rob_re * s_im + rob_im * s_re;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    float vre = fwr[i * 3 + j] * scale + radd_re;
                    float vim = fwi[i * 3 + j] * scale + radd_im;
                    if (self) vre -= 0.25f * tjac * (i == j ? (1.0f / 6.0f) : (1.0f / 12.0f));
                    float2 *dst = &acc[rslot[i] * ldc + cslot[j]];
                    atomicAdd(&dst->x, vre * p.rw);
                    atomicAdd(&dst->y, vim * p.rw);
                }
#pragma unroll 1
                for (int sv = 0; sv < nsrc; ++sv) {
                    const float2 qv = s_q[sv][jj];
                    if (qv.x != 0.f || qv.y != 0.f) {
                        atomicAdd(&rhs[sv * nrows + rslot[i]].x, (s_re * qv.x - s_im * qv.y) * p.rw);
                        atomicAdd(&rhs[sv * nrows + rslot[i]].y, (s_re * qv.y + s_im * qv.x) * p.rw);
                    }
                }
            }
            if (self) continue;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const float s_re = str_[j] * scale, s_im = sti[j] * scale;
                const float radd_re = rob2_re * s_re - rob2_im * s_im;
                const float radd_im = rob2_re * s_im + rob2_im * s_re;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const float vre = tnr[j * 3 + i] * scale + radd_re;
                    const float vim = tni[j * 3 + i] * scale + radd_im;
                    float2 *dst = &acc2[cslot[j] * ldr + rslot[i]];
                    atomicAdd(&dst->x, vre * p.rw);
                    atomicAdd(&dst->y, vim * p.rw);
                }
#pragma unroll 1
                for (int sv = 0; sv < nsrc; ++sv) {
                    const float2 qv = s_tqq[sv][lane];
                    if (qv.x != 0.f || qv.y != 0.f) {
                        atomicAdd(&rhs2[sv * ncols + cslot[j]].x, (s_re * qv.x - s_im * qv.y) * p.rw);
                        atomicAdd(&rhs2[sv * ncols + cslot[j]].y, (s_re * qv.y + s_im * qv.x) * p.rw);
                    }
                }
            }
        }
    }
    __syncthreads();

    float *are_g = p.a_re + (size_t)f * p.a_stride;
    float *aim_g = p.a_im + (size_t)f * p.a_stride;
    for (int e = tid; e < nrows * ncols; e += kAsmThreads) {
        const int r = e / ncols, c = e - r * ncols;
        const float2 v = acc[r * ldc + c];
        if (v.x != 0.f || v.y != 0.f) {
            const size_t off = (size_t)p.rows[r0 + r] * p.lda + p.cols[c0 + c];
            atomicAdd(are_g + off, v.x);
            atomicAdd(aim_g + off, v.y);
        }
    }
    for (int e = tid; e < ncols * nrows; e += kAsmThreads) {
        const int c = e / nrows, r = e - c * nrows;
        const float2 v = acc2[c * ldr + r];
        if (v.x != 0.f || v.y != 0.f) {
            const size_t off = (size_t)p.cols[c0 + c] * p.lda + p.rows[r0 + r];
            atomicAdd(are_g + off, v.x);
            atomicAdd(aim_g + off, v.y);
        }
    }
    if (p.q_re) {
        for (int e = tid; e < nsrc * nrows; e += kAsmThreads) {
            const int sv = e / nrows, r = e - sv * nrows;
            const float2 v = rhs[e];
            if (v.x != 0.f || v.y != 0.f) {
                const size_t off = (size_t)sv * p.b_src_stride + (size_t)f * p.b_stride + p.rows[r0 + r];
                atomicAdd(p.b_re + off, v.x);
                atomicAdd(p.b_im + off, v.y);
            }
        }
        for (int e = tid; e < nsrc * ncols; e += kAsmThreads) {
            const int sv = e / ncols, c = e - sv * ncols;
            const float2 v = rhs2[e];
            if (v.x != 0.f || v.y != 0.f) {
                const size_t off = (size_t)sv * p.b_src_stride + (size_t)f * p.b_stride + p.cols[c0 + c];
                atomicAdd(p.b_re + off, v.x);
                atomicAdd(p.b_im + off, v.y);
            }
        }
    }
}

template <int SYM, bool CK, int MINB>
cudaError_t launch_regular_sym_t(const AsmArgs &a, dim3 grid, size_t smem, cudaStream_t st) {
    auto kern = k_regular_sym<SYM, CK, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kAsmThreads, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool CK>
cudaError_t dispatch_sym_pairs(int sym, const AsmArgs &a, dim3 grid, size_t smem, cudaStream_t st) {
    switch (sym) {
        case 0: return launch_regular_sym_t<0, CK, 2>(a, grid, smem, st);
        case 1: return launch_regular_sym_t<1, CK, 2>(a, grid, smem, st);
        case 2: return launch_regular_sym_t<2, CK, 2>(a, grid, smem, st);
        case 3: return launch_regular_sym_t<3, CK, 2>(a, grid, smem, st);
        default: return launch_regular_sym_t<4, CK, 2>(a, grid, smem, st);
    }
}

template <int SYM, bool CK, int MINB>
cudaError_t launch_regular_t(const AsmArgs &a, dim3 grid, size_t smem, cudaStream_t st) {
    auto kern = k_regular<SYM, CK, MINB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kAsmThreads, smem, st>>>(a);
    return cudaGetLastError();
}

// Resident CTAs per SM for the pair kernel: 2 (128 registers, no spills) or 3
// (80 registers).  HBEM_TUNE_ASM_MINBLOCKS (or the HBEM_ASM_MINBLOCKS
// environment variable) overrides the default.
int regular_min_blocks() {
    const int t = tuning(HBEM_TUNE_ASM_MINBLOCKS);
    if (t == 2 || t == 3) return t;
    static int v = [] {
        const char *e = getenv("HBEM_ASM_MINBLOCKS");
        int m = e ? atoi(e) : 2;
        return (m == 3) ? 3 : 2;
    }();
    return v;
}

template <bool CK, int MINB>
cudaError_t dispatch_sym_m(int sym, const AsmArgs &a, dim3 grid, size_t smem, cudaStream_t st) {
    switch (sym) {
        case 0: return launch_regular_t<0, CK, MINB>(a, grid, smem, st);
        case 1: return launch_regular_t<1, CK, MINB>(a, grid, smem, st);
        case 2: return launch_regular_t<2, CK, MINB>(a, grid, smem, st);
        case 3: return launch_regular_t<3, CK, MINB>(a, grid, smem, st);
        default: return launch_regular_t<4, CK, MINB>(a, grid, smem, st);
    }
}

template <bool CK>
cudaError_t dispatch_sym(int sym, const AsmArgs &a, dim3 grid, size_t smem, cudaStream_t st) {
    return regular_min_blocks() == 3 ? dispatch_sym_m<CK, 3>(sym, a, grid, smem, st)
                                     : dispatch_sym_m<CK, 2>(sym, a, grid, smem, st);
}

// ---------------------------------------------------------------------------
// Duffy corrections: one warp per singular pair.  Lanes stride over the
// pair's Duffy points (+ the 36 regular points, subtracted), each computing
// the image point geometry, one kernel sample and the 3 SLP + 9 DLP basis
// products.  Per-lane partial sums and the warp reduction are FP64, so the
// singular - regular difference is formed in double before the single
// rounding into A and b.
// ---------------------------------------------------------------------------
struct DuffyArgs {
    const DuffyPair *pairs;
    const float4 *rule;
    const float *rule_w;
    const float *verts;
    const int *tris;
    const int *l2g;
    const float *areas;
    const float *normals;
    const float *q_re, *q_im, *beta_re, *beta_im;
    float *a_re, *a_im, *b_re, *b_im;
    long long q_stride, lda, a_stride, b_stride;
    long long q_src_stride, b_src_stride;
    int V, T, n_pairs, n_src;
    int rule_off[3], rule_cnt[3];
    // coupled-baffle projections: ap_local[t] = aperture index or -1.
    // mode 0: A/b (when a_re) and S_ia (when sia); mode 1: S_aa only.
    const int *ap_local;
    float *sia_re, *sia_im, *saa_re, *saa_im;
    long long sia_stride, saa_stride;
    int m_ap, mode, nf;
    float k[kMaxFreqPerLaunch];
    float ki[kMaxFreqPerLaunch];
};

__device__ __forceinline__ float refx(int l) { return l == 1 ? 1.f : 0.f; }
__device__ __forceinline__ float refy(int l) { return l == 2 ? 1.f : 0.f; }

// Map a Duffy point onto the shared edge / vertex of the image triangle
// (main.swift:4213-4231).
// Warp totals of NV values per lane (NV = 32, 16 or 8): after the plain
// butterfly levels h >= NV, each transposing level h < NV halves the values a
// lane holds, sending the half its partner keeps; lane L ends with the total
// of value L & (NV - 1), in NV - 1 + (5 - log2 NV) NV shuffles instead of 5 NV.
template <int NV>
__device__ __forceinline__ double warp_transpose_reduce(double (&v)[NV]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int h = 16; h >= NV; h >>= 1)
#pragma unroll
        for (int i = 0; i < NV; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], h);
#pragma unroll
    for (int h = NV / 2; h >= 1; h >>= 1) {
        const bool hi = (lane & h) != 0;
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const double send = hi ? v[i] : v[i + h];
            const double keep = hi ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, h);
        }
    }
    return v[0];
}

__device__ __forceinline__ void remap(float x, float y, int kind, int l1, int l2, float &ox, float &oy) {
    if (kind == 2) {
        const int vc = 3 - l1 - l2;
        const float ax = refx(l1), ay = refy(l1);
        ox = ax + x * (refx(l2) - ax) + y * (refx(vc) - ax);
        oy = ay + x * (refy(l2) - ay) + y * (refy(vc) - ay);
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

// NF wavenumbers per warp (blockIdx.y = group of NF consecutive wavenumbers;
// a missing last member is computed on a repeated wavenumber and not
// written).  The singular points are summed first (FP32 lane partials, FP64
// warp reduction), then the same registers take the regular points.
template <bool CK, int NF, int MINB>
__global__ void __launch_bounds__(256, MINB) k_duffy(const __grid_constant__ DuffyArgs p) {
    const int lane = threadIdx.x & 31;
    const int pi = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (pi >= p.n_pairs) return;
    const int fg = blockIdx.y * NF;
    const int nfv = min(NF, p.nf - fg);
    const DuffyPair pr = p.pairs[pi];
    const int V = p.V, T = p.T;
    // pairs without an aperture trial (and, for S_aa, an unmirrored aperture
    // test) contribute nothing to the projection-only passes
    if (p.mode == 1 && (pr.test_mask != 0 || p.ap_local[pr.test] < 0 || p.ap_local[pr.trial] < 0)) return;
    if (p.mode == 0 && !p.a_re && (!p.ap_local || p.ap_local[pr.trial] < 0)) return;
    float P[3][3], S[3][3];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int vt = p.tris[l * T + pr.test], vs = p.tris[l * T + pr.trial];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P[l][c] = p.verts[c * V + vt];
            S[l][c] = p.verts[c * V + vs];
        }
    }
    const float tsx = (pr.test_mask & 1) ? -1.f : 1.f, tsy = (pr.test_mask & 2) ? -1.f : 1.f,
                tsz = (pr.test_mask & 4) ? -1.f : 1.f;
    const float ssx = (pr.trial_mask & 1) ? -1.f : 1.f, ssy = (pr.trial_mask & 2) ? -1.f : 1.f,
                ssz = (pr.trial_mask & 4) ? -1.f : 1.f;
    const bool tswap = __popc(pr.test_mask) & 1, sswap = __popc(pr.trial_mask) & 1;
    const float nx = ssx * p.normals[pr.trial], ny = ssy * p.normals[T + pr.trial], nz = ssz * p.normals[2 * T + pr.trial];
    const float jac = (2.f * p.areas[pr.test]) * (2.f * p.areas[pr.trial]);
    // the image triangles as vertex 0 plus edge vectors: a point is x0 + t1 e1 + t2 e2
    {
        const float tsg[3] = {tsx, tsy, tsz}, ssg[3] = {ssx, ssy, ssz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P[1][c] = tsg[c] * (P[1][c] - P[0][c]);
            P[2][c] = tsg[c] * (P[2][c] - P[0][c]);
            P[0][c] = tsg[c] * P[0][c];
            S[1][c] = ssg[c] * (S[1][c] - S[0][c]);
            S[2][c] = ssg[c] * (S[2][c] - S[0][c]);
            S[0][c] = ssg[c] * S[0][c];
        }
    }
    float k[NF], ki[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        const int ff = fg + min(f, nfv - 1);
        k[f] = p.k[ff];
        ki[f] = p.ki[ff];
    }

    // Lane partials as moments over the barycentrics (t0 = s0 = 1, t1, t2, s1,
    // s2): acc[f][0..5] = sum G t_a (a = 0, 1, 2; re, im), acc[f][6 + 2 (3a + b)]
    // = sum D t_a s_b; turned into the P1 entries (tb = 1 - t1 - t2, t1, t2)
    // in FP64 before the warp reduction.
    float acc[NF][24];
    // NF = 2: the two wavenumbers' moments as packed pairs (x: the first, y:
    // the second), one FFMA2 per moment and point
    float2 acc2[24];
    const float2 k2 = make_float2(k[0], k[NF - 1]), nk2 = make_float2(-k[0], -k[NF - 1]);
    const float2 ki2 = make_float2(ki[0], ki[NF - 1]);
    // (txi, teta), (sxi, seta): the point's base-local barycentrics (t1, t2),
    // (s1, s2) on the test and trial triangles
    auto accumulate = [&](float txi, float teta, float sxi, float seta, float w) {
        float d[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float x = fmaf(teta, P[2][c], fmaf(txi, P[1][c], P[0][c]));
            const float y = fmaf(seta, S[2][c], fmaf(sxi, S[1][c], S[0][c]));
            d[c] = y - x;
        }
        if constexpr (NF == 2) {
            float2 dre, dim, gre, gim;
            sample2_w<CK>(d[0], d[1], d[2], nx, ny, nz, k2, nk2, ki2, w, dre, dim, gre, gim);
            const float2 t1 = make_float2(txi, txi), t2 = make_float2(teta, teta);
            const float2 s1 = make_float2(sxi, sxi), s2 = make_float2(seta, seta);
            const float2 tw[3] = {make_float2(1.f, 1.f), t1, t2}, sw[3] = {make_float2(1.f, 1.f), s1, s2};
            const float2 ts[2][2] = {{__fmul2_rn(t1, s1), __fmul2_rn(t1, s2)}, {__fmul2_rn(t2, s1), __fmul2_rn(t2, s2)}};
            acc2[0] = __fadd2_rn(acc2[0], gre);
            acc2[1] = __fadd2_rn(acc2[1], gim);
            acc2[2] = __ffma2_rn(gre, t1, acc2[2]);
            acc2[3] = __ffma2_rn(gim, t1, acc2[3]);
            acc2[4] = __ffma2_rn(gre, t2, acc2[4]);
            acc2[5] = __ffma2_rn(gim, t2, acc2[5]);
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const int e = 6 + 2 * (3 * aa + bb);
                    if (aa == 0 && bb == 0) {
                        acc2[e] = __fadd2_rn(acc2[e], dre);
                        acc2[e + 1] = __fadd2_rn(acc2[e + 1], dim);
                    } else {
                        const float2 wt = aa == 0 ? sw[bb] : (bb == 0 ? tw[aa] : ts[aa - 1][bb - 1]);
                        acc2[e] = __ffma2_rn(dre, wt, acc2[e]);
                        acc2[e + 1] = __ffma2_rn(dim, wt, acc2[e + 1]);
                    }
                }
            return;
        }
        const float ts[2][2] = {{txi * sxi, txi * seta}, {teta * sxi, teta * seta}};
        const float tw[3] = {1.f, txi, teta}, sw[3] = {1.f, sxi, seta};
        float dre[NF], dim[NF], gre[NF], gim[NF];
        sample_nf_w<NF, CK>(d[0], d[1], d[2], nx, ny, nz, k, ki, w, dre, dim, gre, gim);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            acc[f][0] += gre[f];
            acc[f][1] += gim[f];
            acc[f][2] = fmaf(gre[f], txi, acc[f][2]);
            acc[f][3] = fmaf(gim[f], txi, acc[f][3]);
            acc[f][4] = fmaf(gre[f], teta, acc[f][4]);
            acc[f][5] = fmaf(gim[f], teta, acc[f][5]);
#pragma unroll
            for (int aa = 0; aa < 3; ++aa)
#pragma unroll
                for (int bb = 0; bb < 3; ++bb) {
                    const int e = 6 + 2 * (3 * aa + bb);
                    if (aa == 0 && bb == 0) {
                        acc[f][e] += dre[f];
                        acc[f][e + 1] += dim[f];
                    } else {
                        const float wt = aa == 0 ? sw[bb] : (bb == 0 ? tw[aa] : ts[aa - 1][bb - 1]);
                        acc[f][e] = fmaf(dre[f], wt, acc[f][e]);
                        acc[f][e + 1] = fmaf(dim[f], wt, acc[f][e + 1]);
                    }
                }
        }
    };
    // P1 entry e (layout: 0..5 SLP rows (re, im), 6 + 2 (3 i + j) DLP) of
    // wavenumber f from the moments, in FP64
    auto nodal = [&](int f, int e) -> double {
        const int c = e & 1;
        if (e < 6) {
            const int i = e >> 1;
            const double m0 = acc[f][c], m1 = acc[f][2 + c], m2 = acc[f][4 + c];
            return i == 0 ? m0 - m1 - m2 : (i == 1 ? m1 : m2);
        }
        const int ij = (e - 6) >> 1, i = ij / 3, j = ij - 3 * i;
        auto M = [&](int aa, int bb) -> double { return (double)acc[f][6 + 2 * (3 * aa + bb) + c]; };
        auto Tb = [&](int bb) -> double { return i == 0 ? M(0, bb) - M(1, bb) - M(2, bb) : M(i, bb); };
        return j == 0 ? Tb(0) - Tb(1) - Tb(2) : Tb(j);
    };
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int e = 0; e < 24; ++e) acc[f][e] = 0.f;
#pragma unroll
    for (int e = 0; e < 24; ++e) acc2[e] = make_float2(0.f, 0.f);
    // singular (Duffy) points, then the regular 6x6 rule with negated weights
    // (the correction is singular - regular; the coincident self-point is
    // excluded by index exactly as in the regular assembly,
    // main.swift:4323-4336): one accumulation and one reduction per pair
    const int ri = pr.kind - 1;
    const int off = p.rule_off[ri], cnt = p.rule_cnt[ri];
    const bool self_pair = pr.test == pr.trial && pr.test_mask == pr.trial_mask;
    // A rule point (x, y) on the reference triangle reaches the base-local
    // barycentrics through the pair's Duffy remap (anchoring the rule on the
    // shared vertices, image-local order) and, for a mirrored triangle, the
    // swap back to base-local order: one affine map per side, composed here
    // from three evaluations (its coefficients are 0 or +-1, so the composed
    // map reproduces the two steps exactly).
    float tmap[6], smap[6];   // t1 = m0 + m1 x + m2 y, t2 = m3 + m4 x + m5 y
    auto compose = [&](int l1, int l2, bool swp, float (&mm)[6]) {
        float o[3][2];
        const float xs[3] = {0.f, 1.f, 0.f}, ys[3] = {0.f, 0.f, 1.f};
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            remap(xs[e], ys[e], pr.kind, l1, l2, o[e][0], o[e][1]);
            if (swp) { const float t = o[e][0]; o[e][0] = o[e][1]; o[e][1] = t; }
        }
        mm[0] = o[0][0]; mm[1] = o[1][0] - o[0][0]; mm[2] = o[2][0] - o[0][0];
        mm[3] = o[0][1]; mm[4] = o[1][1] - o[0][1]; mm[5] = o[2][1] - o[0][1];
    };
    compose(pr.tl1, pr.tl2, tswap, tmap);
    compose(pr.sl1, pr.sl2, sswap, smap);
    for (int q = lane; q < cnt + 36; q += 32) {
        float t1, t2, s1, s2, w;
        bool skip = false;
        if (q < cnt) {   // warp-uniform: cnt is a multiple of 32
            const float4 r = __ldg(&p.rule[off + q]);
            w = __ldg(&p.rule_w[off + q]);
            t1 = fmaf(tmap[2], r.y, fmaf(tmap[1], r.x, tmap[0]));
            t2 = fmaf(tmap[5], r.y, fmaf(tmap[4], r.x, tmap[3]));
            s1 = fmaf(smap[2], r.w, fmaf(smap[1], r.z, smap[0]));
            s2 = fmaf(smap[5], r.w, fmaf(smap[4], r.z, smap[3]));
        } else {
            const int rq = q - cnt, a = rq / 6, b = rq - 6 * a;
            t1 = tswap ? qy(a) : qx(a);
            t2 = tswap ? qx(a) : qy(a);
            s1 = sswap ? qy(b) : qx(b);
            s2 = sswap ? qx(b) : qy(b);
            w = -(qw(a) * qw(b));
            skip = self_pair && a == b;
        }
        if (!skip) accumulate(t1, t2, s1, s2, w);
    }
    if constexpr (NF == 2) {
#pragma unroll
        for (int e = 0; e < 24; ++e) {
            acc[0][e] = acc2[e].x;
            acc[NF - 1][e] = acc2[e].y;
        }
    }
    // FP64 warp totals of the 24 NF lane partials (value v = 24 f + e): a
    // transpose-reduce leaves value v of the first set in lane v, of the
    // second set in lane v - S0 (and its mirror); then lane e < 9 gathers DLP
    // entry e and lanes 9..11 the SLP rows, (re, im) per wavenumber
    constexpr int S0 = NF == 2 ? 32 : 16, S1 = NF == 2 ? 16 : 8;
    double red0, red1;
    {
        double v0[S0], v1[S1];
#pragma unroll
        for (int i = 0; i < S0; ++i) v0[i] = nodal(i / 24, i % 24);
#pragma unroll
        for (int i = 0; i < S1; ++i) v1[i] = nodal((S0 + i) / 24, (S0 + i) % 24);
        red0 = warp_transpose_reduce<S0>(v0);
        red1 = warp_transpose_reduce<S1>(v1);
    }
    double own_re[NF], own_im[NF];
    {
        const int e_re = lane < 9 ? 6 + 2 * lane : (lane < 12 ? 2 * (lane - 9) : 0);
#pragma unroll
        for (int f = 0; f < NF; ++f) {
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int v = 24 * f + e_re + c;
                const double g0 = __shfl_sync(0xffffffffu, red0, v & (S0 - 1));
                const double g1 = __shfl_sync(0xffffffffu, red1, (v - S0) & (S1 - 1));
                const double g = v < S0 ? g0 : g1;
                if (c == 0) own_re[f] = g;
                else own_im[f] = g;
            }
        }
    }
    const double scale = (double)HBEM_INV4PI * (double)jac * (double)pr.weight;
    const int i_row = lane < 9 ? lane / 3 : lane - 9;
    if (p.mode == 1) {
        // S_aa: sum_i delta_slp_i / area(test), one contribution per unmirrored pair:
        // gather the three SLP rows (lanes 9..11) and let lane 9 write
#pragma unroll
        for (int f = 0; f < NF; ++f) {
            double s_re = (lane >= 9 && lane < 12) ? own_re[f] : 0.0, s_im = (lane >= 9 && lane < 12) ? own_im[f] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                s_re += __shfl_xor_sync(0xffffffffu, s_re, o);
                s_im += __shfl_xor_sync(0xffffffffu, s_im, o);
            }
            if (lane == 9 && f < nfv) {
                const double inv = 1.0 / fmax((double)p.areas[pr.test], 1e-38);
                const size_t o = (size_t)(fg + f) * p.saa_stride + (size_t)p.ap_local[pr.test] * p.m_ap +
                                 p.ap_local[pr.trial];
                atomicAdd(p.saa_re + o, (float)(s_re * (double)HBEM_INV4PI * (double)jac * inv));
                atomicAdd(p.saa_im + o, (float)(s_im * (double)HBEM_INV4PI * (double)jac * inv));
            }
        }
        return;
    }
    // SLP rows (lanes 9..11), broadcast to the DLP lanes of the same row for Robin
#pragma unroll
    for (int f = 0; f < nfv; ++f) {
        const double sr_own = own_re[f] * scale, si_own = own_im[f] * scale;
        const double sr = __shfl_sync(0xffffffffu, sr_own, 9 + i_row);
        const double si = __shfl_sync(0xffffffffu, si_own, 9 + i_row);
        double dr = own_re[f] * scale, di = own_im[f] * scale;
        if (p.sia_re && lane >= 9 && lane < 12) {
            const int t = p.ap_local[pr.trial];
            if (t >= 0) {
                const size_t o = (size_t)(fg + f) * p.sia_stride + (size_t)p.l2g[pr.test * 3 + i_row] * p.m_ap + t;
                atomicAdd(p.sia_re + o, (float)sr);
                atomicAdd(p.sia_im + o, (float)si);
            }
        }
        if (!p.a_re) continue;
        const float br = p.beta_re ? p.beta_re[pr.trial] : 0.f, bi = p.beta_im ? p.beta_im[pr.trial] : 0.f;
        if (lane < 9) {
            const int j = lane - 3 * (lane / 3);
            if (br != 0.f || bi != 0.f) {
                const double ikb_re = -(double)ki[f] * br - (double)k[f] * bi, ikb_im = -(double)ki[f] * bi + (double)k[f] * br;
                dr -= (sr * ikb_re - si * ikb_im) / 3.0;
                di -= (sr * ikb_im + si * ikb_re) / 3.0;
            }
            const size_t o = (size_t)(fg + f) * p.a_stride + (size_t)p.l2g[pr.test * 3 + i_row] * p.lda +
                             p.l2g[pr.trial * 3 + j];
            atomicAdd(p.a_re + o, (float)dr);
            atomicAdd(p.a_im + o, (float)di);
        } else if (lane < 12 && p.q_re) {
            for (int sv = 0; sv < p.n_src; ++sv) {
                const size_t oq = (size_t)sv * p.q_src_stride + (size_t)(fg + f) * p.q_stride + pr.trial;
                const float qr = p.q_re[oq], qi = p.q_im[oq];
                if (qr != 0.f || qi != 0.f) {
                    const size_t o = (size_t)sv * p.b_src_stride + (size_t)(fg + f) * p.b_stride +
                                     p.l2g[pr.test * 3 + i_row];
                    atomicAdd(p.b_re + o, (float)(sr * qr - si * qi));
                    atomicAdd(p.b_im + o, (float)(sr * qi + si * qr));
                }
            }
        }
    }
}

void fill_k(float *k, float *ki, const float *k_re, const float *k_im, int n) {
    for (int f = 0; f < n; ++f) {
        k[f] = k_re[f];
        ki[f] = k_im ? k_im[f] : 0.f;
    }
}

}  // namespace

int launch_regular(Session &s, int n_freq, const float *k_re, const float *k_im, const float *q_re,
                   const float *q_im, long long q_stride, const float *beta_re, const float *beta_im, float *a_re,
                   float *a_im, long long lda, long long a_stride, float *b_re, float *b_im, long long b_stride,
                   cudaStream_t st, int n_src, long long q_src_stride, long long b_src_stride) {
    if (n_src < 1 || n_src > kMaxSources) return fail(HBEM_ERR_ARG, "assembly: 1 .. 8 sources per pass");
    const size_t smem = (size_t)kAsmFreqs * (s.max_rows * (s.max_cols | 1) + s.max_rows) * sizeof(float2);
    const size_t smem_sym = (size_t)(s.max_rows * (s.max_cols | 1) + n_src * s.max_rows +
                                     s.max_cols * (s.max_rows | 1) + n_src * s.max_cols) * sizeof(float2);
    static bool consts_ready[64] = {false};
    if (s.device >= 0 && s.device < 64 && !consts_ready[s.device]) {
        const double QX[6] = {0.4459484909159651, 0.0915762135097710, 0.1081030181680700,
                              0.4459484909159651, 0.8168475729804590, 0.0915762135097710};
        const double QY[6] = {0.4459484909159651, 0.0915762135097700, 0.4459484909159651,
                              0.1081030181680700, 0.0915762135097700, 0.8168475729804580};
        const float QW[6] = {HBEM_QWA, HBEM_QWB, HBEM_QWA, HBEM_QWA, HBEM_QWB, HBEM_QWB};
        float wa[6][3], w[6];
        for (int q = 0; q < 6; ++q) {
            const float x = (float)QX[q], y = (float)QY[q];
            const float b[3] = {1.0f - x - y, x, y};
            for (int i = 0; i < 3; ++i) wa[q][i] = QW[q] * b[i];
            w[q] = QW[q];
        }
        HBEM_CUDA(cudaMemcpyToSymbol(c_wa, wa, sizeof(wa)));
        HBEM_CUDA(cudaMemcpyToSymbol(c_wb, wa, sizeof(wa)));
        HBEM_CUDA(cudaMemcpyToSymbol(c_w, w, sizeof(w)));
        float2 wa2[6][3];
        for (int q = 0; q < 6; ++q)
            for (int i = 0; i < 3; ++i) wa2[q][i] = make_float2(wa[q][i], wa[q][i]);
        HBEM_CUDA(cudaMemcpyToSymbol(c_wa2, wa2, sizeof(wa2)));
        consts_ready[s.device] = true;
    }
    if (smem > 180 * 1024 || smem_sym > 180 * 1024)
        return fail(HBEM_ERR_ARG, "assembly tile needs too much shared memory (mesh ordering too scattered)");
    for (int f0 = 0; f0 < n_freq; f0 += kMaxFreqPerLaunch) {
        const int nf = std::min(kMaxFreqPerLaunch, n_freq - f0);
        AsmArgs a{};
        a.qp = s.d_qp; a.nrm = s.d_nrm; a.tri = s.d_tri; a.test_slot = s.d_test_slot; a.trial_slot = s.d_trial_slot;
        a.row_off = s.d_row_off; a.rows = s.d_rows; a.col_off = s.d_col_off; a.cols = s.d_cols;
        a.q_re = q_re ? q_re + (size_t)f0 * q_stride : nullptr;
        a.q_im = q_im ? q_im + (size_t)f0 * q_stride : nullptr;
        a.beta_re = beta_re; a.beta_im = beta_im;
        a.a_re = a_re + (size_t)f0 * a_stride; a.a_im = a_im + (size_t)f0 * a_stride;
        a.b_re = b_re ? b_re + (size_t)f0 * b_stride : nullptr;
        a.b_im = b_im ? b_im + (size_t)f0 * b_stride : nullptr;
        a.q_stride = q_stride; a.lda = lda; a.a_stride = a_stride; a.b_stride = b_stride;
        a.q_src_stride = q_src_stride; a.b_src_stride = b_src_stride; a.n_src = n_src;
        a.T = s.n_triangles;
        a.rw = (float)(1 << ((s.sym & 1) + ((s.sym >> 1) & 1) + ((s.sym >> 2) & 1)));
        bool ck = false;
        fill_k(a.k, a.ki, k_re + f0, k_im ? k_im + f0 : nullptr, nf);
        for (int f = 0; f < nf; ++f) ck |= a.ki[f] != 0.f;
        if (!a.b_re) a.q_re = a.q_im = nullptr;
        a.nf = nf;
        cudaError_t e;
        if (tuning(HBEM_TUNE_ASM_PAIRS) != 1 || n_src > 1) {
            // unordered pairs, one wavenumber per grid slice
            dim3 grid(s.n_trial_tiles, s.n_test_tiles, nf);
            e = ck ? dispatch_sym_pairs<true>(s.sym, a, grid, smem_sym, st)
                   : dispatch_sym_pairs<false>(s.sym, a, grid, smem_sym, st);
        } else {
            dim3 grid(s.n_trial_tiles, s.n_test_tiles, (nf + kAsmFreqs - 1) / kAsmFreqs);
            e = ck ? dispatch_sym<true>(s.sym, a, grid, smem, st) : dispatch_sym<false>(s.sym, a, grid, smem, st);
        }
        if (e != cudaSuccess) return cuda_fail(e, "k_regular launch");
        count_launch();
        ++s.launches;
    }
    return HBEM_OK;
}

int launch_duffy(Session &s, int n_freq, const float *k_re, const float *k_im, const float *q_re, const float *q_im,
                 long long q_stride, const float *beta_re, const float *beta_im, float *a_re, float *a_im,
                 long long lda, long long a_stride, float *b_re, float *b_im, long long b_stride, cudaStream_t st,
                 const ApertureOut *ap, int n_src, long long q_src_stride, long long b_src_stride) {
    if (s.n_pairs == 0) return HBEM_OK;
    for (int f0 = 0; f0 < n_freq; f0 += kMaxFreqPerLaunch) {
        const int nf = std::min(kMaxFreqPerLaunch, n_freq - f0);
        DuffyArgs a{};
        a.pairs = s.d_pairs; a.rule = s.d_rule; a.rule_w = s.d_rule_w;
        a.verts = s.d_verts; a.tris = s.d_tris; a.l2g = s.d_l2g; a.areas = s.d_areas; a.normals = s.d_normals;
        a.q_re = (q_re && b_re) ? q_re + (size_t)f0 * q_stride : nullptr;
        a.q_im = (q_im && b_re) ? q_im + (size_t)f0 * q_stride : nullptr;
        a.beta_re = beta_re; a.beta_im = beta_im;
        a.a_re = a_re + (size_t)f0 * a_stride; a.a_im = a_im + (size_t)f0 * a_stride;
        a.b_re = b_re ? b_re + (size_t)f0 * b_stride : nullptr;
        a.b_im = b_im ? b_im + (size_t)f0 * b_stride : nullptr;
        a.q_stride = q_stride; a.lda = lda; a.a_stride = a_stride; a.b_stride = b_stride;
        a.q_src_stride = q_src_stride; a.b_src_stride = b_src_stride; a.n_src = n_src;
        a.V = s.n_vertices; a.T = s.n_triangles; a.n_pairs = s.n_pairs;
        for (int r = 0; r < 3; ++r) { a.rule_off[r] = s.rule_off[r]; a.rule_cnt[r] = s.rule_cnt[r]; }
        fill_k(a.k, a.ki, k_re + f0, k_im ? k_im + f0 : nullptr, nf);
        if (ap) {
            a.ap_local = s.d_ap_local;
            a.m_ap = s.m_ap;
            a.mode = ap->mode;
            a.sia_re = ap->sia_re ? ap->sia_re + (size_t)f0 * ap->sia_stride : nullptr;
            a.sia_im = ap->sia_im ? ap->sia_im + (size_t)f0 * ap->sia_stride : nullptr;
            a.saa_re = ap->saa_re ? ap->saa_re + (size_t)f0 * ap->saa_stride : nullptr;
            a.saa_im = ap->saa_im ? ap->saa_im + (size_t)f0 * ap->saa_stride : nullptr;
            a.sia_stride = ap->sia_stride;
            a.saa_stride = ap->saa_stride;
        }
        bool ck = false;
        for (int f = 0; f < nf; ++f) ck |= a.ki[f] != 0.f;
        a.nf = nf;
        // variant: 1 = one wavenumber per warp (3 CTAs/SM), 2 = two (2 CTAs/SM, the default:
        // the faster one on the 1043-dof yz+xz horn at 40 wavenumbers, where it shares the
        // per-point geometry between the two wavenumbers)
        const int var = tuning(HBEM_TUNE_DUFFY) == 1 ? 1 : 2;
        dim3 grid((s.n_pairs + 7) / 8, (nf + var - 1) / var);
        if (var == 2) {
            if (ck) k_duffy<true, 2, 2><<<grid, 256, 0, st>>>(a);
            else k_duffy<false, 2, 2><<<grid, 256, 0, st>>>(a);
        } else {
            if (ck) k_duffy<true, 1, 3><<<grid, 256, 0, st>>>(a);
            else k_duffy<false, 1, 3><<<grid, 256, 0, st>>>(a);
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return cuda_fail(e, "k_duffy launch");
        count_launch();
        ++s.launches;
    }
    return HBEM_OK;
}

}  // namespace hbem

using namespace hbem;

extern "C" int hbem_assemble_multi(hbem_session *h, int n_freq, const float *k_re, const float *k_im, int n_src,
                                   const float *q_re, const float *q_im, long long q_stride, long long q_src_stride,
                                   const float *beta_re, const float *beta_im, float *a_re, float *a_im,
                                   long long lda, long long a_stride, float *b_re, float *b_im, long long b_stride,
                                   long long b_src_stride, int flags, void *stream) {
    Session *s = reinterpret_cast<Session *>(h);
    if (!s) return fail(HBEM_ERR_ARG, "hbem_assemble: NULL session");
    if (n_freq <= 0) return HBEM_OK;
    if (!k_re || !a_re || !a_im) return fail(HBEM_ERR_ARG, "hbem_assemble: NULL k or A pointer");
    if (n_src < 1 || n_src > kMaxSources) return fail(HBEM_ERR_ARG, "hbem_assemble_multi: n_src must be 1 .. 8");
    if (lda < s->n_dof || a_stride < lda * s->n_dof) return fail(HBEM_ERR_ARG, "hbem_assemble: lda/a_stride too small");
    if ((q_re == nullptr) != (q_im == nullptr) || (b_re == nullptr) != (b_im == nullptr))
        return fail(HBEM_ERR_ARG, "hbem_assemble: real/imag pointers must be given together");
    if (q_re && q_stride < s->n_triangles) return fail(HBEM_ERR_ARG, "hbem_assemble: q_stride < n_triangles");
    if (b_re && b_stride < s->n_dof) return fail(HBEM_ERR_ARG, "hbem_assemble: b_stride < n_dof");
    if (n_src > 1 && ((q_re && q_src_stride < q_stride * n_freq) || (b_re && b_src_stride < b_stride * n_freq)))
        return fail(HBEM_ERR_ARG, "hbem_assemble_multi: q_src_stride / b_src_stride overlap the frequencies");
    if ((beta_re == nullptr) != (beta_im == nullptr)) return fail(HBEM_ERR_ARG, "hbem_assemble: beta pointers");
    for (int f = 0; f < n_freq; ++f)
        if (!std::isfinite(k_re[f]) || (k_im && !std::isfinite(k_im[f])))
            return fail(HBEM_ERR_ARG, "hbem_assemble: non-finite wavenumber");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    HBEM_CUDA(cudaSetDevice(s->device));
    if (flags & HBEM_ASM_ZERO) {
        if (a_stride == lda * s->n_dof) {   // one slab (a padded leading dimension is zeroed with it)
            HBEM_CUDA(cudaMemsetAsync(a_re, 0, sizeof(float) * (size_t)a_stride * n_freq, st));
            HBEM_CUDA(cudaMemsetAsync(a_im, 0, sizeof(float) * (size_t)a_stride * n_freq, st));
        } else {
            for (int f = 0; f < n_freq; ++f) {
                HBEM_CUDA(cudaMemset2DAsync(a_re + (size_t)f * a_stride, lda * sizeof(float), 0, s->n_dof * sizeof(float), s->n_dof, st));
                HBEM_CUDA(cudaMemset2DAsync(a_im + (size_t)f * a_stride, lda * sizeof(float), 0, s->n_dof * sizeof(float), s->n_dof, st));
            }
        }
        if (b_re) {
            for (int sv = 0; sv < n_src; ++sv) {
                float *br = b_re + (size_t)sv * b_src_stride, *bi = b_im + (size_t)sv * b_src_stride;
                HBEM_CUDA(cudaMemset2DAsync(br, b_stride * sizeof(float), 0, s->n_dof * sizeof(float), n_freq, st));
                HBEM_CUDA(cudaMemset2DAsync(bi, b_stride * sizeof(float), 0, s->n_dof * sizeof(float), n_freq, st));
            }
        }
    }
    int rc = HBEM_OK;
    if (flags & HBEM_ASM_REGULAR)
        rc = launch_regular(*s, n_freq, k_re, k_im, q_re, q_im, q_stride, beta_re, beta_im, a_re, a_im, lda, a_stride,
                            b_re, b_im, b_stride, st, n_src, q_src_stride, b_src_stride);
    if (rc == HBEM_OK && (flags & HBEM_ASM_DUFFY))
        rc = launch_duffy(*s, n_freq, k_re, k_im, q_re, q_im, q_stride, beta_re, beta_im, a_re, a_im, lda, a_stride,
                          b_re, b_im, b_stride, st, nullptr, n_src, q_src_stride, b_src_stride);
    // near-field subdivision (when the session has it on) with the singular corrections
    if (rc == HBEM_OK && (flags & HBEM_ASM_DUFFY) && s->n_near > 0)
        rc = launch_near(*s, n_freq, k_re, k_im, n_src, q_re, q_im, q_stride, q_src_stride, beta_re, beta_im, a_re,
                         a_im, lda, a_stride, b_re, b_im, b_stride, b_src_stride, st);
    return rc;
}

extern "C" int hbem_assemble(hbem_session *h, int n_freq, const float *k_re, const float *k_im, const float *q_re,
                             const float *q_im, long long q_stride, const float *beta_re, const float *beta_im,
                             float *a_re, float *a_im, long long lda, long long a_stride, float *b_re, float *b_im,
                             long long b_stride, int flags, void *stream) {
    return hbem_assemble_multi(h, n_freq, k_re, k_im, 1, q_re, q_im, q_stride, 0, beta_re, beta_im, a_re, a_im, lda,
                               a_stride, b_re, b_im, b_stride, 0, flags, stream);
}
