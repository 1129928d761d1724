/*
 * TEST INFRASTRUCTURE — CPU oracle for the dense Helmholtz BEM hot path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load this library, and only as the checker or the timed CPU
 * baseline.  The product path (hornlab_metal_bem_b200 + libhbem.so) never
 * calls it.
 *
 * This file restates, in C, the reference's own CPU path for the solve that
 * solve(mesh, native_config(...)) runs (file:line are in the reference's
 * hornlab_metal_bem/metal/native_helper/Sources/HornlabMetalBemNative/main.swift):
 *   - 6-point degree-4 Dunavant triangle rule            main.swift:1472-1489
 *   - Helmholtz G and dG/dn_y kernels, complex k         main.swift:1501-1553
 *   - mirror images for symmetry planes                  main.swift:1555-1604
 *   - regular Galerkin assembly (+ Robin, mass term)     main.swift:1726-1841
 *   - exterior field evaluation                          main.swift:1843-1895
 *   - P1 incidence / Duffy pair list (real + images)     main.swift:2045-2391
 *   - Duffy reduction plan (unique triplets)             main.swift:2560-2613
 *   - Sauter-Schwab style Duffy rules, 4-pt Gauss^4      main.swift:2626-2699
 *   - singular / regular / subdivided pair blocks        main.swift:2701-2973
 *   - CPU Duffy correction with FP64 triplet sums        main.swift:2974-3070
 *   - tag-average surface pressure                       main.swift:807-841
 *   - CHIEF interior collocation rows                    main.swift:1897-2036
 *
 * REAL is float (oracle "f32": same arithmetic type as the reference) or
 * double (oracle "f64": the accuracy oracle).  GREAL, the type of the
 * vertex / area / normal inputs, is float (the reference's geometry buffers)
 * or double (the "g64" build, for FP64 finite differences of the geometry).
 * Functions carry an og32_/og64_/og64g_ prefix chosen by the build.  Parallel loops use OpenMP so the same code is
 * the timed multi-core CPU baseline.
 *
 * Parity pin: geometry/front-end inputs come from the reference's own Python
 * (tests/golden fixtures); Duffy pair-plan counts are the reference tests'
 * known answers; pair blocks are checked against the reference tests' FP64
 * subdivided-quadrature helper and the analytic pulsating sphere.
 */
#include <math.h>
#include <stdint.h>

#ifndef GREAL
#define GREAL float
#endif
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif
#ifndef OGP
#define OGP(name) og64_##name
#endif

typedef struct { REAL re, im; } cplx;

static inline cplx cadd(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx csub(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cplx cmul(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cplx cscale(cplx a, REAL s) { cplx r = {a.re * s, a.im * s}; return r; }

/* Geometry exactly as the session buffers carry it (f32 inputs). */
typedef struct {
    int n_vertices, n_triangles, n_dof, sym;
    const GREAL *verts;    /* (3, V) */
    const int *tris;       /* (3, T) */
    const int *l2g;        /* (T, 3) */
    const GREAL *areas;    /* (T,)   */
    const GREAL *normals;  /* (3, T) */
} og_geom;

/* ---- quadrature ------------------------------------------------------- */
static const double QX[6] = {0.4459484909159651, 0.0915762135097710, 0.1081030181680700,
                             0.4459484909159651, 0.8168475729804590, 0.0915762135097710};
static const double QY[6] = {0.4459484909159651, 0.0915762135097700, 0.4459484909159651,
                             0.1081030181680700, 0.0915762135097700, 0.8168475729804580};
static const double QW[6] = {0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.2233815896780110,
                             0.5 * 0.2233815896780110, 0.5 * 0.1099517436553220, 0.5 * 0.1099517436553220};

static inline int tv(const og_geom *g, int tri, int loc) { return g->tris[loc * g->n_triangles + tri]; }
static inline int dof(const og_geom *g, int tri, int loc) { return g->l2g[tri * 3 + loc]; }

static inline void point_on(const og_geom *g, int tri, REAL xi, REAL eta, REAL out[3]) {
    int V = g->n_vertices;
    int i1 = tv(g, tri, 0), i2 = tv(g, tri, 1), i3 = tv(g, tri, 2);
    REAL b1 = (REAL)1 - xi - eta, b2 = xi, b3 = eta;
    for (int c = 0; c < 3; ++c)
        out[c] = b1 * (REAL)g->verts[c * V + i1] + b2 * (REAL)g->verts[c * V + i2] + b3 * (REAL)g->verts[c * V + i3];
}

static inline void basis(REAL xi, REAL eta, REAL b[3]) { b[0] = (REAL)1 - xi - eta; b[1] = xi; b[2] = eta; }

#define INV4PI ((REAL)0.07957747154594767)

/* G = e^{ikr}/(4 pi r), k = kr + i ki  (main.swift:1505-1519) */
static inline cplx green(REAL dx, REAL dy, REAL dz, REAL kr, REAL ki) {
    REAL r2 = dx * dx + dy * dy + dz * dz;
    cplx z = {0, 0};
    if (r2 <= 0) return z;
    REAL r = sqrt(r2);
    REAL s = exp(-ki * r) * INV4PI / r;
    z.re = cos(kr * r) * s;
    z.im = sin(kr * r) * s;
    return z;
}

/* dG/dn_y = G (ik - 1/r) ((y-x).n)/r  (main.swift:1533-1553) */
static inline cplx dlp(REAL dx, REAL dy, REAL dz, REAL nx, REAL ny, REAL nz, REAL kr, REAL ki) {
    REAL r2 = dx * dx + dy * dy + dz * dz;
    cplx z = {0, 0};
    if (r2 <= 0) return z;
    REAL r = sqrt(r2);
    REAL s = exp(-ki * r) * INV4PI / r;
    REAL gre = cos(kr * r) * s, gim = sin(kr * r) * s;
    REAL proj = (dx * nx + dy * ny + dz * nz) / r;
    REAL fre = (REAL)-1 / r - ki, fim = kr;
    z.re = (gre * fre - gim * fim) * proj;
    z.im = (gre * fim + gim * fre) * proj;
    return z;
}

static int mirror_masks(int sym, int out[3]) {
    if (sym == 1) { out[0] = 1; return 1; }
    if (sym == 2) { out[0] = 2; return 1; }
    if (sym == 4) { out[0] = 4; return 1; }
    if (sym == 3) { out[0] = 1; out[1] = 2; out[2] = 3; return 3; }
    return 0;
}

static inline void mirror(REAL p[3], int mask) {
    if (mask & 1) p[0] = -p[0];
    if (mask & 2) p[1] = -p[1];
    if (mask & 4) p[2] = -p[2];
}

static inline REAL row_weight(int sym) {
    REAL w = 1;
    if (sym & 1) w *= 2;
    if (sym & 2) w *= 2;
    if (sym & 4) w *= 2;
    return w;
}

static inline int mask_is_odd(int mask) { return __builtin_popcount((unsigned)mask) & 1; }

/* image reference coordinates -> original triangle reference coordinates
   (main.swift:2131-2136): an odd mirror reverses the local vertex order. */
static inline void image_to_orig(REAL *xi, REAL *eta, int mask) {
    if (mask_is_odd(mask)) { REAL t = *xi; *xi = *eta; *eta = t; }
}

static inline void atomic_add(REAL *p, REAL v) {
#pragma omp atomic
    *p += v;
}

/* ---- regular assembly (main.swift:1726-1841) -------------------------- */
int OGP(regular_assemble)(const og_geom *g, REAL kr, REAL ki,
                          const float *q_re, const float *q_im,
                          const float *beta_re, const float *beta_im,
                          REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im) {
    int T = g->n_triangles, n = g->n_dof;
    int masks[3];
    int nm = mirror_masks(g->sym, masks);
    REAL rw = row_weight(g->sym);
    cplx iK = {-ki, kr};
#pragma omp parallel for schedule(dynamic, 4)
    for (int test = 0; test < T; ++test) {
        REAL tp[6][3], tb[6][3];
        for (int a = 0; a < 6; ++a) {
            point_on(g, test, (REAL)QX[a], (REAL)QY[a], tp[a]);
            basis((REAL)QX[a], (REAL)QY[a], tb[a]);
        }
        for (int trial = 0; trial < T; ++trial) {
            REAL nn[3] = {g->normals[trial], g->normals[T + trial], g->normals[2 * T + trial]};
            REAL jac = ((REAL)2 * (REAL)g->areas[test]) * ((REAL)2 * (REAL)g->areas[trial]);
            cplx blk[9], slp[3];
            memset(blk, 0, sizeof blk);
            memset(slp, 0, sizeof slp);
            for (int a = 0; a < 6; ++a) {
                for (int b = 0; b < 6; ++b) {
                    REAL sp[3], sb[3];
                    point_on(g, trial, (REAL)QX[b], (REAL)QY[b], sp);
                    basis((REAL)QX[b], (REAL)QY[b], sb);
                    REAL w = (REAL)QW[a] * (REAL)QW[b] * jac;
                    REAL dx = sp[0] - tp[a][0], dy = sp[1] - tp[a][1], dz = sp[2] - tp[a][2];
                    cplx G = green(dx, dy, dz, kr, ki);
                    cplx D = dlp(dx, dy, dz, nn[0], nn[1], nn[2], kr, ki);
                    for (int m = 0; m < nm; ++m) {
                        REAL ip[3] = {sp[0], sp[1], sp[2]}, in[3] = {nn[0], nn[1], nn[2]};
                        mirror(ip, masks[m]);
                        mirror(in, masks[m]);
                        REAL ex = ip[0] - tp[a][0], ey = ip[1] - tp[a][1], ez = ip[2] - tp[a][2];
                        G = cadd(G, green(ex, ey, ez, kr, ki));
                        D = cadd(D, dlp(ex, ey, ez, in[0], in[1], in[2], kr, ki));
                    }
                    for (int i = 0; i < 3; ++i) {
                        slp[i] = cadd(slp[i], cscale(G, tb[a][i] * w));
                        for (int j = 0; j < 3; ++j)
                            blk[i * 3 + j] = cadd(blk[i * 3 + j], cscale(D, tb[a][i] * sb[j] * w));
                    }
                }
            }
            cplx qv = {q_re ? (REAL)q_re[trial] : 0, q_im ? (REAL)q_im[trial] : 0};
            cplx beta = {beta_re ? (REAL)beta_re[trial] : 0, beta_im ? (REAL)beta_im[trial] : 0};
            int robin = beta.re != 0 || beta.im != 0;
            cplx rc = cmul(iK, beta);
            for (int i = 0; i < 3; ++i) {
                int row = dof(g, test, i);
                cplx rv = cscale(cmul(slp[i], qv), rw);
                atomic_add(&b_re[row], rv.re);
                atomic_add(&b_im[row], rv.im);
                for (int j = 0; j < 3; ++j) {
                    int col = dof(g, trial, j);
                    cplx term = blk[i * 3 + j];
                    if (robin) term = csub(term, cscale(cmul(slp[i], rc), (REAL)(1.0 / 3.0)));
                    if (test == trial) {
                        REAL mass = (REAL)g->areas[test] * (i == j ? (REAL)(1.0 / 6.0) : (REAL)(1.0 / 12.0));
                        term.re -= (REAL)0.5 * mass;
                    }
                    atomic_add(&A_re[(size_t)row * n + col], term.re * rw);
                    atomic_add(&A_im[(size_t)row * n + col], term.im * rw);
                }
            }
        }
    }
    return 0;
}

/* ---- Duffy pair list (main.swift:2081-2391) --------------------------- */
typedef struct { int64_t k[3]; int tri; int loc; } key_entry;

static void coord_key(REAL x, REAL y, REAL z, int64_t out[3]) {
    /* 1e-6 lattice, rounding half away from zero (main.swift:2107-2112) */
    out[0] = llround((double)(float)x / 1.0e-6);
    out[1] = llround((double)(float)y / 1.0e-6);
    out[2] = llround((double)(float)z / 1.0e-6);
}

static int key_cmp(const void *pa, const void *pb) {
    const key_entry *a = pa, *b = pb;
    for (int c = 0; c < 3; ++c) {
        if (a->k[c] < b->k[c]) return -1;
        if (a->k[c] > b->k[c]) return 1;
    }
    if (a->tri != b->tri) return a->tri < b->tri ? -1 : 1;
    return a->loc < b->loc ? -1 : (a->loc > b->loc);
}

static int key_lower(const key_entry *e, int n, const int64_t k[3]) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) / 2;
        int c = 0;
        for (int d = 0; d < 3 && !c; ++d) c = e[mid].k[d] < k[d] ? -1 : (e[mid].k[d] > k[d] ? 1 : 0);
        if (c < 0) lo = mid + 1; else hi = mid;
    }
    return lo;
}

static void vertex_point(const og_geom *g, int v, REAL p[3]) {
    int V = g->n_vertices;
    p[0] = g->verts[v]; p[1] = g->verts[V + v]; p[2] = g->verts[2 * V + v];
}

static inline int image_local(int local, int mask) {
    if (!mask_is_odd(mask)) return local;
    return local == 1 ? 2 : (local == 2 ? 1 : local);
}

/* shared vertex detection between image triangles; returns count and the
   first two (test, trial) image-local matches */
static int shared_locals(const og_geom *g, int test, int trial, int tm, int sm, int out[4]) {
    int count = 0;
    out[0] = out[1] = out[2] = out[3] = 0;
    if (tm == 0 && sm == 0) {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                if (tv(g, test, i) == tv(g, trial, j)) {
                    ++count;
                    if (count == 1) { out[0] = i; out[2] = j; } else { out[1] = i; out[3] = j; }
                }
        return count;
    }
    for (int tf = 0; tf < 3; ++tf) {
        REAL p[3];
        vertex_point(g, tv(g, test, image_local(tf, tm)), p);
        mirror(p, tm);
        int64_t kt[3];
        coord_key(p[0], p[1], p[2], kt);
        for (int sf = 0; sf < 3; ++sf) {
            REAL s[3];
            vertex_point(g, tv(g, trial, image_local(sf, sm)), s);
            mirror(s, sm);
            int64_t ks[3];
            coord_key(s[0], s[1], s[2], ks);
            if (kt[0] == ks[0] && kt[1] == ks[1] && kt[2] == ks[2]) {
                ++count;
                if (count == 1) { out[0] = tf; out[2] = sf; } else { out[1] = tf; out[3] = sf; }
            }
        }
    }
    return count;
}

/* Pair record: test, trial, test_mask, trial_mask, kind, tl1, tl2, sl1, sl2. */
#define PAIR_INTS 9

static int append_pair(int *out, int cap, int np, int test, int trial, int tm, int sm, int cnt, const int sh[4], int counts[3]) {
    if (cnt <= 0) return np;
    int kind = cnt == 3 ? 1 : (cnt == 2 ? 2 : 3);
    counts[kind - 1]++;
    if (out && np < cap) {
        int *r = out + (size_t)np * PAIR_INTS;
        r[0] = test; r[1] = trial; r[2] = tm; r[3] = sm; r[4] = kind;
        if (kind == 1) { r[5] = 0; r[6] = 1; r[7] = 0; r[8] = 1; }
        else { r[5] = sh[0]; r[6] = sh[1]; r[7] = sh[2]; r[8] = sh[3]; }
    }
    return np + 1;
}

/* Returns the number of pairs (writes at most cap records when out != NULL). */
int OGP(duffy_pairs)(const og_geom *g, int *out, int cap, int counts[3]) {
    int T = g->n_triangles, V = g->n_vertices;
    int masks[4] = {0, 0, 0, 0};
    int nm = 1 + mirror_masks(g->sym, masks + 1);
    counts[0] = counts[1] = counts[2] = 0;
    int np = 0;
    int *stamp = calloc((size_t)T, sizeof(int));
    int *cand = malloc((size_t)T * sizeof(int));
    int st = 0;
    if (g->sym == 0) {
        /* vertex -> triangle lists in triangle order */
        int *cnt = calloc((size_t)V + 1, sizeof(int));
        for (int t = 0; t < T; ++t) for (int l = 0; l < 3; ++l) cnt[tv(g, t, l) + 1]++;
        for (int v = 0; v < V; ++v) cnt[v + 1] += cnt[v];
        int *fill = calloc((size_t)V, sizeof(int));
        int *lst = malloc((size_t)T * 3 * sizeof(int));
        for (int t = 0; t < T; ++t)
            for (int l = 0; l < 3; ++l) { int v = tv(g, t, l); lst[cnt[v] + fill[v]++] = t; }
        for (int trial = 0; trial < T; ++trial) {
            ++st;
            int nc = 0;
            for (int l = 0; l < 3; ++l) {
                int v = tv(g, trial, l);
                for (int e = cnt[v]; e < cnt[v + 1]; ++e) {
                    int test = lst[e];
                    if (stamp[test] != st) { stamp[test] = st; cand[nc++] = test; }
                }
            }
            for (int c = 0; c < nc; ++c) {
                int sh[4];
                int k = shared_locals(g, cand[c], trial, 0, 0, sh);
                np = append_pair(out, cap, np, cand[c], trial, 0, 0, k, sh, counts);
            }
        }
        free(cnt); free(fill); free(lst);
    } else {
        key_entry *tab[4];
        for (int mi = 0; mi < nm; ++mi) {
            tab[mi] = malloc((size_t)T * 3 * sizeof(key_entry));
            for (int t = 0; t < T; ++t)
                for (int l = 0; l < 3; ++l) {
                    REAL p[3];
                    vertex_point(g, tv(g, t, l), p);
                    mirror(p, masks[mi]);
                    key_entry *e = &tab[mi][t * 3 + l];
                    coord_key(p[0], p[1], p[2], e->k);
                    e->tri = t; e->loc = l;
                }
            qsort(tab[mi], (size_t)T * 3, sizeof(key_entry), key_cmp);
        }
        for (int trial = 0; trial < T; ++trial) {
            for (int si = 0; si < nm; ++si) {
                for (int ti = 0; ti < nm; ++ti) {
                    ++st;
                    int nc = 0;
                    for (int l = 0; l < 3; ++l) {
                        REAL p[3];
                        vertex_point(g, tv(g, trial, l), p);
                        mirror(p, masks[si]);
                        int64_t k[3];
                        coord_key(p[0], p[1], p[2], k);
                        int e = key_lower(tab[ti], T * 3, k);
                        for (; e < T * 3 && tab[ti][e].k[0] == k[0] && tab[ti][e].k[1] == k[1] && tab[ti][e].k[2] == k[2]; ++e) {
                            int test = tab[ti][e].tri;
                            if (stamp[test] != st) { stamp[test] = st; cand[nc++] = test; }
                        }
                    }
                    for (int c = 0; c < nc; ++c) {
                        int sh[4];
                        int cntv = shared_locals(g, cand[c], trial, masks[ti], masks[si], sh);
                        np = append_pair(out, cap, np, cand[c], trial, masks[ti], masks[si], cntv, sh, counts);
                    }
                }
            }
        }
        for (int mi = 0; mi < nm; ++mi) free(tab[mi]);
    }
    free(stamp); free(cand);
    return np;
}

/* Unique (row, col) triplet count of the reduction plan (main.swift:2560-2613). */
static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return x < y ? -1 : (x > y);
}

int OGP(duffy_unique_triplets)(const og_geom *g, const int *pairs, int np) {
    int64_t *keys = malloc((size_t)np * 9 * sizeof(int64_t) + 8);
    for (int p = 0; p < np; ++p) {
        const int *r = pairs + (size_t)p * PAIR_INTS;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                keys[p * 9 + i * 3 + j] = (int64_t)dof(g, r[0], i) + (int64_t)dof(g, r[1], j) * g->n_dof;
    }
    qsort(keys, (size_t)np * 9, sizeof(int64_t), cmp_i64);
    int u = 0;
    for (int i = 0; i < np * 9; ++i) if (i == 0 || keys[i] != keys[i - 1]) ++u;
    free(keys);
    return u;
}

/* ---- Duffy rules (main.swift:2617-2699) ------------------------------- */
#define MAX_GL 16   /* Gauss-Legendre points per Duffy coordinate (the reference uses 4) */

/* m-point Gauss-Legendre nodes (ascending) and weights on [0, 1].  m = 4 uses
   the closed form of the reference's rule; other orders Newton's iteration on
   the Legendre recurrence P_k = ((2k - 1) x P_{k-1} - (k - 1) P_{k-2}) / k
   from the Chebyshev initial guesses (Numerical Recipes' gauleg method). */
static void gauss_legendre01(int m, double *x, double *w) {
    if (m == 4) {
        double a1 = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0)) / 2.0;
        double a2 = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0)) / 2.0;
        double w1 = (18.0 + sqrt(30.0)) / 72.0, w2 = (18.0 - sqrt(30.0)) / 72.0;
        x[0] = 0.5 - a2; x[1] = 0.5 - a1; x[2] = 0.5 + a1; x[3] = 0.5 + a2;
        w[0] = w2; w[1] = w1; w[2] = w1; w[3] = w2;
        return;
    }
    for (int i = 0; i < (m + 1) / 2; ++i) {
        double z = cos(3.14159265358979323846 * (i + 0.75) / (m + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = 0.0;
            for (int k = 1; k <= m; ++k) {
                double p2 = p1;
                p1 = p0;
                p0 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p2) / k;
            }
            dp = m * (z * p0 - p1) / (z * z - 1.0);
            double dz = p0 / dp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        /* z is the i-th largest root on [-1, 1]: map to [0, 1] */
        x[m - 1 - i] = 0.5 * (1.0 + z);
        x[i] = 0.5 * (1.0 - z);
        w[i] = w[m - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
    }
}

/* One rule record per point: test (xi, eta), trial (xi, eta), weight; m
   Gauss-Legendre points per Duffy coordinate ({6, 5, 2} m^4 points). */
static int duffy_rule_m(int kind, int m, REAL *rec) {
    double xd[MAX_GL], wd[MAX_GL];
    gauss_legendre01(m, xd, wd);
    REAL xs[MAX_GL], ws[MAX_GL];
    for (int i = 0; i < m; ++i) { xs[i] = (REAL)xd[i]; ws[i] = (REAL)wd[i]; }
    int n = 0;
#define PUT(TX, TY, SX, SY, W) do { REAL *o = rec + 5 * n++; o[0] = (TX) - (TY); o[1] = (TY); o[2] = (SX) - (SY); o[3] = (SY); o[4] = (W); } while (0)
    for (int a = 0; a < m; ++a)
        for (int b = 0; b < m; ++b)
            for (int c = 0; c < m; ++c)
                for (int d = 0; d < m; ++d) {
                    REAL xi = xs[b], e1 = xs[a], e2 = xs[c], e3 = xs[d];
                    REAL e12 = e1 * e2, e123 = e12 * e3;
                    REAL base = ws[a] * ws[b] * ws[c] * ws[d];
                    if (kind == 1) {
                        REAL w = base * xi * xi * xi * e1 * e1 * e2;
                        PUT(xi, xi * (1 - e1 + e12), xi * (1 - e123), xi * (1 - e1), w);
                        PUT(xi * (1 - e123), xi * (1 - e1), xi, xi * (1 - e1 + e12), w);
                        PUT(xi, xi * (e1 - e12 + e123), xi * (1 - e12), xi * (e1 - e12), w);
                        PUT(xi * (1 - e12), xi * (e1 - e12), xi, xi * (e1 - e12 + e123), w);
                        PUT(xi * (1 - e123), xi * (e1 - e123), xi, xi * (e1 - e12), w);
                        PUT(xi, xi * (e1 - e12), xi * (1 - e123), xi * (e1 - e123), w);
                    } else if (kind == 2) {
                        REAL w = base * xi * xi * xi * e1 * e1;
                        PUT(xi, xi * e1 * e3, xi * (1 - e12), xi * e1 * (1 - e2), w);
                        PUT(xi, xi * e1, xi * (1 - e123), xi * e1 * e2 * (1 - e3), w * e2);
                        PUT(xi * (1 - e12), xi * e1 * (1 - e2), xi, xi * e123, w * e2);
                        PUT(xi * (1 - e123), xi * e12 * (1 - e3), xi, xi * e1, w * e2);
                        PUT(xi * (1 - e123), xi * e1 * (1 - e2 * e3), xi, xi * e12, w * e2);
                    } else {
                        REAL w = base * xi * xi * xi * e2;
                        PUT(xi, xi * e1, xi * e2, xi * e2 * e3, w);
                        PUT(xi * e2, xi * e2 * e3, xi, xi * e1, w);
                    }
                }
#undef PUT
    return n;
}

static int duffy_rule(int kind, REAL *rec) { return duffy_rule_m(kind, 4, rec); }
static size_t rule_len(int m) { return (size_t)6 * m * m * m * m; }

int OGP(duffy_rule_table)(int kind, REAL *rec) { return duffy_rule(kind, rec); }
int OGP(duffy_rule_table_m)(int kind, int m, REAL *rec) {
    if (m < 1 || m > MAX_GL) return -1;
    return duffy_rule_m(kind, m, rec);
}

static inline REAL refx(int l) { return l == 1 ? 1 : 0; }
static inline REAL refy(int l) { return l == 2 ? 1 : 0; }

/* Place a Duffy point on the shared edge / vertex (main.swift:2701-2725). */
static void remap(REAL x, REAL y, int kind, int l1, int l2, REAL *ox, REAL *oy) {
    if (kind == 1) { *ox = x; *oy = y; return; }
    if (kind == 2) {
        int vc = 3 - l1 - l2;
        REAL ax = refx(l1), ay = refy(l1), bx = refx(l2), by = refy(l2), cx = refx(vc), cy = refy(vc);
        *ox = ax + x * (bx - ax) + y * (cx - ax);
        *oy = ay + x * (by - ay) + y * (cy - ay);
        return;
    }
    if (l1 == 0) { *ox = x; *oy = y; }
    else if (l1 == 1) { *ox = 1 - x - y; *oy = y; }
    else { *ox = x; *oy = 1 - x - y; }
}

/* Accumulate one (test, trial) pair block from a list of point pairs given in
   IMAGE reference coordinates.  slp[3], dlp[9] complex (interleaved). */
static void pair_accumulate(const og_geom *g, int test, int trial, int tm, int sm,
                            REAL txi, REAL teta, REAL sxi, REAL seta, REAL w, const REAL nrm[3],
                            REAL kr, REAL ki, cplx slp[3], cplx dl[9]) {
    image_to_orig(&txi, &teta, tm);
    image_to_orig(&sxi, &seta, sm);
    REAL tp[3], sp[3], tb[3], sb[3];
    point_on(g, test, txi, teta, tp);
    mirror(tp, tm);
    point_on(g, trial, sxi, seta, sp);
    mirror(sp, sm);
    basis(txi, teta, tb);
    basis(sxi, seta, sb);
    REAL dx = sp[0] - tp[0], dy = sp[1] - tp[1], dz = sp[2] - tp[2];
    cplx G = cscale(green(dx, dy, dz, kr, ki), w);
    cplx D = cscale(dlp(dx, dy, dz, nrm[0], nrm[1], nrm[2], kr, ki), w);
    for (int i = 0; i < 3; ++i) {
        slp[i] = cadd(slp[i], cscale(G, tb[i]));
        for (int j = 0; j < 3; ++j) dl[i * 3 + j] = cadd(dl[i * 3 + j], cscale(D, tb[i] * sb[j]));
    }
}

/* mode 0: regular 6x6 rule; mode 1: Duffy rule of `kind` with locals; mode 2:
   subdivided regular rule at `level` (main.swift:2768-2971). */
static void pair_blocks(const og_geom *g, int test, int trial, int tm, int sm, int mode,
                        int kind, const int loc[4], int level, const REAL *rule, int nrule,
                        REAL kr, REAL ki, cplx slp[3], cplx dl[9]) {
    int T = g->n_triangles;
    REAL nrm[3] = {g->normals[trial], g->normals[T + trial], g->normals[2 * T + trial]};
    mirror(nrm, sm);
    REAL jac = ((REAL)2 * (REAL)g->areas[test]) * ((REAL)2 * (REAL)g->areas[trial]);
    memset(slp, 0, 3 * sizeof(cplx));
    memset(dl, 0, 9 * sizeof(cplx));
    if (mode == 0) {
        for (int a = 0; a < 6; ++a)
            for (int b = 0; b < 6; ++b)
                pair_accumulate(g, test, trial, tm, sm, (REAL)QX[a], (REAL)QY[a], (REAL)QX[b], (REAL)QY[b],
                                (REAL)QW[a] * (REAL)QW[b] * jac, nrm, kr, ki, slp, dl);
    } else if (mode == 1) {
        for (int q = 0; q < nrule; ++q) {
            const REAL *r = rule + 5 * q;
            REAL tx, ty, sx, sy;
            remap(r[0], r[1], kind, loc[0], loc[1], &tx, &ty);
            remap(r[2], r[3], kind, loc[2], loc[3], &sx, &sy);
            pair_accumulate(g, test, trial, tm, sm, tx, ty, sx, sy, r[4] * jac, nrm, kr, ki, slp, dl);
        }
    } else {
        int nsub = 1;
        for (int l = 0; l < level; ++l) nsub *= 4;
        REAL *sub = malloc((size_t)nsub * 6 * sizeof(REAL));
        REAL *tmp = malloc((size_t)nsub * 6 * sizeof(REAL));
        sub[0] = 0; sub[1] = 0; sub[2] = 1; sub[3] = 0; sub[4] = 0; sub[5] = 1;
        int cur = 1;
        for (int l = 0; l < level; ++l) {
            int m = 0;
            for (int s = 0; s < cur; ++s) {
                REAL *t = sub + 6 * s;
                REAL ab[2] = {(t[0] + t[2]) * (REAL)0.5, (t[1] + t[3]) * (REAL)0.5};
                REAL bc[2] = {(t[2] + t[4]) * (REAL)0.5, (t[3] + t[5]) * (REAL)0.5};
                REAL ca[2] = {(t[4] + t[0]) * (REAL)0.5, (t[5] + t[1]) * (REAL)0.5};
                REAL *o;
                o = tmp + 6 * m++; o[0] = t[0]; o[1] = t[1]; o[2] = ab[0]; o[3] = ab[1]; o[4] = ca[0]; o[5] = ca[1];
                o = tmp + 6 * m++; o[0] = ab[0]; o[1] = ab[1]; o[2] = t[2]; o[3] = t[3]; o[4] = bc[0]; o[5] = bc[1];
                o = tmp + 6 * m++; o[0] = ca[0]; o[1] = ca[1]; o[2] = bc[0]; o[3] = bc[1]; o[4] = t[4]; o[5] = t[5];
                o = tmp + 6 * m++; o[0] = ab[0]; o[1] = ab[1]; o[2] = bc[0]; o[3] = bc[1]; o[4] = ca[0]; o[5] = ca[1];
            }
            memcpy(sub, tmp, (size_t)m * 6 * sizeof(REAL));
            cur = m;
        }
        REAL tj = (REAL)2 * (REAL)g->areas[test], sj = (REAL)2 * (REAL)g->areas[trial];
        for (int ts = 0; ts < cur; ++ts) {
            REAL *A = sub + 6 * ts;
            REAL tdet = fabs((A[2] - A[0]) * (A[5] - A[1]) - (A[3] - A[1]) * (A[4] - A[0]));
            for (int ss = 0; ss < cur; ++ss) {
                REAL *B = sub + 6 * ss;
                REAL sdet = fabs((B[2] - B[0]) * (B[5] - B[1]) - (B[3] - B[1]) * (B[4] - B[0]));
                REAL jj = tj * tdet * sj * sdet;
                for (int a = 0; a < 6; ++a) {
                    REAL tx = A[0] + (REAL)QX[a] * (A[2] - A[0]) + (REAL)QY[a] * (A[4] - A[0]);
                    REAL ty = A[1] + (REAL)QX[a] * (A[3] - A[1]) + (REAL)QY[a] * (A[5] - A[1]);
                    for (int b = 0; b < 6; ++b) {
                        REAL sx = B[0] + (REAL)QX[b] * (B[2] - B[0]) + (REAL)QY[b] * (B[4] - B[0]);
                        REAL sy = B[1] + (REAL)QX[b] * (B[3] - B[1]) + (REAL)QY[b] * (B[5] - B[1]);
                        pair_accumulate(g, test, trial, tm, sm, tx, ty, sx, sy, (REAL)QW[a] * (REAL)QW[b] * jj,
                                        nrm, kr, ki, slp, dl);
                    }
                }
            }
        }
        free(sub); free(tmp);
    }
}

/* Public pair-block probe: out[0..5] = slp re/im, out[6..23] = dlp re/im.
   mode 1 uses the Duffy rule with `level` Gauss-Legendre points per
   coordinate (0: the reference's 4). */
int OGP(pair_blocks)(const og_geom *g, int test, int trial, int tm, int sm, int mode, int kind,
                     const int *locals, int level, REAL kr, REAL ki, REAL *out) {
    static const int zero[4] = {0, 1, 0, 1};
    REAL *rule = NULL;
    int nrule = 0;
    if (mode == 1) {
        int m = level > 0 ? level : 4;
        if (m > MAX_GL) return -1;
        rule = malloc(rule_len(m) * 5 * sizeof(REAL));
        nrule = duffy_rule_m(kind, m, rule);
        level = 0;
    }
    cplx slp[3], dl[9];
    pair_blocks(g, test, trial, tm, sm, mode, kind, locals ? locals : zero, level, rule, nrule, kr, ki, slp, dl);
    for (int i = 0; i < 3; ++i) { out[2 * i] = slp[i].re; out[2 * i + 1] = slp[i].im; }
    for (int i = 0; i < 9; ++i) { out[6 + 2 * i] = dl[i].re; out[7 + 2 * i] = dl[i].im; }
    free(rule);
    return 0;
}

/* CPU Duffy correction (main.swift:2974-3070): adds (singular - regular) for
   every singular pair into A and b at weight 1, Robin coupling included.  The
   per-entry sums are accumulated in double before the final add, as in the
   reference.  Returns the number of unique (row, col) triplets. */
static int duffy_correct_m(const og_geom *g, REAL kr, REAL ki, const float *q_re, const float *q_im,
                           const float *beta_re, const float *beta_im,
                           REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im, int m);

int OGP(duffy_correct)(const og_geom *g, REAL kr, REAL ki, const float *q_re, const float *q_im,
                       const float *beta_re, const float *beta_im,
                       REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im) {
    return duffy_correct_m(g, kr, ki, q_re, q_im, beta_re, beta_im, A_re, A_im, b_re, b_im, 4);
}

/* The same correction with an m-point Gauss-Legendre Duffy rule per
   coordinate: the convergence reference for the reference's 4-point rule. */
int OGP(duffy_correct_m)(const og_geom *g, REAL kr, REAL ki, const float *q_re, const float *q_im,
                         const float *beta_re, const float *beta_im,
                         REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im, int m) {
    if (m < 1 || m > MAX_GL) return -1;
    return duffy_correct_m(g, kr, ki, q_re, q_im, beta_re, beta_im, A_re, A_im, b_re, b_im, m);
}

static int duffy_correct_m(const og_geom *g, REAL kr, REAL ki, const float *q_re, const float *q_im,
                           const float *beta_re, const float *beta_im,
                           REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im, int m) {
    int counts[3];
    int np = OGP(duffy_pairs)(g, NULL, 0, counts);
    int *pairs = malloc((size_t)(np ? np : 1) * PAIR_INTS * sizeof(int));
    OGP(duffy_pairs)(g, pairs, np, counts);
    REAL *rules[3];
    int nr[3];
    for (int k = 0; k < 3; ++k) { rules[k] = malloc(rule_len(m) * 5 * sizeof(REAL)); nr[k] = duffy_rule_m(k + 1, m, rules[k]); }
    int n = g->n_dof;
    double *acc_re = calloc((size_t)n * n, sizeof(double));
    double *acc_im = calloc((size_t)n * n, sizeof(double));
    cplx iK = {-ki, kr};
#pragma omp parallel for schedule(dynamic, 16)
    for (int p = 0; p < np; ++p) {
        const int *r = pairs + (size_t)p * PAIR_INTS;
        int test = r[0], trial = r[1], tm = r[2], sm = r[3], kind = r[4];
        cplx rs[3], rd[9], ss[3], sd[9];
        pair_blocks(g, test, trial, tm, sm, 0, 0, r + 5, 0, NULL, 0, kr, ki, rs, rd);
        pair_blocks(g, test, trial, tm, sm, 1, kind, r + 5, 0, rules[kind - 1], nr[kind - 1], kr, ki, ss, sd);
        cplx qv = {q_re ? (REAL)q_re[trial] : 0, q_im ? (REAL)q_im[trial] : 0};
        cplx beta = {beta_re ? (REAL)beta_re[trial] : 0, beta_im ? (REAL)beta_im[trial] : 0};
        int robin = beta.re != 0 || beta.im != 0;
        cplx rc = cmul(iK, beta);
        for (int i = 0; i < 3; ++i) {
            int row = dof(g, test, i);
            cplx ds = csub(ss[i], rs[i]);
            cplx rv = cmul(ds, qv);
            atomic_add(&b_re[row], rv.re);
            atomic_add(&b_im[row], rv.im);
            for (int j = 0; j < 3; ++j) {
                int col = dof(g, trial, j);
                cplx d = csub(sd[i * 3 + j], rd[i * 3 + j]);
                if (robin) d = csub(d, cscale(cmul(ds, rc), (REAL)(1.0 / 3.0)));
                double *pr = &acc_re[(size_t)row * n + col], *pi = &acc_im[(size_t)row * n + col];
#pragma omp atomic
                *pr += (double)d.re;
#pragma omp atomic
                *pi += (double)d.im;
            }
        }
    }
    for (size_t i = 0; i < (size_t)n * n; ++i) {
        if (acc_re[i] != 0.0 || acc_im[i] != 0.0) {
            A_re[i] += (REAL)acc_re[i];
            A_im[i] += (REAL)acc_im[i];
        }
    }
    int uniq = OGP(duffy_unique_triplets)(g, pairs, np);
    free(acc_re); free(acc_im); free(pairs);
    for (int k = 0; k < 3; ++k) free(rules[k]);
    return uniq;
}

/* ---- near-field subdivision (main.swift:2410-2560, 3072-3202) ---------- */
/* Near, non-touching (test image, trial image) pairs: centroid distance under
   threshold x the longer of the two longest edges (bounding boxes pre-filter),
   no shared vertex; each gets (subdivided block at `level` - regular 6 x 6
   block) added at weight 1 (the image-pair enumeration carries the symmetry
   factor), Robin coupling included.  Returns the number of near pairs. */
typedef struct { double c[3], lo[3], hi[3], edge; } near_metric;

static void near_metrics(const og_geom *g, int tri, int mask, near_metric *m) {
    REAL p[3][3];
    for (int l = 0; l < 3; ++l) {
        vertex_point(g, tv(g, tri, l), p[l]);
        mirror(p[l], mask);
    }
    double e2 = 0;
    for (int c = 0; c < 3; ++c) {
        m->c[c] = ((double)p[0][c] + (double)p[1][c] + (double)p[2][c]) / 3.0;
        m->lo[c] = fmin(p[0][c], fmin(p[1][c], p[2][c]));
        m->hi[c] = fmax(p[0][c], fmax(p[1][c], p[2][c]));
    }
    for (int a = 0; a < 3; ++a) {
        int b = (a + 1) % 3;
        double d2 = 0;
        for (int c = 0; c < 3; ++c) d2 += ((double)p[a][c] - p[b][c]) * ((double)p[a][c] - p[b][c]);
        if (d2 > e2) e2 = d2;
    }
    m->edge = sqrt(e2);
}

static double axis_gap(double alo, double ahi, double blo, double bhi) {
    if (ahi < blo) return blo - ahi;
    if (bhi < alo) return alo - bhi;
    return 0.0;
}

int OGP(near_pairs)(const og_geom *g, double threshold, int *out, int cap) {
    int T = g->n_triangles;
    int masks[4] = {0, 0, 0, 0};
    int nm = 1 + mirror_masks(g->sym, masks + 1);
    near_metric *mt = malloc((size_t)T * nm * sizeof(near_metric));
    for (int mi = 0; mi < nm; ++mi)
        for (int t = 0; t < T; ++t) near_metrics(g, t, masks[mi], &mt[(size_t)mi * T + t]);
    int np = 0;
    for (int trial = 0; trial < T; ++trial)
        for (int si = 0; si < nm; ++si) {
            const near_metric *sm = &mt[(size_t)si * T + trial];
            for (int ti = 0; ti < nm; ++ti)
                for (int test = 0; test < T; ++test) {
                    const near_metric *tm = &mt[(size_t)ti * T + test];
                    double cut = threshold * fmax(tm->edge, sm->edge), cut2 = cut * cut;
                    double gx = axis_gap(tm->lo[0], tm->hi[0], sm->lo[0], sm->hi[0]);
                    double gy = axis_gap(tm->lo[1], tm->hi[1], sm->lo[1], sm->hi[1]);
                    double gz = axis_gap(tm->lo[2], tm->hi[2], sm->lo[2], sm->hi[2]);
                    if (gx * gx + gy * gy + gz * gz > cut2) continue;
                    double dx = tm->c[0] - sm->c[0], dy = tm->c[1] - sm->c[1], dz = tm->c[2] - sm->c[2];
                    if (dx * dx + dy * dy + dz * dz >= cut2) continue;
                    int sh[4];
                    if (shared_locals(g, test, trial, masks[ti], masks[si], sh) > 0) continue;
                    if (out && np < cap) {
                        int *r = out + (size_t)np * 4;
                        r[0] = test; r[1] = trial; r[2] = masks[ti]; r[3] = masks[si];
                    }
                    ++np;
                }
        }
    free(mt);
    return np;
}

int OGP(near_correct)(const og_geom *g, REAL kr, REAL ki, const float *q_re, const float *q_im,
                      const float *beta_re, const float *beta_im, REAL *A_re, REAL *A_im, REAL *b_re, REAL *b_im,
                      int level, double threshold) {
    int np = OGP(near_pairs)(g, threshold, NULL, 0);
    int *pairs = malloc((size_t)(np ? np : 1) * 4 * sizeof(int));
    OGP(near_pairs)(g, threshold, pairs, np);
    int n = g->n_dof;
    double *acc_re = calloc((size_t)n * n, sizeof(double));
    double *acc_im = calloc((size_t)n * n, sizeof(double));
    cplx iK = {-ki, kr};
#pragma omp parallel for schedule(dynamic, 8)
    for (int p = 0; p < np; ++p) {
        const int *r = pairs + (size_t)p * 4;
        int test = r[0], trial = r[1], tm = r[2], sm = r[3];
        cplx rs[3], rd[9], ss[3], sd[9];
        pair_blocks(g, test, trial, tm, sm, 0, 0, NULL, 0, NULL, 0, kr, ki, rs, rd);
        pair_blocks(g, test, trial, tm, sm, 2, 0, NULL, level, NULL, 0, kr, ki, ss, sd);
        cplx qv = {q_re ? (REAL)q_re[trial] : 0, q_im ? (REAL)q_im[trial] : 0};
        cplx beta = {beta_re ? (REAL)beta_re[trial] : 0, beta_im ? (REAL)beta_im[trial] : 0};
        int robin = beta.re != 0 || beta.im != 0;
        cplx rc = cmul(iK, beta);
        for (int i = 0; i < 3; ++i) {
            int row = dof(g, test, i);
            cplx ds = csub(ss[i], rs[i]);
            cplx rv = cmul(ds, qv);
            atomic_add(&b_re[row], rv.re);
            atomic_add(&b_im[row], rv.im);
            for (int j = 0; j < 3; ++j) {
                int col = dof(g, trial, j);
                cplx d = csub(sd[i * 3 + j], rd[i * 3 + j]);
                if (robin) d = csub(d, cscale(cmul(ds, rc), (REAL)(1.0 / 3.0)));
                double *pr = &acc_re[(size_t)row * n + col], *pi = &acc_im[(size_t)row * n + col];
#pragma omp atomic
                *pr += (double)d.re;
#pragma omp atomic
                *pi += (double)d.im;
            }
        }
    }
    for (size_t i = 0; i < (size_t)n * n; ++i) {
        if (acc_re[i] != 0.0 || acc_im[i] != 0.0) {
            A_re[i] += (REAL)acc_re[i];
            A_im[i] += (REAL)acc_im[i];
        }
    }
    free(acc_re); free(acc_im); free(pairs);
    return np;
}

/* ---- exterior field (main.swift:1843-1895) ---------------------------- */
int OGP(field)(const og_geom *g, REAL kr, const REAL *p_re, const REAL *p_im,
               const REAL *q_re, const REAL *q_im, const float *obs3xN, int nobs,
               REAL *out_re, REAL *out_im) {
    int T = g->n_triangles;
    int masks[3];
    int nm = mirror_masks(g->sym, masks);
#pragma omp parallel for schedule(static)
    for (int o = 0; o < nobs; ++o) {
        REAL ox = obs3xN[o], oy = obs3xN[nobs + o], oz = obs3xN[2 * nobs + o];
        cplx acc = {0, 0};
        for (int tri = 0; tri < T; ++tri) {
            REAL nn[3] = {g->normals[tri], g->normals[T + tri], g->normals[2 * T + tri]};
            REAL jac = (REAL)2 * (REAL)g->areas[tri];
            cplx qv = {q_re[tri], q_im[tri]};
            for (int a = 0; a < 6; ++a) {
                REAL sp[3], b[3];
                point_on(g, tri, (REAL)QX[a], (REAL)QY[a], sp);
                basis((REAL)QX[a], (REAL)QY[a], b);
                cplx ps = {0, 0};
                for (int l = 0; l < 3; ++l) {
                    int d = dof(g, tri, l);
                    cplx pv = {p_re[d], p_im[d]};
                    ps = cadd(ps, cscale(pv, b[l]));
                }
                REAL w = (REAL)QW[a] * jac;
                cplx D = dlp(sp[0] - ox, sp[1] - oy, sp[2] - oz, nn[0], nn[1], nn[2], kr, 0);
                cplx G = green(sp[0] - ox, sp[1] - oy, sp[2] - oz, kr, 0);
                acc = cadd(acc, cscale(csub(cmul(D, ps), cmul(G, qv)), w));
                for (int m = 0; m < nm; ++m) {
                    REAL ip[3] = {sp[0], sp[1], sp[2]}, in[3] = {nn[0], nn[1], nn[2]};
                    mirror(ip, masks[m]);
                    mirror(in, masks[m]);
                    cplx Di = dlp(ip[0] - ox, ip[1] - oy, ip[2] - oz, in[0], in[1], in[2], kr, 0);
                    cplx Gi = green(ip[0] - ox, ip[1] - oy, ip[2] - oz, kr, 0);
                    acc = cadd(acc, cscale(csub(cmul(Di, ps), cmul(Gi, qv)), w));
                }
            }
        }
        out_re[o] = acc.re;
        out_im[o] = acc.im;
    }
    return 0;
}

/* ---- CHIEF rows (main.swift:1897-2036) --------------------------------
 * Interior point x_c: one collocation row of the exterior representation,
 * which vanishes inside the body:
 *   sum_tri sum_images int D(x_c, y) p(y) - G(x_c, y) q(y) dy = 0,
 *   q = g + i k beta Pi p  (Robin: Pi p = the triangle's P1 mean).
 * Hence C p = d with C[c][dof] = sum int D phi_dof - (int G) (i k beta) / 3
 * and d[c] = sum_tri (int G) g_tri.  D and G take the real wavenumber (the
 * field kernels); i k of the Robin fold takes the complex one (kr + i ki);
 * no jump term, no symmetry row weight.  C is row-major (m, n_dof).
 * Returns ||C||_inf, the largest row sum of |c|. */
double OGP(chief_rows)(const og_geom *g, const float *pts3xM, int m, REAL kr, REAL ki, const REAL *beta_re,
                       const REAL *beta_im, const REAL *q_re, const REAL *q_im, REAL *c_re, REAL *c_im,
                       REAL *d_re, REAL *d_im) {
    int T = g->n_triangles, n = g->n_dof;
    int masks[3];
    int nm = mirror_masks(g->sym, masks);
    double cnorm = 0;
#pragma omp parallel for schedule(static) reduction(max : cnorm)
    for (int ci = 0; ci < m; ++ci) {
        REAL ox = pts3xM[ci], oy = pts3xM[m + ci], oz = pts3xM[2 * m + ci];
        REAL *cr = c_re + (size_t)ci * n, *cim = c_im + (size_t)ci * n;
        for (int j = 0; j < n; ++j) cr[j] = cim[j] = 0;
        cplx dsum = {0, 0};
        for (int tri = 0; tri < T; ++tri) {
            REAL nn[3] = {g->normals[tri], g->normals[T + tri], g->normals[2 * T + tri]};
            REAL jac = (REAL)2 * (REAL)g->areas[tri];
            cplx dc[3] = {{0, 0}, {0, 0}, {0, 0}}, gs = {0, 0};
            for (int a = 0; a < 6; ++a) {
                REAL sp[3], b[3];
                point_on(g, tri, (REAL)QX[a], (REAL)QY[a], sp);
                basis((REAL)QX[a], (REAL)QY[a], b);
                REAL w = (REAL)QW[a] * jac;
                for (int im = -1; im < nm; ++im) {
                    REAL ip[3] = {sp[0], sp[1], sp[2]}, in[3] = {nn[0], nn[1], nn[2]};
                    if (im >= 0) {
                        mirror(ip, masks[im]);
                        mirror(in, masks[im]);
                    }
                    cplx D = dlp(ip[0] - ox, ip[1] - oy, ip[2] - oz, in[0], in[1], in[2], kr, 0);
                    cplx G = green(ip[0] - ox, ip[1] - oy, ip[2] - oz, kr, 0);
                    for (int l = 0; l < 3; ++l) dc[l] = cadd(dc[l], cscale(D, b[l] * w));
                    gs = cadd(gs, cscale(G, w));
                }
            }
            cplx qv = {q_re ? q_re[tri] : 0, q_im ? q_im[tri] : 0};
            dsum = cadd(dsum, cmul(gs, qv));
            cplx rob = {0, 0};
            if (beta_re && (beta_re[tri] != 0 || beta_im[tri] != 0)) {
                cplx ik = {-ki, kr}, bt = {beta_re[tri], beta_im[tri]};
                rob = cscale(cmul(gs, cmul(ik, bt)), (REAL)1 / 3);
            }
            for (int l = 0; l < 3; ++l) {
                int d = dof(g, tri, l);
                cr[d] += dc[l].re - rob.re;
                cim[d] += dc[l].im - rob.im;
            }
        }
        d_re[ci] = dsum.re;
        d_im[ci] = dsum.im;
        double row = 0;
        for (int j = 0; j < n; ++j) row += hypot((double)cr[j], (double)cim[j]);
        if (row > cnorm) cnorm = row;
    }
    return cnorm;
}

/* ---- tag reduction (main.swift:807-841), FP64 sums -------------------- */
int OGP(tag_average)(const og_geom *g, const int *tags, const REAL *p_re, const REAL *p_im, int tag, double out[3]) {
    double sr = 0, si = 0, ta = 0;
    for (int t = 0; t < g->n_triangles; ++t) {
        if (tags[t] != tag) continue;
        double a = g->areas[t];
        if (a <= 0) continue;
        int d0 = dof(g, t, 0), d1 = dof(g, t, 1), d2 = dof(g, t, 2);
        sr += ((double)p_re[d0] + (double)p_re[d1] + (double)p_re[d2]) / 3.0 * a;
        si += ((double)p_im[d0] + (double)p_im[d1] + (double)p_im[d2]) / 3.0 * a;
        ta += a;
    }
    if (ta < 1e-30) { out[0] = out[1] = out[2] = 0; return 0; }
    out[0] = sr / ta; out[1] = si / ta; out[2] = ta;
    return 0;
}

int OGP(set_threads)(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ---- coupled infinite baffle (main.swift:873-1470, 7504-7595) ---------- */
/* S_ia (n x m): interior SLP projection onto aperture triangles: regular part
   with trial images and the 2^planes row weight (main.swift:1178-1235), plus
   the Duffy SLP deltas of every singular pair whose trial is an aperture
   triangle, at weight 1 (main.swift:1011-1049). */
int OGP(aperture_slp)(const og_geom *g, const int *ap, int m, REAL kr, REAL ki, REAL *S_re, REAL *S_im) {
    int T = g->n_triangles;
    int masks[4] = {0, 0, 0, 0};
    int nm = 1 + mirror_masks(g->sym, masks + 1);
    REAL rw = row_weight(g->sym);
#pragma omp parallel for schedule(dynamic, 8)
    for (int test = 0; test < T; ++test) {
        for (int t = 0; t < m; ++t) {
            cplx slp[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int mi = 0; mi < nm; ++mi) {
                cplx s[3], d[9];
                pair_blocks(g, test, ap[t], 0, masks[mi], 0, 0, NULL, 0, NULL, 0, kr, ki, s, d);
                for (int i = 0; i < 3; ++i) slp[i] = cadd(slp[i], s[i]);
            }
            for (int i = 0; i < 3; ++i) {
                int row = dof(g, test, i);
                atomic_add(&S_re[(size_t)row * m + t], slp[i].re * rw);
                atomic_add(&S_im[(size_t)row * m + t], slp[i].im * rw);
            }
        }
    }
    int counts[3];
    int np = OGP(duffy_pairs)(g, NULL, 0, counts);
    int *pairs = malloc((size_t)(np ? np : 1) * PAIR_INTS * sizeof(int));
    OGP(duffy_pairs)(g, pairs, np, counts);
    int *loc = malloc((size_t)T * sizeof(int));
    for (int i = 0; i < T; ++i) loc[i] = -1;
    for (int t = 0; t < m; ++t) loc[ap[t]] = t;
    REAL *rules[3];
    int nr[3];
    for (int k = 0; k < 3; ++k) { rules[k] = malloc(1536 * 5 * sizeof(REAL)); nr[k] = duffy_rule(k + 1, rules[k]); }
#pragma omp parallel for schedule(dynamic, 16)
    for (int p = 0; p < np; ++p) {
        const int *r = pairs + (size_t)p * PAIR_INTS;
        int t = loc[r[1]];
        if (t < 0) continue;
        cplx rs[3], rd[9], ss[3], sd[9];
        pair_blocks(g, r[0], r[1], r[2], r[3], 0, 0, r + 5, 0, NULL, 0, kr, ki, rs, rd);
        pair_blocks(g, r[0], r[1], r[2], r[3], 1, r[4], r + 5, 0, rules[r[4] - 1], nr[r[4] - 1], kr, ki, ss, sd);
        for (int i = 0; i < 3; ++i) {
            int row = dof(g, r[0], i);
            cplx dlt = csub(ss[i], rs[i]);
            atomic_add(&S_re[(size_t)row * m + t], dlt.re);
            atomic_add(&S_im[(size_t)row * m + t], dlt.im);
        }
    }
    free(pairs); free(loc);
    for (int k = 0; k < 3; ++k) free(rules[k]);
    return 0;
}

/* S_aa (m x m): aperture-averaged SLP at the real field wavenumber, divided
   by the test triangle area (main.swift:1237-1290); Duffy deltas of aperture
   pairs with an unmirrored test triangle (main.swift:1051-1087). */
int OGP(aperture_avg)(const og_geom *g, const int *ap, int m, REAL kr, REAL *S_re, REAL *S_im) {
    int T = g->n_triangles;
    int masks[4] = {0, 0, 0, 0};
    int nm = 1 + mirror_masks(g->sym, masks + 1);
#pragma omp parallel for schedule(dynamic, 4)
    for (int r = 0; r < m; ++r) {
        REAL inv = (REAL)1 / (g->areas[ap[r]] > 0 ? (REAL)g->areas[ap[r]] : (REAL)1e-38);
        for (int c = 0; c < m; ++c) {
            cplx acc = {0, 0};
            for (int mi = 0; mi < nm; ++mi) {
                cplx s[3], d[9];
                pair_blocks(g, ap[r], ap[c], 0, masks[mi], 0, 0, NULL, 0, NULL, 0, kr, 0, s, d);
                for (int i = 0; i < 3; ++i) acc = cadd(acc, s[i]);
            }
            S_re[(size_t)r * m + c] += acc.re * inv;
            S_im[(size_t)r * m + c] += acc.im * inv;
        }
    }
    int counts[3];
    int np = OGP(duffy_pairs)(g, NULL, 0, counts);
    int *pairs = malloc((size_t)(np ? np : 1) * PAIR_INTS * sizeof(int));
    OGP(duffy_pairs)(g, pairs, np, counts);
    int *loc = malloc((size_t)T * sizeof(int));
    for (int i = 0; i < T; ++i) loc[i] = -1;
    for (int t = 0; t < m; ++t) loc[ap[t]] = t;
    REAL *rules[3];
    int nr[3];
    for (int k = 0; k < 3; ++k) { rules[k] = malloc(1536 * 5 * sizeof(REAL)); nr[k] = duffy_rule(k + 1, rules[k]); }
    for (int p = 0; p < np; ++p) {
        const int *q = pairs + (size_t)p * PAIR_INTS;
        if (q[2] != 0 || loc[q[0]] < 0 || loc[q[1]] < 0) continue;
        cplx rs[3], rd[9], ss[3], sd[9];
        pair_blocks(g, q[0], q[1], q[2], q[3], 0, 0, q + 5, 0, NULL, 0, kr, 0, rs, rd);
        pair_blocks(g, q[0], q[1], q[2], q[3], 1, q[4], q + 5, 0, rules[q[4] - 1], nr[q[4] - 1], kr, 0, ss, sd);
        cplx dlt = {0, 0};
        for (int i = 0; i < 3; ++i) dlt = cadd(dlt, csub(ss[i], rs[i]));
        REAL inv = (REAL)1 / (g->areas[q[0]] > 0 ? (REAL)g->areas[q[0]] : (REAL)1e-38);
        S_re[(size_t)loc[q[0]] * m + loc[q[1]]] += dlt.re * inv;
        S_im[(size_t)loc[q[0]] * m + loc[q[1]]] += dlt.im * inv;
    }
    free(pairs); free(loc);
    for (int k = 0; k < 3; ++k) free(rules[k]);
    return 0;
}

/* Rayleigh half-space field of the aperture Neumann data (main.swift:1397-1444):
   p(x) = -2 sum_t q_t sum_q w 2|t| sum_images G(y, x') with x' = (x, y, max(z, 0))
   for z >= -1e-5, zero below the baffle. */
int OGP(rayleigh)(const og_geom *g, const int *ap, int m, REAL kr, const REAL *qa_re, const REAL *qa_im,
                  const float *obs3xN, int nobs, REAL *out_re, REAL *out_im) {
    int masks[3];
    int nm = mirror_masks(g->sym, masks);
#pragma omp parallel for schedule(static)
    for (int o = 0; o < nobs; ++o) {
        REAL ox = obs3xN[o], oy = obs3xN[nobs + o], oz = obs3xN[2 * nobs + o];
        out_re[o] = 0; out_im[o] = 0;
        if (oz < (REAL)-1e-5) continue;
        REAL ez = oz < 0 ? 0 : oz;
        cplx acc = {0, 0};
        for (int t = 0; t < m; ++t) {
            cplx qv = {qa_re[t], qa_im[t]};
            if (qv.re == 0 && qv.im == 0) continue;
            REAL jac = (REAL)2 * (REAL)g->areas[ap[t]];
            for (int a = 0; a < 6; ++a) {
                REAL sp[3];
                point_on(g, ap[t], (REAL)QX[a], (REAL)QY[a], sp);
                REAL w = (REAL)QW[a] * jac;
                acc = cadd(acc, cscale(cmul(green(sp[0] - ox, sp[1] - oy, sp[2] - ez, kr, 0), qv), w));
                for (int mi = 0; mi < nm; ++mi) {
                    REAL ip[3] = {sp[0], sp[1], sp[2]};
                    mirror(ip, masks[mi]);
                    acc = cadd(acc, cscale(cmul(green(ip[0] - ox, ip[1] - oy, ip[2] - ez, kr, 0), qv), w));
                }
            }
        }
        out_re[o] = acc.re * (REAL)-2;
        out_im[o] = acc.im * (REAL)-2;
    }
    return 0;
}
