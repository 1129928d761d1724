// Session lifecycle, host-side plans (spatial tiling, Duffy pair list, rule
// tables) and the small C-ABI utilities.
//
// Reference counterparts (main.swift of m3gnus/hornlab-metal-bem):
//   ResidentMetalContext set-up  5370-5507  (P1 incidence, pair list, upload)
//   buildDuffyPairList          2266-2391  (real and image pair enumeration)
//   buildDuffyReductionPlan     2560-2613  (unique (row, col) triplets)
//   duffyRule                   2652-2699  (Sauter-Schwab style rules)
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <set>
#include <tuple>
#include <unordered_map>

#include "hbem_internal.h"

namespace hbem {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return e == cudaErrorMemoryAllocation ? HBEM_ERR_NOMEM : HBEM_ERR_CUDA;
}

void count_launch(long long n) { g_launches += n; }

// Kernel attributes belong to a kernel on one device: raise the dynamic
// shared-memory limit (and, when asked, allow non-portable cluster sizes) the
// first time a kernel runs on each device, under a lock.
int func_opt_in(const void *func, int smem_bytes, bool nonportable_cluster) {
    static std::mutex mu;
    static std::set<std::tuple<int, const void *, int, bool>> done;
    int dev = 0;
    HBEM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(dev, func, smem_bytes, nonportable_cluster);
    if (done.count(key)) return HBEM_OK;
    HBEM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes));
    if (nonportable_cluster) HBEM_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    done.insert(key);
    return HBEM_OK;
}

// Stream-ordered allocations (workspaces of the LU, refinement, condition
// estimate) come from the device's default memory pool; by default that pool
// hands freed memory back to the driver at every synchronisation, so the
// next allocation maps memory again.  Keep it cached instead (process-local
// setting of this process's pool, like a caching allocator).
void keep_pool_memory() {
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    const unsigned long long bit = 1ull << dev;
    if (done.load() & bit) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.fetch_or(bit);
}

// Tuning knobs (HBEM_TUNE_*), process-wide; 0 = the built-in choice.
static std::atomic<int> g_tuning[HBEM_TUNE_COUNT];
int tuning(int key) { return (key >= 0 && key < HBEM_TUNE_COUNT) ? g_tuning[key].load() : 0; }

// ---------------------------------------------------------------------------
// Duffy rules: 4-point Gauss-Legendre on [0,1] in each of four Duffy
// coordinates; 6 / 5 / 2 sub-regions for coincident / edge / vertex pairs.
// Each record: test (xi, eta), trial (xi, eta), weight on the reference
// triangle 0 <= eta <= 1 - xi.  The sub-region maps are the published
// Sauter-Schwab formulas (Sauter & Schwab, Boundary Element Methods, 2011,
// ch. 5), laid out in the reference's order (main.swift:2652-2699) so the
// tables are point-for-point identical.
// ---------------------------------------------------------------------------
void duffy_rule_table(int kind, std::vector<float> &rec) {
    const double a1 = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
    const double a2 = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0)) / 2.0;
    const double w1 = (18.0 + std::sqrt(30.0)) / 72.0, w2 = (18.0 - std::sqrt(30.0)) / 72.0;
    // Nodes/weights rounded to float first, then combined in float, matching
    // the FP32 arithmetic of the reference's rule construction.
    const float xs[4] = {float(0.5 - a2), float(0.5 - a1), float(0.5 + a1), float(0.5 + a2)};
    const float ws[4] = {float(w2), float(w1), float(w1), float(w2)};
    rec.clear();
    auto put = [&](float tx, float ty, float sx, float sy, float w) {
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
                    float xi = xs[b], e1 = xs[a], e2 = xs[c], e3 = xs[d];
                    float e12 = e1 * e2, e123 = e12 * e3;
                    float base = ws[a] * ws[b] * ws[c] * ws[d];
                    if (kind == 1) {
                        float w = base * xi * xi * xi * e1 * e1 * e2;
                        put(xi, xi * (1 - e1 + e12), xi * (1 - e123), xi * (1 - e1), w);
                        put(xi * (1 - e123), xi * (1 - e1), xi, xi * (1 - e1 + e12), w);
                        put(xi, xi * (e1 - e12 + e123), xi * (1 - e12), xi * (e1 - e12), w);
                        put(xi * (1 - e12), xi * (e1 - e12), xi, xi * (e1 - e12 + e123), w);
                        put(xi * (1 - e123), xi * (e1 - e123), xi, xi * (e1 - e12), w);
                        put(xi, xi * (e1 - e12), xi * (1 - e123), xi * (e1 - e123), w);
                    } else if (kind == 2) {
                        float w = base * xi * xi * xi * e1 * e1;
                        put(xi, xi * e1 * e3, xi * (1 - e12), xi * e1 * (1 - e2), w);
                        put(xi, xi * e1, xi * (1 - e123), xi * e1 * e2 * (1 - e3), w * e2);
                        put(xi * (1 - e12), xi * e1 * (1 - e2), xi, xi * e123, w * e2);
                        put(xi * (1 - e123), xi * e12 * (1 - e3), xi, xi * e1, w * e2);
                        put(xi * (1 - e123), xi * e1 * (1 - e2 * e3), xi, xi * e12, w * e2);
                    } else {
                        float w = base * xi * xi * xi * e2;
                        put(xi, xi * e1, xi * e2, xi * e2 * e3, w);
                        put(xi * e2, xi * e2 * e3, xi, xi * e1, w);
                    }
                }
}

// ---------------------------------------------------------------------------
// Singular pair enumeration.  Two (image) triangles form a singular pair when
// they share 3 / 2 / 1 vertices; with symmetry planes every (test image,
// trial image) mask combination is enumerated and vertices are matched on the
// 1e-6 lattice of their mirrored coordinates (main.swift:2107-2112, 2152-2193,
// 2316-2380).  An odd mirror reverses local vertex order.
// ---------------------------------------------------------------------------
namespace {

struct Key3 {
    long long x, y, z;
    bool operator==(const Key3 &o) const { return x == o.x && y == o.y && z == o.z; }
};
struct Key3Hash {
    size_t operator()(const Key3 &k) const {
        uint64_t h = (uint64_t)k.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)k.y + 0x632BE59BD9B4E019ull + (h << 6) + (h >> 2);
        h ^= (uint64_t)k.z + 0x85157AF5ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

inline bool odd(int m) { return __builtin_popcount((unsigned)m) & 1; }
inline int image_local(int l, int m) { return odd(m) ? (l == 1 ? 2 : (l == 2 ? 1 : l)) : l; }

Key3 key_of(const Session &s, int v, int mask) {
    const int V = s.n_vertices;
    float x = s.verts[v], y = s.verts[V + v], z = s.verts[2 * V + v];
    if (mask & 1) x = -x;
    if (mask & 2) y = -y;
    if (mask & 4) z = -z;
    return Key3{llround((double)x / 1.0e-6), llround((double)y / 1.0e-6), llround((double)z / 1.0e-6)};
}

inline int tvert(const Session &s, int t, int l) { return s.tris[l * s.n_triangles + t]; }

int shared(const Session &s, int test, int trial, int tm, int sm, int loc[4]) {
    int count = 0;
    loc[0] = loc[1] = loc[2] = loc[3] = 0;
    for (int tf = 0; tf < 3; ++tf) {
        int vt = tvert(s, test, image_local(tf, tm));
        Key3 kt = key_of(s, vt, tm);
        for (int sf = 0; sf < 3; ++sf) {
            int vs = tvert(s, trial, image_local(sf, sm));
            bool match = (tm == 0 && sm == 0) ? (vt == vs) : (kt == key_of(s, vs, sm));
            if (match) {
                ++count;
                if (count == 1) { loc[0] = tf; loc[2] = sf; } else { loc[1] = tf; loc[3] = sf; }
            }
        }
    }
    return count;
}

}  // namespace

int build_duffy_pairs(Session &s, std::vector<DuffyPair> &pairs) {
    const int T = s.n_triangles;
    std::vector<int> masks = {0};
    if (s.sym == 1) masks.push_back(1);
    if (s.sym == 2) masks.push_back(2);
    if (s.sym == 4) masks.push_back(4);
    if (s.sym == 3) { masks.push_back(1); masks.push_back(2); masks.push_back(3); }
    const int nm = (int)masks.size();
    // per test mask: mirrored-vertex key -> triangles (ascending)
    std::vector<std::unordered_map<Key3, std::vector<int>, Key3Hash>> table(nm);
    for (int mi = 0; mi < nm; ++mi) {
        auto &tab = table[mi];
        tab.reserve((size_t)s.n_vertices * 2);
        for (int t = 0; t < T; ++t)
            for (int l = 0; l < 3; ++l) tab[key_of(s, tvert(s, t, l), masks[mi])].push_back(t);
    }
    std::vector<int> stamp(T, 0), cand;
    cand.reserve(64);
    int st = 0;
    pairs.clear();
    pairs.reserve((size_t)T * 13 * nm);
    for (int trial = 0; trial < T; ++trial) {
        for (int si = 0; si < nm; ++si) {
            for (int ti = 0; ti < nm; ++ti) {
                if (s.sym == 0 && (si | ti)) continue;
                ++st;
                cand.clear();
                for (int l = 0; l < 3; ++l) {
                    auto it = table[ti].find(key_of(s, tvert(s, trial, l), masks[si]));
                    if (it == table[ti].end()) continue;
                    for (int test : it->second)
                        if (stamp[test] != st) { stamp[test] = st; cand.push_back(test); }
                }
                for (int test : cand) {
                    int loc[4];
                    int c = shared(s, test, trial, masks[ti], masks[si], loc);
                    if (c <= 0) continue;
                    DuffyPair p{};
                    p.test = test; p.trial = trial; p.test_mask = masks[ti]; p.trial_mask = masks[si];
                    p.kind = c == 3 ? 1 : (c == 2 ? 2 : 3);
                    if (p.kind == 1) { p.tl1 = 0; p.tl2 = 1; p.sl1 = 0; p.sl2 = 1; }
                    else { p.tl1 = loc[0]; p.tl2 = loc[1]; p.sl1 = loc[2]; p.sl2 = loc[3]; }
                    pairs.push_back(p);
                }
            }
        }
    }
    return HBEM_OK;
}

// Vertices an image pair of triangles shares (matched on the 1e-6 lattice of
// the mirrored coordinates, as for the singular pairs).
int image_shared_vertices(const Session &s, int test, int trial, int test_mask, int trial_mask) {
    int loc[4];
    return shared(s, test, trial, test_mask, trial_mask, loc);
}

}  // namespace hbem

using namespace hbem;

// ---------------------------------------------------------------------------
// Session creation
// ---------------------------------------------------------------------------
namespace {

uint32_t spread10(uint32_t v) {
    v &= 0x3FF;
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

template <typename T>
int upload(T **dst, const T *src, size_t count) {
    if (count == 0) count = 1;
    HBEM_CUDA(cudaMalloc((void **)dst, count * sizeof(T)));
    if (src) HBEM_CUDA(cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
    return HBEM_OK;
}

void free_session(Session *s) {
    if (!s) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    void *ptrs[] = {s->d_qp, s->d_nrm, s->d_tri, s->d_test_slot, s->d_trial_slot, s->d_row_off, s->d_rows,
                    s->d_col_off, s->d_cols, s->d_verts, s->d_tris, s->d_l2g, s->d_tags, s->d_areas,
                    s->d_normals, s->d_fqp, s->d_fnrm, s->d_pairs, s->d_rule, s->d_rule_w, s->d_status, s->ws,
                    s->d_ap_tris, s->d_ap_local, s->d_sing_bits, s->d_geo64, s->d_near, s->d_subrule};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (s->pinned) cudaFreeHost(s->pinned);
    if (s->aux_fork) cudaEventDestroy(s->aux_fork);
    if (s->aux_join) cudaEventDestroy(s->aux_join);
    if (s->aux) cudaStreamDestroy(s->aux);
    cudaSetDevice(prev);
    delete s;
}

const double kQX[6] = {0.4459484909159651, 0.0915762135097710, 0.1081030181680700,
                       0.4459484909159651, 0.8168475729804590, 0.0915762135097710};
const double kQY[6] = {0.4459484909159651, 0.0915762135097700, 0.4459484909159651,
                       0.1081030181680700, 0.0915762135097700, 0.8168475729804580};

// Build the test/trial tile dof lists of consecutive sorted triangles.
void tile_plan(const Session &s, int tile, std::vector<int> &off, std::vector<int> &list,
               std::vector<uchar4> &slot, int &max_count) {
    const int T = s.n_triangles;
    const int ntiles = (T + tile - 1) / tile;
    off.assign(ntiles + 1, 0);
    list.clear();
    slot.assign(T, make_uchar4(0, 0, 0, 0));
    max_count = 1;
    std::vector<int> d;
    for (int t = 0; t < ntiles; ++t) {
        d.clear();
        for (int i = t * tile; i < std::min(T, (t + 1) * tile); ++i)
            for (int l = 0; l < 3; ++l) d.push_back(s.l2g[s.order[i] * 3 + l]);
        std::sort(d.begin(), d.end());
        d.erase(std::unique(d.begin(), d.end()), d.end());
        off[t] = (int)list.size();
        list.insert(list.end(), d.begin(), d.end());
        max_count = std::max(max_count, (int)d.size());
        for (int i = t * tile; i < std::min(T, (t + 1) * tile); ++i) {
            unsigned char sl[3];
            for (int l = 0; l < 3; ++l)
                sl[l] = (unsigned char)(std::lower_bound(d.begin(), d.end(), s.l2g[s.order[i] * 3 + l]) - d.begin());
            slot[i] = make_uchar4(sl[0], sl[1], sl[2], 0);
        }
    }
    off[ntiles] = (int)list.size();
}

}  // namespace

extern "C" int hbem_version(void) { return 100; }

extern "C" int hbem_last_error(char *buf, size_t len) {
    if (buf && len) {
        std::snprintf(buf, len, "%s", g_last_error.c_str());
    }
    return (int)g_last_error.size();
}

extern "C" long long hbem_launch_count(void) { return g_launches.load(); }

extern "C" int hbem_set_tuning(int key, int value) {
    switch (key) {
        case HBEM_TUNE_ASM_MINBLOCKS:
            if (value != 0 && value != 2 && value != 3) return fail(HBEM_ERR_ARG, "HBEM_TUNE_ASM_MINBLOCKS: 0, 2 or 3");
            break;
        case HBEM_TUNE_LU_PANEL:
            if (value != 0 && value != 16 && value != 32 && value != 64)
                return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_PANEL: 0, 16, 32 or 64");
            break;
        case HBEM_TUNE_LU_SOLVE:
            if (value < 0 || value > 3) return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_SOLVE: 0, 1, 2 or 3");
            break;
        case HBEM_TUNE_ASM_PAIRS:
            if (value < 0 || value > 1) return fail(HBEM_ERR_ARG, "HBEM_TUNE_ASM_PAIRS: 0 or 1");
            break;
        case HBEM_TUNE_DUFFY:
            if (value < 0 || value > 2) return fail(HBEM_ERR_ARG, "HBEM_TUNE_DUFFY: 0, 1 or 2");
            break;
        case HBEM_TUNE_LU_LOOKAHEAD:
            if (value < 0 || value > 1) return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_LOOKAHEAD: 0 or 1");
            break;
        case HBEM_TUNE_LU_RESERVE:
            if (value < 0 || value > 1024) return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_RESERVE: 0 .. 1024");
            break;
        case HBEM_TUNE_WAVE_SPIN:
            if (value < 0 || value > (1 << 22)) return fail(HBEM_ERR_ARG, "HBEM_TUNE_WAVE_SPIN: 0 .. 4194304");
            break;
        case HBEM_TUNE_LU_UPDATE:
            if (value < 0 || value > 2) return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_UPDATE: 0, 1 or 2");
            break;
        case HBEM_TUNE_LU_BLOCK:
            if (value != 0 && value != 32 && value != 64 && value != 128)
                return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_BLOCK: 0, 32, 64 or 128");
            break;
        case HBEM_TUNE_LU_PANEL_KERNEL:
            if (value < 0 || value > 1) return fail(HBEM_ERR_ARG, "HBEM_TUNE_LU_PANEL_KERNEL: 0 or 1");
            break;
        default:
            return fail(HBEM_ERR_ARG, "hbem_set_tuning: unknown key " + std::to_string(key));
    }
    g_tuning[key].store(value);
    return HBEM_OK;
}

extern "C" int hbem_get_tuning(int key) { return tuning(key); }

extern "C" int hbem_session_create(const float *vertices_3xv, int n_vertices, const int *triangles_3xt,
                                   int n_triangles, const int *l2g, int n_dof, const int *tags,
                                   const float *areas, const float *normals_3xt, int sym_code, int device,
                                   hbem_session **out) {
    if (!out) return fail(HBEM_ERR_ARG, "hbem_session_create: out is NULL");
    *out = nullptr;
    if (!vertices_3xv || !triangles_3xt || !l2g || !tags || !areas || !normals_3xt)
        return fail(HBEM_ERR_ARG, "hbem_session_create: NULL geometry pointer");
    if (n_vertices <= 0 || n_triangles <= 0 || n_dof <= 0)
        return fail(HBEM_ERR_ARG, "hbem_session_create: empty geometry");
    if (!(sym_code == 0 || sym_code == 1 || sym_code == 2 || sym_code == 3 || sym_code == 4))
        return fail(HBEM_ERR_ARG, "hbem_session_create: sym_code must be 0, 1, 2, 3 or 4");
    for (long long i = 0; i < 3LL * n_triangles; ++i) {
        if (triangles_3xt[i] < 0 || triangles_3xt[i] >= n_vertices)
            return fail(HBEM_ERR_ARG, "hbem_session_create: triangle vertex index out of range");
        if (l2g[i] < 0 || l2g[i] >= n_dof)
            return fail(HBEM_ERR_ARG, "p1_local2global contains out-of-range DOF " + std::to_string(l2g[i]));
    }
    for (int t = 0; t < n_triangles; ++t)
        if (!(areas[t] > 0.0f) || !std::isfinite(areas[t]))
            return fail(HBEM_ERR_ARG, "hbem_session_create: triangle " + std::to_string(t) + " has non-positive area");
    int ndev = 0;
    HBEM_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(HBEM_ERR_ARG, "hbem_session_create: bad device index");
    HBEM_CUDA(cudaSetDevice(device));
    keep_pool_memory();

    Session *s = new Session();
    s->device = device;
    s->n_vertices = n_vertices;
    s->n_triangles = n_triangles;
    s->n_dof = n_dof;
    s->sym = sym_code;
    const int T = n_triangles, V = n_vertices;
    s->verts.assign(vertices_3xv, vertices_3xv + 3LL * V);
    s->tris.assign(triangles_3xt, triangles_3xt + 3LL * T);
    s->l2g.assign(l2g, l2g + 3LL * T);
    s->tags.assign(tags, tags + T);
    s->areas.assign(areas, areas + T);
    s->normals.assign(normals_3xt, normals_3xt + 3LL * T);

    // quadrature points in double, original order
    std::vector<float4> qp((size_t)T * 6), nrm(T);
    std::vector<double> cx(T), cy(T), cz(T);
    for (int t = 0; t < T; ++t) {
        double P[3][3];
        for (int l = 0; l < 3; ++l) {
            int v = s->tris[l * T + t];
            for (int c = 0; c < 3; ++c) P[l][c] = s->verts[c * V + v];
        }
        for (int q = 0; q < 6; ++q) {
            double b1 = 1.0 - kQX[q] - kQY[q], b2 = kQX[q], b3 = kQY[q];
            double x[3];
            for (int c = 0; c < 3; ++c) x[c] = b1 * P[0][c] + b2 * P[1][c] + b3 * P[2][c];
            qp[(size_t)t * 6 + q] = make_float4((float)x[0], (float)x[1], (float)x[2], 0.f);
        }
        cx[t] = (P[0][0] + P[1][0] + P[2][0]) / 3;
        cy[t] = (P[0][1] + P[1][1] + P[2][1]) / 3;
        cz[t] = (P[0][2] + P[1][2] + P[2][2]) / 3;
        nrm[t] = make_float4(s->normals[t], s->normals[T + t], s->normals[2 * T + t], 2.0f * s->areas[t]);
    }

    // Morton order of centroids keeps tiles spatially compact, so a tile of
    // 32 / 64 triangles touches few distinct dofs.
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int t = 0; t < T; ++t) {
        double c[3] = {cx[t], cy[t], cz[t]};
        for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], c[k]); hi[k] = std::max(hi[k], c[k]); }
    }
    double span = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-30});
    std::vector<uint32_t> code(T);
    for (int t = 0; t < T; ++t) {
        uint32_t ix = (uint32_t)std::min(1023.0, (cx[t] - lo[0]) / span * 1023.0);
        uint32_t iy = (uint32_t)std::min(1023.0, (cy[t] - lo[1]) / span * 1023.0);
        uint32_t iz = (uint32_t)std::min(1023.0, (cz[t] - lo[2]) / span * 1023.0);
        code[t] = spread10(ix) | (spread10(iy) << 1) | (spread10(iz) << 2);
    }
    s->order.resize(T);
    std::iota(s->order.begin(), s->order.end(), 0);
    std::stable_sort(s->order.begin(), s->order.end(), [&](int a, int b) { return code[a] < code[b]; });

    std::vector<float4> sqp((size_t)T * 6), snrm(T);
    std::vector<int4> stri(T);
    for (int i = 0; i < T; ++i) {
        int t = s->order[i];
        for (int q = 0; q < 6; ++q) sqp[(size_t)i * 6 + q] = qp[(size_t)t * 6 + q];
        snrm[i] = nrm[t];
        stri[i] = make_int4(s->l2g[t * 3], s->l2g[t * 3 + 1], s->l2g[t * 3 + 2], t);
    }
    std::vector<int> row_off, rows, col_off, cols;
    std::vector<uchar4> test_slot, trial_slot;
    tile_plan(*s, kTestTile, row_off, rows, test_slot, s->max_rows);
    tile_plan(*s, kTrialTile, col_off, cols, trial_slot, s->max_cols);
    s->n_test_tiles = (int)row_off.size() - 1;
    s->n_trial_tiles = (int)col_off.size() - 1;

    // Duffy pairs, sorted by kind (coincident, edge, vertex)
    std::vector<DuffyPair> pairs;
    build_duffy_pairs(*s, pairs);
    for (auto &p : pairs) {
        if (p.kind == 1) ++s->n_coincident;
        else if (p.kind == 2) ++s->n_edge;
        else ++s->n_vertex;
        if (p.test_mask || p.trial_mask) ++s->n_image_pairs;
        p.weight = 1;
    }
    {
        // unique (row, col) triplets of the full enumeration (main.swift:2560-2613)
        std::vector<long long> keys;
        keys.reserve((size_t)pairs.size() * 9);
        for (auto &p : pairs)
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    keys.push_back((long long)s->l2g[p.test * 3 + i] + (long long)s->l2g[p.trial * 3 + j] * n_dof);
        std::sort(keys.begin(), keys.end());
        s->n_unique_triplets = (long long)(std::unique(keys.begin(), keys.end()) - keys.begin());
    }
    if (sym_code == 3) {
        // With both yz and xz planes, mirroring a (test image, trial image) pair
        // by the even mask 3 (a rotation by pi about z) maps it onto the pair
        // (test_mask ^ 3, trial_mask ^ 3) with identical local numbering and
        // bitwise-identical kernel samples (sign flips are exact).  The pair
        // list holds both twins; keep one with weight 2.
        std::vector<DuffyPair> kept;
        kept.reserve(pairs.size() / 2 + 1);
        for (auto &p : pairs)
            if (p.test_mask == 0 || p.test_mask == 1) {
                p.weight = 2;
                kept.push_back(p);
            }
        pairs.swap(kept);
    }
    std::stable_sort(pairs.begin(), pairs.end(), [](const DuffyPair &a, const DuffyPair &b) { return a.kind < b.kind; });
    s->n_pairs = (int)pairs.size();

    std::vector<float4> rule;
    std::vector<float> rule_w;
    for (int kind = 1; kind <= 3; ++kind) {
        std::vector<float> rec;
        duffy_rule_table(kind, rec);
        s->rule_off[kind - 1] = (int)rule.size();
        s->rule_cnt[kind - 1] = (int)(rec.size() / 5);
        for (size_t q = 0; q < rec.size() / 5; ++q) {
            rule.push_back(make_float4(rec[5 * q], rec[5 * q + 1], rec[5 * q + 2], rec[5 * q + 3]));
            rule_w.push_back(rec[5 * q + 4]);
        }
    }

    int rc = HBEM_OK;
    auto U = [&](int r) { if (rc == HBEM_OK) rc = r; };
    U(upload(&s->d_qp, sqp.data(), sqp.size()));
    U(upload(&s->d_nrm, snrm.data(), snrm.size()));
    U(upload(&s->d_tri, stri.data(), stri.size()));
    U(upload(&s->d_test_slot, test_slot.data(), test_slot.size()));
    U(upload(&s->d_trial_slot, trial_slot.data(), trial_slot.size()));
    U(upload(&s->d_row_off, row_off.data(), row_off.size()));
    U(upload(&s->d_rows, rows.data(), rows.size()));
    U(upload(&s->d_col_off, col_off.data(), col_off.size()));
    U(upload(&s->d_cols, cols.data(), cols.size()));
    U(upload(&s->d_verts, s->verts.data(), s->verts.size()));
    U(upload(&s->d_tris, s->tris.data(), s->tris.size()));
    U(upload(&s->d_l2g, s->l2g.data(), s->l2g.size()));
    U(upload(&s->d_tags, s->tags.data(), s->tags.size()));
    U(upload(&s->d_areas, s->areas.data(), s->areas.size()));
    U(upload(&s->d_normals, s->normals.data(), s->normals.size()));
    U(upload(&s->d_fqp, qp.data(), qp.size()));
    U(upload(&s->d_fnrm, nrm.data(), nrm.size()));
    U(upload(&s->d_pairs, pairs.data(), pairs.size()));
    U(upload(&s->d_rule, rule.data(), rule.size()));
    U(upload(&s->d_rule_w, rule_w.data(), rule_w.size()));
    U(upload(&s->d_status, (const int *)nullptr, 4));
    if (rc == HBEM_OK) {
        cudaError_t e = cudaMemset(s->d_status, 0, 4 * sizeof(int));
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemset(status)");
    }
    if (rc != HBEM_OK) {
        std::string msg = g_last_error;
        free_session(s);
        return fail(rc, msg);
    }
    *out = reinterpret_cast<hbem_session *>(s);
    return HBEM_OK;
}

extern "C" int hbem_session_destroy(hbem_session *h) {
    free_session(reinterpret_cast<Session *>(h));
    return HBEM_OK;
}

extern "C" int hbem_session_query(const hbem_session *h, int key, long long *value) {
    const Session *s = reinterpret_cast<const Session *>(h);
    if (!s || !value) return fail(HBEM_ERR_ARG, "hbem_session_query: NULL argument");
    const long long T = s->n_triangles;
    const long long M = s->sym == 3 ? 4 : (s->sym ? 2 : 1);
    switch (key) {
        case HBEM_Q_N_DOF: *value = s->n_dof; break;
        case HBEM_Q_N_TRIANGLES: *value = T; break;
        case HBEM_Q_N_PAIRS: *value = s->n_pairs; break;
        case HBEM_Q_PAIRS_COINCIDENT: *value = s->n_coincident; break;
        case HBEM_Q_PAIRS_EDGE: *value = s->n_edge; break;
        case HBEM_Q_PAIRS_VERTEX: *value = s->n_vertex; break;
        case HBEM_Q_IMAGE_PAIRS: *value = s->n_image_pairs; break;
        case HBEM_Q_UNIQUE_TRIPLETS: *value = s->n_unique_triplets; break;
        case HBEM_Q_SYMMETRY: *value = s->sym; break;
        case HBEM_Q_APERTURE_TRIANGLES: *value = s->m_ap; break;
        case HBEM_Q_NEAR_PAIRS: *value = s->n_near; break;
        case HBEM_Q_KERNEL_LAUNCHES: *value = s->launches; break;
        case HBEM_Q_REGULAR_EVALS: *value = T * T * 36 * M; break;
        case HBEM_Q_DUFFY_EVALS: {
            // evaluated after exact twin folding
            const long long fold = s->sym == 3 ? 2 : 1;
            *value = (s->n_coincident * (1536 + 36) + s->n_edge * (1280 + 36) + s->n_vertex * (512 + 36)) / fold;
            break;
        }
        default: return fail(HBEM_ERR_ARG, "hbem_session_query: unknown key");
    }
    return HBEM_OK;
}
