// Internal declarations shared by the libhbem.so translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/hbem.h"

namespace hbem {

// ---- error plumbing ------------------------------------------------------
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
void count_launch(long long n = 1);
int tuning(int key);   // HBEM_TUNE_* value, 0 = built-in choice
void keep_pool_memory();   // cache freed stream-ordered allocations of the current device
// raise a kernel's dynamic shared-memory limit once per device (thread-safe)
int func_opt_in(const void *func, int smem_bytes, bool nonportable_cluster = false);

#define HBEM_CUDA(call)                                        \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return ::hbem::cuda_fail(_e, #call); \
    } while (0)

#define HBEM_LAUNCH_CHECK(name)                                \
    do {                                                       \
        cudaError_t _e = cudaGetLastError();                   \
        if (_e != cudaSuccess) return ::hbem::cuda_fail(_e, name); \
        ::hbem::count_launch();                                \
    } while (0)

#ifdef __CUDACC__
// 4-byte asynchronous copy global -> shared; src_bytes 0 writes a zero
__device__ __forceinline__ void cp_async4(float *dst, const float *src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(dst))),
                 "l"(src), "r"(src_bytes)
                 : "memory");
}
#endif

// ---- assembly tiling constants -------------------------------------------
constexpr int kTestTile = 32;    // test triangles per CTA (one per lane)
constexpr int kTrialTile = 64;   // trial triangles per CTA (split over 8 warps)
constexpr int kAsmThreads = 256;

// Duffy pair record (device), 3 x int4.
struct DuffyPair {
    int test, trial, test_mask, trial_mask;   // original triangle ids, image masks
    int kind, tl1, tl2, sl1;                  // 1 coincident, 2 edge, 3 vertex; image-local ids
    int sl2, weight, col_base, pad;           // weight: exact image twins folded into one pair
};

struct Session {
    int device = 0;
    int n_vertices = 0, n_triangles = 0, n_dof = 0, sym = 0;
    // host copies (original order)
    std::vector<float> verts;      // (3, V)
    std::vector<int> tris;         // (3, T)
    std::vector<int> l2g;          // (T, 3)
    std::vector<int> tags;         // (T,)
    std::vector<float> areas;      // (T,)
    std::vector<float> normals;    // (3, T)

    // spatial order used by the tiled assembly: sorted position -> original id
    std::vector<int> order;
    int n_test_tiles = 0, n_trial_tiles = 0;
    int max_rows = 0, max_cols = 0;  // distinct dofs per test / trial tile

    // device geometry, sorted order
    float4 *d_qp = nullptr;         // (T, 6) quadrature points (x, y, z, 0)
    float4 *d_nrm = nullptr;        // (T) normal xyz + jacobian 2*area
    int4 *d_tri = nullptr;          // (T) dof0, dof1, dof2, original id
    uchar4 *d_test_slot = nullptr;  // (T) slot of each local dof within its test tile
    uchar4 *d_trial_slot = nullptr; // (T) slot within its trial tile
    int *d_row_off = nullptr;       // (n_test_tiles + 1)
    int *d_rows = nullptr;          // concatenated dof lists of test tiles
    int *d_col_off = nullptr;       // (n_trial_tiles + 1)
    int *d_cols = nullptr;

    // device geometry, original order (Duffy, field, reductions)
    float *d_verts = nullptr;       // (3, V)
    int *d_tris = nullptr;          // (3, T)
    int *d_l2g = nullptr;           // (T, 3)
    int *d_tags = nullptr;          // (T)
    float *d_areas = nullptr;       // (T)
    float *d_normals = nullptr;     // (3, T)
    float4 *d_fqp = nullptr;        // (T, 6) quadrature points, original order
    float4 *d_fnrm = nullptr;       // (T) normal + jac, original order

    // Duffy pairs (sorted by kind) + rule tables
    int n_pairs = 0;
    long long n_coincident = 0, n_edge = 0, n_vertex = 0, n_image_pairs = 0, n_unique_triplets = 0;
    int kind_begin[4] = {0, 0, 0, 0};
    DuffyPair *d_pairs = nullptr;
    float4 *d_rule = nullptr;       // test(x,y), trial(x,y) for kinds 1,2,3 concatenated
    float *d_rule_w = nullptr;
    int rule_off[3] = {0, 0, 0}, rule_cnt[3] = {0, 0, 0};

    int *d_status = nullptr;        // device-side status word (bounds / wait failures)
    unsigned *d_sing_bits = nullptr; // T x T bitmap of touching pairs (shape gradients, built on first use)
    double *d_geo64 = nullptr;      // FP64 path (built on first use): (T, 9) vertices per triangle,
                                    // (T, 4) normal + area, then the Duffy rules as 5 doubles per point

    // coupled infinite baffle: aperture triangles (ascending ids) and their
    // local index per triangle (-1 elsewhere)
    int aperture_tag = 0, m_ap = 0;
    std::vector<int> ap_tris;
    int *d_ap_tris = nullptr;
    int *d_ap_local = nullptr;

    // near-field subdivision (the reference's optional near quadrature): near,
    // non-touching image pairs and the subdivided 6-point rule of the level
    int near_level = 0;
    double near_threshold = 0.0;
    int n_near = 0, n_sub = 0;
    int4 *d_near = nullptr;         // test, trial, test mask, trial mask
    float4 *d_subrule = nullptr;    // (xi, eta, weight, 0) of the subdivided rule

    // sweep workspace (grown on demand)
    void *ws = nullptr;
    size_t ws_bytes = 0;
    // second stream of the sweep (the condition estimate beside the solves)
    // and its fork / join events, created on first use
    cudaStream_t aux = nullptr;
    cudaEvent_t aux_fork = nullptr, aux_join = nullptr;
    void *pinned = nullptr;
    size_t pinned_bytes = 0;

    long long launches = 0;
};

// ---- pieces implemented in separate translation units ---------------------
int build_duffy_pairs(Session &s, std::vector<DuffyPair> &pairs);
int image_shared_vertices(const Session &s, int test, int trial, int test_mask, int trial_mask);
int launch_near(Session &s, int n_freq, const float *k_re, const float *k_im, int n_src, const float *q_re,
                const float *q_im, long long q_stride, long long q_src_stride, const float *beta_re,
                const float *beta_im, float *a_re, float *a_im, long long lda, long long a_stride, float *b_re,
                float *b_im, long long b_stride, long long b_src_stride, cudaStream_t st);
void duffy_rule_table(int kind, std::vector<float> &rec);  // 5 floats per point
void duffy_rule_table64(int kind, std::vector<double> &rec);  // the same rule in double

int launch_regular(Session &s, int n_freq, const float *k_re, const float *k_im,
                   const float *q_re, const float *q_im, long long q_stride,
                   const float *beta_re, const float *beta_im,
                   float *a_re, float *a_im, long long lda, long long a_stride,
                   float *b_re, float *b_im, long long b_stride, cudaStream_t st,
                   int n_src = 1, long long q_src_stride = 0, long long b_src_stride = 0);
struct ApertureOut {
    int mode;                        // 0: S_ia (with or without A/b), 1: S_aa
    float *sia_re, *sia_im, *saa_re, *saa_im;
    long long sia_stride, saa_stride;
};
int launch_duffy(Session &s, int n_freq, const float *k_re, const float *k_im,
                 const float *q_re, const float *q_im, long long q_stride,
                 const float *beta_re, const float *beta_im,
                 float *a_re, float *a_im, long long lda, long long a_stride,
                 float *b_re, float *b_im, long long b_stride, cudaStream_t st,
                 const ApertureOut *ap, int n_src = 1, long long q_src_stride = 0, long long b_src_stride = 0);

}  // namespace hbem

// Dunavant 6-point degree-4 rule on the reference triangle (xi, eta), weights
// summing to 1/2 (reference main.swift:1472-1489).
#define HBEM_QX0 0.4459484909159651f
#define HBEM_QX1 0.0915762135097710f
#define HBEM_QX2 0.1081030181680700f
#define HBEM_QX3 0.4459484909159651f
#define HBEM_QX4 0.8168475729804590f
#define HBEM_QX5 0.0915762135097710f
#define HBEM_QY0 0.4459484909159651f
#define HBEM_QY1 0.0915762135097700f
#define HBEM_QY2 0.4459484909159651f
#define HBEM_QY3 0.1081030181680700f
#define HBEM_QY4 0.0915762135097700f
#define HBEM_QY5 0.8168475729804580f
#define HBEM_QWA 0.1116907948390055f
#define HBEM_QWB 0.0549758718276610f
#define HBEM_INV4PI 0.07957747154594767f
