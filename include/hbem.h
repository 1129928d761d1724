/*
 * hbem.h — C ABI of libhbem.so, the B200 (sm_100a) dense Helmholtz BEM hot path.
 *
 * Conventions
 *   - Every entry point returns an int status: HBEM_OK (0) on success, a
 *     negative HBEM_ERR_* code on failure (message via hbem_last_error), or a
 *     positive value for a numerical condition (singular pivot).
 *   - No C++ exception crosses this ABI; no torch type appears in it.
 *   - Complex arrays are planar: separate real and imaginary float32 arrays
 *     (the reference's IPC layout, docs/native-ipc.md "real_f32"/"imag_f32").
 *   - Dense matrices are row-major with a leading dimension `lda` (>= n) and a
 *     batch stride between consecutive matrices, all in elements.
 *   - "device" pointers are caller-owned CUDA device memory on the session's
 *     device; "host" pointers are ordinary host memory.  `stream` is a
 *     cudaStream_t passed as void* (NULL = legacy default stream).
 *   - A session is not thread-safe: use it from one host thread and one stream
 *     at a time.  Distinct sessions are independent.
 *
 * The reference (m3gnus/hornlab-metal-bem) crosses this boundary as a
 * subprocess with JSON manifests and planar float32 files
 * (hornlab_metal_bem/metal/native.py:252-377, 737-1203;
 *  hornlab_metal_bem/metal/session.py:21-389).  Each entry point below names
 * the reference operation it replaces.
 */
#ifndef HBEM_H
#define HBEM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HBEM_OK 0
#define HBEM_ERR_ARG (-1)      /* invalid argument / shape / index */
#define HBEM_ERR_CUDA (-2)     /* CUDA runtime or launch failure */
#define HBEM_ERR_NOMEM (-3)    /* device or host allocation failed */
#define HBEM_ERR_STATE (-4)    /* session misuse or device-side status flag set */
#define HBEM_SINGULAR 1        /* LU hit an exactly zero pivot (info > 0) */

/* Assembly flags */
#define HBEM_ASM_REGULAR 1     /* 6x6 Dunavant regular quadrature, all pairs */
#define HBEM_ASM_DUFFY 2       /* Duffy singular corrections (coincident/edge/vertex pairs) */
#define HBEM_ASM_ZERO 4        /* zero A (a whole slab, padding columns included, when a_stride = lda * n)
                                  and b before accumulating */
#define HBEM_ASM_CORRECTED (HBEM_ASM_REGULAR | HBEM_ASM_DUFFY | HBEM_ASM_ZERO)

/* LU precision */
#define HBEM_PREC_PLAIN 0      /* FP32 LU (complex64 cgesv semantics); HBEM_TUNE_LU_UPDATE = 2 moves its
                                  look-ahead bulk update to the tensor cores (TF32x3) */
#define HBEM_PREC_MIXED 1      /* BF16x3 tensor-core trailing updates; pair with hbem_refine */
#define HBEM_PREC_FP64 2       /* hbem_solve_batch only: complex128 LU of the widened FP32 system (zgesv semantics) */
#define HBEM_PREC_TF32X3 3     /* hbem_lu_factor only: the FP32 LU with its look-ahead bulk update on the tensor
                                  cores as TF32x3 split products (22 significand bits per operand: backward error
                                  a few times the FP32 LU's); for callers that refine with FP64 residuals, as
                                  hbem_solve_batch's plain path does when refinement is on */

/* Solve transposition */
#define HBEM_TRANS_N 0
#define HBEM_TRANS_T 1
#define HBEM_TRANS_C 2

/* hbem_session_query keys */
#define HBEM_Q_N_DOF 0
#define HBEM_Q_N_TRIANGLES 1
#define HBEM_Q_N_PAIRS 2
#define HBEM_Q_PAIRS_COINCIDENT 3
#define HBEM_Q_PAIRS_EDGE 4
#define HBEM_Q_PAIRS_VERTEX 5
#define HBEM_Q_IMAGE_PAIRS 6
#define HBEM_Q_UNIQUE_TRIPLETS 7
#define HBEM_Q_SYMMETRY 8
#define HBEM_Q_KERNEL_LAUNCHES 9   /* cumulative launches of this library's kernels on the session */
#define HBEM_Q_REGULAR_EVALS 10    /* kernel evaluations per frequency, regular part */
#define HBEM_Q_DUFFY_EVALS 11      /* kernel evaluations per frequency, Duffy part */
#define HBEM_Q_APERTURE_TRIANGLES 12  /* m: aperture triangles of the coupled baffle (0 when unset) */
#define HBEM_Q_NEAR_PAIRS 13       /* near, non-touching image pairs of the near-field option (0 when off) */

typedef struct hbem_session hbem_session;

/* Library version (major*10000 + minor*100 + patch). */
int hbem_version(void);

/* Copy the calling thread's last error message into buf (always NUL-terminated).
   Returns the message length. */
int hbem_last_error(char *buf, size_t len);

/* Number of kernel launches this library issued in the calling process. */
long long hbem_launch_count(void);

/*
 * Process-wide tuning knobs, read at launch time (so a CUDA graph captured
 * after a change keeps the variant it captured).  0 restores the built-in
 * choice.  Used by the autotuner of batched sweeps; no counterpart in the
 * reference.
 *   HBEM_TUNE_ASM_MINBLOCKS: resident CTAs per SM of the pair-assembly kernel
 *                            (2: 128 registers, 3: 80 registers)
 *   HBEM_TUNE_LU_PANEL:      inner sub-panel width of the LU (16: always;
 *                            32: wherever an 8-CTA cluster holds the
 *                            sub-panel; 0: the whole 64-column block where
 *                            one CTA holds it, else 32 where one CTA holds
 *                            it, else 16 where one CTA holds it, else 32 in
 *                            a cluster; 64: as 0, but the whole block also
 *                            in an 8-CTA cluster where that holds it)
 *   HBEM_TUNE_LU_SOLVE:      triangular solves (1: one CTA per right-hand
 *                            side, 2: blocked multi-CTA steps, 3: wavefront,
 *                            one CTA per 32-row block; 0: one CTA per
 *                            right-hand side for n <= 128, else wavefront)
 *   HBEM_TUNE_ASM_PAIRS:     regular assembly (0: unordered pairs, both
 *                            orders from one kernel evaluation; 1: ordered
 *                            pairs, two wavenumbers per evaluation)
 *   HBEM_TUNE_DUFFY:         singular corrections (1: one wavenumber per
 *                            warp, 2: two wavenumbers per warp)
 *   HBEM_TUNE_LU_LOOKAHEAD:  LU schedule (0: look-ahead, the block after
 *                            the panel is updated first and the rest of the
 *                            trailing update overlaps the next panel on a
 *                            second stream; 1: one stream)
 *   HBEM_TUNE_LU_RESERVE:    SMs the look-ahead's persistent tensor-core
 *                            update leaves to the factorisation chain
 *                            (v >= 1: v - 1 SMs, at most half; 0: built-in,
 *                            none)
 *   HBEM_TUNE_WAVE_SPIN:     polls (of >= 32 ns) a wavefront-solve warp waits
 *                            for an earlier block before it gives up (0: the
 *                            built-in 2^22); a wait that runs out makes the
 *                            launch abort, writes NaN into the unfinished x
 *                            and is reported by hbem_solve_status and the
 *                            synchronising entry points as HBEM_ERR_STATE
 *   HBEM_TUNE_LU_UPDATE:     the K = 64 trailing update of the FP32 LU
 *                            beside the factorisation chain (0: built-in,
 *                            CUDA cores for HBEM_PREC_PLAIN and tensor cores
 *                            for HBEM_PREC_TF32X3; 1: CUDA cores, exact FP32
 *                            products, for both; 2: tensor cores, TF32x3
 *                            split products, for both)
 *   HBEM_TUNE_LU_BLOCK:      column block of the mixed (BF16x3) LU and the K
 *                            of its tensor-core update (64 or 128; 0: the
 *                            built-in 128 for n > 16000, else 64); for the
 *                            FP32 LU's TF32x3 bulk, the K of one tensor-core
 *                            pass over a 64-column block (32: two passes, 64:
 *                            one; 0: the built-in 32 for n < 12000, else 64)
 *   HBEM_TUNE_LU_PANEL_KERNEL: sub-panels with their rows in shared memory
 *                            (0, built-in) or, where one row per thread fits,
 *                            in registers (1: 64 columns up to 384 rows, 32
 *                            up to 768, 16 up to 1024); the factors are the
 *                            same bits
 */
#define HBEM_TUNE_ASM_MINBLOCKS 0
#define HBEM_TUNE_LU_PANEL 1
#define HBEM_TUNE_LU_SOLVE 2
#define HBEM_TUNE_ASM_PAIRS 3
#define HBEM_TUNE_DUFFY 4
#define HBEM_TUNE_LU_LOOKAHEAD 5
#define HBEM_TUNE_LU_RESERVE 6
#define HBEM_TUNE_WAVE_SPIN 7
#define HBEM_TUNE_LU_UPDATE 8
#define HBEM_TUNE_LU_BLOCK 9
#define HBEM_TUNE_LU_PANEL_KERNEL 10
#define HBEM_TUNE_COUNT 11
int hbem_set_tuning(int key, int value);
int hbem_get_tuning(int key);

/*
 * Create a session on `device` from host geometry buffers.
 * Replaces: MetalNativeStandardSession.create_session
 *   (hornlab_metal_bem/metal/native.py:252-377) and the helper's
 *   ResidentMetalContext set-up (main.swift:5370-5507: P1 incidence, Duffy
 *   pair list, reduction plan, rules, geometry upload).
 * Inputs (host): vertices (3, n_vertices) f32; triangles (3, n_triangles) i32;
 *   p1_local2global (n_triangles, 3) i32 with values < n_dof; tags (n_triangles,);
 *   areas (n_triangles,) f32; normals (3, n_triangles) f32;
 *   sym_code 0 none, 1 yz, 2 xz, 3 yz+xz, 4 xy (main.swift:703-717).
 */
int hbem_session_create(const float *vertices_3xv, int n_vertices,
                        const int *triangles_3xt, int n_triangles,
                        const int *p1_local2global_tx3, int n_dof,
                        const int *tags, const float *areas, const float *normals_3xt,
                        int sym_code, int device, hbem_session **out);

/*
 * Near-field subdivision of the regular quadrature: for every pair of (image)
 * triangles that share no vertex and whose centroids are closer than
 * threshold x the longer of their longest edges, the assembly adds (the
 * 6-point rule on each of the 4^level sub-triangles of both - the 6 x 6 rule)
 * to A and the right-hand sides, with the Robin coupling, on every following
 * hbem_assemble / hbem_assemble_multi / hbem_solve_batch call that includes
 * HBEM_ASM_DUFFY.  level 0 turns it off; level 1 or 2; threshold > 0 (the
 * reference's default 1.5).  The pair count is HBEM_Q_NEAR_PAIRS.
 * Replaces: HORNLAB_METAL_BEM_NATIVE_NEAR_QUADRATURE = "<level>[:<threshold>]"
 *   (main.swift:5024-5054 parsing, 2471-2556 pair list, 2840-2912 subdivided
 *   blocks, 3072-3202 correction).  The FP64 path and the shape gradients do
 *   not include it.
 */
int hbem_session_set_near_quadrature(hbem_session *s, int level, double threshold);

/* Release a session and its device memory. */
int hbem_session_destroy(hbem_session *s);

/* Read one HBEM_Q_* property. */
int hbem_session_query(const hbem_session *s, int key, long long *value);

/*
 * Assemble A (P1 x P1 Galerkin, DLP - 1/2 mass, image method, Robin) and the
 * right-hand side b = SLP q for `n_freq` wavenumbers in one launch set.
 * Replaces: assemble_standard_neumann[_batch] ops
 *   (main.swift:3993-4133 pair kernel, 3698-3736 RHS kernel, 4246-4431 Duffy
 *   kernel, 6498-6561 CPU delta reduction).
 * k_re/k_im: host (n_freq,).  q_re/q_im: device (n_freq, n_triangles), row
 * stride q_stride.  beta_re/beta_im: device (n_triangles,) Robin admittance or
 * NULL.  A: device, frequency f at A + f*a_stride, row-major with lda.
 * b: device, frequency f at b + f*b_stride.
 */
int hbem_assemble(hbem_session *s, int n_freq, const float *k_re, const float *k_im,
                  const float *q_re, const float *q_im, long long q_stride,
                  const float *beta_re, const float *beta_im,
                  float *a_re, float *a_im, long long lda, long long a_stride,
                  float *b_re, float *b_im, long long b_stride,
                  int flags, void *stream);

/*
 * hbem_assemble for n_src right-hand sides (velocity sources) at once: one
 * pass assembles A (shared) and b_s = SLP q_s for every source s (1 .. 8),
 * the kernel samples shared by all of them.  Source s reads q at
 * q + s * q_src_stride (then frequency f at + f * q_stride) and writes b at
 * b + s * b_src_stride (+ f * b_stride).
 * Replaces: the reference's extra-source right-hand-side dispatches and their
 *   Duffy deltas (main.swift:6348-6368, 6467-6496), which evaluate the kernel
 *   once per source.
 */
int hbem_assemble_multi(hbem_session *s, int n_freq, const float *k_re, const float *k_im, int n_src,
                        const float *q_re, const float *q_im, long long q_stride, long long q_src_stride,
                        const float *beta_re, const float *beta_im,
                        float *a_re, float *a_im, long long lda, long long a_stride,
                        float *b_re, float *b_im, long long b_stride, long long b_src_stride,
                        int flags, void *stream);

/*
 * Batched in-place complex LU with partial pivoting (LAPACK getrf semantics:
 * unit-lower L and U overwrite A; piv[i] = 0-based row swapped with row i).
 * Replaces: cgesv_/cgetrf_ in solveDenseAccelerateCgesvMulti
 *   (main.swift:7834-7941, 8015-8020).
 * info: device int per matrix; 0 or the 1-based index of the first zero pivot.
 * precision: HBEM_PREC_PLAIN, HBEM_PREC_TF32X3 or HBEM_PREC_MIXED.
 * Returns HBEM_OK even when a pivot is zero (read info).  Does not
 * synchronise `stream`: a timed-out barrier wait of the tensor-core updates
 * (mixed precision, or the FP32 LU's TF32x3 bulk) is reported as
 * HBEM_ERR_STATE by hbem_solve_status, hbem_refine or hbem_solve_batch.
 */
int hbem_lu_factor(int n, int batch, float *a_re, float *a_im, long long lda, long long a_stride,
                   int *piv, long long piv_stride, int *info, int precision, void *stream);

/*
 * Solve op(A) X = B with the factors of hbem_lu_factor; B (n, nrhs) row-major
 * with leading dimension ldb, overwritten by X.  trans = HBEM_TRANS_N/T/C.
 * Replaces: cgetrs_ / the back-substitution inside cgesv_.
 */
int hbem_lu_solve(int n, int nrhs, int batch, const float *lu_re, const float *lu_im, long long lda,
                  long long a_stride, const int *piv, long long piv_stride,
                  float *b_re, float *b_im, long long ldb, long long b_stride, int trans, void *stream);

/*
 * Synchronise `stream` and report the device-side status of the asynchronous
 * solves issued before it: HBEM_ERR_STATE when a wavefront triangular-solve
 * wait timed out since the last report (that solve's unfinished x is NaN), or
 * the tensor-core update of a factorisation did,
 * else HBEM_OK.  Clears the status.  hbem_refine, hbem_lu_rcond and
 * hbem_solve_batch report it themselves.  No counterpart in the reference,
 * whose LAPACK solves are synchronous.
 */
int hbem_solve_status(void *stream);

/*
 * FP64-residual iterative refinement of X for A X = B (nrhs = 1 per matrix):
 * r = b - A x in FP64 from the ORIGINAL matrix, d = LU \ r, x += d, until
 * ||r||_2 / ||b||_2 <= tol, max_iter passes, or a pass that no longer lowers
 * the residual (as the reference stops).  The LU factors are read with A's
 * leading dimension lda (lu_stride >= lda * n).  iters/resid: device per
 * matrix, either may be NULL.
 * Replaces: refineDenseSolveSolution (main.swift:6964-7070).
 */
int hbem_refine(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                const float *lu_re, const float *lu_im, long long lu_stride,
                const int *piv, long long piv_stride,
                const float *b_re, const float *b_im, long long b_stride,
                float *x_re, float *x_im, long long x_stride,
                double tol, int max_iter, int *iters, double *resid, void *stream);

/*
 * hbem_refine without host synchronisation: same arguments, same stopping
 * rule, applied on the device.  All max_iter passes are issued; a matrix that
 * has stopped skips the rest of them (residual, wavefront solve blocks,
 * update).  The call can be captured in a CUDA graph (its scratch is a
 * stream-ordered allocation).  A timed-out wait of its triangular solves is
 * reported by hbem_solve_status.  No counterpart in the reference, whose
 * refinement runs on the host after a synchronous LAPACK solve.
 */
int hbem_refine_async(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                      const float *lu_re, const float *lu_im, long long lu_stride,
                      const int *piv, long long piv_stride,
                      const float *b_re, const float *b_im, long long b_stride,
                      float *x_re, float *x_im, long long x_stride,
                      double tol, int max_iter, int *iters, double *resid, void *stream);

/*
 * CHIEF least squares (reference assembleChiefRows + solveDenseLeastSquaresZgels,
 * main.swift:1897-2036, 7186-7409): for each of n_freq assembled systems
 * A x = b (FP32, as hbem_assemble leaves them, n_src right-hand sides) and m
 * interior points, the collocation rows C p = d of the vanishing exterior
 * representation (D, G at the real wavenumber, images, the Robin fold
 * -(int G) (i k beta) / 3 per P1 column with the complex one; d = sum (int G) g)
 * are built in FP64 and  min || [A; s C] p - [b; s d] ||_2,  s = weight *
 * ||A||_inf / ||C||_inf, is solved in complex128 by Householder QR; x =
 * (float) p.  q (device, (n_src, n_freq, T)): the driving Neumann data g;
 * beta (device, (T,)) or NULL; k_re/k_im host (k_im may be NULL);
 * chief_3xm host (3, m) float.  resid (device (n_src, n_freq), optional):
 * ||s (C p - d)||_2 / ||b||_2 (the reference's chief_residual_rel); scale_out
 * (device (n_freq,), optional): s.  Asynchronous on `stream`.
 */
int hbem_chief_lstsq(hbem_session *s, int n_freq, int n_src, const float *k_re, const float *k_im,
                     const float *q_re, const float *q_im, long long q_stride, long long q_src_stride,
                     const float *beta_re, const float *beta_im,
                     const float *a_re, const float *a_im, long long lda, long long a_stride,
                     const float *b_re, const float *b_im, long long b_stride, long long b_src_stride,
                     const float *chief_3xm, int m, double weight,
                     float *x_re, float *x_im, long long x_stride, long long x_src_stride,
                     double *resid, double *scale_out, void *stream);

/*
 * 1-norm condition estimate, as LAPACK cgecon (norm '1') on the factors.
 * hbem_matrix_norm1: anorm[f] = ||A_f||_1 = max_j sum_i |a_ij| (clange '1'),
 *   device float (batch,), of the matrix BEFORE factorisation.
 * hbem_lu_rcond: rcond[f] = 1 / (anorm[f] * est ||(L U)^-1||_1), device double
 *   (batch,), by Hager's method in Higham's formulation (CLACN2) with solves
 *   by L U and (L U)^H; 0 when the estimate or the norm is 0.
 * Replaces: matrixOneNorm / estimateReciprocalCondition (main.swift:463-503,
 *   called per case at 7886 and 7898).
 * Both are asynchronous on `stream` (no host synchronisation: the estimate
 * runs a fixed six rounds, matrices that finish earlier drop out on the
 * device), so the estimate can run on a second stream beside the solves; a
 * timed-out triangular-solve wait inside it is reported by hbem_solve_status.
 */
int hbem_matrix_norm1(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                      float *anorm, void *stream);
int hbem_lu_rcond(int n, int batch, const float *lu_re, const float *lu_im, long long lda, long long a_stride,
                  const float *anorm, double *rcond, void *stream);

/*
 * hbem_refine without any device allocation: same arguments, same results.
 * No counterpart in the reference, which allocates nothing on a device.
 * For callers that may not allocate device memory, such as a process whose
 * device memory is held by another caching allocator (a stream-ordered
 * allocation inside hbem_refine can then fail), or a loop that must never
 * enter an allocator.  Its scratch is one fixed device array of 12 MiB per
 * device, in this library's module.  Limits: batch <= 256 and
 * batch * x_stride <= 524288 complex elements; larger calls return
 * HBEM_ERR_ARG.  The first call on each device looks the array up (and may
 * load the module there), so make it before any stream capture.  Every call
 * shares the array, which keeps the last call's contents: calls on different
 * streams or threads that overlap in time race and give wrong results;
 * serialise them.
 */
int hbem_refine_noalloc(int n, int batch, const float *a_re, const float *a_im, long long lda, long long a_stride,
                        const float *lu_re, const float *lu_im, long long lu_stride,
                        const int *piv, long long piv_stride,
                        const float *b_re, const float *b_im, long long b_stride,
                        float *x_re, float *x_im, long long x_stride,
                        double tol, int max_iter, int *iters, double *resid, void *stream);

/*
 * Exterior field p(x_o) = sum_tri sum_q w [dG/dn_y p(y_q) - G q_tri] (+ images)
 * for n_freq cases at once.  Replaces: evaluate_field_regular / evaluateExterior
 *   (main.swift:4135-4203, 8312-8424; Python forces the GPU field,
 *   hornlab_metal_bem/sweep.py:114-115).
 * p: device (n_freq, n_dof) with stride p_stride; q: device (n_freq, n_triangles).
 * obs: device (3, n_obs).  out: device (n_freq, n_obs) with stride out_stride.
 */
int hbem_field(hbem_session *s, int n_freq, const float *k_re,
               const float *p_re, const float *p_im, long long p_stride,
               const float *q_re, const float *q_im, long long q_stride,
               const float *obs_3xn, int n_obs,
               float *out_re, float *out_im, long long out_stride, void *stream);

/*
 * Area-weighted average of the P1 surface pressure over the faces of each tag,
 * FP64 sums.  out: device (n_freq, n_tags, 2) double (re, im).
 * Replaces: averageSurfacePressureForTag / nativePressureReductionPayload
 *   (main.swift:807-871).
 */
int hbem_reduce_tag_avg(hbem_session *s, int n_freq, const float *p_re, const float *p_im, long long p_stride,
                        const int *tags_host, int n_tags, double *out, void *stream);
/* hbem_reduce_tag_avg with the tag list in device memory (n_tags ints): no
 * host copy or allocation, so it can be captured in a CUDA graph. */
int hbem_reduce_tag_avg_device(hbem_session *s, int n_freq, const float *p_re, const float *p_im, long long p_stride,
                               const int *tags_device, int n_tags, double *out, void *stream);

/*
 * One-call batched sweep over host buffers: host->device copies, assembly,
 * LU, solve, optional refinement, field and tag reductions, device->host
 * copies.  Replaces: MetalNativeStandardSession.
 *   assemble_solve_evaluate_standard_neumann_batch
 *   (hornlab_metal_bem/metal/native.py:737-1203; helper op
 *    main.swift:8869-9878).
 * Host inputs: k_re, k_im (n_freq,); q_re, q_im (n_freq, n_triangles);
 *   obs (3, n_obs); tags (n_tags,).
 * Host outputs: field (n_freq, n_obs) planar; tag_avg (n_freq, n_tags, 2)
 *   double; surface (n_freq, n_dof) planar or NULL; info (n_freq,);
 *   refine_iters (n_freq,) or NULL; refine_resid (n_freq,) or NULL;
 *   rcond (n_freq,) or NULL: 1-norm reciprocal condition estimate of each
 *   matrix (as cgecon; NULL skips the estimate);
 *   timings_ms (4,) = assembly, solve, field, total (device event times) or NULL.
 * precision: HBEM_PREC_PLAIN, HBEM_PREC_MIXED (with refinement) or
 *   HBEM_PREC_FP64 (dense_solve_dtype "float64": the FP32-assembled system
 *   widened to complex128, factored and solved in FP64, the solution narrowed
 *   to complex64 for the field; rcond from the factors narrowed to FP32).
 */
int hbem_solve_batch(hbem_session *s, int n_freq, const float *k_re, const float *k_im,
                     const float *q_re, const float *q_im,
                     const float *obs_3xn, int n_obs,
                     const int *tags, int n_tags,
                     int precision, double refine_tol, int refine_max_iter,
                     float *field_re, float *field_im, double *tag_avg,
                     float *surface_re, float *surface_im,
                     int *info, int *refine_iters, double *refine_resid, double *rcond,
                     float *timings_ms, void *stream);

/*
 * hbem_solve_batch for n_src velocity sources (1 .. 8) sharing each
 * frequency's matrix: one assembly pass (hbem_assemble_multi), one LU per
 * frequency, one solve (and refinement) per source.  Host arrays are
 * source-major: q (n_src, n_freq, n_triangles); field (n_src, n_freq, n_obs);
 * tag_avg (n_src, n_freq, n_tags, 2); surface (n_src, n_freq, n_dof);
 * refine_iters, refine_resid (n_src, n_freq); info and rcond (n_freq,) as the
 * matrix is shared.  n_src = 1 is hbem_solve_batch.
 * Replaces: the multi-RHS batch op (extra_neumann_dp0 of
 *   assemble_solve_evaluate_standard_neumann_batch,
 *   hornlab_metal_bem/metal/native.py:760-779; cgesv with nrhs = sources,
 *   main.swift:7887).
 */
int hbem_solve_batch_multi(hbem_session *s, int n_freq, int n_src, const float *k_re, const float *k_im,
                           const float *q_re, const float *q_im,
                           const float *obs_3xn, int n_obs,
                           const int *tags, int n_tags,
                           int precision, double refine_tol, int refine_max_iter,
                           float *field_re, float *field_im, double *tag_avg,
                           float *surface_re, float *surface_im,
                           int *info, int *refine_iters, double *refine_resid, double *rcond,
                           float *timings_ms, void *stream);

/*
 * Coupled infinite baffle (interior BIE + Rayleigh half-space through the
 * aperture at z = 0).  Replaces: buildApertureGeometry / buildCoupledIBCoupling
 * / solveCoupledIBDenseMultiSchur / evaluateCoupledIBRayleighReference
 * (main.swift:915-964, 1295-1385, 7597-7789, 1397-1444).
 *
 * hbem_session_set_aperture: select the aperture faces (physical tag); m is
 *   then readable with HBEM_Q_APERTURE_TRIANGLES.
 * hbem_aperture_assemble: S_ia (n_freq, n, m) = P1-test x DP0-aperture-trial
 *   single layer at k (images, 2^planes row weight, Duffy deltas), and
 *   S_aa (n_freq, m, m) = aperture-averaged single layer at the real field
 *   wavenumber kf (Duffy deltas of unmirrored test triangles), both device.
 * hbem_coupled_ib_schur: A <- A - S_ia (2 S_aa)^-1 P_avg in place (P_avg: 1/3
 *   on the three dofs of each aperture triangle); writes M = (2 S_aa)^-1
 *   (n_freq, m, m).  S_aa is overwritten by its LU factors.
 * hbem_coupled_ib_field: q_a = M (P_avg p) (n_freq, m) and the Rayleigh field
 *   -2 sum G(y, x') q_a with x' = (x, y, max(z, 0)) for z >= -1e-5, 0 below.
 *   With minv_re = minv_im = NULL, q_a is an input (p is not read).
 * hbem_coupled_ib_augment: the augmented twin (main.swift:7504-7595) for
 *   large apertures: K (n_freq, N, N), N = m + n, rows beta [-2 alpha S_aa |
 *   P_avg] then [-alpha S_ia | A], with per-frequency block scales alpha =
 *   max|A| / max|S_ia| and beta = max|A| / (2 alpha max|S_aa|) written to
 *   alpha (device, n_freq).  Call it after hbem_assemble has written the A
 *   block in place (a = K + m * ldk + m, lda = ldk); it fills every other
 *   entry.  K [q~; p] = [0; b] gives the Schur solution p and q_a = alpha q~.
 */
int hbem_session_set_aperture(hbem_session *s, int aperture_tag);
int hbem_aperture_assemble(hbem_session *s, int n_freq, const float *k_re, const float *k_im, const float *kf_re,
                           float *sia_re, float *sia_im, float *saa_re, float *saa_im, void *stream);
int hbem_coupled_ib_schur(hbem_session *s, int n_freq, float *a_re, float *a_im, const float *sia_re,
                          const float *sia_im, float *saa_re, float *saa_im, float *minv_re, float *minv_im,
                          int *info, void *stream);
int hbem_coupled_ib_field(hbem_session *s, int n_freq, const float *kf_re, const float *p_re, const float *p_im,
                          const float *minv_re, const float *minv_im, const float *obs_3xn, int n_obs,
                          float *qa_re, float *qa_im, float *out_re, float *out_im, void *stream);
int hbem_coupled_ib_augment(hbem_session *s, int n_freq, const float *sia_re, const float *sia_im,
                            const float *saa_re, const float *saa_im, float *k_re, float *k_im, long long ldk,
                            long long k_stride, float *alpha, void *stream);

/*
 * Shape gradients (adjoint of the forward map vertices -> A, b -> p -> field),
 * sessions without symmetry planes, real wavenumbers.  With g (n_freq, n_obs)
 * = dL/dRe F + i dL/dIm F of a real objective L of the field F:
 *   hbem_field_adjoint:    g_p = Fp^H g (n_freq, n_dof), F = Fp p + Fq q;
 *   then lambda = A^-H g_p with hbem_lu_solve(..., HBEM_TRANS_C) on the
 *   forward's factors;
 *   hbem_field_backward:   grad += d/dX Re g^H F at fixed p;
 *   hbem_assemble_backward: grad += -Re lambda^H (dA/dX) p + Re lambda^H (db/dX),
 *   recomputing the forward's quadrature (regular 6x6 on far pairs, the Duffy
 *   rules on touching pairs, the mass term) pair by pair.
 * grad_3xv: device float64 (3, n_vertices), accumulated (zero it first).
 * No dA/dX is stored.  hbem_session_set_vertices moves the vertices of a
 * session in place (same topology), with areas and unit normals as at
 * creation.  No counterpart in the reference, which has no adjoint; the
 * forward they differentiate is main.swift:3443-3480, 4090-4120, 4246-4431,
 * 4135-4203.
 */
int hbem_session_set_vertices(hbem_session *s, const float *vertices_3xv, const float *areas,
                              const float *normals_3xt);
int hbem_field_adjoint(hbem_session *s, int n_freq, const float *k_re, const float *obs_3xn, int n_obs,
                       const float *g_re, const float *g_im, long long g_stride, float *gp_re, float *gp_im,
                       long long gp_stride, void *stream);
int hbem_field_backward(hbem_session *s, int n_freq, const float *k_re, const float *obs_3xn, int n_obs,
                        const float *g_re, const float *g_im, long long g_stride, const float *p_re,
                        const float *p_im, long long p_stride, const float *q_re, const float *q_im,
                        long long q_stride, double *grad_3xv, void *stream);
int hbem_assemble_backward(hbem_session *s, int n_freq, const float *k_re, const float *k_im,
                           const float *lam_re, const float *lam_im, long long lam_stride,
                           const float *p_re, const float *p_im, long long p_stride,
                           const float *q_re, const float *q_im, long long q_stride,
                           double *grad_3xv, void *stream);

/*
 * FP64 path: the corrected assembly, the exterior field and a complex128 LU in
 * double precision on the GPU.  Same discretisation as the FP32 entry points
 * (6-point rule on far pairs with images, row weight, mass and Robin terms,
 * the 4^4-point Duffy rules on touching pairs, built in double), evaluated in
 * double from the session's float32 geometry: the difference between an FP32
 * result and its FP64 twin is the FP32 arithmetic error, which every result
 * line states.  Replaces the reference's own FP64 checks: the assembly parity
 * gate (main.swift:8257-8307) and the float64 dense solve (zgesv on the
 * widened system, main.swift:7101-7185).
 *
 * hbem_assemble_f64: as hbem_assemble with double buffers (k on the host, q,
 *   beta, A, b on the device).
 * hbem_field_f64: as hbem_field with double p, q and output (obs stays float).
 * hbem_lu_factor_f64: batched in-place complex128 LU with partial pivoting
 *   (getrf semantics: first maximum of |re| + |im|; piv 0-based; info 0 or the
 *   1-based index of the first zero pivot), n <= 131072, batch <= 65535.
 * hbem_lu_solve_f64: op(A) X = B with those factors, HBEM_TRANS_N only;
 *   B (n, nrhs) row-major with leading dimension ldb; batch * nrhs <= 65535.
 */
int hbem_assemble_f64(hbem_session *s, int n_freq, const double *k_re, const double *k_im,
                      const double *q_re, const double *q_im, long long q_stride,
                      const double *beta_re, const double *beta_im,
                      double *a_re, double *a_im, long long lda, long long a_stride,
                      double *b_re, double *b_im, long long b_stride, int flags, void *stream);
int hbem_field_f64(hbem_session *s, int n_freq, const double *k_re,
                   const double *p_re, const double *p_im, long long p_stride,
                   const double *q_re, const double *q_im, long long q_stride,
                   const float *obs_3xn, int n_obs,
                   double *out_re, double *out_im, long long out_stride, void *stream);
int hbem_lu_factor_f64(int n, int batch, double *a_re, double *a_im, long long lda, long long a_stride,
                       int *piv, long long piv_stride, int *info, void *stream);
int hbem_lu_solve_f64(int n, int nrhs, int batch, const double *lu_re, const double *lu_im, long long lda,
                      long long a_stride, const int *piv, long long piv_stride,
                      double *b_re, double *b_im, long long ldb, long long b_stride, int trans, void *stream);
/*
 * The coupled infinite baffle on the FP64 path: hbem_aperture_assemble_f64
 * writes S_ia (n_freq, n, m) and S_aa (n_freq, m, m) as hbem_aperture_assemble
 * does (double buffers, k and kf on the host; zeroed first), and
 * hbem_coupled_ib_field_f64 the Rayleigh field -2 sum G(y, x') q_a from given
 * aperture data q_a (n_freq, m) (x' = (x, y, max(z, 0)) for z >= -1e-5, 0
 * below; n_obs <= 65535).  With hbem_assemble_f64 and hbem_lu_*_f64 they
 * solve the augmented system [[A, -S_ia], [P_avg, -2 S_aa]] [p; q_a] = [b; 0]
 * in FP64 (main.swift:7504-7595), the error reference of the coupled sweeps.
 */
int hbem_aperture_assemble_f64(hbem_session *s, int n_freq, const double *k_re, const double *k_im,
                               const double *kf_re, double *sia_re, double *sia_im, double *saa_re,
                               double *saa_im, void *stream);
int hbem_coupled_ib_field_f64(hbem_session *s, int n_freq, const double *kf_re, const double *qa_re,
                              const double *qa_im, const float *obs_3xn, int n_obs, double *out_re,
                              double *out_im, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* HBEM_H */
