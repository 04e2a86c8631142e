/*
 * unwrap_b200.h — C ABI of the B200 (sm_100a) DCT+IRLS L1 2-D phase unwrapper.
 *
 * Drop-in boundary for insardev's `irls_unwrap_2d`
 * (insardev/insardev/utils_unwrap2d.py:1082-1766).  All pointers are device
 * pointers unless stated; all calls are thread safe (every piece of mutable
 * state lives in the caller's workspace) and run on the caller's CUDA stream.
 * Calls that must read a device scalar to decide what to do next (bounding
 * box, IRLS convergence, component count) synchronise that stream.
 *
 * Return codes: 0 ok; negative = error (see UNW_E_*), message via
 * unw_last_error().  UNW_W_NUMERIC (>0) is the reference's "NaN/inf produced"
 * outcome (utils_unwrap2d.py:1659-1665): outputs are all-NaN / all-zero and a
 * caller mirroring the reference raises RuntimeWarning.
 */
#ifndef UNWRAP_B200_H
#define UNWRAP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define UNW_API __attribute__((visibility("default")))
#else
#define UNW_API
#endif

#define UNW_ABI_VERSION 2

enum {
    UNW_OK = 0,
    UNW_W_NUMERIC = 1,      /* non-finite solution on valid pixels: NaN output  */
    UNW_E_ARG = -1,         /* bad argument (null pointer, shape, pitch)        */
    UNW_E_WORKSPACE = -2,   /* workspace too small                              */
    UNW_E_CUDA = -3,        /* CUDA runtime error                               */
    UNW_E_UNSUPPORTED = -4, /* grid dimension beyond the transform limits       */
    UNW_E_OVERFLOW = -5     /* > 65535 kept components (uint16 labels)           */
};

/* Solver parameters: same names and meaning as the reference keywords
 * (utils_unwrap2d.py:1082-1083).  `flags` holds UNW_F_* bits. */
typedef struct unw_params {
    int32_t max_iter;       /* IRLS iterations (reference default 50)          */
    float tol;              /* IRLS relative-change tolerance (1e-3)           */
    int32_t cg_max_iter;    /* PCG iterations per IRLS step (20)               */
    float cg_tol;           /* absolute PCG residual-norm tolerance (1e-4)     */
    float epsilon;          /* L1 smoothing (1e-2)                             */
    int32_t conncomp_size;  /* minimum kept component size (30)                */
    int32_t flags;
    int32_t check_every;    /* IRLS iterations enqueued between host checks    */
} unw_params;

#define UNW_F_CONGRUENT 1   /* output phase + 2*pi*k instead of the smooth solution */
#define UNW_F_NO_GRAPH  2   /* launch kernels one by one instead of a CUDA graph    */
#define UNW_F_PROFILE   4   /* time every kernel launch with CUDA events (unw_stats.prof_*) */
#define UNW_F_FIXED_ITERS 8 /* run max_iter IRLS x cg_max_iter PCG iterations: the tol and
                               cg_tol stop tests are off, the numerical breaks stay (for
                               comparing throughput at identical work)                      */
#define UNW_F_MIXED 16      /* mixed-precision form: for grids of at most 1024 rows the column
                               DCT / scaling / inverse DCT of the preconditioner may run as
                               split-precision bf16 products on the tensor cores, where an
                               autotuner (timing both on the first call for a shape) finds
                               them faster than the float32 FFT pass; unw_stats reports the
                               choice and the float64 residual of the final system         */
#define UNW_F_COL_TC 32     /* with UNW_F_MIXED: always the tensor-core column pass (else
                               UNW_E_UNSUPPORTED), no autotuning                             */
#define UNW_F_COL_FFT 64    /* with UNW_F_MIXED: always the float32 FFT column pass          */
#define UNW_F_COL_NO_TMA 128 /* power-of-two column pass at H = 2048 / 4096 with plain
                               loads and stores, never TMA copies of the column slab (the
                               same arithmetic and bits); by default an autotuner times both
                               per shape on the first call and keeps the faster               */
#define UNW_F_COL_TMA 256    /* always the TMA-staged column pass where it applies           */
#define UNW_F_MV_NO_TMA 512  /* matvec with plain loads instead of TMA-staged halo tiles (the
                               same arithmetic and bits; for comparison)                     */

/* Kernel families timed under UNW_F_PROFILE (index into unw_stats.prof_*). */
enum {
    UNW_PROF_BBOX = 0, UNW_PROF_SETUP, UNW_PROF_ROW_RHO, UNW_PROF_COL, UNW_PROF_ROW_INV,
    UNW_PROF_MATVEC, UNW_PROF_ROW_UPD, UNW_PROF_ROW_R0, UNW_PROF_HEAD, UNW_PROF_ELEM,
    UNW_PROF_POST, UNW_PROF_N
};

/* Per-solve statistics (the reference prints these under debug=True). */
typedef struct unw_stats {
    int32_t irls_iters;     /* IRLS iterations run                              */
    int32_t cg_iters_total; /* PCG iterations summed over IRLS iterations        */
    int32_t cg_iters_last;  /* PCG iterations of the last IRLS iteration         */
    int32_t n_components;   /* kept components (labels 1..n)                    */
    int32_t n_labels;       /* 4-connected components before the size filter    */
    int32_t status;         /* UNW_S_* bits                                     */
    int32_t bbox[4];        /* r0, r1, c0, c1 of the valid bounding box          */
    double rel_change;      /* last IRLS relative change                         */
    double best_residual;   /* best sum of squared gradient residuals            */
    double k_median;        /* median 2-pi cycle shift applied                   */
    int32_t cg_iters[64];   /* PCG iterations of the first 64 IRLS iterations    */
    float prof_ms[16];      /* summed kernel time per family (UNW_F_PROFILE)     */
    int32_t prof_launches[16]; /* launches per family (UNW_F_PROFILE)            */
    int32_t col_path;       /* column pass used: 0 float32 FFT, 1 tensor cores  */
    float tune_ms[2];       /* autotuner: FFT / tensor-core column pass, ms per
                               launch (UNW_F_MIXED, 0 when not timed)          */
    int32_t col_tma;        /* 1: the power-of-two column pass moved its slab by TMA */
    double resid_rel;       /* ||b - A u|| / ||b|| of the final weighted system
                               in float64 (UNW_F_MIXED; 0 otherwise): the error
                               of the result against an exact solve of the last
                               IRLS system                                     */
} unw_stats;

#define UNW_S_DCT_INIT_NONFINITE 1   /* DCT init produced NaN/inf (zero-filled)  */
#define UNW_S_REVERTED           2   /* reverted to the best iterate             */
#define UNW_S_NONFINITE_OUT      4   /* non-finite output: NaN result            */
#define UNW_S_ALL_NAN            8   /* input all NaN                            */
#define UNW_S_TC_TIMEOUT        16   /* a TMA-staged column pass (tensor-core or
                                        power-of-two) gave up waiting on its copies
                                        (bounded wait); result not valid        */

/* One grid of a batched solve (unw_solve_batch).  Pitches are in elements. */
typedef struct unw_grid {
    const float* phase;     int64_t phase_pitch;
    const float* weight;    int64_t weight_pitch;   /* NULL = uniform weights   */
    int64_t H, W;
    float* out_u;           int64_t out_u_pitch;
    uint16_t* out_cc;       int64_t out_cc_pitch;
} unw_grid;

UNW_API int unw_abi_version(void);

/* Thread-local text of the last error on this thread. */
UNW_API const char* unw_last_error(void);

/* Device workspace bytes needed to solve one H x W grid. */
UNW_API size_t unw_workspace_bytes(int64_t H, int64_t W);

/* Device workspace bytes for a batch of n grids solved together. */
UNW_API size_t unw_batch_workspace_bytes(int32_t n, const int64_t* H, const int64_t* W);

/*
 * Unwrap one grid.  Replaces utils_unwrap2d.py:1082 irls_unwrap_2d.
 *   phase  [H][phase_pitch]  float32, NaN = invalid (device)
 *   weight [H][weight_pitch] float32 or NULL (device)
 *   out_u  [H][out_u_pitch]  float32 (device): unwrapped phase, NaN where invalid
 *   out_cc [H][out_cc_pitch] uint16  (device): 0 invalid/small, 1 largest, ...
 *   stats  host pointer or NULL.
 */
UNW_API int unw_solve_f32(const float* phase, int64_t phase_pitch,
                  const float* weight, int64_t weight_pitch,
                  int64_t H, int64_t W, const unw_params* params,
                  float* out_u, int64_t out_u_pitch,
                  uint16_t* out_cc, int64_t out_cc_pitch,
                  void* workspace, size_t workspace_bytes,
                  unw_stats* stats, void* cuda_stream);

/*
 * Unwrap n independent grids of any sizes in one launch sequence: every kernel
 * covers all still-active grids, each grid stops on its own convergence test.
 * Replaces the per-pair loop of Stack_unwrap2d.py:102-130 (_irls_overlap_kernel)
 * and the per-task calls of Stack_unwrap2d.py:32-71.  stats: n entries or NULL.
 */
UNW_API int unw_solve_batch(int32_t n, const unw_grid* grids, const unw_params* params,
                    void* workspace, size_t workspace_bytes,
                    unw_stats* stats, void* cuda_stream);

/*
 * Operator entry points (one H x W grid, dense pitch = W, device pointers).
 * They expose single steps of the solver for verification.
 */

/* Wrapped gradients and edge weights, utils_unwrap2d.py:1228-1275.
 * Outputs gx, gy, wx, wy: [H][W] float32; valid: [H][W] uint8. */
UNW_API int unw_setup_gradients(const float* phase, const float* weight, int64_t H, int64_t W,
                        float* gx, float* gy, float* wx, float* wy, uint8_t* valid,
                        void* workspace, size_t workspace_bytes, void* cuda_stream);

/* Weighted-Laplacian matvec Ax = -div(w grad x), utils_unwrap2d.py:1367-1388. */
UNW_API int unw_apply_laplacian(const float* x, const float* wx, const float* wy,
                        int64_t H, int64_t W, float* Ax,
                        void* workspace, size_t workspace_bytes, void* cuda_stream);

/* DCT preconditioner z = IDCT2(-DCT2(r)/lambda), DC term zeroed,
 * utils_unwrap2d.py:1390-1403 (also the DCT initial solve :1478-1513). */
UNW_API int unw_apply_preconditioner(const float* r, int64_t H, int64_t W, float* z,
                             void* workspace, size_t workspace_bytes, void* cuda_stream);

/* The same operator in the mixed-precision form: col_path 1 runs the column
 * DCT / scaling / inverse DCT as split-precision bf16 products on the tensor
 * cores (H <= 1024 and W a multiple of 4, else UNW_E_UNSUPPORTED), 0 the float32
 * FFT pass, -1 lets the autotuner choose.  Returns the path used (0 or 1) or a
 * negative error code.  It has no counterpart in the reference (which has one
 * float32 DCT path, utils_unwrap2d.py:1316-1365). */
UNW_API int unw_apply_preconditioner_mixed(const float* r, int64_t H, int64_t W, float* z, int32_t col_path,
                                           void* workspace, size_t workspace_bytes, void* cuda_stream);

/*
 * Gradients through the unwrap (frozen-weight implicit adjoint).  It has no
 * counterpart in the reference, whose solve is not differentiable.
 *
 * The differentiated map is the unwrap with what the forward solution fixes
 * held constant: the valid mask, its 4-connected components, the median
 * 2-pi shift and the IRLS scale 1/sqrt(r^2 + eps^2) of every edge at u
 * (utils_unwrap2d.py:1560-1574).  What remains is differentiable: the wrapped
 * phase differences, the coherence edge weights, the weighted Poisson solve
 * A(wI) u* = b (utils_unwrap2d.py:1367-1388, :1576-1581) and the per-component
 * circular-mean alignment (utils_unwrap2d.py:1694-1716).  The call first
 * refines u to u* on that frozen system (one PCG solve from u, then float64
 * residual-refinement passes, each correction from the same PCG), then solves
 * the adjoint system with the same DCT-preconditioned PCG, then forms the
 * gradients in float64.
 *   phase, weight   the forward call's inputs (device, NaN = invalid)
 *   u               the forward call's unwrapped output (device)
 *   grad_u          dL/du (device; ignored where phase is NaN)
 *   params          epsilon as in the forward call; cg_max_iter caps each of
 *                   the two PCG solves; cg_tol is RELATIVE to the initial
 *                   residual norm of each solve (e.g. 1e-6)
 *   grad_phase      dL/dphase (device), 0 where phase is NaN
 *   grad_weight     dL/dweight (device) or NULL; needs weight
 *   stats           cg_iters[0] / [1]: first u* / adjoint PCG iterations,
 *                   cg_iters[2..4]: PCG iterations of the refinement passes,
 *                   rel_change: final relative residual of the adjoint solve,
 *                   resid_rel: float64 ||b - A u*|| / ||b|| of the final u*
 * Returns UNW_W_NUMERIC (gradients 0) when the refinement is not finite.
 */
UNW_API size_t unw_adjoint_workspace_bytes(int64_t H, int64_t W);
UNW_API int unw_adjoint_f32(const float* phase, int64_t phase_pitch,
                            const float* weight, int64_t weight_pitch,
                            int64_t H, int64_t W, const unw_params* params,
                            const float* u, int64_t u_pitch,
                            const float* grad_u, int64_t grad_u_pitch,
                            float* grad_phase, int64_t grad_phase_pitch,
                            float* grad_weight, int64_t grad_weight_pitch,
                            void* workspace, size_t workspace_bytes,
                            unw_stats* stats, void* cuda_stream);

/*
 * Batched form of unw_adjoint_f32: the adjoints of n grids (each with its own
 * forward output and dL/du) in one launch sequence per launch shape, every
 * kernel covering all grids of its group and each grid's PCG solves stopping on
 * their own tolerance.  Same arguments per grid as unw_adjoint_f32 (pitches in
 * elements); stats is an array of n (or NULL).  No reference counterpart (the
 * reference has no differentiable path); the autograd function of
 * core_b200.irls_unwrap_2d_diff uses it for (B, H, W) batches.  Returns
 * UNW_W_NUMERIC when the refinement of any grid is not finite (that grid's
 * gradients are 0).
 */
typedef struct unw_adj_grid {
    const float* phase;   int64_t phase_pitch;
    const float* weight;  int64_t weight_pitch;       /* may be NULL */
    int64_t H, W;
    const float* u;       int64_t u_pitch;            /* forward output */
    const float* grad_u;  int64_t grad_u_pitch;       /* dL/du */
    float* grad_phase;    int64_t grad_phase_pitch;
    float* grad_weight;   int64_t grad_weight_pitch;  /* may be NULL; needs weight */
} unw_adj_grid;

UNW_API size_t unw_adjoint_batch_workspace_bytes(int32_t n, const int64_t* H, const int64_t* W);
UNW_API int unw_adjoint_batch(int32_t n, const unw_adj_grid* grids, const unw_params* params,
                              void* workspace, size_t workspace_bytes, unw_stats* stats,
                              void* cuda_stream);

/*
 * Goldstein adaptive phase filter on one grid.  Replaces the GPU path of
 * insardev's filter, goldstein_pytorch (utils_goldstein.py:157-330, dispatched
 * from Batch.py:2023-2027): psize_y x psize_x patches at half-patch steps,
 * spectrum weighted by max(|F|, 1e-10)^alpha, alpha = 1 - taper-weighted mean
 * coherence, taper and overlap-add divided by the number of valid patches
 * (a patch is valid with at least int(psize_y * psize_x * threshold) non-NaN
 * pixels); NaN where the input is NaN or no valid patch covers the pixel.
 *   phase [H][phase_pitch] interleaved complex64 (device), corr [H][corr_pitch]
 *   float32 (device, NaN allowed), out [H][out_pitch] complex64 (device).
 * Patch sizes: powers of two in [4, 64] (UNW_E_UNSUPPORTED otherwise).
 */
UNW_API size_t unw_goldstein_workspace_bytes(int64_t H, int64_t W, int32_t psize_y, int32_t psize_x);
UNW_API int unw_goldstein_c64(const float* phase, int64_t phase_pitch, const float* corr, int64_t corr_pitch,
                              int64_t H, int64_t W, int32_t psize_y, int32_t psize_x, float threshold,
                              float* out, int64_t out_pitch, void* workspace, size_t workspace_bytes,
                              void* cuda_stream);

/*
 * Component linking: integer 2-pi offsets between separately unwrapped
 * components.  Replaces the geometry of find_component_connections_fast
 * (insardev/insardev/utils_unwrap2d.py:195-444) and the raster updates of
 * connect_components_ilp_fast (:886-1040), as driven by _link_2d
 * (Stack_unwrap2d.py:325-407); the reference's cv2 contours and shapely
 * measures become pixel-lattice geometry (boundary = border pixels, polygon =
 * their convex hull, distances between pixel centres).  The greedy choice of
 * connections and the integer program run on the host between the two calls.
 *
 * unw_link_pairs_f32: components from labels (uint16 IRLS labels, label
 * order; NULL = 4-connected components of the non-NaN pixels, size order),
 * kept when they have >= min_size pixels; then every candidate pair (each
 * component with its max_neighbors nearest by hull distance) with its closest
 * border pixels, whether the segment between them meets a third component's
 * hull, and np.nanmean of each side's values in a (2*(window/2)+1)^2 window.
 * Outputs go to host arrays; when comp_cap or pair_cap is too small the call
 * returns UNW_E_WORKSPACE with the needed counts in *n_comp / *n_pairs.
 * For the mask path comp_label holds the raster index of the component's
 * first pixel.  The workspace keeps the component raster for
 * unw_link_apply_f32, which writes phase + 2*pi*k[c] on component c, NaN on
 * labelled pixels of components below min_size, and phase elsewhere; call it
 * with the same workspace, shape and min_size.
 */
typedef struct unw_link_params {
    int32_t min_size;       /* the reference uses max(conncomp_size, 4)             */
    int32_t max_neighbors;  /* conncomp_linkcount (<= 256 unless >= components - 1) */
    int32_t window;         /* conncomp_linksize, 0..31                             */
    int32_t flags;          /* reserved, 0                                          */
} unw_link_params;

#define UNW_LINK_C_LINE 1   /* component in one row or column: no contour polygon */

typedef struct unw_link_pair {
    int32_t comp_i, comp_j;       /* component indices, comp_i < comp_j             */
    int32_t yi, xi, yj, xj;       /* closest border pixels (ties: smallest yi,xi,yj,xj) */
    int64_t d2;                   /* their squared distance                          */
    int32_t blocked;              /* the segment meets a third component's hull      */
    int32_t n_i, n_j;             /* window pixels of each component                 */
    int32_t nf_i, nf_j;           /* ... of which finite                             */
    float mean_i, mean_j;         /* np.nanmean of the window values (NaN if none)   */
    int32_t pad;
} unw_link_pair;

UNW_API size_t unw_link_workspace_bytes(int64_t H, int64_t W, int32_t min_size);
UNW_API int unw_link_pairs_f32(const float* phase, int64_t phase_pitch,
                               const uint16_t* labels, int64_t label_pitch,
                               int64_t H, int64_t W, const unw_link_params* params,
                               int64_t* comp_label, int64_t* comp_size, int32_t* comp_flags,
                               int32_t comp_cap, int32_t* n_comp,
                               unw_link_pair* pairs, int32_t pair_cap, int32_t* n_pairs,
                               void* workspace, size_t workspace_bytes, void* cuda_stream);
UNW_API int unw_link_apply_f32(const float* phase, int64_t phase_pitch, int64_t H, int64_t W,
                               const int32_t* k, int32_t n_comp, float* out, int64_t out_pitch,
                               void* workspace, size_t workspace_bytes, int32_t min_size,
                               void* cuda_stream);

/*
 * Integer offsets for the linking connections (host code, no GPU): the program
 * connect_components_ilp_fast gives to CP-SAT (utils_unwrap2d.py:933-970),
 * minimise sum_e w[e] |s (k[ei[e]] - k[ej[e]]) - off[e]| with k[0] = 0,
 * k in [-100, 100], |s (k_i - k_j) - off| <= 200, s = +1 (sign >= 0, the
 * reference) or -1; among optimal assignments the least sum |k| (exact).
 * w[e] in [0, 2^31], off[e] in [-200, 200].  Writes k_out[0..n).
 */
UNW_API int unw_link_offsets(int32_t n, int32_t m, const int32_t* ei, const int32_t* ej, const int32_t* off,
                             const int64_t* w, int32_t sign, int32_t* k_out);

/*
 * Allocation-free variant of unw_apply_preconditioner.  It has no counterpart
 * in the reference.  It is for callers that cannot allocate device memory
 * where they need the operator: C or Fortran codes with no device allocator
 * of their own, and real-time loops that must not allocate after start-up.
 * Its scratch is one 16 MiB device array that the library holds on every GPU
 * that loads it, so the caller passes only r and z (dense, pitch W, device
 * pointers, 16-byte aligned, else UNW_E_ARG).  Limit: H * W <= 3932160 and
 * transform lengths <= 16384, otherwise UNW_E_UNSUPPORTED.  All calls on a
 * device share the array: calls that overlap on the GPU race (order them on
 * one stream).  The first call on a device looks up the array's address and
 * caches it for the life of the process; it is not valid after
 * cudaDeviceReset.
 */
UNW_API int unw_apply_preconditioner_noalloc(const float* r, int64_t H, int64_t W, float* z,
                                             void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* UNWRAP_B200_H */
