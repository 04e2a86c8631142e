// Host-side declarations of the kernel launchers (implemented in the .cu files).
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "unw_internal.cuh"

// Raises a kernel's dynamic shared-memory limit to the most one CTA can have on the
// current device (the opt-in maximum less the kernel's static shared memory), once per
// kernel and device.  Launches may then pass any dynamic size up to that.  Kernels whose
// launches use different dynamic sizes use this instead of setting the limit to each
// launch's size: with launches from several host threads (a batch's launch groups run
// concurrently) a smaller setting from one thread could land between another thread's
// setting and its launch, which then fails.
inline cudaError_t unw_smem_limit(const void* kfn) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({kfn, dev})) return cudaSuccess;
    cudaFuncAttributes a;
    int optin = 0;
    if ((e = cudaFuncGetAttributes(&a, kfn)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
    if (e == cudaSuccess) done[{kfn, dev}] = 1;
    return e;
}

struct UnwScalars {
    int max_iter;
    int cg_max_iter;
    float tol;
    float cg_tol;
    float eps2;
    int conncomp_size;
    float cg_rel;     // > 0: PCG tolerance relative to the initial residual norm (adjoint solves)
};

enum {
    UNW_K_STATE_INIT = 0,
    UNW_K_SETUP,
    UNW_K_MATVEC,
    UNW_K_HEAD,
    UNW_K_MEAN,
    UNW_K_INIT_RECENTRE,
    UNW_K_COPY_BEST,
    UNW_K_REL,
    UNW_K_LAP_APPLY,
    UNW_K_RESID
};

// records the thread-local error text returned by unw_last_error(); returns code
int unw_set_error(int code, const char* msg);

// solver kernels
cudaError_t unw_launch_tables(const FftPlanDev& f, const DctPlanDev& d, float* sv, int Ncos,
                              cudaStream_t s);
cudaError_t unw_launch_hspec(int T, int emax, const DctPlanDev& d, cudaStream_t s);
cudaError_t unw_launch_row_fwd(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                               const GridDev* gd, const int* starts, int n, int it, int cgk);
cudaError_t unw_launch_row_inv(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                               const GridDev* gd, const int* starts, int n);
cudaError_t unw_launch_col(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                           const GridDev* gd, const int* starts, int n);
cudaError_t unw_launch_simple(int which, int nblk, cudaStream_t s, const GridDev* gd,
                              const int* starts, int n, int it, UnwScalars sc);

// power-of-two register-FFT DCT passes (N = 256 .. 16384)
int unw_p2_col_nseq(int N);
cudaError_t unw_launch_rowf_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n, int it, int cgk);
cudaError_t unw_launch_rowi_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n);
cudaError_t unw_launch_col_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                              int n);

// Bluestein-on-register-FFT DCT passes for other lengths (M = power of two >= 2N - 1)
int unw_bl_col_nseq(int M);
cudaError_t unw_launch_rowf_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n, int it, int cgk);
cudaError_t unw_launch_rowi_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n);
cudaError_t unw_launch_col_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                              int n);

// tensor-core (tcgen05, split-precision bf16) column pass for grids of H <= UNW_TC_MAX_H rows
#define UNW_TC_MAX_H 1024
struct TcMaps {                       // four CUtensorMap (128 bytes each): C hi / lo, E hi / lo
    alignas(64) unsigned char c_hi[128];
    alignas(64) unsigned char c_lo[128];
    alignas(64) unsigned char e_hi[128];
    alignas(64) unsigned char e_lo[128];
};
size_t unw_tc_table_bytes(int H);     // workspace bytes of the split DCT matrices (0 if H > UNW_TC_MAX_H)
int unw_tc_ctas(int H, int W);        // CTAs of one grid's tensor-core column pass
cudaError_t unw_tc_prepare(int H, void* tab, TcMaps* maps, cudaStream_t s);
// per-grid tensor maps of the pass's float32 sources T and Y (p1), H x W with pitch P:
// two 128-byte CUtensorMap objects written to out2 (64-byte aligned host memory)
bool unw_tc_data_maps(const float* T, const float* Y, int H, int W, int P, void* out2);
cudaError_t unw_launch_col_tc(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                              const TcMaps* maps, const void* bmaps);

// bounding box of valid pixels on the caller's full grid
cudaError_t unw_launch_bbox(const float* phase, long long pitch, int H0, int W0, int* rowany,
                            int* colany, int* bbox, cudaStream_t s);

// post-processing
enum {
    UNW_P_KSTATS = 0,   // non-finite count, min/max cycle count
    UNW_P_HIST,         // histogram of cycle counts
    UNW_P_MEDIAN,       // median -> shift (one CTA per grid)
    UNW_P_SHIFT_CCINIT, // apply shift, NaN restore, union-find init
    UNW_P_UNION,        // union with right/down neighbours
    UNW_P_FLATTEN,      // root per pixel, roots per tile
    UNW_P_TILESCAN,     // exclusive scan of tile counts (one CTA per grid)
    UNW_P_LABEL,        // compact labels of roots
    UNW_P_ACCUM,        // per-label sin/cos sums and counts
    UNW_P_ADJUST,       // per-label circular-mean adjustment
    UNW_P_WRITE,        // outputs into the caller's full grid
    UNW_P_FILL          // NaN / 0 outside the crop and for failed grids
};
cudaError_t unw_launch_post(int which, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                            int n, const UnwScalars& sc, const GridDev* host_grids);

// Per-grid tensor maps of the TMA-staged passes (one 128-byte CUtensorMap each): the
// column pass's two (tensor-core T / p1, or power-of-two even / odd rows of T) at
// UNW_MAP_COL, the matvec's three (p, wIx, wIy) at UNW_MAP_MV.
#define UNW_MAPS_PER_GRID 8
#define UNW_MAP_BYTES (128 * UNW_MAPS_PER_GRID)
#define UNW_MAP_COL 0
#define UNW_MAP_MV 2
bool unw_mv_tma_maps(const float* p, const float* wIx, const float* wIy, int H, int W, int P, void* out);
cudaError_t unw_launch_matvec_tma(int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                                  const void* maps);

// power-of-two column pass with the slab moved by TMA (unw_dct_p2_tma.cu), H = 2048 / 4096
int unw_p2_tma_nseq(int N);
bool unw_p2_tma_maps(const float* T, int H, int W, int P, int nseq, void* out);
cudaError_t unw_launch_col_p2_tma(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                                  int n, const void* maps);

// frozen-weight adjoint (KS_ELEM shapes except REARM)
#define UNW_ADJ_REFINE 3    // refinement passes of u* (each stops early below 1e-13 residual)
#define UNW_ADJ_CHUNK 8     // adjoint PCG iterations enqueued between reads of the instance state
enum {
    UNW_A_LOAD = 0,     // forward output and dL/dout into the crop
    UNW_A_LSUM,         // per-component sum of dL/dout
    UNW_A_RHS,          // adjoint right-hand side, x0 = 0
    UNW_A_REARM,        // solver state for the adjoint PCG
    UNW_A_GRAD,         // dL/dphase, dL/dweight
    UNW_A_REFINE,       // float64 residual of the frozen system at u* -> correction right-hand side
    UNW_A_ADDD          // u* += correction (pass k)
};
cudaError_t unw_launch_adj(int which, int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                           int k = 0);
