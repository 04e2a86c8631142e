// Internal device-side structures and helpers of the B200 unwrapper.
//
// Memory model: every grid of a (batched) solve owns a block of the caller's
// workspace holding its float32 work arrays (row pitch P floats, 128-byte
// aligned rows), its FFT tables, its scalar state and its reduction scratch.
// Kernels cover all grids of a batch: a CTA finds its grid through a prefix
// array of per-grid CTA counts (one prefix array per kernel shape).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define UNW_MAX_PASSES 16
#define UNW_NPART 4          // doubles of reduction partials per CTA
#define UNW_MAX_LOG 64       // per-IRLS-iteration CG counts kept in the state

// Kernel shapes; each has its own CTA prefix array.
enum { KS_ROWPAIR = 0, KS_COL = 1, KS_STEN = 2, KS_ELEM = 3, KS_ONE = 4, KS_MATVEC = 5, KS_TC = 6, KS_NKIND = 7 };

struct FftPlanDev {
    int n;                      // transform length
    int npass;
    int radix[UNW_MAX_PASSES];
    const float2* tw;           // n entries, exp(-2*pi*i*m/n)
};

// Length-N DFT used by the DCT passes: a direct mixed-radix FFT when N is
// 7-smooth, otherwise Bluestein's chirp-z convolution through a smooth FFT of
// length M >= 2N-1.
struct DctPlanDev {
    int N;
    int blue;
    int stride;                 // float2 slots per sequence in shared memory
    FftPlanDev fft;             // length N (direct) or M (Bluestein)
    const float2* dctw;         // N entries, exp(-i*pi*k/(2N))
    const float2* chirp;        // N entries, exp(+i*pi*m^2/N)      (Bluestein)
    const float2* hspec;        // M entries, FFT(chirp filter) / M (Bluestein)
};

// Scalar state of one grid's solve.  Written only by the last CTA of a
// reducing kernel (or by single-CTA kernels), read by the following kernels.
struct InstState {
    // PCG (utils_unwrap2d.py:1405-1474)
    double rz;
    double pAp;
    double rnorm;
    float alpha, beta;
    int cg_active;
    int cg_iter;
    // IRLS (utils_unwrap2d.py:1529-1632)
    int irls_active;
    int irls_iter;
    int max_iter;
    int best_update;
    int revert;
    int u_index;                // which U buffer holds the current iterate
    int status;                 // UNW_S_* bits
    double vcount;              // number of valid pixels
    double mean;
    double residual;
    double best_residual;
    double rel_change;
    double resid_rel;           // ||b - A u|| / ||b|| of the final system in float64 (k_resid)
    float tol, cg_tol, eps2;
    float cg_rel;               // > 0: cg_tol = cg_rel * ||r0|| at the PCG start
    double refine_scale;        // adjoint refinement: scale of the correction's right-hand side
    int cg_max_iter;
    int cg_total;
    int cg_log[UNW_MAX_LOG];
    // post-processing (utils_unwrap2d.py:1659-1746)
    int n_nonfinite;
    int kmin, kmax;
    int hist_ok;
    float kmed;
    float shift;
    int n_labels;
    int n_kneg, n_kpos;         // valid pixels whose cycle count is -inf / +inf (infinite phase)
    int pad_;
};


struct GridDev {
    int H, W, P;                // cropped grid, pitch of work arrays
    int H0, W0;                 // caller's full grid
    int r0, c0;                 // crop origin
    const float* phase;  long long phase_pitch;   // points at the crop origin
    const float* weight; long long weight_pitch;  // may be null
    float* out_u;        long long out_u_pitch;   // full-grid origin
    uint16_t* out_cc;    long long out_cc_pitch;
    int congruent;
    int col_nseq;               // complex sequences (column pairs) per column CTA
    int col_ctas;               // CTA cap of the persistent column pass
    int sten_rows;              // rows per stencil CTA
    int sten_tiles_x;           // column tiles per stencil row strip
    float *gx, *gy, *wx, *wy;
    float *wIx, *wIy, *b, *r, *z, *p0, *p1, *Ap, *T;
    // The IRLS iterate u is a float32 pair U + L with U = fl32(u) and |L| <= ulp(U)/2
    // (about 48 significant bits): U0/L0 and U1/L1 ping-pong per IRLS iteration, Ub/Lb
    // hold the best iterate.  The PCG accumulates its correction x - x0 in D (float32,
    // zeroed at the PCG start); the IRLS tail adds it to the pair in float64.
    float *U0, *U1, *Ub;
    float *L0, *L1, *Lb, *D;
    uint8_t* valid;
    // Neumann-Laplacian eigenvalue parts: lambda(k, j) = -(sH[k] + sW[j]) with
    // sH[k] = 4 sin^2(pi k / 2H), sW[j] = 4 sin^2(pi j / 2W), each computed in
    // float64 and rounded once.  Equal to 2cos(pi k/H) + 2cos(pi j/W) - 4
    // (utils_unwrap2d.py:1284-1289) without its cancellation near k = j = 0.
    const float* sH;
    const float* sW;
    DctPlanDev prow, pcol;
    InstState* st;
    double* part;               // reduction partials [max CTAs][UNW_NPART]
    unsigned* counter;          // last-CTA arrival counter
    // post-processing scratch (aliases dead solver buffers)
    int* parent;                // union-find parent / component label per pixel
    int* lab;                   // compact label of each root
    double* csum;               // [4][cap] sin/cos sums per label
    int* ccount;                // [cap] pixel count per label
    int* remap;                 // [cap] size-ranked output label
    double* adj;                // [cap] per-label adjustment
    int* hist;                  // histogram of cycle counts
    int hist_cap;
    int lab_cap;
    int* tilecnt;               // roots per scan tile
    int ntiles;
    // frozen-weight adjoint: the caller's full grids (forward output, dL/du in; gradients out)
    const float* a_u;  long long a_u_pitch;
    const float* a_gu; long long a_gu_pitch;
    float* a_gph;      long long a_gph_pitch;
    float* a_gw;       long long a_gw_pitch;    // may be null
};

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ int find_grid(const int* __restrict__ starts, int n, int bid) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&starts[mid]) <= bid) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// Reference-faithful float32 arithmetic: one rounding per operation, no FMA
// contraction (the reference applies separate torch elementwise ops).
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
// torch.clamp semantics: NaN propagates.
__device__ __forceinline__ float clampf_nan(float x, float lo, float hi) {
    return x < lo ? lo : (x > hi ? hi : x);
}

// Block-wide sum of NV doubles; the result is valid in thread 0.
// Fixed reduction tree: deterministic for a given blockDim.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* sm /* >= 32*NV */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) sm[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? sm[q * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[q] = x;
        }
    }
    __syncthreads();
}

// Writes this CTA's partials, then returns true in exactly one CTA per grid:
// the last to arrive.  That CTA then reads all partials (finish_sum).
template <int NV>
__device__ __forceinline__ bool arrive(const GridDev& G, int local, int nctas, double (&v)[NV],
                                       double* sm) {
    __shared__ int s_last;
    block_sum<NV>(v, sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) G.part[(size_t)local * UNW_NPART + q] = v[q];
        __threadfence();
        unsigned prev = atomicAdd(G.counter, 1u);
        s_last = (prev == (unsigned)(nctas - 1));
    }
    __syncthreads();
    return s_last != 0;
}

// Sums all CTAs' partials in a fixed order (deterministic); result in thread 0,
// and resets the arrival counter for the next kernel.
template <int NV>
__device__ __forceinline__ void finish_sum(const GridDev& G, int nctas, double (&v)[NV], double* sm) {
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = 0.0;
    for (int c = threadIdx.x; c < nctas; c += blockDim.x) {
#pragma unroll
        for (int q = 0; q < NV; q++) v[q] += __ldcg(&G.part[(size_t)c * UNW_NPART + q]);
    }
    block_sum<NV>(v, sm);
    if (threadIdx.x == 0) *G.counter = 0u;
}

// Splits a float64 value into the float32 pair (hi, lo), hi = fl32(v), lo = fl32(v - hi).
__device__ __forceinline__ void split_pair(double v, float& hi, float& lo) {
    hi = __double2float_rn(v);
    lo = isfinite(hi) ? __double2float_rn(v - (double)hi) : 0.f;
}
__device__ __forceinline__ double pair_val(float hi, float lo) { return (double)hi + (double)lo; }

// Makhoul's even/odd reordering: x_n sits at position perm(n) of the sequence
// whose DFT yields the DCT-II (J. Makhoul, IEEE TASSP 28(1), 1980).
__device__ __forceinline__ int mk_perm(int n, int N) {
    return (n & 1) ? (N - 1 - (n >> 1)) : (n >> 1);
}
