// Column pass of the power-of-two DCT preconditioner with the column slab moved by TMA
// (H = 2048 and 4096): the column DCT-II, the -1/lambda scaling and the column DCT-III
// (utils_unwrap2d.py:1390-1403, the column half of dct_2d/idct_2d at :1316-1365), the
// same arithmetic as k_col_p2 in unw_dct_p2.cu, so the result is bit-identical.
//
// What changes is how the slab (2*NSEQ columns x H rows of T) reaches the registers.  A
// row of the slab is only 16 (NSEQ = 2 column pairs) or 32 (NSEQ = 4) bytes, so a warp's
// plain loads and stores touch 16 (8) rows each: one L1 wavefront per row, which at
// H = 4096 made the L1 data pipe the busiest unit of the pass (59% of peak, 60% of its
// wavefronts from these accesses).  Here one thread issues 2-D TMA copies of the slab into shared memory and
// back: the even rows and the odd rows through two tensor maps (row strides 2P), so that
// Makhoul's reordering of the DCT-II (FFT position m holds row 2m for m < H/2 and row
// 2H-1-2m above) becomes position m of the even half or position H-1-m of the odd half:
// a warp's 16 consecutive positions are 256 contiguous bytes, read and written without
// bank conflicts.  The staged slab shares the transform buffers (it is read into
// registers before the first FFT pass writes them, and written back after the last
// pass has read them).
//
// Synchronisation: one mbarrier with the slab's byte count per load (phase = slab parity);
// before the next load into the buffer, the issuing thread waits until the previous
// slab's bulk stores have read it.  Every mbarrier wait is bounded by the global timer
// (2 s): a wait that runs out sets UNW_S_TC_TIMEOUT in the grid's state and the CTA
// stops (after a bounded wait for the copy it issued).  No multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "unw_kernels.h"
#include "unw_regfft.cuh"
#include "unw_rowops.cuh"
#include "unw_colspec.cuh"

namespace {

constexpr unsigned long long CT_WAIT_NS = 2000000000ull;  // 2 s per wait at most
constexpr int CT_BOX_ROWS = 256;                           // rows per TMA box
constexpr int CT_STATUS_TIMEOUT = 16;                      // UNW_S_TC_TIMEOUT

__device__ __forceinline__ uint32_t ct_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long ct_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool ct_wait(uint64_t* b, uint32_t parity) {
    const unsigned long long t0 = ct_timer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(ct_smem(b)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (ct_timer() - t0 > CT_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void ct_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(ct_smem(dst)), "l"((unsigned long long)map), "r"(ct_smem(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void ct_store(const CUtensorMap* map, const void* src, int x, int y) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];"
                 ::"l"((unsigned long long)map), "r"(ct_smem(src)), "r"(x), "r"(y)
                 : "memory");
}

template <int NT>
constexpr int ct_min_blocks() { return NT >= 1024 ? 1 : 1024 / NT; }

template <int N, int NSEQ, int MODE>
__global__ void __launch_bounds__(N / 16 * NSEQ, ct_min_blocks<N / 16 * NSEQ>()) k_col_p2_tma(
    const GridDev* __restrict__ grids, const int* __restrict__ starts, int n, const CUtensorMap* __restrict__ maps) {
    constexpr int T = N / 16;
    constexpr int ROWB = 8 * NSEQ;                 // bytes of one slab row (2 NSEQ floats)
    constexpr int HALF = N / 2 * ROWB;             // bytes of the slab's even (or odd) rows
    constexpr int NBOX = N / 2 / CT_BOX_ROWS;      // TMA boxes per half
    static_assert(2 * HALF <= NSEQ * RegFft<N>::SEQ_STRIDE * (int)sizeof(float2), "slab fits the buffers");
    static_assert(N / 2 % CT_BOX_ROWS == 0, "whole boxes");
    extern __shared__ unsigned char ct_raw[];
    __shared__ double red[32];
    __shared__ __align__(8) uint64_t bar;
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (MODE >= 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W;
    const int s = threadIdx.x % NSEQ, t = threadIdx.x / NSEQ;
    unsigned char* const base = (unsigned char*)(((size_t)ct_raw + 127) & ~(size_t)127);
    float2* sms = reinterpret_cast<float2*>(base) + s * RegFft<N>::SEQ_STRIDE;
    const CUtensorMap* me = maps + UNW_MAPS_PER_GRID * g + UNW_MAP_COL;  // even rows of T
    const CUtensorMap* mo = me + 1;        // odd rows of T
    const float2* __restrict__ tw = G.pcol.fft.tw;
    const float2* __restrict__ dw = G.pcol.dctw;
    const float* __restrict__ sH = G.sH;
    const float negs = -1.0f / (4.0f * (float)N * (float)W);
    const int nslab = (W + 2 * NSEQ - 1) / (2 * NSEQ);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(ct_smem(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((unsigned long long)me) : "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((unsigned long long)mo) : "memory");
    }
    __syncthreads();
    double acc[1] = {0.0};
    bool failed = false;
    int it = 0;
    for (int slab = local; slab < nslab; slab += nct, it++) {
        const int j0 = 2 * NSEQ * slab;
        if (threadIdx.x == 0) {
            // the previous slab's bulk stores have read the buffer
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(ct_smem(&bar)),
                         "r"((uint32_t)(2 * HALF))
                         : "memory");
#pragma unroll 1
            for (int b = 0; b < NBOX; b++) {
                ct_load(base + b * CT_BOX_ROWS * ROWB, me, &bar, j0, b * CT_BOX_ROWS);
                ct_load(base + HALF + b * CT_BOX_ROWS * ROWB, mo, &bar, j0, b * CT_BOX_ROWS);
            }
        }
        const bool ok = ct_wait(&bar, (uint32_t)(it & 1));
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        const int ja = j0 + 2 * s;
        const bool hasa = ja < W, hasb = ja + 1 < W;
        // FFT position m = t + T q: even row 2m at position m of the even half (q < 8), odd
        // row 2N-1-2m at position N-1-m of the odd half (q >= 8); columns beyond W are zeros
        const unsigned char* col = base + 8 * s;
        float2 v[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int m = t + T * q;
            v[q] = *reinterpret_cast<const float2*>(col + (q < 8 ? m * ROWB : HALF + (N - 1 - m) * ROWB));
        }
        __syncthreads();  // every staged read done before the transform writes the buffer
        io_fft<N, true, false>(v, sms, t, tw);
        const float ca = hasa ? G.sW[ja] : 1.0f, cb = hasb ? G.sW[ja + 1] : 1.0f;
        col_spectral_p2<N, MODE>(sms, t, dw, sH, ca, cb, ja == 0, hasb, negs, acc[0]);
        __syncthreads();
        io_fft<N, false, true>(v, sms, t, tw);
        __syncthreads();  // every transform read of the buffer done before the slab is staged back
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int m = t + T * q;
            *reinterpret_cast<float2*>(base + 8 * s + (q < 8 ? m * ROWB : HALF + (N - 1 - m) * ROWB)) =
                make_float2(v[q].x, -v[q].y);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the bulk copies
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll 1
            for (int b = 0; b < NBOX; b++) {
                ct_store(me, base + b * CT_BOX_ROWS * ROWB, j0, b * CT_BOX_ROWS);
                ct_store(mo, base + HALF + b * CT_BOX_ROWS * ROWB, j0, b * CT_BOX_ROWS);
            }
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
    }
    if (threadIdx.x == 0) {
        if (failed) {
            // the copy of the slab that timed out may still land: wait for it once more (bounded)
            ct_wait(&bar, (uint32_t)(it & 1));
            atomicOr(&st->status, CT_STATUS_TIMEOUT);
        }
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");  // stores complete before exit
    }
    if (MODE == 0) return;
    // every CTA arrives (a failed one with its partial r.z: the status bit marks the result)
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) col_finalize<MODE>(st, acc[0]);
    }
}

// Column pairs per CTA: those of the plain-load pass at the same length (two at H = 4096,
// 16-byte rows; four at H = 2048, 32-byte rows).  Which of the two passes is faster depends
// on the shape (measured on B200, CUDA-event time per column pass, bit-identical results:
// 4096 x 4096 92.4 us TMA / 101.8 us plain, 4096 x 1000 35.7 / 35.3, 2048 x 2048 34.8 / 31.4),
// so the solver's autotuner times both per shape and keeps the faster.
template <int N>
constexpr int ct_nseq() { return N == 2048 ? 4 : 2; }

template <int N>
cudaError_t ct_launch(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n,
                      const CUtensorMap* maps) {
    constexpr int NS = ct_nseq<N>();
    const size_t smem = sizeof(float2) * RegFft<N>::SEQ_STRIDE * NS + 128;
    auto go = [&](auto kfn) {
        const cudaError_t e = unw_smem_limit((const void*)kfn);
        if (e != cudaSuccess) return e;
        kfn<<<nblk, N / 16 * NS, smem, s>>>(gd, st, n, maps);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_col_p2_tma<N, NS, 0>);
        case 1: return go(k_col_p2_tma<N, NS, 1>);
        default: return go(k_col_p2_tma<N, NS, 2>);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 ct_encode_fn() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

}  // namespace

// Column sequences (pairs) per CTA of the TMA column pass; 0 where it does not apply.
int unw_p2_tma_nseq(int N) {
    switch (N) {
        case 2048: return ct_nseq<2048>();
        case 4096: return ct_nseq<4096>();
        default: return 0;
    }
}

// Two tensor maps (even rows, odd rows) of the float32 H x W array T with a row pitch of
// P floats, box 2*nseq columns x 256 rows, no swizzle; reads beyond W are zero-filled and
// stores beyond W are dropped.  False where the layout does not allow TMA (alignment) or
// the driver entry point is missing.
bool unw_p2_tma_maps(const float* T, int H, int W, int P, int nseq, void* out) {
    auto fn = ct_encode_fn();
    if (!fn || nseq <= 0 || (H & 1) || H / 2 < CT_BOX_ROWS || (P & 3) || ((size_t)T & 15)) return false;
    CUtensorMap* m = (CUtensorMap*)out;
    for (int par = 0; par < 2; par++) {
        cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)(H / 2)};
        cuuint64_t strides[1] = {(cuuint64_t)P * 2 * 4};
        cuuint32_t box[2] = {(cuuint32_t)(2 * nseq), (cuuint32_t)CT_BOX_ROWS};
        cuuint32_t estr[2] = {1, 1};
        if (fn(&m[par], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(T + (size_t)par * P), dims, strides,
               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

cudaError_t unw_launch_col_p2_tma(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                                  int n, const void* maps) {
    if (nblk <= 0) return cudaSuccess;
    const CUtensorMap* m = (const CUtensorMap*)maps;
    switch (N) {
        case 2048: return ct_launch<2048>(mode, nblk, s, gd, starts, n, m);
        case 4096: return ct_launch<4096>(mode, nblk, s, gd, starts, n, m);
        default: return cudaErrorInvalidValue;
    }
}
