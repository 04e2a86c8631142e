// Weighted-Laplacian matvec of the PCG, Ap = A p and pAp = p.Ap
// (utils_unwrap2d.py:1367-1388, :1433-1442), on TMA-staged halo tiles.
//
// Same tiles, thread mapping and arithmetic as k_matvec (unw_solver_kernels.cu), so the
// results are bit-identical; what changes is how the operands arrive.  A CTA of 16 warps
// computes 128-column x 16-row output tiles (one warp per row, four columns per lane) in a
// persistent loop.  Per tile, one thread issues three 2-D TMA copies into shared memory:
//   p    rows i0-1 .. i0+16, columns j0-4 .. j0+131 (the halo rows above and below, and
//        the column on each side, rounded out to 16-byte boundaries)
//   wIx  rows i0 .. i0+15,   columns j0-4 .. j0+131 (the weight of the left edge)
//   wIy  rows i0-1 .. i0+15, columns j0 .. j0+127   (the weight of the upper edge)
// Coordinates outside the grid (rows outside 0..H-1, columns outside 0..P-1) read as zeros; the
// stencil masks those terms as before, and columns W..P-1 hold what k_matvec reads there.
// Three stages: the copies of the tile three ahead are issued as soon as every warp is done
// with the current one, so each warp's operands are in shared memory when it starts a tile
// and no warp waits on DRAM latency (k_matvec: 8.8 long-scoreboard stalls per issue).  Every
// mbarrier wait is bounded by the global timer (2 s): a wait that runs out sets
// UNW_S_TC_TIMEOUT in the grid's state and the CTA stops (after a bounded wait for the copies
// it issued).  No multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "unw_kernels.h"
#include "unw_rowops.cuh"

namespace {

constexpr int MV_TW = 128;                     // output columns per tile
constexpr int MV_TH = 16;                      // output rows per tile (one warp each)
constexpr int MV_BW = MV_TW + 8;               // staged columns: j0-4 .. j0+131
constexpr int MV_THREADS = 32 * MV_TH;
constexpr uint32_t MV_P_BYTES = (MV_TH + 2) * MV_BW * 4;      // 9792
constexpr uint32_t MV_WX_BYTES = MV_TH * MV_BW * 4;           // 8704
constexpr uint32_t MV_WY_BYTES = (MV_TH + 1) * MV_TW * 4;     // 8704
constexpr uint32_t MV_P_OFF = 0;
constexpr uint32_t MV_WX_OFF = (MV_P_BYTES + 127) / 128 * 128;
constexpr uint32_t MV_WY_OFF = MV_WX_OFF + MV_WX_BYTES;
constexpr uint32_t MV_STAGE = (MV_WY_OFF + MV_WY_BYTES + 127) / 128 * 128;
// stages in flight (measured on B200, 4096^2 fault grid, CUDA-event time per launch, same
// bits: 2 stages 55.7 us, 3 stages 53.0 us, 4 stages 54.1 us; k_matvec 55.7 us)
constexpr int MV_NST = 3;
constexpr size_t MV_SMEM = MV_NST * (size_t)MV_STAGE + 128;
constexpr unsigned long long MV_WAIT_NS = 2000000000ull;
constexpr int MV_STATUS_TIMEOUT = 16;          // UNW_S_TC_TIMEOUT
static_assert(MV_WX_BYTES % 128 == 0 && MV_WY_BYTES % 128 == 0, "128-byte regions");

__device__ __forceinline__ uint32_t mv_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long mv_timer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mv_wait(uint64_t* b, uint32_t parity) {
    const unsigned long long t0 = mv_timer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(mv_smem(b)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (mv_timer() - t0 > MV_WAIT_NS) return false;
    }
}

__device__ __forceinline__ void mv_load(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(mv_smem(dst)), "l"((unsigned long long)map), "r"(mv_smem(bar)), "r"(x), "r"(y)
        : "memory");
}

// the three copies of one tile into a stage, completing on the stage's mbarrier
__device__ __forceinline__ void mv_issue(unsigned char* stage, uint64_t* bar, const CUtensorMap* maps, int i0,
                                         int j0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mv_smem(bar)),
                 "r"(MV_P_BYTES + MV_WX_BYTES + MV_WY_BYTES)
                 : "memory");
    mv_load(stage + MV_P_OFF, maps + 0, bar, j0 - 4, i0 - 1);
    mv_load(stage + MV_WX_OFF, maps + 1, bar, j0 - 4, i0);
    mv_load(stage + MV_WY_OFF, maps + 2, bar, j0, i0 - 1);
}

__global__ void __launch_bounds__(MV_THREADS, 2) k_matvec_tma(const GridDev* __restrict__ grids,
                                                              const int* __restrict__ starts, int n,
                                                              const CUtensorMap* __restrict__ allmaps) {
    extern __shared__ unsigned char mv_raw[];
    __shared__ double red[32 * 1];
    __shared__ __align__(8) uint64_t bar[MV_NST];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* const base = (unsigned char*)(((size_t)mv_raw + 127) & ~(size_t)127);
    const CUtensorMap* maps = allmaps + UNW_MAPS_PER_GRID * g + UNW_MAP_MV;
    const int ntiles = G.sten_tiles_x * ((H + 15) / 16);
    // tile k of this CTA (bottom rows first, as k_matvec: the row-inverse pass that formed p
    // ends at the bottom and the row-forward pass that reads Ap next starts at the top)
    auto tile_ij = [&](int tile, int& i0, int& j0) {
        const int tr = ntiles - 1 - tile;
        j0 = (tr % G.sten_tiles_x) * MV_TW;
        i0 = (tr / G.sten_tiles_x) * MV_TH;
    };
    int issued = 0;
    if (threadIdx.x == 0) {
        for (int k = 0; k < MV_NST; k++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mv_smem(&bar[k])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        for (int m = 0; m < 3; m++)
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((unsigned long long)(maps + m))
                         : "memory");
        for (int k = 0; k < MV_NST; k++) {
            const int tile = local + k * nct;
            if (tile >= ntiles) break;
            int i0, j0;
            tile_ij(tile, i0, j0);
            mv_issue(base + k * MV_STAGE, &bar[k], maps, i0, j0);
            issued++;
        }
    }
    __syncthreads();
    double acc[1] = {0.0};
    bool failed = false;
    int it = 0;
    for (int tile = local; tile < ntiles; tile += nct, it++) {
        const int sidx = it % MV_NST;
        const bool ok = mv_wait(&bar[sidx], (uint32_t)((it / MV_NST) & 1));
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        const unsigned char* stage = base + sidx * MV_STAGE;
        const float* __restrict__ ps = reinterpret_cast<const float*>(stage + MV_P_OFF);
        const float* __restrict__ wxs = reinterpret_cast<const float*>(stage + MV_WX_OFF);
        const float* __restrict__ wys = reinterpret_cast<const float*>(stage + MV_WY_OFF);
        int i0, j0;
        tile_ij(tile, i0, j0);
        const int jj = lane * 4;           // column of the lane within the tile
        const int j = j0 + jj;
        const int i = i0 + warp;
        const bool on = i < H && j < W;
        const bool hu = i > 0, hd = i < H - 1;
        // staged row r of p is grid row i0 - 1 + r; staged column c is grid column j0 - 4 + c
        const float4 cur = *reinterpret_cast<const float4*>(ps + (warp + 1) * MV_BW + 4 + jj);
        const float4 up = *reinterpret_cast<const float4*>(ps + warp * MV_BW + 4 + jj);
        const float4 dn = *reinterpret_cast<const float4*>(ps + (warp + 2) * MV_BW + 4 + jj);
        const float4 wx = *reinterpret_cast<const float4*>(wxs + warp * MV_BW + 4 + jj);
        const float4 wy = *reinterpret_cast<const float4*>(wys + (warp + 1) * MV_TW + jj);
        const float4 wyu = *reinterpret_cast<const float4*>(wys + warp * MV_TW + jj);
        const float c4[4] = {cur.x, cur.y, cur.z, cur.w};
        const float u4[4] = {up.x, up.y, up.z, up.w};
        const float d4[4] = {dn.x, dn.y, dn.z, dn.w};
        const float x4[4] = {wx.x, wx.y, wx.z, wx.w};
        const float y4[4] = {wy.x, wy.y, wy.z, wy.w};
        const float yu4[4] = {wyu.x, wyu.y, wyu.z, wyu.w};
        float pl = __shfl_up_sync(0xffffffffu, c4[3], 1);
        float wll = __shfl_up_sync(0xffffffffu, x4[3], 1);
        float pr = __shfl_down_sync(0xffffffffu, c4[0], 1);
        if (lane == 0) {
            pl = ps[(warp + 1) * MV_BW + 3];
            wll = wxs[warp * MV_BW + 3];
        }
        if (lane == 31) pr = ps[(warp + 1) * MV_BW + 4 + MV_TW];
        if (on) {
            float ap[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int jc = j + c;
                const float pc = c4[c];
                const float pleft = c == 0 ? pl : c4[c - 1];
                const float pright = c == 3 ? pr : c4[c + 1];
                const float wleft = c == 0 ? wll : x4[c - 1];
                float res = 0.f;
                if (jc > 0) res = fsub(res, fmul(fsub(pc, pleft), wleft));
                if (jc < W - 1) res = fadd(res, fmul(fsub(pright, pc), x4[c]));
                if (hu) res = fsub(res, fmul(fsub(pc, u4[c]), yu4[c]));
                if (hd) res = fadd(res, fmul(fsub(d4[c], pc), y4[c]));
                ap[c] = -res;
                if (jc < W) acc[0] += (double)pc * (double)ap[c];
            }
            *reinterpret_cast<float4*>(G.Ap + (size_t)i * P + j) = make_float4(ap[0], ap[1], ap[2], ap[3]);
        }
        __syncthreads();  // every warp is done with this stage
        if (threadIdx.x == 0) {
            const int next = tile + MV_NST * nct;
            if (next < ntiles) {
                int ni0, nj0;
                tile_ij(next, ni0, nj0);
                mv_issue(base + sidx * MV_STAGE, &bar[sidx], maps, ni0, nj0);
                issued++;
            }
        }
    }
    if (failed && threadIdx.x == 0) {
        // copies issued for tiles it .. issued-1 may still land: wait for them (bounded)
        for (int k = it; k < issued; k++) mv_wait(&bar[k % MV_NST], (uint32_t)((k / MV_NST) & 1));
        atomicOr(&st->status, MV_STATUS_TIMEOUT);
    }
    // every CTA arrives (a failed one with its partial pAp: the status bit marks the result)
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) matvec_finalize(st, acc[0]);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 mv_encode_fn() {
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

// H rows of P floats (the whole pitch, as k_matvec reads it: a lane whose first column is
// below W reads all four of its columns), box box_w x box_h; reads outside are zeros
bool mv_map(CUtensorMap* m, const float* a, int H, int P, int box_w, int box_h) {
    auto fn = mv_encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)P, (cuuint64_t)H};
    cuuint64_t strides[1] = {(cuuint64_t)P * 4};
    cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(a), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

// Tensor maps of p, wIx and wIy for the TMA matvec (three consecutive maps at `out`); false
// where the layout does not allow TMA (alignment) or the driver entry point is missing.
bool unw_mv_tma_maps(const float* p, const float* wIx, const float* wIy, int H, int W, int P, void* out) {
    if ((P & 3) || ((size_t)p & 15) || ((size_t)wIx & 15) || ((size_t)wIy & 15) || H < 1 || W < 1) return false;
    CUtensorMap* m = (CUtensorMap*)out;
    return mv_map(&m[0], p, H, P, MV_BW, MV_TH + 2) && mv_map(&m[1], wIx, H, P, MV_BW, MV_TH) &&
           mv_map(&m[2], wIy, H, P, MV_TW, MV_TH + 1);
}

cudaError_t unw_launch_matvec_tma(int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                                  const void* maps) {
    if (nblk <= 0) return cudaSuccess;
    const cudaError_t e = unw_smem_limit((const void*)k_matvec_tma);  // once per device
    if (e != cudaSuccess) return e;
    k_matvec_tma<<<nblk, MV_THREADS, MV_SMEM, s>>>(gd, starts, n, (const CUtensorMap*)maps);
    return cudaGetLastError();
}
