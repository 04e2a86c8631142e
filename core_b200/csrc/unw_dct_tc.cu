// Tensor-core column pass for grids of at most 1024 rows (the mixed-precision
// form): the column DCT-II, the -1/lambda scaling and the column DCT-III of the
// preconditioner (utils_unwrap2d.py:1390-1403, the column half of
// dct_2d/idct_2d at :1316-1365) as two dense matrix products per grid,
//     X = C T        C[k][i] = 2 cos(pi k (2i+1) / 2H)           (DCT-II)
//     Y = S .* X     S[k][j] = -1 / (4 H W lambda(k, j)), Y[0][0] = 0
//     T' = E Y       E[i][k] = c_k cos(pi k (2i+1) / 2H), c_0 = 1, c_k = 2
// (E and the 4HW factor match the FFT column pass, so the row passes around it
// are unchanged), plus r.z by Parseval's identity from X and Y.
//
// Arithmetic: split-precision BF16 on the 5th-generation tensor cores.  Every
// operand is split into hi = bf16(v) and lo = bf16(v - hi); each product is
// A_hi B_hi + A_hi B_lo + A_lo B_hi (three tcgen05.mma kind::f16 issues into one
// float32 accumulator in tensor memory), about 16 significant bits per term.
// The DCT matrices are split once per solve into the workspace and staged by
// TMA (128-byte swizzle); the float32 data are staged by TMA too and split by the
// CTA's threads in shared memory, so no extra pass over HBM is needed.
//
// Tiling: one CTA per 128 x 64 output tile; K runs in stages of 64 through a
// three-stage ring (the bf16 A tiles and the float32 B tile by TMA), with one warp
// loading, one issuing the MMAs and four splitting B into the MMA layout and then
// reading the accumulator (128 lanes x 64 columns of TMEM) back with tcgen05.ld.  Every
// wait on an mbarrier is bounded by the global timer: a wait that runs out sets
// UNW_S_TC_TIMEOUT in the grid's state, the CTA stops issuing, waits (bounded)
// for the MMAs it committed, frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <mutex>

#include "unw_kernels.h"
#include "unw_rowops.cuh"

namespace {

constexpr int TC_M = 128;                    // output rows per tile (TMEM lanes)
constexpr int TC_N = 64;                     // output columns per tile (TMEM columns)
constexpr int TC_K = 64;                     // K per stage: one 128-byte bf16 swizzle row
constexpr int TC_STAGES = 3;
constexpr int TC_THREADS = 192;                 // warp 0 loads, warp 1 MMAs, warps 2-5 split / epilogue
constexpr int TC_CONV_THREADS = 128;
constexpr uint32_t TC_A_TILE = TC_M * TC_K * 2;            // 16 KB per split (bf16, TMA, swizzled)
constexpr uint32_t TC_R_TILE = TC_K * TC_N * 4;            // 16 KB float32 B tile (TMA, row-major)
constexpr uint32_t TC_B_TILE = TC_K * TC_N * 2;            // 8 KB per split (bf16, MMA layout)
constexpr uint32_t TC_STAGE = 2 * TC_A_TILE + TC_R_TILE + 2 * TC_B_TILE;
constexpr size_t TC_SMEM = (size_t)TC_STAGES * TC_STAGE + 1024;  // + alignment slack
constexpr unsigned long long TC_WAIT_NS = 2000000000ull;   // 2 s per wait at most
constexpr int TC_STATUS_TIMEOUT = 16;                       // UNW_S_TC_TIMEOUT

// ---------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

// Waits for the phase with the given parity to complete; false after TC_WAIT_NS.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity) {
    const unsigned long long t0 = gtimer();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(smem_u32(b)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (gtimer() - t0 > TC_WAIT_NS) return false;
    }
}

// 2-D tiled TMA load (no multicast) of box (x, y) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((unsigned long long)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem desc] * B[smem desc], kind::f16 (bf16 operands, f32 accumulator)
__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d), "l"(a), "l"(b), "r"(idesc), "r"(accum)
        : "memory");
}

// the mbarrier completes once every MMA this thread issued before has finished
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2), sm100 version bit.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor: f32 accumulator, bf16 A (K-major) and B (MN-major), M x N.
constexpr uint32_t tc_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (0u << 15) | (1u << 16) | ((uint32_t)(TC_N >> 3) << 17) |
           ((uint32_t)(TC_M >> 4) << 24);
}

// 16 consecutive accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// ---------------------------------------------------------------- tables
// C (forward) and E (inverse) matrices of length H, zero-padded to Hp x Hp, split
// into bf16 hi / lo planes: tab = [C_hi | C_lo | E_hi | E_lo], each Hp x Hp row-major.
__global__ void k_tc_tables(int H, int Hp, __nv_bfloat16* __restrict__ tab) {
    const size_t plane = (size_t)Hp * Hp;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < plane; q += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(q / Hp), c = (int)(q % Hp);
        double cv = 0.0, ev = 0.0;
        if (r < H && c < H) {
            // C[k = r][i = c]: cos(pi k (2i+1) / 2H) with the angle index reduced exactly mod 4H
            const long long ac = ((long long)r * (2LL * c + 1)) % (4LL * H);
            cv = 2.0 * cospi((double)ac / (2.0 * H));
            // E[i = r][k = c]
            const long long ae = ((long long)c * (2LL * r + 1)) % (4LL * H);
            ev = (c == 0 ? 1.0 : 2.0) * cospi((double)ae / (2.0 * H));
        }
        const float cf = (float)cv, ef = (float)ev;
        const __nv_bfloat16 ch = __float2bfloat16_rn(cf), eh = __float2bfloat16_rn(ef);
        tab[q] = ch;
        tab[plane + q] = __float2bfloat16_rn(cf - __bfloat162float(ch));
        tab[2 * plane + q] = eh;
        tab[3 * plane + q] = __float2bfloat16_rn(ef - __bfloat162float(eh));
    }
}

// ---------------------------------------------------------------- the GEMM
// EPI 0: first product (X = C T): Y = S .* X -> p1, r.z (MODE >= 1), scalar step
// EPI 1: second product (T' = E Y): -> T
//
// Warp roles (192 threads), no block barrier inside the K loop:
//   warp 0      one thread issues the TMA loads of each stage (A hi / lo tiles and the
//               float32 B tile on the stage's `full` mbarrier), TC_STAGES steps ahead,
//               waiting only for the stage's `empty` mbarrier (its previous MMAs done);
//   warp 1      one thread waits for the stage's `conv` mbarrier, issues its 12 MMAs and
//               commits them to `empty`; after the last step it commits to `done`;
//   warps 2-5   wait for `full`, split the float32 B tile into bf16 hi / lo in the MMA
//               layout, arrive on `conv`; then the epilogue (warp w reads TMEM lanes
//               32 (w % 4) .. +31).
template <int EPI, int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1) k_col_tc(const GridDev* __restrict__ grids,
                                                          const int* __restrict__ starts, int n,
                                                          const __grid_constant__ CUtensorMap a_hi,
                                                          const __grid_constant__ CUtensorMap a_lo,
                                                          const CUtensorMap* __restrict__ bmaps) {
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ uint64_t full_bar[TC_STAGES], conv_bar[TC_STAGES], empty_bar[TC_STAGES], done_bar;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_fail;
    __shared__ volatile int s_issued;  // K steps whose loads the producer issued
    __shared__ double red[32];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (MODE >= 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int Hp = (H + TC_M - 1) / TC_M * TC_M;
    const int MT = Hp / TC_M;
    const int mt = local % MT, nt = local / MT;
    const int m0 = mt * TC_M, n0 = nt * TC_N;
    const int nk = Hp / TC_K;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    unsigned char* smem = (unsigned char*)(((uintptr_t)tc_smem_raw + 1023) & ~(uintptr_t)1023);
    // the float32 source of B: T (first product) or Y in p1 (second), one map per grid
    const CUtensorMap* bmap = bmaps + UNW_MAPS_PER_GRID * g + UNW_MAP_COL + EPI;

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&conv_bar[s], TC_CONV_THREADS);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&done_bar, 1);
        s_fail = 0;
        s_issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"((unsigned long long)bmap)
                     : "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    int committed = -1;  // (warp 1) K steps whose MMAs were committed

    if (warp == 0) {
        if (lane == 0) {
            for (int ks = 0; ks < nk && !s_fail; ks++) {
                const int s = ks % TC_STAGES;
                if (ks >= TC_STAGES && !mbar_wait(&empty_bar[s], (uint32_t)((ks / TC_STAGES - 1) & 1))) {
                    s_fail = 1;
                    break;
                }
                unsigned char* sa = smem + s * TC_STAGE;
                mbar_expect_tx(&full_bar[s], 2 * TC_A_TILE + TC_R_TILE);
                tma_load_2d(sa, &a_hi, &full_bar[s], ks * TC_K, m0);
                tma_load_2d(sa + TC_A_TILE, &a_lo, &full_bar[s], ks * TC_K, m0);
                tma_load_2d(sa + 2 * TC_A_TILE, bmap, &full_bar[s], n0, ks * TC_K);  // rows ks*64.., cols n0..
                s_issued = ks + 1;
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = tc_idesc();
            committed = 0;
            for (int ks = 0; ks < nk && !s_fail; ks++) {
                const int s = ks % TC_STAGES;
                if (!mbar_wait(&conv_bar[s], (uint32_t)((ks / TC_STAGES) & 1))) {
                    s_fail = 1;
                    break;
                }
                tc_fence_after();
                unsigned char* sa = smem + s * TC_STAGE;
                const uint32_t a0 = smem_u32(sa), b0 = smem_u32(sa + 2 * TC_A_TILE + TC_R_TILE);
#pragma unroll
                for (int kk = 0; kk < TC_K / 16; kk++) {
                    // A: +32 bytes per 16 K inside the swizzle row; B: +2 swizzle atoms (16 rows)
                    const uint64_t ah = sw128_desc(a0 + kk * 32, 16, 1024);
                    const uint64_t al = sw128_desc(a0 + TC_A_TILE + kk * 32, 16, 1024);
                    const uint64_t bh = sw128_desc(b0 + kk * 2048, TC_B_TILE, 1024);
                    const uint64_t bl = sw128_desc(b0 + TC_B_TILE + kk * 2048, TC_B_TILE, 1024);
                    const uint32_t acc0 = (ks > 0 || kk > 0) ? 1u : 0u;
                    umma(tmem, ah, bh, idesc, acc0);
                    umma(tmem, ah, bl, idesc, 1u);
                    umma(tmem, al, bh, idesc, 1u);
                }
                umma_commit(&empty_bar[s]);
                committed = ks + 1;
            }
            umma_commit(&done_bar);  // completes once every MMA issued above has finished
        }
    } else {
        // split B: row kk, 16-byte chunk c8 (8 columns) -> MN-major, 128-byte swizzle:
        // (kk / 8) * 1024 + (kk % 8) * 128 + ((c8 ^ (kk % 8)) * 16)
        const int ct = tid - 64;
        for (int ks = 0; ks < nk; ks++) {
            const int s = ks % TC_STAGES;
            if (s_fail || !mbar_wait(&full_bar[s], (uint32_t)((ks / TC_STAGES) & 1))) {
                s_fail = 1;
                break;
            }
            unsigned char* sa = smem + s * TC_STAGE;
            const unsigned char* sr = sa + 2 * TC_A_TILE;
            unsigned char* sb = sa + 2 * TC_A_TILE + TC_R_TILE;
#pragma unroll
            for (int q = 0; q < (TC_K * TC_N / 8) / TC_CONV_THREADS; q++) {
                const int c = ct + q * TC_CONV_THREADS;
                const int kk = c >> 3, c8 = c & 7;
                const float4 x0 = *reinterpret_cast<const float4*>(sr + kk * 256 + c8 * 32);
                const float4 x1 = *reinterpret_cast<const float4*>(sr + kk * 256 + c8 * 32 + 16);
                const float v[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
                float r[8];
#pragma unroll
                for (int e = 0; e < 8; e++) r[e] = v[e] - __bfloat162float(__float2bfloat16_rn(v[e]));
                uint4 hi, lo;
                hi.x = pack_bf16(v[0], v[1]); hi.y = pack_bf16(v[2], v[3]);
                hi.z = pack_bf16(v[4], v[5]); hi.w = pack_bf16(v[6], v[7]);
                lo.x = pack_bf16(r[0], r[1]); lo.y = pack_bf16(r[2], r[3]);
                lo.z = pack_bf16(r[4], r[5]); lo.w = pack_bf16(r[6], r[7]);
                const uint32_t off = (uint32_t)((kk >> 3) * 1024 + (kk & 7) * 128 + ((c8 ^ (kk & 7)) << 4));
                *reinterpret_cast<uint4*>(sb + off) = hi;
                *reinterpret_cast<uint4*>(sb + TC_B_TILE + off) = lo;
            }
            fence_proxy_async();
            mbar_arrive(&conv_bar[s]);
        }
    }
    // every MMA issued has finished once `done` completes (bounded); a failed run also
    // waits (bounded) for the loads it issued, so nothing is in flight when TMEM is freed
    if (warp == 1 && lane == 0 && committed >= 0) {
        if (!mbar_wait(&done_bar, 0)) s_fail = 1;
    }
    __syncthreads();
    if (s_fail) {
        if (tid == 0) {
            // the last load issued into each stage completes that stage's phase
            // (ks / TC_STAGES) & 1; earlier phases of the stage have completed already
            const int issued = s_issued;
            for (int ks = issued - TC_STAGES < 0 ? 0 : issued - TC_STAGES; ks < issued; ks++)
                mbar_wait(&full_bar[ks % TC_STAGES], (uint32_t)((ks / TC_STAGES) & 1));
            atomicOr(&st->status, TC_STATUS_TIMEOUT);
        }
        __syncthreads();
    }
    tc_fence_after();
    double acc[1] = {0.0};
    if (!s_fail && warp >= 2) {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 = output rows m0 + that range
        const int quarter = warp & 3;
        const int row = m0 + quarter * 32 + lane;
        const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16);
        if (EPI == 0) {
            const float negs = -1.0f / (4.0f * (float)H * (float)W);
            const float ck = row < H ? __ldg(&G.sH[row]) : 1.f;
            float* __restrict__ ydst = G.p1 + (size_t)row * P;
#pragma unroll 1
            for (int c0 = 0; c0 < TC_N; c0 += 16) {
                float x[16];
                tmem_ld16(tbase + c0, x);
                if (row < H) {
#pragma unroll
                    for (int e = 0; e < 16; e += 4) {
                        const int j = n0 + c0 + e;
                        if (j >= W) break;
                        float y[4];
#pragma unroll
                        for (int q = 0; q < 4; q++) {
                            const int jj = j + q;
                            float yv = 0.f;
                            if (jj < W && !(row == 0 && jj == 0)) yv = x[e + q] * (negs / -(ck + __ldg(&G.sW[jj])));
                            y[q] = yv;
                            if (MODE >= 1 && jj < W) {
                                const float w = (row == 0 ? 0.5f : 1.f) * (jj == 0 ? 0.5f : 1.f);
                                acc[0] += (double)(w * x[e + q]) * (double)yv;
                            }
                        }
                        if (j + 3 < W) {
                            *reinterpret_cast<float4*>(ydst + j) = make_float4(y[0], y[1], y[2], y[3]);
                        } else {
                            for (int q = 0; q < 4 && j + q < W; q++) ydst[j + q] = y[q];
                        }
                    }
                }
            }
        } else {
            float* __restrict__ tdst = G.T + (size_t)row * P;
#pragma unroll 1
            for (int c0 = 0; c0 < TC_N; c0 += 16) {
                float x[16];
                tmem_ld16(tbase + c0, x);
                if (row < H) {
#pragma unroll
                    for (int e = 0; e < 16; e += 4) {
                        const int j = n0 + c0 + e;
                        if (j >= W) break;
                        if (j + 3 < W) {
                            *reinterpret_cast<float4*>(tdst + j) = make_float4(x[e], x[e + 1], x[e + 2], x[e + 3]);
                        } else {
                            for (int q = 0; q < 4 && j + q < W; q++) tdst[j + q] = x[e + q];
                        }
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_N));
    if (EPI == 0 && MODE >= 1) {
        if (arrive<1>(G, local, nct, acc, red)) {
            finish_sum<1>(G, nct, acc, red);
            if (threadIdx.x == 0) col_finalize<MODE>(st, acc[0]);
        }
    }
}

// ---------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// Hp x Hp bf16 plane, box 64 (K, inner) x 128 (M), 128-byte swizzle
bool make_map(CUtensorMap* m, const void* plane, int Hp) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)Hp, (cuuint64_t)Hp};
    cuuint64_t strides[1] = {(cuuint64_t)Hp * 2};
    cuuint32_t box[2] = {(cuuint32_t)TC_K, (cuuint32_t)TC_M};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(plane), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// float32 H x W array with a row pitch of P floats, box 64 (columns) x 64 (rows), no
// swizzle; reads beyond the array are zero-filled
bool make_data_map(CUtensorMap* m, const float* base, int H, int W, int P) {
    auto fn = encode_fn();
    if (!fn) return false;
    cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
    cuuint64_t strides[1] = {(cuuint64_t)P * 4};
    cuuint32_t box[2] = {(cuuint32_t)TC_N, (cuuint32_t)TC_K};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int EPI, int MODE>
cudaError_t go(int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n, const CUtensorMap& hi,
               const CUtensorMap& lo, const CUtensorMap* bmaps) {
    auto kfn = k_col_tc<EPI, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM);
    if (e != cudaSuccess) return e;
    kfn<<<nblk, TC_THREADS, TC_SMEM, s>>>(gd, starts, n, hi, lo, bmaps);
    return cudaGetLastError();
}

}  // namespace

size_t unw_tc_table_bytes(int H) {
    if (H <= 0 || H > UNW_TC_MAX_H) return 0;
    const size_t Hp = (size_t)(H + TC_M - 1) / TC_M * TC_M;
    return 4 * Hp * Hp * sizeof(__nv_bfloat16);
}

int unw_tc_ctas(int H, int W) {
    const int Hp = (H + TC_M - 1) / TC_M * TC_M;
    return (Hp / TC_M) * ((W + TC_N - 1) / TC_N);
}

cudaError_t unw_tc_prepare(int H, void* tab, TcMaps* maps, cudaStream_t s) {
    if (H <= 0 || H > UNW_TC_MAX_H || !tab || ((uintptr_t)tab & 127)) return cudaErrorInvalidValue;
    const int Hp = (H + TC_M - 1) / TC_M * TC_M;
    const size_t plane = (size_t)Hp * Hp;
    k_tc_tables<<<592, 256, 0, s>>>(H, Hp, (__nv_bfloat16*)tab);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const __nv_bfloat16* t = (const __nv_bfloat16*)tab;
    if (!make_map((CUtensorMap*)maps->c_hi, t, Hp) || !make_map((CUtensorMap*)maps->c_lo, t + plane, Hp) ||
        !make_map((CUtensorMap*)maps->e_hi, t + 2 * plane, Hp) || !make_map((CUtensorMap*)maps->e_lo, t + 3 * plane, Hp))
        return cudaErrorNotSupported;
    return cudaSuccess;
}

bool unw_tc_data_maps(const float* T, const float* Y, int H, int W, int P, void* out2) {
    if ((P & 3) || ((uintptr_t)T & 15) || ((uintptr_t)Y & 15)) return false;
    CUtensorMap* m = (CUtensorMap*)out2;
    return make_data_map(m, T, H, W, P) && make_data_map(m + 1, Y, H, W, P);
}

cudaError_t unw_launch_col_tc(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                              const TcMaps* maps, const void* bmaps) {
    if (nblk <= 0) return cudaSuccess;
    const CUtensorMap& ch = *(const CUtensorMap*)maps->c_hi;
    const CUtensorMap& cl = *(const CUtensorMap*)maps->c_lo;
    const CUtensorMap& eh = *(const CUtensorMap*)maps->e_hi;
    const CUtensorMap& el = *(const CUtensorMap*)maps->e_lo;
    const CUtensorMap* bm = (const CUtensorMap*)bmaps;
    cudaError_t e;
    switch (mode) {
        case 0: e = go<0, 0>(nblk, s, gd, starts, n, ch, cl, bm); if (e == cudaSuccess) e = go<1, 0>(nblk, s, gd, starts, n, eh, el, bm); break;
        case 1: e = go<0, 1>(nblk, s, gd, starts, n, ch, cl, bm); if (e == cudaSuccess) e = go<1, 1>(nblk, s, gd, starts, n, eh, el, bm); break;
        default: e = go<0, 2>(nblk, s, gd, starts, n, ch, cl, bm); if (e == cudaSuccess) e = go<1, 2>(nblk, s, gd, starts, n, eh, el, bm); break;
    }
    return e;
}
