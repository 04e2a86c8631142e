// Row DCT passes for row lengths N that are not powers of two (64 < N <= 8192):
// the same row-pair structure as the power-of-two kernels (two real rows are
// one complex sequence, Makhoul's reordering is a scatter/gather through
// shared memory), with the length-N DFT done by Bluestein on the register FFT
// of length M >= 2N - 1, a power of two or three times one (unw_bluestein.cuh).
// M / 16 threads per CTA; the CTA loops over row pairs.
#include "unw_bluestein.cuh"
#include "unw_rowops.cuh"
#include "unw_kernels.h"

namespace {

template <int T>
constexpr int bl_min_blocks() { return T >= 1024 ? 1 : (1024 / T > 16 ? 16 : 1024 / T); }

__device__ __forceinline__ float4 ld4v(const float* __restrict__ a, size_t o) {
    return *reinterpret_cast<const float4*>(a + o);
}
__device__ __forceinline__ void st4v(float* __restrict__ a, size_t o, float4 v) {
    *reinterpret_cast<float4*>(a + o) = v;
}
__device__ __forceinline__ float f4at(const float4& v, int c) {
    return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}

// x += alpha p, r -= alpha Ap at columns j..j+3 of row i (the reference's PCG
// update, utils_unwrap2d.py:1445-1459, same operations as rowfwd_value mode 2;
// x is the PCG correction D).
// Rows are 128-byte aligned with a pitch of whole float4 groups, so a group
// starting below W stays inside the row; columns >= W are updated but do not
// enter the norms.
__device__ __forceinline__ float4 upd4(const GridDev& G, float* __restrict__ U, const float* __restrict__ pk,
                                       float alpha, int i, int j, int W, double (&acc)[2]) {
    const size_t o = (size_t)i * G.P + j;
    const float4 x = ld4v(U, o), p = ld4v(pk, o), r = ld4v(G.r, o), ap = ld4v(G.Ap, o);
    float4 xn, rn;
    xn.x = fmaf(alpha, p.x, x.x); xn.y = fmaf(alpha, p.y, x.y);
    xn.z = fmaf(alpha, p.z, x.z); xn.w = fmaf(alpha, p.w, x.w);
    rn.x = fmaf(-alpha, ap.x, r.x); rn.y = fmaf(-alpha, ap.y, r.y);
    rn.z = fmaf(-alpha, ap.z, r.z); rn.w = fmaf(-alpha, ap.w, r.w);
    st4v(U, o, xn);
    st4v(G.r, o, rn);
#pragma unroll
    for (int c = 0; c < 4; c++) {
        if (j + c < W) {
            const float v = f4at(rn, c);
            acc[0] += (double)v * (double)v;
            acc[1] += isfinite(f4at(xn, c)) ? 0.0 : 1.0;
        }
    }
    return rn;
}

// the PCG-start pass (mode 1, once per IRLS iteration) takes half the resident CTAs for
// the registers of the iterate pair's stencil
template <int T, int MODE>
constexpr int bl_rowf_blocks() {
    return MODE == 1 ? (bl_min_blocks<T>() / 2 > 0 ? bl_min_blocks<T>() / 2 : 1) : bl_min_blocks<T>();
}

template <class BL, int MODE>
__global__ void __launch_bounds__(BL::T, (bl_rowf_blocks<BL::T, MODE>())) k_rowf_bl(const GridDev* __restrict__ grids,
                                                                           const int* __restrict__ starts, int n,
                                                                           int it, int cgk) {
    constexpr int T = BL::T;
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowfwd_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int t = threadIdx.x;
    float* U = rowfwd_x<MODE>(G, it);  // x0 of this IRLS iteration, or D in mode 2
    const float* Lo = rowfwd_lo(G, it);
    const float* pk = (MODE == 2) ? G.p0 : nullptr;
    const float alpha = (MODE == 2) ? st->alpha : 0.f;
    const float2* __restrict__ dw = G.prow.dctw;
    double acc[2] = {0.0, 0.0};
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
        const int i0 = 2 * pair, i1 = i0 + 1;
        const bool has1 = i1 < H;
        __syncthreads();  // previous row pair's reads of sm are done
        if (MODE == 2) {
            for (int j = 4 * t; j < W; j += 4 * T) {
                const float4 a = upd4(G, U, pk, alpha, i0, j, W, acc);
                const float4 b = has1 ? upd4(G, U, pk, alpha, i1, j, W, acc) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (j + c < W) sm[BL::pos(mk_perm(j + c, W))] = make_float2(f4at(a, c), f4at(b, c));
            }
        } else {
            for (int j = t; j < W; j += T) {
                const float a = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i0, j, acc);
                const float b = has1 ? rowfwd_value<MODE>(G, U, Lo, pk, alpha, i1, j, acc) : 0.f;
                sm[BL::pos(mk_perm(j, W))] = make_float2(a, b);
            }
        }
        __syncthreads();
        BL::dft(sm, t, W, G.prow);
        // two real rows from one complex DFT, then X_k = Re(exp(-i pi k/2W) V_k)
        float* __restrict__ Ta = G.T + (size_t)i0 * P;
        float* __restrict__ Tb = G.T + (size_t)i1 * P;
        for (int k = t; k < W; k += T) {
            const float2 C = sm[BL::pos(k)];
            const float2 Cm = sm[BL::pos(k == 0 ? 0 : W - k)];
            const float2 w = __ldg(&dw[k]);
            const float2 Va = make_float2(C.x + Cm.x, C.y - Cm.y);
            const float2 Vb = make_float2(C.y + Cm.y, Cm.x - C.x);
            Ta[k] = w.x * Va.x - w.y * Va.y;
            if (has1) Tb[k] = w.x * Vb.x - w.y * Vb.y;
        }
    }
    if (MODE == 0 || MODE == 3) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowfwd_finalize<MODE>(st, acc);
    }
}

template <class BL, int MODE>
__global__ void __launch_bounds__(BL::T, bl_min_blocks<BL::T>()) k_rowi_bl(const GridDev* __restrict__ grids,
                                                                           const int* __restrict__ starts, int n) {
    constexpr int T = BL::T;
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowinv_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int t = threadIdx.x;
    const float2* __restrict__ dw = G.prow.dctw;
    const float beta = MODE == 2 ? st->beta : 0.f;
    double acc[2] = {0.0, 0.0};
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
        const int i0 = 2 * pair, i1 = i0 + 1;
        const bool has1 = i1 < H;
        const float* __restrict__ Ta = G.T + (size_t)i0 * P;
        const float* __restrict__ Tb = G.T + (size_t)i1 * P;
        __syncthreads();  // previous row pair's reads of sm are done
        // DCT-III pre-twiddle: V'_k = conj(w_k) (Y_k - i Y_{W-k}), Y_W = 0; store conj(C')
        for (int k = t; k < W; k += T) {
            const float ya = Ta[k], yb = has1 ? Tb[k] : 0.f;
            const float yam = k ? Ta[W - k] : 0.f;
            const float ybm = (k && has1) ? Tb[W - k] : 0.f;
            const float2 wc = cconj(__ldg(&dw[k]));
            const float2 Pa = cmul(wc, make_float2(ya, -yam));
            const float2 Pb = cmul(wc, make_float2(yb, -ybm));
            sm[BL::pos(k)] = cconj(make_float2(Pa.x - Pb.y, Pa.y + Pb.x));
        }
        __syncthreads();
        BL::dft(sm, t, W, G.prow);
        if (MODE == 2) {
            // p = z + beta p in float4 groups (columns >= W of a group are padding)
            for (int j = 4 * t; j < W; j += 4 * T) {
                float za[4], zb[4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float2 v = j + c < W ? sm[BL::pos(mk_perm(j + c, W))] : make_float2(0.f, 0.f);
                    za[c] = v.x;
                    zb[c] = -v.y;
                }
                const size_t oa = (size_t)i0 * P + j;
                const float4 pa = ld4v(G.p0, oa);
                st4v(G.p0, oa, make_float4(fadd(fmul(pa.x, beta), za[0]), fadd(fmul(pa.y, beta), za[1]),
                                           fadd(fmul(pa.z, beta), za[2]), fadd(fmul(pa.w, beta), za[3])));
                if (has1) {
                    const size_t ob = oa + P;
                    const float4 pb = ld4v(G.p0, ob);
                    st4v(G.p0, ob, make_float4(fadd(fmul(pb.x, beta), zb[0]), fadd(fmul(pb.y, beta), zb[1]),
                                               fadd(fmul(pb.z, beta), zb[2]), fadd(fmul(pb.w, beta), zb[3])));
                }
            }
        } else {
            for (int j = t; j < W; j += T) {
                const float2 v = sm[BL::pos(mk_perm(j, W))];
                rowinv_store<MODE>(G, i0, j, v.x, beta, acc);
                if (has1) rowinv_store<MODE>(G, i1, j, -v.y, beta, acc);
            }
        }
    }
    if (MODE != 0) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowinv_finalize_initu(st, acc);
    }
}

template <class BL>
cudaError_t rowf_bl_m(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n, int it, int cgk) {
    const size_t smem = sizeof(float2) * BL::SLOTS;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, BL::T, smem, s>>>(gd, st, n, it, cgk);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_rowf_bl<BL, 0>);
        case 1: return go(k_rowf_bl<BL, 1>);
        case 2: return go(k_rowf_bl<BL, 2>);
        default: return go(k_rowf_bl<BL, 3>);
    }
}

template <class BL>
cudaError_t rowi_bl_m(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n) {
    const size_t smem = sizeof(float2) * BL::SLOTS;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, BL::T, smem, s>>>(gd, st, n);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_rowi_bl<BL, 0>);
        case 1: return go(k_rowi_bl<BL, 1>);
        case 2: return go(k_rowi_bl<BL, 2>);
        default: return go(k_rowi_bl<BL, 3>);
    }
}

}  // namespace

// Bluestein lengths: powers of two 256..16384 and three times powers of two 768..12288
#define UNW_BL_SWITCH(M, CALL)                    \
    switch (M) {                                  \
        case 256: return CALL(BlP2<256>);         \
        case 512: return CALL(BlP2<512>);         \
        case 1024: return CALL(BlP2<1024>);       \
        case 2048: return CALL(BlP2<2048>);       \
        case 4096: return CALL(BlP2<4096>);       \
        case 8192: return CALL(BlP2<8192>);       \
        case 16384: return CALL(BlP2<16384>);     \
        case 768: return CALL(BlMix3<256>);       \
        case 1536: return CALL(BlMix3<512>);      \
        case 3072: return CALL(BlMix3<1024>);     \
        case 6144: return CALL(BlMix3<2048>);     \
        case 12288: return CALL(BlMix3<4096>);    \
        default: return cudaErrorInvalidValue;    \
    }

cudaError_t unw_launch_rowf_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n, int it, int cgk) {
    if (nblk <= 0) return cudaSuccess;
#define CALL(BB) rowf_bl_m<BB>(mode, nblk, s, gd, starts, n, it, cgk)
    UNW_BL_SWITCH(M, CALL)
#undef CALL
}

cudaError_t unw_launch_rowi_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n) {
    if (nblk <= 0) return cudaSuccess;
#define CALL(BB) rowi_bl_m<BB>(mode, nblk, s, gd, starts, n)
    UNW_BL_SWITCH(M, CALL)
#undef CALL
}
