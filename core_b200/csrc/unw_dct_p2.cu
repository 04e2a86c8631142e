// DCT passes for power-of-two grid dimensions on the register/shared-memory
// radix-16 FFT (unw_regfft.cuh).
//
// Row passes: one CTA of N/16 threads per pair of rows (two real rows are the
// real and imaginary parts of one complex length-N sequence).  Global I/O is
// coalesced float4; Makhoul's even/odd reordering (x_n sits at FFT position
// n/2 for even n, N-1-(n-1)/2 for odd n) is a scatter into / gather from
// shared memory, so it costs no extra pass over HBM.
//
// Column pass: NSEQ column pairs per CTA; forward FFT, spectral step on
// frequency pairs (k, N-k) in shared memory (DCT-II extraction, -1/lambda
// scaling, DCT-III pre-twiddle), inverse FFT, store.
#include "unw_regfft.cuh"
#include "unw_rowops.cuh"
#include "unw_colspec.cuh"
#include "unw_kernels.h"

template <int T>
constexpr int min_blocks() { return T >= 1024 ? 1 : (1024 / T > 16 ? 16 : 1024 / T); }

__device__ __forceinline__ int mk_pos(int n, int N) { return (n & 1) ? N - 1 - (n >> 1) : (n >> 1); }

__device__ __forceinline__ float4 ld4f(const float* __restrict__ a, size_t o) {
    return *reinterpret_cast<const float4*>(a + o);
}
__device__ __forceinline__ void st4f(float* __restrict__ a, size_t o, float4 v) {
    *reinterpret_cast<float4*>(a + o) = v;
}
__device__ __forceinline__ float f4get(const float4& v, int c) {
    return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}

// Four consecutive source values of row i (columns j..j+3) of the row-forward pass.
template <int MODE>
__device__ __forceinline__ float4 rowf_vals4(const GridDev& G, float* __restrict__ U, const float* __restrict__ Lo,
                                             const float* __restrict__ pk, float alpha, int i, int j,
                                             double (&acc)[2]) {
    const size_t o = (size_t)i * G.P + j;
    if (MODE == 2) {
        const float4 x = ld4f(U, o), p = ld4f(pk, o), r = ld4f(G.r, o), ap = ld4f(G.Ap, o);
        float4 xn, rn;
        xn.x = fmaf(alpha, p.x, x.x); xn.y = fmaf(alpha, p.y, x.y);
        xn.z = fmaf(alpha, p.z, x.z); xn.w = fmaf(alpha, p.w, x.w);
        rn.x = fmaf(-alpha, ap.x, r.x); rn.y = fmaf(-alpha, ap.y, r.y);
        rn.z = fmaf(-alpha, ap.z, r.z); rn.w = fmaf(-alpha, ap.w, r.w);
        st4f(U, o, xn);
        st4f(G.r, o, rn);
        acc[0] += (double)rn.x * rn.x + (double)rn.y * rn.y + (double)rn.z * rn.z + (double)rn.w * rn.w;
        acc[1] += (isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z) && isfinite(xn.w)) ? 0.0 : 1.0;
        return rn;
    } else if (MODE == 3) {
        return ld4f(G.r, o);
    } else if (MODE == 1) {
        // r = b - A x0 at columns j..j+3, neighbour differences from the pair (rowfwd_value mode 1)
        const int H = G.H, W = G.W, P = G.P;
        const float4 x4 = ld4f(U, o), l4 = ld4f(Lo, o), b4 = ld4f(G.b, o), wx4 = ld4f(G.wIx, o), wy4 = ld4f(G.wIy, o);
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 xu4 = i > 0 ? ld4f(U, o - P) : z4, lu4 = i > 0 ? ld4f(Lo, o - P) : z4;
        const float4 wyu4 = i > 0 ? ld4f(G.wIy, o - P) : z4;
        const float4 xd4 = i < H - 1 ? ld4f(U, o + P) : z4, ld4 = i < H - 1 ? ld4f(Lo, o + P) : z4;
        const float xl = j > 0 ? U[o - 1] : 0.f, ll = j > 0 ? Lo[o - 1] : 0.f;
        const float wxl = j > 0 ? G.wIx[o - 1] : 0.f;
        const float xr = j + 4 < W ? U[o + 4] : 0.f, lr = j + 4 < W ? Lo[o + 4] : 0.f;
        const double xs[6] = {pair_val(xl, ll), pair_val(x4.x, l4.x), pair_val(x4.y, l4.y), pair_val(x4.z, l4.z),
                              pair_val(x4.w, l4.w), pair_val(xr, lr)};
        const float wxs[5] = {wxl, wx4.x, wx4.y, wx4.z, wx4.w};
        float out[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int jj = j + q;
            const double xc = xs[q + 1];
            float res = 0.f;
            if (jj > 0) res = fsub(res, fmul(dpair_diff(xc, xs[q]), wxs[q]));
            if (jj < W - 1) res = fadd(res, fmul(dpair_diff(xs[q + 2], xc), wxs[q + 1]));
            if (i > 0) res = fsub(res, fmul(dpair_diff(xc, pair_val(f4get(xu4, q), f4get(lu4, q))), f4get(wyu4, q)));
            if (i < H - 1) res = fadd(res, fmul(dpair_diff(pair_val(f4get(xd4, q), f4get(ld4, q)), xc), f4get(wy4, q)));
            const float val = fsub(f4get(b4, q), -res);
            out[q] = val;
            acc[0] += isfinite(val) ? 0.0 : 1.0;
            acc[1] += (double)val * (double)val;
        }
        const float4 r4 = make_float4(out[0], out[1], out[2], out[3]);
        st4f(G.r, o, r4);
        st4f(G.D, o, z4);
        return r4;
    } else {
        float4 v;
        v.x = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i, j, acc);
        v.y = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i, j + 1, acc);
        v.z = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i, j + 2, acc);
        v.w = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i, j + 3, acc);
        return v;
    }
}

// The PCG-start pass (mode 1) forms b - A x0 from the iterate pair (eleven float4 rows
// in flight): it runs once per IRLS iteration and takes half the resident CTAs for the
// registers that keep it from spilling.
template <int T, int MODE>
constexpr int rowf_blocks() { return MODE == 1 ? (min_blocks<T>() / 2 > 0 ? min_blocks<T>() / 2 : 1) : min_blocks<T>(); }

template <int N, int MODE>
__global__ void __launch_bounds__(N / 16, (rowf_blocks<N / 16, MODE>())) k_rowf_p2(const GridDev* __restrict__ grids,
                                                                         const int* __restrict__ starts, int n,
                                                                         int it, int cgk) {
    constexpr int T = N / 16;
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowfwd_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, P = G.P;
    const int t = threadIdx.x;
    float* U = rowfwd_x<MODE>(G, it);  // x0 of this IRLS iteration, or D in mode 2
    const float* Lo = rowfwd_lo(G, it);
    const float* pk = (MODE == 2) ? G.p0 : nullptr;
    const float alpha = (MODE == 2) ? st->alpha : 0.f;
    double acc[2] = {0.0, 0.0};
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
    const int i0 = 2 * pair, i1 = i0 + 1;
    const bool has1 = i1 < H;
    __syncthreads();  // previous row pair's reads of sm are done
#ifndef UNW_ROWF_UNROLL
#define UNW_ROWF_UNROLL 1
#endif
    if (MODE == 2 && UNW_ROWF_UNROLL) {
        // the thread's four 16-byte groups per row as one unrolled sequence (a fixed trip
        // count), so that the loads of later groups can be issued before earlier ones are used
#pragma unroll
        for (int m = 0; m < N / (4 * T); m++) {
            const int j = 4 * (t + m * T);
            const float4 a = rowf_vals4<MODE>(G, U, Lo, pk, alpha, i0, j, acc);
            const float4 b = has1 ? rowf_vals4<MODE>(G, U, Lo, pk, alpha, i1, j, acc) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 4; c++) sm[pad16(mk_pos(j + c, N))] = make_float2(f4get(a, c), f4get(b, c));
        }
    } else {
        for (int c4 = t; c4 < N / 4; c4 += T) {
            const int j = 4 * c4;
            const float4 a = rowf_vals4<MODE>(G, U, Lo, pk, alpha, i0, j, acc);
            const float4 b = has1 ? rowf_vals4<MODE>(G, U, Lo, pk, alpha, i1, j, acc) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int c = 0; c < 4; c++) sm[pad16(mk_pos(j + c, N))] = make_float2(f4get(a, c), f4get(b, c));
        }
    }
    __syncthreads();
    smem_fft<N>(sm, t, G.prow.fft.tw);
    // two real rows from one complex DFT, then X_k = Re(exp(-i pi k/2N) V_k)
    const float2* __restrict__ dw = G.prow.dctw;
    float* __restrict__ Ta = G.T + (size_t)i0 * P;
    float* __restrict__ Tb = G.T + (size_t)i1 * P;
    for (int c4 = t; c4 < N / 4; c4 += T) {
        float xa[4], xb[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = 4 * c4 + c;
            const float2 C = sm[pad16(k)];
            const float2 Cm = sm[pad16((N - k) & (N - 1))];
            const float2 w = __ldg(&dw[k]);
            const float2 Va = make_float2(C.x + Cm.x, C.y - Cm.y);
            const float2 Vb = make_float2(C.y + Cm.y, Cm.x - C.x);
            xa[c] = w.x * Va.x - w.y * Va.y;
            xb[c] = w.x * Vb.x - w.y * Vb.y;
        }
        st4f(Ta, 4 * c4, make_float4(xa[0], xa[1], xa[2], xa[3]));
        if (has1) st4f(Tb, 4 * c4, make_float4(xb[0], xb[1], xb[2], xb[3]));
    }
    }
    if (MODE == 0 || MODE == 3) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowfwd_finalize<MODE>(st, acc);
    }
}

// Epilogue of the row-inverse pass for columns j..j+3 of row i.
template <int MODE>
__device__ __forceinline__ void rowi_store4(const GridDev& G, int i, int j, float4 z, float beta,
                                            double (&acc)[2]) {
    const size_t o = (size_t)i * G.P + j;
    if (MODE == 3) {
        st4f(G.z, o, z);
    } else if (MODE == 0) {
        float4 u;
        u.x = isfinite(z.x) ? z.x : 0.f; u.y = isfinite(z.y) ? z.y : 0.f;
        u.z = isfinite(z.z) ? z.z : 0.f; u.w = isfinite(z.w) ? z.w : 0.f;
        acc[1] += (isfinite(z.x) && isfinite(z.y) && isfinite(z.z) && isfinite(z.w)) ? 0.0 : 1.0;
        st4f(G.U0, o, u);
        const uchar4 v = *reinterpret_cast<const uchar4*>(G.valid + o);
        acc[0] += (double)(u.x * (v.x ? 1.f : 0.f)) + (double)(u.y * (v.y ? 1.f : 0.f)) +
                  (double)(u.z * (v.z ? 1.f : 0.f)) + (double)(u.w * (v.w ? 1.f : 0.f));
    } else if (MODE == 1) {
        st4f(G.p0, o, z);
    } else {
        const float4 p = ld4f(G.p0, o);
        st4f(G.p0, o, make_float4(fadd(fmul(p.x, beta), z.x), fadd(fmul(p.y, beta), z.y),
                                  fadd(fmul(p.z, beta), z.z), fadd(fmul(p.w, beta), z.w)));
    }
}

#ifndef UNW_ROWI_STAGED
#define UNW_ROWI_STAGED 1
#endif
#ifndef UNW_ROWI_REGIN
#define UNW_ROWI_REGIN 1
#endif
#ifndef UNW_ROWI_QB
#define UNW_ROWI_QB 4
#endif
template <int N, int MODE>
__global__ void __launch_bounds__(N / 16, min_blocks<N / 16>()) k_rowi_p2(const GridDev* __restrict__ grids,
                                                                         const int* __restrict__ starts, int n) {
    constexpr int T = N / 16;
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowinv_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, P = G.P;
    const int t = threadIdx.x;
    const float2* __restrict__ dw = G.prow.dctw;
    const float beta = MODE == 2 ? st->beta : 0.f;
    double acc[2] = {0.0, 0.0};
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
    const int i0 = 2 * pair, i1 = i0 + 1;
    const bool has1 = i1 < H;
    const float* __restrict__ Ta = G.T + (size_t)i0 * P;
    const float* __restrict__ Tb = G.T + (size_t)i1 * P;
    if (MODE == 2) {
        // the epilogue reads p of these rows after the FFT: start them towards L2 now
        const float* ra = G.p0 + (size_t)i0 * P;
        for (int c = t * 32; c < N; c += T * 32) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(ra + c));
            if (has1) asm volatile("prefetch.global.L2 [%0];" ::"l"(ra + P + c));
        }
    }
    if constexpr (UNW_ROWI_REGIN && MODE == 2) {
    // DCT-III pre-twiddle formed straight into the register layout of the FFT's first pass:
    // thread t holds k = t + T q (q = 0..15) and reads Y_k and its mirror Y_{N-k} of both rows
    // (each a coalesced warp-wide run of the row), V'_k = conj(w_k) (Y_k - i Y_{N-k}), Y_N = 0;
    // v[q] = conj(C'_k).  Same arithmetic per element as the staged form below.
    float2 v[16];
#pragma unroll
    for (int h = 0; h < 16 / UNW_ROWI_QB; h++) {
        float ya[UNW_ROWI_QB], yam[UNW_ROWI_QB], yb[UNW_ROWI_QB], ybm[UNW_ROWI_QB];
#pragma unroll
        for (int e = 0; e < UNW_ROWI_QB; e++) {
            const int k = t + (UNW_ROWI_QB * h + e) * T;
            ya[e] = Ta[k];
            yam[e] = k ? Ta[N - k] : 0.f;
            yb[e] = has1 ? Tb[k] : 0.f;
            ybm[e] = (has1 && k) ? Tb[N - k] : 0.f;
        }
#pragma unroll
        for (int e = 0; e < UNW_ROWI_QB; e++) {
            const int k = t + (UNW_ROWI_QB * h + e) * T;
            const float2 wk = cconj(__ldg(&dw[k]));
            const float2 Pa = cmul(wk, make_float2(ya[e], -yam[e]));
            const float2 Pb = cmul(wk, make_float2(yb[e], -ybm[e]));
            v[UNW_ROWI_QB * h + e] = cconj(make_float2(Pa.x - Pb.y, Pa.y + Pb.x));
        }
    }
    __syncthreads();  // previous row pair's reads of sm are done
    io_fft<N, true, false>(v, sm, t, G.prow.fft.tw);
    } else {
#if UNW_ROWI_STAGED
    // the row pair's T values: all eight 16-byte loads of a thread issued together, then
    // (Y_a[k], Y_b[k]) into sm[pad16(k)]
    float4 ya[N / (4 * T)], yb[N / (4 * T)];
#pragma unroll
    for (int m = 0; m < N / (4 * T); m++) {
        const int c4 = t + m * T;
        ya[m] = ld4f(Ta, 4 * c4);
        yb[m] = has1 ? ld4f(Tb, 4 * c4) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();  // previous row pair's reads of sm are done
#pragma unroll
    for (int m = 0; m < N / (4 * T); m++) {
        const int k = 4 * (t + m * T);
#pragma unroll
        for (int c = 0; c < 4; c++) sm[pad16(k + c)] = make_float2(f4get(ya[m], c), f4get(yb[m], c));
    }
    __syncthreads();
    // DCT-III pre-twiddle in place, one frequency pair (k, N-k) per step (both outputs read
    // only this pair): V'_k = conj(w_k) (Y_k - i Y_{N-k}), Y_N = 0; store conj(C')
    for (int k = t; k <= N / 2; k += T) {
        const int km = N - k;
        const float2 yk = sm[pad16(k)];
        const float2 ym = k ? sm[pad16(km)] : make_float2(0.f, 0.f);
        const float2 wk = cconj(__ldg(&dw[k]));
        const float2 Pa = cmul(wk, make_float2(yk.x, -ym.x));
        const float2 Pb = cmul(wk, make_float2(yk.y, -ym.y));
        if (k && km != k) {
            const float2 wm = cconj(__ldg(&dw[km]));
            const float2 Qa = cmul(wm, make_float2(ym.x, -yk.x));
            const float2 Qb = cmul(wm, make_float2(ym.y, -yk.y));
            sm[pad16(km)] = cconj(make_float2(Qa.x - Qb.y, Qa.y + Qb.x));
        }
        sm[pad16(k)] = cconj(make_float2(Pa.x - Pb.y, Pa.y + Pb.x));
    }
#else
    __syncthreads();  // previous row pair's reads of sm are done
    // DCT-III pre-twiddle: V'_k = conj(w_k) (Y_k - i Y_{N-k}), Y_N = 0; store conj(C')
    for (int c4 = t; c4 < N / 4; c4 += T) {
        const float4 ya = ld4f(Ta, 4 * c4);
        const float4 yb = has1 ? ld4f(Tb, 4 * c4) : make_float4(0.f, 0.f, 0.f, 0.f);
        // mirrors N-k of k = 4c4..4c4+3: N-4c4 (.x of the chunk at N-4c4, none for
        // c4 = 0) and N-4c4-1..N-4c4-3 (.w .z .y of the chunk at N-4c4-4)
        const float4 za = ld4f(Ta, N - 4 * c4 - 4);
        const float4 zb = has1 ? ld4f(Tb, N - 4 * c4 - 4) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float xa0 = c4 ? Ta[N - 4 * c4] : 0.f;
        const float xb0 = (c4 && has1) ? Tb[N - 4 * c4] : 0.f;
        const float ma[4] = {xa0, za.w, za.z, za.y};
        const float mb[4] = {xb0, zb.w, zb.z, zb.y};
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = 4 * c4 + c;
            const float yam = ma[c], ybm = mb[c];
            const float2 wc = cconj(__ldg(&dw[k]));
            const float2 Pa = cmul(wc, make_float2(f4get(ya, c), -yam));
            const float2 Pb = cmul(wc, make_float2(f4get(yb, c), -ybm));
            sm[pad16(k)] = cconj(make_float2(Pa.x - Pb.y, Pa.y + Pb.x));
        }
    }
#endif
    __syncthreads();
    smem_fft<N>(sm, t, G.prow.fft.tw);
    }
#if UNW_ROWI_STAGED
    if constexpr (MODE == 2) {
        // p = z + beta p: the thread's p loads (L2-prefetched above) all issued before the
        // first use
        float4 pa[N / (4 * T)], pb[N / (4 * T)];
#pragma unroll
        for (int m = 0; m < N / (4 * T); m++) {
            const size_t o = (size_t)i0 * P + 4 * (t + m * T);
            pa[m] = ld4f(G.p0, o);
            pb[m] = has1 ? ld4f(G.p0, o + P) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int m = 0; m < N / (4 * T); m++) {
            const int j = 4 * (t + m * T);
            float za[4], zb[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float2 v = sm[pad16(mk_pos(j + c, N))];
                za[c] = fadd(fmul(f4get(pa[m], c), beta), v.x);
                zb[c] = fadd(fmul(f4get(pb[m], c), beta), -v.y);
            }
            const size_t o = (size_t)i0 * P + j;
            st4f(G.p0, o, make_float4(za[0], za[1], za[2], za[3]));
            if (has1) st4f(G.p0, o + P, make_float4(zb[0], zb[1], zb[2], zb[3]));
        }
    } else
#endif
    {
        for (int c4 = t; c4 < N / 4; c4 += T) {
            const int j = 4 * c4;
            float za[4], zb[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float2 v = sm[pad16(mk_pos(j + c, N))];
                za[c] = v.x;
                zb[c] = -v.y;
            }
            rowi_store4<MODE>(G, i0, j, make_float4(za[0], za[1], za[2], za[3]), beta, acc);
            if (has1) rowi_store4<MODE>(G, i1, j, make_float4(zb[0], zb[1], zb[2], zb[3]), beta, acc);
        }
    }
    }
    if (MODE != 0) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowinv_finalize_initu(st, acc);
    }
}

// MODE 0: DCT initial solve (always runs); MODE 1 / 2: PCG (gated), also
// r.z by Parseval and its scalar step (col_finalize).
template <int N, int NSEQ, int MODE>
__global__ void __launch_bounds__(N / 16 * NSEQ, min_blocks<N / 16 * NSEQ>()) k_col_p2(
    const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    constexpr int T = N / 16;
    extern __shared__ float2 sm[];
    __shared__ double red[32];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (MODE >= 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const int s = threadIdx.x % NSEQ, t = threadIdx.x / NSEQ;
    float2* sms = sm + s * RegFft<N>::SEQ_STRIDE;
    float* __restrict__ Tm = G.T;
    const float2* __restrict__ tw = G.pcol.fft.tw;
    const float2* __restrict__ dw = G.pcol.dctw;
    const float* __restrict__ sH = G.sH;
    const float negs = -1.0f / (4.0f * (float)N * (float)W);
    const int nslab = (W + 2 * NSEQ - 1) / (2 * NSEQ);
    double acc[1] = {0.0};
    for (int slab = local; slab < nslab; slab += nct) {
    const int ja = 2 * NSEQ * slab + 2 * s;
    const bool hasa = ja < W, hasb = ja + 1 < W;
    const bool vec = hasb && !(P & 1);
    // FFT position m = t + T q reads source row 2m (q < 8) or 2N-1-2m (q >= 8):
    // rows lo + q*step and hi - (q-8)*step with step = 2T rows
    const size_t step = (size_t)(2 * T) * P;
    float* const lo = Tm + (size_t)(2 * t) * P + ja;
    float* const hi = Tm + (size_t)(N - 1 - 2 * t) * P + ja;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const float* a = q < 8 ? lo + q * step : hi - (q - 8) * step;
        float2 x = make_float2(0.f, 0.f);
        if (vec) x = *reinterpret_cast<const float2*>(a);
        else if (hasb) x = make_float2(a[0], a[1]);
        else if (hasa) x.x = a[0];
        v[q] = x;
    }
    __syncthreads();  // previous slab's reads of sm are done
    io_fft<N, true, false>(v, sms, t, tw);
    const float ca = hasa ? G.sW[ja] : 1.0f, cb = hasb ? G.sW[ja + 1] : 1.0f;
    col_spectral_p2<N, MODE>(sms, t, dw, sH, ca, cb, ja == 0, hasb, negs, acc[0]);
    __syncthreads();
    io_fft<N, false, true>(v, sms, t, tw);
#pragma unroll
    for (int q = 0; q < 16; q++) {
        float* a = q < 8 ? lo + q * step : hi - (q - 8) * step;
        if (vec) *reinterpret_cast<float2*>(a) = make_float2(v[q].x, -v[q].y);
        else if (hasb) { a[0] = v[q].x; a[1] = -v[q].y; }
        else if (hasa) a[0] = v[q].x;
    }
    }
    if (MODE == 0) return;
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) col_finalize<MODE>(st, acc[0]);
    }
}

// ------------------------------------------------------------------ launchers
template <int N>
static cudaError_t rowf_p2_n(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n, int it,
                             int cgk) {
    const size_t smem = sizeof(float2) * RegFft<N>::SMEM;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, N / 16, smem, s>>>(gd, st, n, it, cgk);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_rowf_p2<N, 0>);
        case 1: return go(k_rowf_p2<N, 1>);
        case 2: return go(k_rowf_p2<N, 2>);
        default: return go(k_rowf_p2<N, 3>);
    }
}

template <int N>
static cudaError_t rowi_p2_n(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n) {
    const size_t smem = sizeof(float2) * RegFft<N>::SMEM;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, N / 16, smem, s>>>(gd, st, n);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_rowi_p2<N, 0>);
        case 1: return go(k_rowi_p2<N, 1>);
        case 2: return go(k_rowi_p2<N, 2>);
        default: return go(k_rowi_p2<N, 3>);
    }
}

// column pairs per CTA: from N = 2048 up, UNW_COL_P2_THREADS threads (512: two pairs at
// N = 4096, 16-byte row segments; at least one pair, at most eight); below, four pairs,
// which gives short columns enough CTAs (measured on B200: at N = 1024, 18.8 us per launch
// against 27.0 us with eight pairs; at N = 512, 13.7 us against 16.5 us)
#ifndef UNW_COL_P2_THREADS
#define UNW_COL_P2_THREADS 512
#endif
template <int N>
constexpr int col_nseq_p2() {
    return N < 2048 ? 4
                    : (UNW_COL_P2_THREADS / (N / 16) < 1
                           ? 1
                           : (UNW_COL_P2_THREADS / (N / 16) > 8 ? 8 : UNW_COL_P2_THREADS / (N / 16)));
}

template <int N>
static cudaError_t col_p2_n(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n) {
    constexpr int NS = col_nseq_p2<N>();
    const size_t smem = sizeof(float2) * RegFft<N>::SEQ_STRIDE * NS;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, N / 16 * NS, smem, s>>>(gd, st, n);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_col_p2<N, NS, 0>);
        case 1: return go(k_col_p2<N, NS, 1>);
        default: return go(k_col_p2<N, NS, 2>);
    }
}

int unw_p2_col_nseq(int N) {
    switch (N) {
        case 256: return col_nseq_p2<256>();
        case 512: return col_nseq_p2<512>();
        case 1024: return col_nseq_p2<1024>();
        case 2048: return col_nseq_p2<2048>();
        case 4096: return col_nseq_p2<4096>();
        case 8192: return col_nseq_p2<8192>();
        case 16384: return col_nseq_p2<16384>();
        default: return 0;
    }
}

#define UNW_P2_SWITCH(N, CALL)                 \
    switch (N) {                               \
        case 256: return CALL(256);            \
        case 512: return CALL(512);            \
        case 1024: return CALL(1024);          \
        case 2048: return CALL(2048);          \
        case 4096: return CALL(4096);          \
        case 8192: return CALL(8192);          \
        case 16384: return CALL(16384);        \
        default: return cudaErrorInvalidValue; \
    }

cudaError_t unw_launch_rowf_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n, int it, int cgk) {
    if (nblk <= 0) return cudaSuccess;
#define CALL(NN) rowf_p2_n<NN>(mode, nblk, s, gd, starts, n, it, cgk)
    UNW_P2_SWITCH(N, CALL)
#undef CALL
}

cudaError_t unw_launch_rowi_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                               int n) {
    if (nblk <= 0) return cudaSuccess;
#define CALL(NN) rowi_p2_n<NN>(mode, nblk, s, gd, starts, n)
    UNW_P2_SWITCH(N, CALL)
#undef CALL
}

cudaError_t unw_launch_col_p2(int N, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                              int n) {
    if (nblk <= 0) return cudaSuccess;
#define CALL(NN) col_p2_n<NN>(mode, nblk, s, gd, starts, n)
    UNW_P2_SWITCH(N, CALL)
#undef CALL
}
