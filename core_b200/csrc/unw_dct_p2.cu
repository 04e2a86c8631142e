// DCT passes for power-of-two grid dimensions on the register-resident FFT.
//
// Row passes: one CTA of N/16 threads per pair of rows (two real rows are the
// real and imaginary parts of one complex length-N sequence).  Thread t
// handles FFT positions m = t + (N/16) q, whose source column is Makhoul's
// n(m) = 2m (m < N/2) or 2N-1-2m, so the even/odd reordering costs nothing:
// it is just the address each thread loads (and, for the inverse, stores).
//
// Column pass: NSEQ column pairs per CTA; forward FFT, spectral step
// (DCT-II extraction, -1/lambda scaling, DCT-III pre-twiddle) done in
// registers for k with C_{N-k} read from shared memory, inverse FFT, store.
#include "unw_regfft.cuh"
#include "unw_rowops.cuh"
#include "unw_kernels.h"

template <int N, int MODE>
__global__ void __launch_bounds__(N / 16) k_rowf_p2(const GridDev* __restrict__ grids,
                                                    const int* __restrict__ starts, int n, int it, int cgk) {
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
    const int i0 = 2 * local, i1 = i0 + 1;
    const bool has1 = i1 < H;
    const int t = threadIdx.x;
    float* U = (it & 1) ? G.U0 : G.U1;
    const float* pk = (MODE == 2) ? ((cgk & 1) ? G.p1 : G.p0) : nullptr;
    const float alpha = (MODE == 2) ? st->alpha : 0.f;
    double acc[2] = {0.0, 0.0};
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int j = mk_src<N>(t + T * q);
        const float a = rowfwd_value<MODE>(G, U, pk, alpha, i0, j, acc);
        const float b = has1 ? rowfwd_value<MODE>(G, U, pk, alpha, i1, j, acc) : 0.f;
        v[q] = make_float2(a, b);
    }
    reg_fft<N>(v, sm, t, G.prow.fft.tw);
#pragma unroll
    for (int q = 0; q < 16; q++) sm[pad16(t + T * q)] = v[q];
    __syncthreads();
    const float2* __restrict__ dw = G.prow.dctw;
    float* __restrict__ Ta = G.T + (size_t)i0 * P;
    float* __restrict__ Tb = G.T + (size_t)i1 * P;
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = t + T * q;
        const float2 C = v[q];
        const float2 Cm = sm[pad16((N - k) & (N - 1))];
        const float2 w = __ldg(&dw[k]);
        const float2 Va = make_float2(C.x + Cm.x, C.y - Cm.y);
        const float2 Vb = make_float2(C.y + Cm.y, Cm.x - C.x);
        Ta[k] = w.x * Va.x - w.y * Va.y;
        if (has1) Tb[k] = w.x * Vb.x - w.y * Vb.y;
    }
    if (MODE == 0 || MODE == 3) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowfwd_finalize<MODE>(st, acc);
    }
}

template <int N, int MODE>
__global__ void __launch_bounds__(N / 16) k_rowi_p2(const GridDev* __restrict__ grids,
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
    const int i0 = 2 * local, i1 = i0 + 1;
    const bool has1 = i1 < H;
    const int t = threadIdx.x;
    const float* __restrict__ Ta = G.T + (size_t)i0 * P;
    const float* __restrict__ Tb = G.T + (size_t)i1 * P;
    const float2* __restrict__ dw = G.prow.dctw;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = t + T * q;
        const int km = (N - k) & (N - 1);
        const float yak = Ta[k], ybk = has1 ? Tb[k] : 0.f;
        const float yam = k ? Ta[km] : 0.f, ybm = (k && has1) ? Tb[km] : 0.f;
        const float2 wc = cconj(__ldg(&dw[k]));
        const float2 Pa = cmul(wc, make_float2(yak, -yam));
        const float2 Pb = cmul(wc, make_float2(ybk, -ybm));
        v[q] = cconj(make_float2(Pa.x - Pb.y, Pa.y + Pb.x));
    }
    reg_fft<N>(v, sm, t, G.prow.fft.tw);
    double acc[2] = {0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int j = mk_src<N>(t + T * q);
        rowinv_store<MODE>(G, i0, j, v[q].x, acc);
        if (has1) rowinv_store<MODE>(G, i1, j, -v[q].y, acc);
    }
    if (MODE == 3) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowinv_finalize<MODE>(st, acc);
    }
}

// MODE 0: DCT initial solve (always runs); MODE 1: PCG (gated).
template <int N, int NSEQ, int MODE>
__global__ void __launch_bounds__(N / 16 * NSEQ) k_col_p2(const GridDev* __restrict__ grids,
                                                          const int* __restrict__ starts, int n) {
    constexpr int T = N / 16;
    extern __shared__ float2 sm[];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (MODE == 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int W = G.W, P = G.P;
    const int s = threadIdx.x % NSEQ, t = threadIdx.x / NSEQ;
    const int ja = 2 * NSEQ * local + 2 * s;
    const bool hasa = ja < W, hasb = ja + 1 < W;
    float2* sms = sm + s * RegFft<N>::SMEM;
    float* __restrict__ Tm = G.T;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const size_t o = (size_t)mk_src<N>(t + T * q) * P + ja;
        float2 x = make_float2(0.f, 0.f);
        if (hasb && !(P & 1)) x = *reinterpret_cast<const float2*>(Tm + o);
        else if (hasb) x = make_float2(Tm[o], Tm[o + 1]);
        else if (hasa) x.x = Tm[o];
        v[q] = x;
    }
    const float2* __restrict__ tw = G.pcol.fft.tw;
    reg_fft<N>(v, sms, t, tw);
#pragma unroll
    for (int q = 0; q < 16; q++) sms[pad16(t + T * q)] = v[q];
    __syncthreads();
    const float2* __restrict__ dw = G.pcol.dctw;
    const double* __restrict__ cH = G.cosH;
    const double ca = hasa ? G.cosW[ja] : 1.0, cb = hasb ? G.cosW[ja + 1] : 1.0;
    const float negs = -1.0f / (4.0f * (float)N * (float)W);
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = t + T * q;
        const int km = (N - k) & (N - 1);
        const float2 Cm = sms[pad16(km)];
        v[q] = col_spectral(v[q], Cm, k, km, __ldg(&dw[k]), __ldg(&dw[km]), cH[k], cH[km], ca, cb, ja == 0, hasb,
                            negs);
    }
    __syncthreads();
    reg_fft<N>(v, sms, t, tw);
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const size_t o = (size_t)mk_src<N>(t + T * q) * P + ja;
        if (hasb && !(P & 1)) *reinterpret_cast<float2*>(Tm + o) = make_float2(v[q].x, -v[q].y);
        else if (hasb) { Tm[o] = v[q].x; Tm[o + 1] = -v[q].y; }
        else if (hasa) Tm[o] = v[q].x;
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

// column pairs per CTA: 512 threads and ~70 KB of shared memory up to N = 8192
template <int N>
constexpr int col_nseq_p2() { return N >= 8192 ? 1 : (8192 / N > 8 ? 8 : 8192 / N); }

template <int N>
static cudaError_t col_p2_n(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n) {
    constexpr int NS = col_nseq_p2<N>();
    const size_t smem = sizeof(float2) * RegFft<N>::SMEM * NS;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, N / 16 * NS, smem, s>>>(gd, st, n);
        return cudaGetLastError();
    };
    return mode == 0 ? go(k_col_p2<N, NS, 0>) : go(k_col_p2<N, NS, 1>);
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

#define UNW_P2_SWITCH(N, CALL)          \
    switch (N) {                        \
        case 256: return CALL(256);     \
        case 512: return CALL(512);     \
        case 1024: return CALL(1024);   \
        case 2048: return CALL(2048);   \
        case 4096: return CALL(4096);   \
        case 8192: return CALL(8192);   \
        case 16384: return CALL(16384); \
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
