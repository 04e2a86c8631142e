// Spectral step of the power-of-two column pass (column DCT-II spectrum -> scaling by
// -1/(4 H W lambda) -> DCT-III pre-twiddle, with r.z by Parseval), shared by the plain-load and
// the TMA-staged column kernels.  The spectrum of the column pair sits in `sms` (natural order,
// padded addresses) and is overwritten in place by the pre-twiddled input of the inverse FFT.
#pragma once
#include "unw_regfft.cuh"
#include "unw_rowops.cuh"

#ifndef UNW_COLSPEC_UNROLL
#define UNW_COLSPEC_UNROLL 2
#endif

template <int N, int MODE>
__device__ __forceinline__ void col_spectral_k(float2* __restrict__ sms, int k, const float2* __restrict__ dw,
                                               const float* __restrict__ sH, float ca, float cb, bool ja0,
                                               bool hasb, float negs, double& rz) {
    const int km = (N - k) & (N - 1);
    const float2 C = sms[pad16(k)], Cm = sms[pad16(km)];
    const float2 wk = __ldg(&dw[k]), wm = __ldg(&dw[km]);
    const float ck = __ldg(&sH[k]), cm = __ldg(&sH[km]);
    float2 ok, om;
    col_spectral_pair<(MODE >= 1)>(C, Cm, k, km, wk, wm, ck, cm, ca, cb, ja0, hasb, negs, ok, om, rz);
    if (km != k) sms[pad16(km)] = om;
    sms[pad16(k)] = ok;
}

template <int N, int MODE>
__device__ __forceinline__ void col_spectral_p2(float2* __restrict__ sms, int t, const float2* __restrict__ dw,
                                                const float* __restrict__ sH, float ca, float cb, bool ja0,
                                                bool hasb, float negs, double& rz) {
    constexpr int T = N / 16;
#if UNW_COLSPEC_UNROLL
    // thread t owns the frequencies k = t + T i with their mirrors N - k: i < 8 for every
    // thread (k < N/2) and k = N/2 for thread 0 alone, after the others (the order of a loop
    // over k, so r.z accumulates in the same order).  The fixed trip count lets the table
    // loads of the next frequencies issue before the current ones are used.
    constexpr int U = UNW_COLSPEC_UNROLL;
#pragma unroll U
    for (int i = 0; i < 8; i++) col_spectral_k<N, MODE>(sms, t + T * i, dw, sH, ca, cb, ja0, hasb, negs, rz);
    if (t == 0) col_spectral_k<N, MODE>(sms, N / 2, dw, sH, ca, cb, ja0, hasb, negs, rz);
#else
    for (int k = t; k <= N / 2; k += T) col_spectral_k<N, MODE>(sms, k, dw, sH, ca, cb, ja0, hasb, negs, rz);
#endif
}
