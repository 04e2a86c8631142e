// Length-N DFT for lengths that are not powers of two, by Bluestein's chirp-z
// algorithm (L. Bluestein, IEEE Trans. Audio Electroacoust. 18(4), 1970) on the
// register radix-16 FFT of a power-of-two length M >= 2N - 1:
//   X_k = conj(c_k) * sum_m (x_m conj(c_m)) c_{k-m},  c_m = exp(i pi m^2 / N),
// the convolution done as FFT_M, a product with the precomputed spectrum of the
// chirp filter (scaled by 1/M), and a second forward FFT of the conjugate.
// Every DCT pass of a non-power-of-two axis runs on this, so those axes use
// the same conflict-free register/shared-memory FFT as the power-of-two ones.
#pragma once
#include "unw_regfft.cuh"

// x_m in sm[pad16(m)], m < N (written and synchronised by the caller) ->
// X_k in sm[pad16(k)], k < N, synchronised on return.  M / 16 threads per
// sequence, t = this thread's index within its sequence; every thread of the
// CTA must call (the FFT passes synchronise the CTA).
template <int M>
__device__ __forceinline__ void blue_fft(float2* __restrict__ sm, int t, int N, const DctPlanDev& P) {
    constexpr int T = M / 16;
    const float2* __restrict__ ch = P.chirp;
    const float2* __restrict__ hs = P.hspec;
    for (int m = t; m < M; m += T) {
        const int a = pad16(m);
        sm[a] = m < N ? cmul(sm[a], cconj(__ldg(&ch[m]))) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 v[16];
    io_fft<M, false, true>(v, sm, t, P.fft.tw);
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = cconj(cmul(v[q], __ldg(&hs[t + T * q])));
    // the last pass above synchronised after its reads: sm may be overwritten
    io_fft<M, true, false>(v, sm, t, P.fft.tw);
    for (int k = t; k < N; k += T) {
        const int a = pad16(k);
        sm[a] = cmul(cconj(sm[a]), cconj(__ldg(&ch[k])));
    }
    __syncthreads();
}
