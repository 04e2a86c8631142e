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
// CTA must call (the FFT passes synchronise the CTA).  The data stays in shared
// memory between the steps (measured faster than carrying it in registers
// across the two FFTs, which spills at these thread counts).
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
    smem_fft<M>(sm, t, P.fft.tw);
    for (int m = t; m < M; m += T) {
        const int a = pad16(m);
        sm[a] = cconj(cmul(sm[a], __ldg(&hs[m])));
    }
    __syncthreads();
    smem_fft<M>(sm, t, P.fft.tw);
    for (int k = t; k < N; k += T) {
        const int a = pad16(k);
        sm[a] = cmul(cconj(sm[a]), cconj(__ldg(&ch[k])));
    }
    __syncthreads();
}

// Bluestein length M = 3 * M3 (M3 a power of two >= 256).  The two length-M FFTs
// are split into a radix-3 stage and three register FFTs of length M3, so
// that no permutation pass is needed:
//   FFT 1, decimation in frequency: natural order in three contiguous thirds ->
//     radix-3 butterflies across the thirds with twiddles W_M^{s m} -> three
//     FFTs of length M3 -> third s holds X_{3k+s} at index k;
//   the filter spectrum is applied in that order (index 3k + s);
//   FFT 2, decimation in time: third r holds the sub-sequence x_{3m+r} ->
//     three FFTs of length M3 -> radix-3 butterflies with W_M^{r k} ->
//     natural order in three contiguous thirds.
template <int M3>
__device__ __forceinline__ void blue_fft3(float2* __restrict__ sm, int t, int N, const DctPlanDev& P) {
    constexpr int M = 3 * M3;
    constexpr int T3 = M3 / 16, T = 3 * T3;
    constexpr int R = RegFft<M3>::SEQ_STRIDE;      // slots per third
    constexpr int L3 = ilog2c(M3);
    const float2* __restrict__ ch = P.chirp;
    const float2* __restrict__ hs = P.hspec;
    const float2* __restrict__ tw = P.fft.tw;       // exp(-2 pi i m / M), m < M
    const int grp = t / T3, tt = t - grp * T3;
    for (int m = t; m < M; m += T) {
        const int a = (m >> L3) * R + pad16(m & (M3 - 1));
        sm[a] = m < N ? cmul(sm[a], cconj(__ldg(&ch[m]))) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int m = t; m < M3; m += T) {
        const int a = pad16(m);
        float2 v[3] = {sm[a], sm[R + a], sm[2 * R + a]};
        Dft<3>::run(v);
        sm[a] = v[0];
        sm[R + a] = cmul(v[1], __ldg(&tw[m]));
        sm[2 * R + a] = cmul(v[2], __ldg(&tw[2 * m]));
    }
    __syncthreads();
    smem_fft<M3, 3>(sm + grp * R, tt, tw);
    for (int q = t; q < M; q += T) {
        const int s3 = q >> L3, k = q & (M3 - 1);
        const int a = s3 * R + pad16(k);
        sm[a] = cconj(cmul(sm[a], __ldg(&hs[3 * k + s3])));
    }
    __syncthreads();
    smem_fft<M3, 3>(sm + grp * R, tt, tw);
    for (int k = t; k < M3; k += T) {
        const int a = pad16(k);
        float2 v[3] = {sm[a], cmul(sm[R + a], __ldg(&tw[k])), cmul(sm[2 * R + a], __ldg(&tw[2 * k]))};
        Dft<3>::run(v);
        sm[a] = v[0];
        sm[R + a] = v[1];
        sm[2 * R + a] = v[2];
    }
    __syncthreads();
    for (int k = t; k < N; k += T) {
        const int a = (k >> L3) * R + pad16(k & (M3 - 1));
        sm[a] = cmul(cconj(sm[a]), cconj(__ldg(&ch[k])));
    }
    __syncthreads();
}

// The two Bluestein FFT shapes as one interface for the DCT kernels:
// threads per sequence, shared-memory slots per sequence (with the bank offset
// between sequences), the slot of natural index m, and the length-N DFT.
template <int M>
struct BlP2 {
    static constexpr int LEN = M;
    static constexpr int T = M / 16;
    static constexpr int SLOTS = RegFft<M>::SEQ_STRIDE;
    static __device__ __forceinline__ int pos(int m) { return pad16(m); }
    static __device__ __forceinline__ void dft(float2* sm, int t, int N, const DctPlanDev& P) {
        blue_fft<M>(sm, t, N, P);
    }
};

template <int M3>
struct BlMix3 {
    static constexpr int LEN = 3 * M3;
    static constexpr int T = 3 * (M3 / 16);
    static constexpr int R = RegFft<M3>::SEQ_STRIDE;
    static constexpr int SLOTS = 3 * R;
    static constexpr int L3 = ilog2c(M3);
    static __device__ __forceinline__ int pos(int m) { return (m >> L3) * R + pad16(m & (M3 - 1)); }
    static __device__ __forceinline__ void dft(float2* sm, int t, int N, const DctPlanDev& P) {
        blue_fft3<M3>(sm, t, N, P);
    }
};
