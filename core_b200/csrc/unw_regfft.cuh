// Register-resident Stockham FFT for power-of-two lengths N (256..16384).
//
// N/16 threads cooperate on one sequence; thread t holds the 16 elements
// x[t + (N/16) q], q = 0..15, on entry, and X[t + (N/16) q] on exit (the same
// "stride-T" layout, so the first pass reads registers and the last pass
// leaves the spectrum in registers).  Passes are radix 16 except a final
// radix 2/4/8 pass when log2(N) is not a multiple of 4.  Between passes the
// data goes through shared memory with one padding slot per 16 entries, which
// makes every exchange pattern free of bank conflicts for 8-byte accesses.
// Everything is resolved at compile time: no integer division, no dynamic
// register indexing.
#pragma once
#include "unw_fft.cuh"

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n / 2); }

template <int N>
struct RegFft {
    static_assert((N & (N - 1)) == 0 && N >= 256 && N <= 16384, "power of two in [256, 16384]");
    static constexpr int LOG = ilog2c(N);
    static constexpr int T = N / 16;              // threads per sequence
    static constexpr int NP16 = LOG / 4;          // radix-16 passes
    static constexpr int REM = LOG % 4;           // log2 of the final small radix (0 = none)
    static constexpr int NPASS = NP16 + (REM ? 1 : 0);
    static constexpr int SMEM = N + N / 16;       // float2 slots per sequence
    // distance between sequences sharing a CTA: SMEM + 8 float2, so that lanes of
    // two sequences at the same position fall on different banks (16 words apart)
    static constexpr int SEQ_STRIDE = SMEM + 8;
};

// Multiplies w[r] by w1^r, r = 1..R-1, from a single table twiddle w1: powers
// by squaring (w2, w4, w8) and one extra product each, so every power carries
// at most a few roundings (relative error below 1e-6).
template <int R>
__device__ __forceinline__ void twiddle_row(float2* w, float2 w1) {
    float2 p[R];
    p[1] = w1;
    if (R > 2) p[2] = cmul(w1, w1);
    if (R > 3) p[3] = cmul(p[2], w1);
    if (R > 4) {
        p[4] = cmul(p[2], p[2]);
        p[5] = cmul(p[4], w1);
        p[6] = cmul(p[4], p[2]);
        p[7] = cmul(p[4], p[3]);
    }
    if (R > 8) {
        p[8] = cmul(p[4], p[4]);
#pragma unroll
        for (int r = 9; r < R; r++) p[r] = cmul(p[8], p[r - 8]);
    }
#pragma unroll
    for (int r = 1; r < R; r++) w[r] = cmul(w[r], p[r]);
}

// One Stockham pass of radix R with NS = product of earlier radices.
// Butterfly j = t + b*T (b < 16/R) reads elements j + r*(N/R) and writes
// (j - k)*R + k + r*NS, k = j mod NS.  The twiddle table holds exp(-2 pi i m / (N*TS)):
// TS > 1 lets a length-N transform use the table of a TS times longer one.
template <int N, int R, int NS, bool FIRST, bool LAST, int TS = 1>
__device__ __forceinline__ void reg_pass(float2 (&v)[16], float2* __restrict__ sm, int t,
                                         const float2* __restrict__ tw) {
    constexpr int T = N / 16;
    constexpr int NB = 16 / R;
    constexpr int NR = N / R;
    constexpr int S = N / (NS * R);
    // padded addresses with compile-time strides: pad16(a + 16 c) = pad16(a) + 17 c
    static_assert(T % 16 == 0 && NR % 16 == 0, "strides must be multiples of 16");
    float2 w[NB][R];
    const int rd = pad16(t);
#pragma unroll
    for (int b = 0; b < NB; b++) {
#pragma unroll
        for (int r = 0; r < R; r++) {
            if (FIRST) w[b][r] = v[b + r * NB];
            else w[b][r] = sm[rd + b * (T + T / 16) + r * (NR + NR / 16)];
        }
    }
    if (!FIRST) __syncthreads();  // every read of this exchange done before it is overwritten
#pragma unroll
    for (int b = 0; b < NB; b++) {
        const int j = t + b * T;
        const int k = j & (NS - 1);
        if (NS > 1) twiddle_row<R>(w[b], __ldg(&tw[k * S * TS]));
        Dft<R>::run(w[b]);
        if (LAST) {
#pragma unroll
            for (int r = 0; r < R; r++) v[b + r * NB] = w[b][r];
        } else {
            const int base = (j - k) * R + k;
            if (NS == 1) {
                static_assert(NS > 1 || R == 16, "first pass is radix 16");
                // pad16(16 j + r) = 17 j + r for r < 16
#pragma unroll
                for (int r = 0; r < R; r++) sm[17 * j + r] = w[b][r];
            } else {
                const int wb = pad16(base);
#pragma unroll
                for (int r = 0; r < R; r++) sm[wb + r * (NS + NS / 16)] = w[b][r];
            }
        }
    }
    if (!LAST) __syncthreads();
}

template <int N, int P, int NS>
__device__ __forceinline__ void reg_fft_rec(float2 (&v)[16], float2* sm, int t, const float2* tw) {
    if constexpr (P < RegFft<N>::NPASS) {
        constexpr int R = (P < RegFft<N>::NP16) ? 16 : (1 << RegFft<N>::REM);
        reg_pass<N, R, NS, P == 0, P == RegFft<N>::NPASS - 1>(v, sm, t, tw);
        reg_fft_rec<N, P + 1, NS * R>(v, sm, t, tw);
    }
}

template <int N, int P, int NS, int TS = 1>
__device__ __forceinline__ void smem_fft_rec(float2* sm, int t, const float2* tw) {
    if constexpr (P < RegFft<N>::NPASS) {
        constexpr int R = (P < RegFft<N>::NP16) ? 16 : (1 << RegFft<N>::REM);
        float2 v[16];
        reg_pass<N, R, NS, false, false, TS>(v, sm, t, tw);
        smem_fft_rec<N, P + 1, NS * R, TS>(sm, t, tw);
    }
}

template <int N, int P, int NS, bool IN_REG, bool OUT_REG>
__device__ __forceinline__ void io_fft_rec(float2 (&v)[16], float2* sm, int t, const float2* tw) {
    if constexpr (P < RegFft<N>::NPASS) {
        constexpr int R = (P < RegFft<N>::NP16) ? 16 : (1 << RegFft<N>::REM);
        reg_pass<N, R, NS, IN_REG && P == 0, OUT_REG && P == RegFft<N>::NPASS - 1>(v, sm, t, tw);
        io_fft_rec<N, P + 1, NS * R, IN_REG, OUT_REG>(v, sm, t, tw);
    }
}

// Forward FFT with the input in registers (stride-T layout) or in shared memory
// (natural order), and the output likewise; the other side goes through `sm`.
template <int N, bool IN_REG, bool OUT_REG>
__device__ __forceinline__ void io_fft(float2 (&v)[16], float2* sm, int t, const float2* tw) {
    io_fft_rec<N, 0, 1, IN_REG, OUT_REG>(v, sm, t, tw);
}

// Forward FFT of the sequence held in shared memory (natural order, padded
// addresses pad16(i)), result in place.  Registers are used only inside each
// pass.  The caller synchronises before the call (inputs written) and the
// result is visible to all threads on return.
template <int N, int TS = 1>
__device__ __forceinline__ void smem_fft(float2* sm, int t, const float2* tw) {
    smem_fft_rec<N, 0, 1, TS>(sm, t, tw);
}

// Forward FFT (exp(-2 pi i nk/N)) in place in the stride-T register layout.
// `sm` (RegFft<N>::SMEM float2) must not be read by other threads of this
// sequence while the call runs; the caller synchronises before reusing it.
template <int N>
__device__ __forceinline__ void reg_fft(float2 (&v)[16], float2* sm, int t, const float2* tw) {
    reg_fft_rec<N, 0, 1>(v, sm, t, tw);
}

// FFT position m of the Makhoul reordering holds source sample n(m).
template <int N>
__device__ __forceinline__ int mk_src(int m) {
    return m < N / 2 ? 2 * m : 2 * N - 1 - 2 * m;
}
