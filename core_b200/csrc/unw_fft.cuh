// Shared-memory mixed-radix FFT (Stockham autosort, radices 2,3,4,5,7,8,16)
// and the length-N DFT used by the DCT passes (direct, or Bluestein chirp-z
// for lengths with a prime factor above 7).
//
// All threads of a CTA cooperate on `nseq` sequences stored at
// buf + s*stride.  Each pass first reads every butterfly's inputs into
// registers, synchronises, then writes the outputs, so a pass runs in place
// with one shared buffer (no ping-pong copy).  EMAX bounds the complex
// elements a thread holds in one pass; the host picks (T, EMAX) so that
// nseq * n <= T * (EMAX/R)*R for every radix R of the plan.
#pragma once
#include "unw_internal.cuh"

// ------------------------------------------------------------ butterflies
// Forward DFT of R points in registers: X_k = sum_n v_n exp(-2*pi*i*n*k/R).
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)

__device__ __forceinline__ void bf2(float2& a, float2& b) {
    float2 t = a;
    a = make_float2(t.x + b.x, t.y + b.y);
    b = make_float2(t.x - b.x, t.y - b.y);
}

__device__ __forceinline__ void dft4(float2& v0, float2& v1, float2& v2, float2& v3) {
    float2 t0 = make_float2(v0.x + v2.x, v0.y + v2.y);
    float2 t1 = make_float2(v0.x - v2.x, v0.y - v2.y);
    float2 t2 = make_float2(v1.x + v3.x, v1.y + v3.y);
    float2 t3 = mul_mi(make_float2(v1.x - v3.x, v1.y - v3.y));
    v0 = make_float2(t0.x + t2.x, t0.y + t2.y);
    v2 = make_float2(t0.x - t2.x, t0.y - t2.y);
    v1 = make_float2(t1.x + t3.x, t1.y + t3.y);
    v3 = make_float2(t1.x - t3.x, t1.y - t3.y);
}

template <int R> struct Dft;

template <> struct Dft<2> {
    static __device__ __forceinline__ void run(float2* v) { bf2(v[0], v[1]); }
};
template <> struct Dft<4> {
    static __device__ __forceinline__ void run(float2* v) { dft4(v[0], v[1], v[2], v[3]); }
};
template <> struct Dft<8> {
    static __device__ __forceinline__ void run(float2* v) {
        const float c = 0.70710678118654752f;
        float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4(e0, e1, e2, e3);
        dft4(o0, o1, o2, o3);
        o1 = make_float2(c * (o1.x + o1.y), c * (o1.y - o1.x));   // * exp(-i pi/4)
        o2 = mul_mi(o2);                                            // * exp(-i pi/2)
        o3 = make_float2(c * (o3.y - o3.x), -c * (o3.x + o3.y));  // * exp(-3i pi/4)
        v[0] = make_float2(e0.x + o0.x, e0.y + o0.y); v[4] = make_float2(e0.x - o0.x, e0.y - o0.y);
        v[1] = make_float2(e1.x + o1.x, e1.y + o1.y); v[5] = make_float2(e1.x - o1.x, e1.y - o1.y);
        v[2] = make_float2(e2.x + o2.x, e2.y + o2.y); v[6] = make_float2(e2.x - o2.x, e2.y - o2.y);
        v[3] = make_float2(e3.x + o3.x, e3.y + o3.y); v[7] = make_float2(e3.x - o3.x, e3.y - o3.y);
    }
};
// 16 = 4 x 4 Cooley-Tukey: n = 4*n1 + n2, k = k1 + 4*k2.
template <> struct Dft<16> {
    static __device__ __forceinline__ void run(float2* v) {
        const float c1 = 0.92387953251128674f, s1 = 0.38268343236508978f, c2 = 0.70710678118654752f;
#pragma unroll
        for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]);
        // v[n2 + 4*k1] now holds Y[n2][k1]; twiddle by W16^(n2*k1)
        const float2 w1 = make_float2(c1, -s1), w2 = make_float2(c2, -c2), w3 = make_float2(s1, -c1);
        const float2 w6 = make_float2(-c2, -c2), w9 = make_float2(-c1, s1);
        v[1 + 4] = cmul(v[1 + 4], w1);
        v[1 + 8] = cmul(v[1 + 8], w2);
        v[1 + 12] = cmul(v[1 + 12], w3);
        v[2 + 4] = cmul(v[2 + 4], w2);
        v[2 + 8] = mul_mi(v[2 + 8]);
        v[2 + 12] = cmul(v[2 + 12], w6);
        v[3 + 4] = cmul(v[3 + 4], w3);
        v[3 + 8] = cmul(v[3 + 8], w6);
        v[3 + 12] = cmul(v[3 + 12], w9);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
        // v[4*k1 + k2] = X[k1 + 4*k2]: transpose 4x4 into natural order
        float2 t[16];
#pragma unroll
        for (int i = 0; i < 16; i++) t[i] = v[i];
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++)
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = t[4 * k1 + k2];
    }
};
template <> struct Dft<3> {
    static __device__ __forceinline__ void run(float2* v) {
        const float h = 0.86602540378443865f;  // sqrt(3)/2
        float2 a = v[0], b = v[1], c = v[2];
        float2 t1 = make_float2(b.x + c.x, b.y + c.y);
        float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
        float2 t3 = make_float2(h * (b.y - c.y), -h * (b.x - c.x));  // (b - c) * (-i sqrt3/2)
        v[0] = make_float2(a.x + t1.x, a.y + t1.y);
        v[1] = make_float2(t2.x + t3.x, t2.y + t3.y);
        v[2] = make_float2(t2.x - t3.x, t2.y - t3.y);
    }
};
// Odd prime radix by symmetric pairs: X_k = v0 + sum_n (s_n cos - i d_n sin).
template <int R>
__device__ __forceinline__ void dft_odd(float2* v, const float* cs, const float* sn) {
    constexpr int h = (R - 1) / 2;
    float2 s[h], d[h];
#pragma unroll
    for (int n = 1; n <= h; n++) {
        s[n - 1] = make_float2(v[n].x + v[R - n].x, v[n].y + v[R - n].y);
        d[n - 1] = make_float2(v[n].x - v[R - n].x, v[n].y - v[R - n].y);
    }
    float2 x0 = v[0];
    float2 X0 = x0;
#pragma unroll
    for (int n = 0; n < h; n++) { X0.x += s[n].x; X0.y += s[n].y; }
#pragma unroll
    for (int k = 1; k <= h; k++) {
        float2 A = x0, B = make_float2(0.f, 0.f);
#pragma unroll
        for (int n = 1; n <= h; n++) {
            const int m = (n * k) % R;  // angle index; cos symmetric, sin antisymmetric
            const float c = cs[m <= h ? m : R - m];
            const float sg = m <= h ? sn[m] : -sn[R - m];
            A.x += s[n - 1].x * c; A.y += s[n - 1].y * c;
            B.x += d[n - 1].x * sg; B.y += d[n - 1].y * sg;
        }
        v[k] = make_float2(A.x + B.y, A.y - B.x);       // A - i B
        v[R - k] = make_float2(A.x - B.y, A.y + B.x);   // A + i B
    }
    v[0] = X0;
}
template <> struct Dft<5> {
    static __device__ __forceinline__ void run(float2* v) {
        const float cs[3] = {1.f, 0.30901699437494742f, -0.80901699437494742f};
        const float sn[3] = {0.f, 0.95105651629515357f, 0.58778525229247313f};
        dft_odd<5>(v, cs, sn);
    }
};
template <> struct Dft<7> {
    static __device__ __forceinline__ void run(float2* v) {
        const float cs[4] = {1.f, 0.62348980185873353f, -0.22252093395631440f, -0.90096886790241913f};
        const float sn[4] = {0.f, 0.78183148246802981f, 0.97492791218182361f, 0.43388373911755812f};
        dft_odd<7>(v, cs, sn);
    }
};

// ------------------------------------------------------------ one pass
template <int R, int T, int EMAX>
__device__ __forceinline__ void fft_pass(float2* buf, int nseq, int stride, int n, int Ns,
                                         const float2* __restrict__ tw) {
    constexpr int MB = EMAX / R;
    static_assert(MB >= 1, "EMAX too small for radix");
    const int nb = n / R;
    const int total = nseq * nb;
    float2 v[MB][R];
#pragma unroll
    for (int q = 0; q < MB; q++) {
        const int t = threadIdx.x + q * T;
        if (t < total) {
            const int s = t / nb, j = t - s * nb;
            const float2* src = buf + s * stride + j;
#pragma unroll
            for (int r = 0; r < R; r++) v[q][r] = src[r * nb];
        }
    }
    __syncthreads();
    const int twstep = n / (Ns * R);
#pragma unroll
    for (int q = 0; q < MB; q++) {
        const int t = threadIdx.x + q * T;
        if (t < total) {
            const int s = t / nb, j = t - s * nb;
            const int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[q][r] = cmul(v[q][r], __ldg(&tw[r * k * twstep]));
            }
            Dft<R>::run(v[q]);
            float2* dst = buf + s * stride + (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) dst[r * Ns] = v[q][r];
        }
    }
    __syncthreads();
}

// Forward FFT (exp(-2 pi i nk/n)) of nseq sequences in shared memory.
template <int T, int EMAX>
__device__ void fft_smem(float2* buf, int nseq, int stride, const FftPlanDev& pl) {
    int Ns = 1;
    const int n = pl.n;
    for (int p = 0; p < pl.npass; p++) {
        const int R = pl.radix[p];
        switch (R) {
            case 16: fft_pass<16, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 8:  fft_pass<8, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 4:  fft_pass<4, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 2:  fft_pass<2, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 3:  fft_pass<3, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 5:  fft_pass<5, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            case 7:  fft_pass<7, T, EMAX>(buf, nseq, stride, n, Ns, pl.tw); break;
            default: break;
        }
        Ns *= R;
    }
}

// Forward length-N DFT of nseq sequences (first N slots of each are input).
template <int T, int EMAX>
__device__ void dft_n(float2* buf, int nseq, const DctPlanDev& P) {
    if (!P.blue) {
        fft_smem<T, EMAX>(buf, nseq, P.stride, P.fft);
        return;
    }
    const int M = P.fft.n, N = P.N, st = P.stride;
    for (int i = threadIdx.x; i < nseq * M; i += T) {
        const int s = i / M, m = i - s * M;
        float2* e = buf + s * st + m;
        *e = (m < N) ? cmul(*e, cconj(__ldg(&P.chirp[m]))) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    fft_smem<T, EMAX>(buf, nseq, st, P.fft);
    for (int i = threadIdx.x; i < nseq * M; i += T) {
        const int s = i / M, m = i - s * M;
        float2* e = buf + s * st + m;
        *e = cconj(cmul(*e, __ldg(&P.hspec[m])));
    }
    __syncthreads();
    fft_smem<T, EMAX>(buf, nseq, st, P.fft);
    for (int i = threadIdx.x; i < nseq * N; i += T) {
        const int s = i / N, k = i - s * N;
        float2* e = buf + s * st + k;
        *e = cmul(cconj(*e), cconj(__ldg(&P.chirp[k])));
    }
    __syncthreads();
}
