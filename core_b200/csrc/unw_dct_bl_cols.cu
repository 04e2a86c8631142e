// Column pass (column DCT-II -> -1/lambda scaling -> column DCT-III, in place
// on T) for column lengths N that are not powers of two (64 < N <= 8192):
// NSEQ column pairs per CTA, each pair one complex sequence handled by M / 16
// threads, the length-N DFTs by Bluestein on the register FFT of length
// M >= 2N - 1, a power of two or three times one (unw_bluestein.cuh).  MODE 0: DCT initial
// solve; MODE 1 / 2: PCG (gated), with r.z by Parseval (col_spectral_pair)
// and its scalar step (col_finalize).
#include "unw_bluestein.cuh"
#include "unw_rowops.cuh"
#include "unw_kernels.h"

namespace {

template <int T>
constexpr int bl_min_blocks() { return T >= 1024 ? 1 : (1024 / T > 16 ? 16 : 1024 / T); }

// column pairs per CTA: about 512 threads per CTA, at most 8 pairs; at M = 6144 two pairs
// (768 threads, 16-byte rows) rather than one (measured on B200 at 2436 x 5911: 381 us vs 393 us
// per column pass, same bits)
constexpr int bl_col_nseq_len(int M) {
    return M == 6144 ? 2 : (M >= 8192 ? 1 : (8192 / M > 8 ? 8 : (8192 / M < 1 ? 1 : 8192 / M)));
}

template <class BL, int NSEQ, int MODE>
__global__ void __launch_bounds__(BL::T * NSEQ, bl_min_blocks<BL::T * NSEQ>()) k_col_bl(
    const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    constexpr int T = BL::T;
    extern __shared__ float2 sm[];
    __shared__ double red[32];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (MODE >= 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int s = threadIdx.x % NSEQ, t = threadIdx.x / NSEQ;
    float2* sms = sm + s * BL::SLOTS;
    float* __restrict__ Tm = G.T;
    const float2* __restrict__ dw = G.pcol.dctw;
    const float* __restrict__ sH = G.sH;
    const float negs = -1.0f / (4.0f * (float)H * (float)W);
    const int nslab = (W + 2 * NSEQ - 1) / (2 * NSEQ);
    double acc[1] = {0.0};
    for (int slab = local; slab < nslab; slab += nct) {
        const int ja = 2 * NSEQ * slab + 2 * s;
        const bool hasa = ja < W, hasb = ja + 1 < W;
        // the pair as one 8-byte access (ja is even): one L1 request per row instead of two
        // (column pass 392.8 vs 439.6 us at 2436 x 5911, 147.6 vs 160.3 at 1838 x 4122, same bits)
        const bool vec = hasb && !(P & 1);
        __syncthreads();  // previous slab's reads of sm are done
        // column pair (ja, ja+1): row i goes to DFT position perm(i)
        for (int i = t; i < H; i += T) {
            const float* a = Tm + (size_t)i * P + ja;
            float2 x = make_float2(0.f, 0.f);
            if (vec) x = *reinterpret_cast<const float2*>(a);
            else if (hasb) x = make_float2(a[0], a[1]);
            else if (hasa) x.x = a[0];
            sms[BL::pos(mk_perm(i, H))] = x;
        }
        __syncthreads();
        BL::dft(sms, t, H, G.pcol);
        const float ca = hasa ? G.sW[ja] : 1.0f, cb = hasb ? G.sW[ja + 1] : 1.0f;
        for (int k = t; k <= H / 2; k += T) {
            const int km = k == 0 ? 0 : H - k;
            const float2 C = sms[BL::pos(k)], Cm = sms[BL::pos(km)];
            const float2 wk = __ldg(&dw[k]), wm = __ldg(&dw[km]);
            const float ck = __ldg(&sH[k]), cm = __ldg(&sH[km]);
            float2 ok, om;
            col_spectral_pair<(MODE >= 1)>(C, Cm, k, km, wk, wm, ck, cm, ca, cb, ja == 0, hasb, negs, ok, om,
                                           acc[0]);
            if (km != k) sms[BL::pos(km)] = om;
            sms[BL::pos(k)] = ok;
        }
        __syncthreads();
        BL::dft(sms, t, H, G.pcol);
        for (int i = t; i < H; i += T) {
            const float2 v = sms[BL::pos(mk_perm(i, H))];
            float* a = Tm + (size_t)i * P + ja;
            if (vec) *reinterpret_cast<float2*>(a) = make_float2(v.x, -v.y);
            else if (hasb) { a[0] = v.x; a[1] = -v.y; }
            else if (hasa) a[0] = v.x;
        }
    }
    if (MODE == 0) return;
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) col_finalize<MODE>(st, acc[0]);
    }
}

template <class BL>
cudaError_t col_bl_m(int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* st, int n) {
    constexpr int NS = bl_col_nseq_len(BL::LEN);
    const size_t smem = sizeof(float2) * (size_t)BL::SLOTS * NS;
    auto go = [&](auto kfn) {
        cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        kfn<<<nblk, BL::T * NS, smem, s>>>(gd, st, n);
        return cudaGetLastError();
    };
    switch (mode) {
        case 0: return go(k_col_bl<BL, NS, 0>);
        case 1: return go(k_col_bl<BL, NS, 1>);
        default: return go(k_col_bl<BL, NS, 2>);
    }
}

}  // namespace

int unw_bl_col_nseq(int M) {
    switch (M) {
        case 256: case 512: case 1024: case 2048: case 4096: case 8192: case 16384:
        case 768: case 1536: case 3072: case 6144: case 12288: return bl_col_nseq_len(M);
        default: return 0;
    }
}

cudaError_t unw_launch_col_bl(int M, int mode, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                              int n) {
    if (nblk <= 0) return cudaSuccess;
    switch (M) {
        case 256: return col_bl_m<BlP2<256>>(mode, nblk, s, gd, starts, n);
        case 512: return col_bl_m<BlP2<512>>(mode, nblk, s, gd, starts, n);
        case 1024: return col_bl_m<BlP2<1024>>(mode, nblk, s, gd, starts, n);
        case 2048: return col_bl_m<BlP2<2048>>(mode, nblk, s, gd, starts, n);
        case 4096: return col_bl_m<BlP2<4096>>(mode, nblk, s, gd, starts, n);
        case 8192: return col_bl_m<BlP2<8192>>(mode, nblk, s, gd, starts, n);
        case 16384: return col_bl_m<BlP2<16384>>(mode, nblk, s, gd, starts, n);
        case 768: return col_bl_m<BlMix3<256>>(mode, nblk, s, gd, starts, n);
        case 1536: return col_bl_m<BlMix3<512>>(mode, nblk, s, gd, starts, n);
        case 3072: return col_bl_m<BlMix3<1024>>(mode, nblk, s, gd, starts, n);
        case 6144: return col_bl_m<BlMix3<2048>>(mode, nblk, s, gd, starts, n);
        case 12288: return col_bl_m<BlMix3<4096>>(mode, nblk, s, gd, starts, n);
        default: return cudaErrorInvalidValue;
    }
}
