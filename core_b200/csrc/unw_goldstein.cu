// Goldstein adaptive phase filter, the code path insardev runs on CUDA devices
// (goldstein_pytorch, insardev/insardev/utils_goldstein.py:157-330):
// overlapping psize_y x psize_x patches at half-patch steps, each patch's 2-D
// spectrum weighted by max(|F|, 1e-10)^alpha with alpha = 1 - weighted mean
// coherence, inverse transform, triangular taper, overlap-add, division by the
// number of valid patches covering a pixel.
//
// One CTA per patch: the patch goes to shared memory once, both 2-D FFTs run
// there (radix-2 Stockham along x then y, ping-pong buffers), and the tapered
// result is added into a padded accumulator.  Patches of one parity class
// (patch row parity, patch column parity) never overlap, so the four classes
// run as four launches with plain (non-atomic) read-add-write: deterministic.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

namespace {

struct GsArgs {
    const float2* phase; long long pp;
    const float* corr; long long cp;
    int ny, nx;             // input grid
    int H, W;               // padded grid (accumulator pitch W)
    int py, px, sy, sx;     // patch size and step
    int lpy, lpx;           // log2 of the patch size
    int npy, npx;           // patches per axis
    int min_valid;
    const float* wgt;       // [py][px] taper, and its float32 sum at wgt[py*px]
    float2* acc;            // [H][W] overlap-add of tapered patches
    float* cnt;             // [H][W] valid patches covering each pixel
};

// Taper (utils_goldstein.py:198-203): separable tent over half a patch, built in
// float64 and rounded once; sum accumulated in float64 and rounded.
__global__ void k_gs_weights(float* wgt, int py, int px) {
    const int n = py * px;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int y = e / px, x = e % px;
        const int hy = py / 2, hx = px / 2;
        const int qy = y < hy ? y : py - 1 - y;   // mirrored quadrant index
        const int qx = x < hx ? x : px - 1 - x;
        const double cy = py / 2.0 - 1.0, cx = px / 2.0 - 1.0;
        const double wy = 1.0 - fabs((double)qy - cy) / cy;
        const double wx = 1.0 - fabs((double)qx - cx) / cx;
        wgt[e] = (float)(wy * wx);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int e = 0; e < n; e++) s += (double)wgt[e];
        wgt[n] = (float)s;
    }
}

// Radix-2 Stockham pass sequence along one axis of a py x px array in shared
// memory; returns the buffer that holds the result.  sign -1: forward.
__device__ float2* fft_axis(float2* src, float2* dst, int lpy, int lpx, bool along_x, float sign) {
    const int ln = along_x ? lpx : lpy;       // log2 transform length
    const int lm = along_x ? lpy : lpx;       // log2 number of sequences
    const int n = 1 << ln, half = n >> 1;
    const int estride = along_x ? 1 : (1 << lpx);
    const int sstride = along_x ? (1 << lpx) : 1;
    const int nb = half << lm;                // butterflies per pass
    for (int Ns = 1, lNs = 0; Ns < n; Ns <<= 1, lNs++) {
        for (int idx = threadIdx.x; idx < nb; idx += blockDim.x) {
            int s, jj;
            if (along_x) { s = idx >> (ln - 1); jj = idx & (half - 1); }   // consecutive threads: consecutive x
            else { s = idx & ((1 << lm) - 1); jj = idx >> lm; }            // consecutive threads: consecutive columns
            const int k = jj & (Ns - 1);
            const float2 a = src[s * sstride + jj * estride];
            const float2 b = src[s * sstride + (jj + half) * estride];
            float sn, cs;
            sincospif(sign * (float)k / (float)Ns, &sn, &cs);   // exp(sign i pi k / Ns)
            const float2 wb = make_float2(cs * b.x - sn * b.y, cs * b.y + sn * b.x);
            const int o = ((jj - k) << 1) + k;
            dst[s * sstride + o * estride] = make_float2(a.x + wb.x, a.y + wb.y);
            dst[s * sstride + (o + Ns) * estride] = make_float2(a.x - wb.x, a.y - wb.y);
        }
        __syncthreads();
        float2* t = src; src = dst; dst = t;
    }
    return src;
}

__global__ void __launch_bounds__(256) k_gs_patch(GsArgs a, int ci, int cj) {
    extern __shared__ float2 sm[];
    __shared__ float rw[8];
    __shared__ int rv[8];
    const int n = a.py * a.px;
    const int nci = (a.npy - ci + 1) / 2, ncj = (a.npx - cj + 1) / 2;
    const float wsum = a.wgt[n];
    const float inv_n = 1.0f / (float)n;
    for (int pid = blockIdx.x; pid < nci * ncj; pid += gridDim.x) {
        const int pi = ci + 2 * (pid / ncj), pj = cj + 2 * (pid % ncj);
        const int y0 = pi * a.sy, x0 = pj * a.sx;
        float2* b0 = sm;
        float2* b1 = sm + n;
        // load (padding and NaN -> 0; utils_goldstein.py:214-230)
        float wc = 0.f;
        int vc = 0;
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const int y = e >> a.lpx, x = e & (a.px - 1);
            const int gy = y0 + y, gx = x0 + x;
            float2 v = make_float2(0.f, 0.f);
            float c = 0.f;
            if (gy < a.ny && gx < a.nx) {
                v = a.phase[(long long)gy * a.pp + gx];
                const bool ok = !(isnan(v.x) || isnan(v.y));
                if (!ok) v = make_float2(0.f, 0.f);
                vc += ok ? 1 : 0;
                c = a.corr[(long long)gy * a.cp + gx];
                if (isnan(c)) c = 0.f;
            }
            b0[e] = v;
            wc = fmaf(a.wgt[e], c, wc);
        }
        // block sums of the weighted coherence and the valid count
        for (int o = 16; o > 0; o >>= 1) {
            wc += __shfl_down_sync(0xffffffffu, wc, o);
            vc += __shfl_down_sync(0xffffffffu, vc, o);
        }
        if ((threadIdx.x & 31) == 0) { rw[threadIdx.x >> 5] = wc; rv[threadIdx.x >> 5] = vc; }
        __syncthreads();
        float W8 = 0.f;
        int V8 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { W8 += rw[w]; V8 += rv[w]; }
        const float alpha = 1.0f - W8 / wsum;      // utils_goldstein.py:259-262
        const bool valid = V8 >= a.min_valid;      // :264-267
        __syncthreads();                            // rw/rv reads done before the next patch
        if (!valid) continue;                       // uniform over the CTA
        float2* f = fft_axis(b0, b1, a.lpy, a.lpx, true, -1.f);
        float2* g = fft_axis(f, f == b0 ? b1 : b0, a.lpy, a.lpx, false, -1.f);
        // spectrum weight max(|F|, 1e-10)^alpha (:270-276)
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const float2 F = g[e];
            const float m = fmaxf(sqrtf(F.x * F.x + F.y * F.y), 1e-10f);
            const float s = powf(m, alpha);
            g[e] = make_float2(F.x * s, F.y * s);
        }
        __syncthreads();
        f = fft_axis(g, g == b0 ? b1 : b0, a.lpy, a.lpx, true, 1.f);
        g = fft_axis(f, f == b0 ? b1 : b0, a.lpy, a.lpx, false, 1.f);
        // taper, overlap-add, coverage count (:283-307); this class's patches are disjoint
        for (int e = threadIdx.x; e < n; e += blockDim.x) {
            const int y = e >> a.lpx, x = e & (a.px - 1);
            const size_t o = (size_t)(y0 + y) * a.W + (x0 + x);
            const float w = a.wgt[e] * inv_n;
            const float2 v = g[e];
            float2 s = a.acc[o];
            s.x = fmaf(w, v.x, s.x);
            s.y = fmaf(w, v.y, s.y);
            a.acc[o] = s;
            a.cnt[o] += 1.0f;
        }
        __syncthreads();  // shared buffers reused by the next patch
    }
}

// normalisation and NaN restore (:308-320)
__global__ void k_gs_final(GsArgs a, float2* out, long long op) {
    const long long n = (long long)a.ny * a.nx;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n;
         q += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(q / a.nx), x = (int)(q - (long long)y * a.nx);
        const size_t o = (size_t)y * a.W + x;
        const float c = a.cnt[o];
        const float2 in = a.phase[(long long)y * a.pp + x];
        float2 v;
        if (isnan(in.x) || isnan(in.y) || c < 1e-6f) {
            v = make_float2(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000));
        } else {
            const float d = fmaxf(c, 1.0f);
            v = make_float2(a.acc[o].x / d, a.acc[o].y / d);
        }
        out[(long long)y * op + x] = v;
    }
}

int ilog2i(int v) {
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

struct GsLayout {
    int H, W;
    size_t wgt, acc, cnt, total;
};

GsLayout gs_layout(long long ny, long long nx, int py, int px) {
    GsLayout L{};
    const int sy = py / 2, sx = px / 2;
    const long long pad_y = py - sy, pad_x = px - sx;
    const long long ey = (sy - ((ny + pad_y - py) % sy)) % sy;
    const long long ex = (sx - ((nx + pad_x - px) % sx)) % sx;
    L.H = (int)(ny + pad_y + ey);
    L.W = (int)(nx + pad_x + ex);
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    size_t o = 0;
    L.wgt = o; o = up(o + sizeof(float) * ((size_t)py * px + 1));
    L.acc = o; o = up(o + sizeof(float2) * (size_t)L.H * L.W);
    L.cnt = o; o = up(o + sizeof(float) * (size_t)L.H * L.W);
    L.total = o + 256;
    return L;
}

bool gs_psize_ok(int p) { return p >= 4 && p <= 64 && (p & (p - 1)) == 0; }

}  // namespace

extern "C" {

size_t unw_goldstein_workspace_bytes(int64_t H, int64_t W, int32_t psize_y, int32_t psize_x) {
    if (H <= 0 || W <= 0 || !gs_psize_ok(psize_y) || !gs_psize_ok(psize_x)) return 0;
    return gs_layout(H, W, psize_y, psize_x).total;
}

int unw_goldstein_c64(const float* phase, int64_t phase_pitch, const float* corr, int64_t corr_pitch, int64_t H,
                      int64_t W, int32_t psize_y, int32_t psize_x, float threshold, float* out, int64_t out_pitch,
                      void* workspace, size_t workspace_bytes, void* cuda_stream) {
    if (!phase || !corr || !out) return unw_set_error(UNW_E_ARG, "goldstein: null pointer");
    if (H <= 0 || W <= 0) return unw_set_error(UNW_E_ARG, "goldstein: bad shape");
    if (phase_pitch < W || corr_pitch < W || out_pitch < W)
        return unw_set_error(UNW_E_ARG, "goldstein: pitch smaller than width");
    if (!gs_psize_ok(psize_y) || !gs_psize_ok(psize_x))
        return unw_set_error(UNW_E_UNSUPPORTED, "goldstein: patch sizes must be powers of two in [4, 64]");
    if (!(threshold >= 0.f) || !(threshold <= 1.f)) return unw_set_error(UNW_E_ARG, "goldstein: threshold in [0, 1]");
    if (!workspace) return unw_set_error(UNW_E_ARG, "goldstein: workspace is NULL");
    const GsLayout L = gs_layout(H, W, psize_y, psize_x);
    char* base = (char*)(((size_t)workspace + 255) / 256 * 256);
    if ((size_t)(base - (char*)workspace) + L.total - 256 > workspace_bytes)
        return unw_set_error(UNW_E_WORKSPACE, "goldstein: workspace too small");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    GsArgs a{};
    a.phase = (const float2*)phase; a.pp = phase_pitch;
    a.corr = corr; a.cp = corr_pitch;
    a.ny = (int)H; a.nx = (int)W; a.H = L.H; a.W = L.W;
    a.py = psize_y; a.px = psize_x; a.sy = psize_y / 2; a.sx = psize_x / 2;
    a.lpy = ilog2i(psize_y); a.lpx = ilog2i(psize_x);
    a.npy = (L.H - psize_y) / a.sy + 1;
    a.npx = (L.W - psize_x) / a.sx + 1;
    a.min_valid = (int)((double)psize_y * (double)psize_x * (double)threshold);
    a.wgt = (const float*)(base + L.wgt);
    a.acc = (float2*)(base + L.acc);
    a.cnt = (float*)(base + L.cnt);
    cudaError_t e;
    if ((e = cudaMemsetAsync(a.acc, 0, sizeof(float2) * (size_t)L.H * L.W, s)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.cnt, 0, sizeof(float) * (size_t)L.H * L.W, s)) != cudaSuccess)
        return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    k_gs_weights<<<1, 256, 0, s>>>(const_cast<float*>(a.wgt), psize_y, psize_x);
    const size_t smem = 2 * sizeof(float2) * (size_t)psize_y * psize_x;
    unw_smem_limit((const void*)k_gs_patch);
    for (int c = 0; c < 4; c++) {
        const int ci = c >> 1, cj = c & 1;
        const long long np = (long long)((a.npy - ci + 1) / 2) * ((a.npx - cj + 1) / 2);
        if (np <= 0) continue;
        const int grid = (int)(np < 148 * 16 ? np : 148 * 16);
        k_gs_patch<<<grid, 256, smem, s>>>(a, ci, cj);
    }
    const long long npx = (long long)H * W;
    const int gf = (int)((npx + 255) / 256 < 148 * 32 ? (npx + 255) / 256 : 148 * 32);
    k_gs_final<<<gf, 256, 0, s>>>(a, (float2*)out, out_pitch);
    if ((e = cudaGetLastError()) != cudaSuccess) return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    return UNW_OK;
}

}  // extern "C"
