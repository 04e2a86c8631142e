// Post-processing kernels (utils_unwrap2d.py:1659-1757 and the numba kernels
// at :24-75), all on the device:
//   non-finite test and 2-pi cycle statistics -> histogram -> median shift,
//   4-connected components by lock-free union-find (root = first pixel in
//   raster order, so labels come out in the same order as
//   cv2.connectedComponents), per-component float64 sin/cos sums, circular
//   mean alignment, size-ranked relabel and un-crop into the caller's grid.
#include <climits>
#include "unw_kernels.h"

#define UNW_TILE_PX 4096      // pixels per scan tile (256 threads x 16)
#define UNW_UF_LIMIT (1 << 24)

__device__ __forceinline__ float* ufinal(const GridDev& G, const InstState* st) {
    return st->u_index == 2 ? G.Ub : (st->u_index == 1 ? G.U1 : G.U0);
}

__device__ __forceinline__ bool post_ok(const InstState* st) {
    return st->n_nonfinite == 0 && st->hist_ok;
}

// k = round((u - phase) / 2pi) in float32, as numpy does for the reference's
// float32 arrays (utils_unwrap2d.py:1673-1674); 2*pi rounds to 6.2831855f.
__device__ __forceinline__ float cycles_f(float u, float ph) {
    return rintf(__fdiv_rn(__fsub_rn(u, ph), 6.28318548202514648f));
}

// ---------------------------------------------------------------- stats
// Non-finite solution count (utils_unwrap2d.py:1659-1665) and the range of the
// cycle counts k.  An infinite input phase on a valid pixel gives k = -inf or
// +inf there (u is finite by now); those are counted apart and enter the median
// as the smallest / largest values, as they do in np.median.
__global__ void p_kstats(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ double red[32 * 3];
    __shared__ int smin, smax;
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const long long npx = (long long)G.H * W;
    const float* __restrict__ U = ufinal(G, st);
    if (threadIdx.x == 0) { smin = INT_MAX; smax = INT_MIN; }
    __syncthreads();
    int kmn = INT_MAX, kmx = INT_MIN;
    double acc[3] = {0.0, 0.0, 0.0};
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        if (!G.valid[(size_t)i * P + j]) continue;
        const float u = U[(size_t)i * P + j];
        if (!isfinite(u)) { acc[0] += 1.0; continue; }
        float k = cycles_f(u, G.phase[(long long)i * G.phase_pitch + j]);
        if (!isfinite(k)) { acc[k < 0.f ? 1 : 2] += 1.0; continue; }
        k = fminf(fmaxf(k, -1073741824.f), 1073741824.f);
        const int ki = (int)k;
        kmn = min(kmn, ki);
        kmx = max(kmx, ki);
    }
    for (int o = 16; o > 0; o >>= 1) {
        kmn = min(kmn, __shfl_down_sync(0xffffffffu, kmn, o));
        kmx = max(kmx, __shfl_down_sync(0xffffffffu, kmx, o));
    }
    if ((threadIdx.x & 31) == 0) { atomicMin(&smin, kmn); atomicMax(&smax, kmx); }
    __syncthreads();
    if (threadIdx.x == 0) { atomicMin(&st->kmin, smin); atomicMax(&st->kmax, smax); }
    if (arrive<3>(G, local, nct, acc, red)) {
        finish_sum<3>(G, nct, acc, red);
        if (threadIdx.x == 0) {
            st->n_nonfinite = (int)acc[0];
            st->n_kneg = (int)acc[1];
            st->n_kpos = (int)acc[2];
            const double nfin = st->vcount - acc[1] - acc[2];
            bool ok;
            if (nfin > 0.0) {
                const int kmin = __ldcg(&st->kmin), kmax = __ldcg(&st->kmax);
                const long long range = (long long)kmax - (long long)kmin + 1;
                ok = range >= 1 && range <= G.hist_cap;
            } else {
                st->kmin = 0;  // no finite count: empty histogram
                st->kmax = -1;
                ok = st->vcount > 0;
            }
            st->hist_ok = (acc[0] == 0.0 && ok) ? 1 : 0;
        }
    }
}

__global__ void p_hist(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ int sh[2048];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const long long npx = (long long)G.H * W;
    const float* __restrict__ U = ufinal(G, st);
    const int kmin = st->kmin, range = st->kmax - st->kmin + 1;
    if (range <= 0) return;
    const bool small = range <= 2048;
    if (small) {
        for (int b = threadIdx.x; b < range; b += blockDim.x) sh[b] = 0;
        __syncthreads();
    }
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        if (!G.valid[(size_t)i * P + j]) continue;
        const float kf = cycles_f(U[(size_t)i * P + j], G.phase[(long long)i * G.phase_pitch + j]);
        if (!isfinite(kf)) continue;  // counted as -inf / +inf by p_kstats
        const int k = (int)kf - kmin;
        if (k < 0 || k >= range) continue;
        if (small) atomicAdd(&sh[k], 1); else atomicAdd(&G.hist[k], 1);
    }
    if (small) {
        __syncthreads();
        for (int b = threadIdx.x; b < range; b += blockDim.x)
            if (sh[b]) atomicAdd(&G.hist[b], sh[b]);
    }
}

// One CTA per grid: order statistics of the sorted cycle counts -> np.median
// semantics (mean of the two middle values), shift = float32(float32(2*kmed) *
// float32(pi)).  The sorted order is n_kneg times -inf, the histogram, then
// n_kpos times +inf.
__global__ void p_median(const GridDev* __restrict__ grids, int n) {
    __shared__ int s_lo, s_hi;
    __shared__ int wsum[32];
    const GridDev& G = grids[blockIdx.x];
    InstState* st = G.st;
    if (!post_ok(st)) return;
    const long long nv = (long long)st->vcount;
    const long long nneg = st->n_kneg, nfin = nv - st->n_kneg - st->n_kpos;
    const long long plo = (nv - 1) / 2, phi = nv / 2;
    const long long qlo = plo - nneg, qhi = phi - nneg;  // positions inside the histogram
    const bool need_lo = qlo >= 0 && qlo < nfin, need_hi = qhi >= 0 && qhi < nfin;
    const int range = st->kmax - st->kmin + 1;
    if (threadIdx.x == 0) { s_lo = -1; s_hi = -1; }
    __syncthreads();
    long long base = 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int c0 = 0; c0 < range; c0 += blockDim.x) {
        const int b = c0 + threadIdx.x;
        const int v = b < range ? G.hist[b] : 0;
        int x = v;  // inclusive warp scan
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = lane < nw ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < nw) wsum[lane] = w;
        }
        __syncthreads();
        const long long incl = base + x + (wid > 0 ? wsum[wid - 1] : 0);
        const long long excl = incl - v;
        if (v > 0) {
            if (qlo >= excl && qlo < incl) s_lo = b;
            if (qhi >= excl && qhi < incl) s_hi = b;
        }
        base += wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float inf = __int_as_float(0x7f800000);
        const float klo = need_lo ? (float)(s_lo + st->kmin) : (qlo < 0 ? -inf : inf);
        const float khi = need_hi ? (float)(s_hi + st->kmin) : (qhi < 0 ? -inf : inf);
        const float kmed = __fdiv_rn(__fadd_rn(klo, khi), 2.0f);
        st->kmed = kmed;
        st->shift = __fmul_rn(__fmul_rn(kmed, 2.0f), 3.14159274101257324f);
        if ((need_lo && s_lo < 0) || (need_hi && s_hi < 0)) st->hist_ok = 0;
    }
}

// ---------------------------------------------------------------- components
__device__ __forceinline__ int uf_find(int* parent, int x) {
    for (int guard = 0; guard < UNW_UF_LIMIT; guard++) {
        const int p = __ldcg(&parent[x]);
        if (p == x) return x;
        const int gp = __ldcg(&parent[p]);
        if (gp != p) parent[x] = gp;  // path halving: gp is an ancestor of x
        x = gp;
    }
    return -1;
}

// Read-only walk to the root.  The flatten pass must not compress paths: a
// halving store could overwrite another thread's final parent[x] = root with
// an intermediate ancestor, leaving a pixel that points at a non-root.
__device__ __forceinline__ int uf_root(const int* parent, int x) {
    for (int guard = 0; guard < UNW_UF_LIMIT; guard++) {
        const int p = __ldcg(&parent[x]);
        if (p == x) return x;
        x = p;
    }
    return -1;
}

__device__ __forceinline__ bool uf_union(int* parent, int a, int b) {
    for (int guard = 0; guard < UNW_UF_LIMIT; guard++) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a < 0 || b < 0) return false;
        if (a == b) return true;
        if (a > b) { const int t = a; a = b; b = t; }
        const int old = atomicCAS(&parent[b], b, a);  // hook the larger root under the smaller
        if (old == b) return true;
    }
    return false;
}

__global__ void p_shift_ccinit(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const long long npx = (long long)G.H * W;
    float* __restrict__ U = ufinal(G, st);
    const float sh = st->shift;
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        const size_t o = (size_t)i * P + j;
        if (G.valid[o]) {
            U[o] = __fsub_rn(U[o], sh);
            G.parent[q] = (int)q;
        } else {
            U[o] = __int_as_float(0x7fc00000);
            G.parent[q] = -1;
        }
    }
}

__global__ void p_union(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const long long npx = (long long)H * W;
    bool ok = true;
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        const size_t o = (size_t)i * P + j;
        if (!G.valid[o]) continue;
        if (j < W - 1 && G.valid[o + 1]) ok &= uf_union(G.parent, (int)q, (int)q + 1);
        if (i < H - 1 && G.valid[o + P]) ok &= uf_union(G.parent, (int)q, (int)q + W);
    }
    if (!ok) st->hist_ok = 0;
}

// One CTA per tile of UNW_TILE_PX pixels: every valid pixel points at its root
// afterwards (only its own entry is written), and roots are counted per tile.
__global__ void p_flatten(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ int cnt;
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!post_ok(st)) return;
    const int tile = blockIdx.x - starts[g];
    const long long npx = (long long)G.H * G.W;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int c = 0;
    bool ok = true;
    const long long b0 = (long long)tile * UNW_TILE_PX;
    for (int t = threadIdx.x; t < UNW_TILE_PX; t += blockDim.x) {
        const long long q = b0 + t;
        if (q >= npx) break;
        if (G.parent[q] < 0) continue;
        const int r = uf_root(G.parent, (int)q);
        if (r < 0) { ok = false; continue; }
        G.parent[q] = r;
        c += (r == (int)q) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&cnt, c);
    if (!ok) st->hist_ok = 0;
    __syncthreads();
    if (threadIdx.x == 0) G.tilecnt[tile] = cnt;
}

// One CTA per grid: exclusive scan of roots per tile.
__global__ void p_tilescan(const GridDev* __restrict__ grids, int n) {
    __shared__ int wsum[32];
    const GridDev& G = grids[blockIdx.x];
    InstState* st = G.st;
    if (!post_ok(st)) return;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int base = 0;
    for (int c0 = 0; c0 < G.ntiles; c0 += blockDim.x) {
        const int b = c0 + threadIdx.x;
        const int v = b < G.ntiles ? G.tilecnt[b] : 0;
        int x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = lane < nw ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < nw) wsum[lane] = w;
        }
        __syncthreads();
        const int excl = base + x - v + (wid > 0 ? wsum[wid - 1] : 0);
        if (b < G.ntiles) G.tilecnt[b] = excl;
        base += wsum[nw - 1];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        st->n_labels = base;
        if (base + 1 > G.lab_cap) st->hist_ok = 0;
    }
}

// One CTA per tile: compact label (1-based, raster order of roots) for each
// root; also zeroes the per-label accumulators.
__global__ void p_label(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ int wsum[32];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int tile = blockIdx.x - starts[g];
    const int ntile = starts[g + 1] - starts[g];
    const long long npx = (long long)G.H * G.W;
    const int nl = st->n_labels + 1;
    for (int L = tile * blockDim.x + threadIdx.x; L < nl; L += ntile * blockDim.x) {
        G.csum[L] = 0.0;
        G.csum[(size_t)G.lab_cap + L] = 0.0;
        G.csum[2 * (size_t)G.lab_cap + L] = 0.0;
        G.csum[3 * (size_t)G.lab_cap + L] = 0.0;
        G.ccount[L] = 0;
    }
    constexpr int PER = UNW_TILE_PX / 256;
    const long long b0 = (long long)tile * UNW_TILE_PX + (long long)threadIdx.x * PER;
    int c = 0;
    for (int t = 0; t < PER; t++) {
        const long long q = b0 + t;
        if (q < npx && G.parent[q] == (int)q) c++;
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < nw ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) wsum[lane] = w;
    }
    __syncthreads();
    int lbl = G.tilecnt[tile] + x - c + (wid > 0 ? wsum[wid - 1] : 0) + 1;
    for (int t = 0; t < PER; t++) {
        const long long q = b0 + t;
        if (q < npx && G.parent[q] == (int)q) G.lab[q] = lbl++;
    }
}

// Per-label sums of sin/cos of the input phase and of the shifted solution
// (float32 sin/cos accumulated in float64, like the numba kernel at :24-65).
__global__ void p_accum(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const long long npx = (long long)G.H * W;
    const float* __restrict__ U = ufinal(G, st);
    const size_t cap = (size_t)G.lab_cap;
    const int nlab = st->n_labels;
    bool bad = false;
    for (long long q0 = (long long)local * blockDim.x; q0 < npx; q0 += (long long)nct * blockDim.x) {
        const long long q = q0 + threadIdx.x;
        int L = 0;
        double si = 0, ci = 0, so = 0, co = 0;
        if (q < npx) {
            const int i = (int)(q / W), j = (int)(q - (long long)i * W);
            const size_t o = (size_t)i * P + j;
            if (G.valid[o]) {
                L = G.lab[G.parent[q]];
                if (L < 1 || L > nlab) { bad = true; L = 0; }
                const float ph = G.phase[(long long)i * G.phase_pitch + j];
                const float u = U[o];
                si = (double)sinf(ph); ci = (double)cosf(ph);
                so = (double)sinf(u); co = (double)cosf(u);
            }
        }
        __syncwarp();
        if (q < npx) {
            const int i = (int)(q / W), j = (int)(q - (long long)i * W);
            if (G.valid[(size_t)i * P + j]) G.parent[q] = L;  // parent now holds the label
        }
        const int L0 = __shfl_sync(0xffffffffu, L, 0);
        const bool uniform = __all_sync(0xffffffffu, L == L0);
        if (uniform) {
            if (L0 == 0) continue;
            int c = 1;
            for (int o = 16; o > 0; o >>= 1) {
                si += __shfl_down_sync(0xffffffffu, si, o);
                ci += __shfl_down_sync(0xffffffffu, ci, o);
                so += __shfl_down_sync(0xffffffffu, so, o);
                co += __shfl_down_sync(0xffffffffu, co, o);
                c += __shfl_down_sync(0xffffffffu, c, o);
            }
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(&G.csum[L0], si);
                atomicAdd(&G.csum[cap + L0], ci);
                atomicAdd(&G.csum[2 * cap + L0], so);
                atomicAdd(&G.csum[3 * cap + L0], co);
                atomicAdd(&G.ccount[L0], c);
            }
        } else if (L > 0) {
            atomicAdd(&G.csum[L], si);
            atomicAdd(&G.csum[cap + L], ci);
            atomicAdd(&G.csum[2 * cap + L], so);
            atomicAdd(&G.csum[3 * cap + L], co);
            atomicAdd(&G.ccount[L], 1);
        }
    }
    if (bad) G.st->hist_ok = 0;
}

// adjust = wrap(circmean(phase) - circmean(u)) per label (utils_unwrap2d.py:1704-1716)
__global__ void p_adjust(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const size_t cap = (size_t)G.lab_cap;
    const int nl = st->n_labels + 1;
    for (int L = local * blockDim.x + threadIdx.x; L < nl; L += nct * blockDim.x) {
        if (L == 0) { G.adj[0] = 0.0; continue; }
        double c = (double)G.ccount[L];
        if (c == 0.0) c = 1.0;
        const double im = atan2(G.csum[L] / c, G.csum[cap + L] / c);
        const double om = atan2(G.csum[2 * cap + L] / c, G.csum[3 * cap + L] / c);
        const double d = im - om;
        G.adj[L] = atan2(sin(d), cos(d));
    }
}

// Final outputs in the caller's full grid (crop offset r0, c0).
__global__ void p_write(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!post_ok(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int W = G.W, P = G.P;
    const long long npx = (long long)G.H * W;
    const float* __restrict__ U = ufinal(G, st);
    const int nlab = st->n_labels;
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        const size_t o = (size_t)i * P + j;
        float u = __int_as_float(0x7fc00000);
        uint16_t cc = 0;
        if (G.valid[o]) {
            int L = G.parent[q];
            L = (L >= 1 && L <= nlab) ? L : 0;
            u = (float)((double)U[o] + G.adj[L]);
            cc = (uint16_t)G.remap[L];
            if (G.congruent) {
                const float ph = G.phase[(long long)i * G.phase_pitch + j];
                const float k = rintf(__fdiv_rn(__fsub_rn(u, ph), 6.28318548202514648f));
                u = (float)((double)ph + 6.283185307179586 * (double)k);
            }
        }
        const long long oi = (long long)(G.r0 + i), oj = (long long)(G.c0 + j);
        G.out_u[oi * G.out_u_pitch + oj] = u;
        G.out_cc[oi * G.out_cc_pitch + oj] = cc;
    }
}

// NaN / 0 outside the crop; the whole grid when the solve failed.
__global__ void p_fill(const GridDev* __restrict__ grids, int n) {
    const int g = blockIdx.y;
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    const bool failed = (G.H == 0) || st == nullptr || !post_ok(st);
    const long long npx = (long long)G.H0 * G.W0;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < npx; q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q / G.W0), j = (int)(q - (long long)i * G.W0);
        const bool inside = i >= G.r0 && i < G.r0 + G.H && j >= G.c0 && j < G.c0 + G.W;
        if (inside && !failed) continue;
        G.out_u[(long long)i * G.out_u_pitch + j] = __int_as_float(0x7fc00000);
        G.out_cc[(long long)i * G.out_cc_pitch + j] = 0;
    }
}

// ---------------------------------------------------------------- bbox
// Valid rows / columns of the caller's full grid (utils_unwrap2d.py:1204-1209).
__global__ void p_bbox_tiles(const float* __restrict__ phase, long long pitch, int H0, int W0,
                             int* rowany, int* colany) {
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int i0 = blockIdx.y * 64;
    int cany = 0;
    for (int i = i0 + (threadIdx.x >> 5); i < min(H0, i0 + 64); i += blockDim.x >> 5) {
        const bool v = j < W0 && !isnan(phase[(long long)i * pitch + j]);
        cany |= v;
        if (__any_sync(0xffffffffu, v) && (threadIdx.x & 31) == 0) rowany[i] = 1;
    }
    if (cany && j < W0) colany[j] = 1;
}

__global__ void p_bbox_final(const int* __restrict__ rowany, const int* __restrict__ colany, int H0, int W0,
                             int* bbox) {
    __shared__ int r0, r1, c0, c1;
    if (threadIdx.x == 0) { r0 = INT_MAX; r1 = -1; c0 = INT_MAX; c1 = -1; }
    __syncthreads();
    for (int i = threadIdx.x; i < H0; i += blockDim.x)
        if (rowany[i]) { atomicMin(&r0, i); atomicMax(&r1, i); }
    for (int j = threadIdx.x; j < W0; j += blockDim.x)
        if (colany[j]) { atomicMin(&c0, j); atomicMax(&c1, j); }
    __syncthreads();
    if (threadIdx.x == 0) {
        const bool any = r1 >= 0;
        bbox[0] = any ? r0 : 0;
        bbox[1] = any ? r1 + 1 : 0;
        bbox[2] = any ? c0 : 0;
        bbox[3] = any ? c1 + 1 : 0;
    }
}

cudaError_t unw_launch_bbox(const float* phase, long long pitch, int H0, int W0, int* rowany,
                            int* colany, int* bbox, cudaStream_t s) {
    cudaMemsetAsync(rowany, 0, sizeof(int) * (size_t)H0, s);
    cudaMemsetAsync(colany, 0, sizeof(int) * (size_t)W0, s);
    dim3 grid((W0 + 31) / 32, (H0 + 63) / 64);
    p_bbox_tiles<<<grid, 256, 0, s>>>(phase, pitch, H0, W0, rowany, colany);
    p_bbox_final<<<1, 1024, 0, s>>>(rowany, colany, H0, W0, bbox);
    return cudaGetLastError();
}

cudaError_t unw_launch_post(int which, int nblk, cudaStream_t s, const GridDev* gd, const int* starts,
                            int n, const UnwScalars& sc, const GridDev* host_grids) {
    (void)sc;
    if (nblk <= 0 && which != UNW_P_MEDIAN && which != UNW_P_TILESCAN && which != UNW_P_FILL)
        return cudaSuccess;
    switch (which) {
        case UNW_P_KSTATS: p_kstats<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_HIST: p_hist<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_MEDIAN: p_median<<<n, 1024, 0, s>>>(gd, n); break;
        case UNW_P_SHIFT_CCINIT: p_shift_ccinit<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_UNION: p_union<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_FLATTEN: p_flatten<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_TILESCAN: p_tilescan<<<n, 1024, 0, s>>>(gd, n); break;
        case UNW_P_LABEL: p_label<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_ACCUM: p_accum<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_ADJUST: p_adjust<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_WRITE: p_write<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_P_FILL: {
            long long mx = 1;
            for (int g = 0; g < n; g++) {
                const long long np = (long long)host_grids[g].H0 * host_grids[g].W0;
                mx = np > mx ? np : mx;
            }
            long long nb = (mx + 1023) / 1024;
            nb = nb > 1184 ? 1184 : nb;
            p_fill<<<dim3((unsigned)nb, (unsigned)n), 256, 0, s>>>(gd, n);
            break;
        }
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
