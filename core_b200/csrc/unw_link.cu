// Component linking: integer 2-pi offsets between separately unwrapped
// components (insardev/insardev/utils_unwrap2d.py:195-444, :886-1040, driven by
// Stack_unwrap2d.py:325-407).  The geometry the reference builds with cv2
// contours and shapely runs here on the pixel lattice:
//   * components: the IRLS labels (label order) or a union-find labelling of
//     the valid mask (size order); cid[p] = component index, -1 = keep the
//     pixel as it is (label 0), -2 = labelled component below min_size (NaN);
//   * border pixels (a 4-neighbour outside the component or the raster) per
//     component, grouped by row and sorted by x: one warp walks each image row
//     left to right, so the lists come out in raster order without a sort;
//   * convex hulls from the per-row extreme border pixels (two monotone
//     chains, one thread per component);
//   * neighbour ranking by exact hull distance, the closest border-pixel pair
//     of each candidate pair (row-indexed search: binary search in the rows
//     within the current best distance), the blocking test of the connecting
//     segment against third hulls, and the window means, summed in float32 in
//     numpy's pairwise order so that they equal np.nanmean bit for bit.
// The greedy choice of connections and the integer program stay on the host.
#include <cuda_runtime.h>
#include <stdint.h>
#include <limits.h>
#include <math.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

namespace {

constexpr int LK_LABELS = 65536;
constexpr int LK_PAIR_CHUNK = 1 << 18;   // candidate pairs per device pass
constexpr int LK_NBR_CHUNK = 1 << 22;    // neighbour-table entries per pass
constexpr int LK_MAX_K = 256;            // ranked neighbours per component
constexpr int LK_MAX_WIN = 31;           // window side (conncomp_linksize)
constexpr int SCAN_TILE = 4096;          // items per block in the scan
constexpr unsigned FULL = 0xffffffffu;
static_assert(sizeof(unw_link_pair) == 64, "unw_link_pair layout (mirrored by the ctypes binding)");

struct LkComp {
    int y0, y1, x0, x1;      // bounding box (inclusive)
    int size;                // pixels
    int rowoff;              // first per-row slot (rows y0..y1)
    int bstart, nb;          // border pixels in bpts[bstart, bstart + nb)
    int hoff, hn;            // hull vertices hv[hoff, hoff + hn), counter-clockwise
    int flags;               // UNW_LINK_C_*
    int pad;
};

struct LkLayout {
    size_t cid, par, rows, hv, comps, hist, map, roots, rsz, cnt, scan, nbr, pin, pout, kf, total;
    long long N, RS;          // pixels; row-slot capacity
    int NC;                   // component capacity
};

__host__ __device__ inline unsigned pack_yx(int y, int x) { return ((unsigned)y << 16) | (unsigned)x; }
__device__ inline int py_(unsigned v) { return (int)(v >> 16); }
__device__ inline int px_(unsigned v) { return (int)(v & 0xffffu); }

// ---------------------------------------------------------------------------- warp-grouped updates
// All 32 lanes call these with the same loop trip count; `act` marks lanes
// with a key.  Each distinct key in the warp is handled once by its lowest lane.
__device__ __forceinline__ void grp_count(int* ctr, int key, bool act) {
    const int lane = threadIdx.x & 31;
    unsigned pend = __ballot_sync(FULL, act);
    while (pend) {
        const int leader = __ffs(pend) - 1;
        const int lk = __shfl_sync(FULL, key, leader);
        const unsigned grp = __ballot_sync(FULL, act && key == lk);
        if (lane == leader) atomicAdd(&ctr[lk], __popc(grp));
        pend &= ~grp;
    }
}

__device__ __forceinline__ void grp_bbox(LkComp* C, int key, bool act, int y, int x) {
    const int lane = threadIdx.x & 31;
    unsigned pend = __ballot_sync(FULL, act);
    while (pend) {
        const int leader = __ffs(pend) - 1;
        const int lk = __shfl_sync(FULL, key, leader);
        const bool mine = act && key == lk;
        const unsigned grp = __ballot_sync(FULL, mine);
        const int ymin = __reduce_min_sync(FULL, mine ? y : INT_MAX);
        const int ymax = __reduce_max_sync(FULL, mine ? y : INT_MIN);
        const int xmin = __reduce_min_sync(FULL, mine ? x : INT_MAX);
        const int xmax = __reduce_max_sync(FULL, mine ? x : INT_MIN);
        if (lane == leader) {
            atomicMin(&C[lk].y0, ymin);
            atomicMax(&C[lk].y1, ymax);
            atomicMin(&C[lk].x0, xmin);
            atomicMax(&C[lk].x1, xmax);
        }
        pend &= ~grp;
    }
}

// ---------------------------------------------------------------------------- components
__global__ void k_lk_hist(const uint16_t* __restrict__ lab, long long lp, int H, int W, int* hist) {
    const long long N = (long long)H * W;
    for (long long b = (long long)blockIdx.x * blockDim.x; b < N; b += (long long)gridDim.x * blockDim.x) {
        const long long p = b + threadIdx.x;
        const bool act = p < N;
        const int key = act ? (int)lab[(p / W) * lp + p % W] : 0;
        grp_count(hist, key, act);
    }
}

__global__ void k_lk_cid_labels(const uint16_t* __restrict__ lab, long long lp, int H, int W,
                                const int* __restrict__ map, int* cid, LkComp* C) {
    const long long N = (long long)H * W;
    for (long long b = (long long)blockIdx.x * blockDim.x; b < N; b += (long long)gridDim.x * blockDim.x) {
        const long long p = b + threadIdx.x;
        const bool in = p < N;
        const int y = in ? (int)(p / W) : 0, x = in ? (int)(p % W) : 0;
        const int c = in ? map[lab[(long long)y * lp + x]] : -1;
        if (in) cid[p] = c;
        grp_bbox(C, c, c >= 0, y, x);
    }
}

__device__ __forceinline__ int uf_find(int* par, int x) {
    while (true) {
        const int q = par[x];
        if (q == x) return x;
        const int g = par[q];
        if (g != q) par[x] = g;   // path halving; g is an ancestor of x
        x = q;
    }
}

__device__ __forceinline__ void uf_unite(int* par, int a, int b) {
    while (true) {
        a = uf_find(par, a);
        b = uf_find(par, b);
        if (a == b) return;
        if (a > b) { const int t = a; a = b; b = t; }
        const int old = atomicCAS(&par[b], b, a);   // the larger root goes under the smaller
        if (old == b) return;
        b = old;
    }
}

__global__ void k_lk_uf_init(const float* __restrict__ ph, long long pp, int H, int W, int* par) {
    const long long N = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        const float v = ph[(p / W) * pp + p % W];
        par[p] = isnan(v) ? -1 : (int)p;
    }
}

__global__ void k_lk_uf_union(int H, int W, int* par) {
    const long long N = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        if (par[p] < 0) continue;
        const int x = (int)(p % W);
        if (x + 1 < W && par[p + 1] >= 0) uf_unite(par, (int)p, (int)p + 1);
        if (p + W < N && par[p + W] >= 0) uf_unite(par, (int)p, (int)(p + W));
    }
}

// After the unions: every pixel points at its root.  The walk only reads, so
// the one store to par[p] is this thread's and is never overwritten by another
// thread's path halving (which could leave p pointing at an inner node).
__global__ void k_lk_uf_flatten(int H, int W, int* par, int* cnt_px) {
    const long long N = (long long)H * W;
    for (long long b = (long long)blockIdx.x * blockDim.x; b < N; b += (long long)gridDim.x * blockDim.x) {
        const long long p = b + threadIdx.x;
        int r = -1;
        if (p < N && par[p] >= 0) {
            r = (int)p;
            for (int q = par[r]; q != r; q = par[r]) r = q;
            par[p] = r;
        }
        grp_count(cnt_px, r, r >= 0);     // component sizes at the root's slot
    }
}

__global__ void k_lk_roots(int H, int W, const int* __restrict__ par, const int* __restrict__ cnt_px, int min_size,
                           int* roots, int* rsz, int* nroot, int cap) {
    const long long N = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        if (par[p] != (int)p || cnt_px[p] < min_size) continue;
        const int s = atomicAdd(nroot, 1);
        if (s < cap) { roots[s] = (int)p; rsz[s] = cnt_px[p]; }
    }
}

// cid at every root: -2 (a component below min_size) ...
__global__ void k_lk_rootmark(int H, int W, const int* __restrict__ par, int* cid) {
    const long long N = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x)
        if (par[p] == (int)p) cid[p] = -2;
}

// ... then the component index at the kept roots (in size order) ...
__global__ void k_lk_rootmap(const int* __restrict__ roots_sorted, int n, int* cid) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) cid[roots_sorted[s]] = s;
}

// ... then every other pixel copies its root's value (roots are not written here).
__global__ void k_lk_cid_mask(int H, int W, const int* __restrict__ par, int* cid, LkComp* C) {
    const long long N = (long long)H * W;
    for (long long b = (long long)blockIdx.x * blockDim.x; b < N; b += (long long)gridDim.x * blockDim.x) {
        const long long p = b + threadIdx.x;
        int c = -1;
        int y = 0, x = 0;
        if (p < N) {
            y = (int)(p / W); x = (int)(p % W);
            const int r = par[p];
            if (r < 0) cid[p] = -1;
            else if (r == (int)p) c = cid[p];
            else { c = cid[r]; cid[p] = c; }
        }
        grp_bbox(C, c, c >= 0, y, x);
    }
}

__global__ void k_lk_comp_init(LkComp* C, int n) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        LkComp v{};
        v.y0 = INT_MAX; v.y1 = INT_MIN; v.x0 = INT_MAX; v.x1 = INT_MIN;
        C[c] = v;
    }
}

// ---------------------------------------------------------------------------- border lists
__global__ void k_lk_rows_init(int* xmin, int* xmax, int* cnt, long long RS) {
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s <= RS; s += (long long)gridDim.x * blockDim.x) {
        xmin[s] = INT_MAX;
        xmax[s] = -1;
        cnt[s] = 0;
    }
}

// One warp per image row, left to right in 32-pixel steps.  COUNT: per
// (component, row) slot the border count and the first / last border x.
// SCATTER: border pixels to bpts in x order from the slot's cursor.
template <bool SCATTER>
__global__ void k_lk_rows(const int* __restrict__ cid, int H, int W, const LkComp* __restrict__ C, int* xmin,
                          int* xmax, int* cnt, int* cur, unsigned* bpts) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int y = warp; y < H; y += nwarps) {
        const long long row = (long long)y * W;
        for (int x0 = 0; x0 < W; x0 += 32) {
            const int x = x0 + lane;
            const int c = x < W ? cid[row + x] : -1;
            bool b = false;
            if (c >= 0) {
                b = x == 0 || x == W - 1 || y == 0 || y == H - 1 || cid[row + x - 1] != c || cid[row + x + 1] != c ||
                    cid[row - W + x] != c || cid[row + W + x] != c;
            }
            unsigned pend = __ballot_sync(FULL, b);
            while (pend) {
                const int leader = __ffs(pend) - 1;
                const int lc = __shfl_sync(FULL, c, leader);
                const bool mine = b && c == lc;
                const unsigned grp = __ballot_sync(FULL, mine);
                const int s = C[lc].rowoff + (y - C[lc].y0);
                if (!SCATTER) {
                    if (lane == leader) {
                        if (xmin[s] == INT_MAX) xmin[s] = x;
                        cnt[s] += __popc(grp);
                    }
                    if (lane == 31 - __clz(grp)) xmax[s] = x;
                } else {
                    int base = 0;
                    if (lane == leader) base = cur[s];
                    base = __shfl_sync(FULL, base, leader);
                    if (mine) bpts[base + __popc(grp & ((1u << lane) - 1u))] = pack_yx(y, x);
                    if (lane == leader) cur[s] = base + __popc(grp);
                }
                pend &= ~grp;
            }
        }
    }
}

// Exclusive scan of a[0, n) in place, SCAN_TILE items per block; tile sums to sums[].
__global__ void k_scan_tiles(int* a, long long n, int* sums) {
    __shared__ int wsum[32];
    const long long base = (long long)blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    int v[4];
    int t = 0;
    for (int k = 0; k < 4; k++) {
        v[k] = base + k < n ? a[base + k] : 0;
        const int e = t;
        t += v[k];
        v[k] = e;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int inc = t;
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        int s = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += u;
        }
        wsum[lane] = s;
    }
    __syncthreads();
    const int off = (w > 0 ? wsum[w - 1] : 0) + inc - t;
    for (int k = 0; k < 4; k++)
        if (base + k < n) a[base + k] = v[k] + off;
    if (threadIdx.x == blockDim.x - 1 && sums) sums[blockIdx.x] = wsum[(blockDim.x >> 5) - 1];
}

__global__ void k_scan_add(int* a, long long n, const int* __restrict__ sums) {
    const long long base = (long long)blockIdx.x * SCAN_TILE;
    const int add = sums[blockIdx.x];
    for (int k = threadIdx.x; k < SCAN_TILE; k += blockDim.x)
        if (base + k < n) a[base + k] += add;
}

int scan_levels(int* a, long long n, int* scratch, cudaStream_t s) {
    const long long tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    k_scan_tiles<<<(unsigned)tiles, SCAN_TILE / 4, 0, s>>>(a, n, tiles > 1 ? scratch : nullptr);
    if (tiles > 1) {
        scan_levels(scratch, tiles, scratch + tiles, s);
        k_scan_add<<<(unsigned)tiles, 256, 0, s>>>(a, n, scratch);
    }
    return 0;
}

long long scan_scratch(long long n) {
    long long t = 0;
    while (n > 1) {
        n = (n + SCAN_TILE - 1) / SCAN_TILE;
        t += n;
    }
    return t + 4;
}

// ---------------------------------------------------------------------------- hulls
__device__ __forceinline__ long long crs(int ox, int oy, int ax, int ay, int bx, int by) {
    return (long long)(ax - ox) * (by - oy) - (long long)(ay - oy) * (bx - ox);
}
__device__ __forceinline__ long long crs_u(unsigned o, unsigned a, unsigned b) {
    return crs(px_(o), py_(o), px_(a), py_(a), px_(b), py_(b));
}

// One thread per component: right chain (x = last border x per row) and left
// chain (first border x per row) top to bottom, then the polygon right chain +
// reversed left chain, with collinear and duplicate junction vertices removed.
__global__ void k_lk_hull(LkComp* C, int n, const int* __restrict__ xmin, const int* __restrict__ xmax,
                          const int* __restrict__ rstart, unsigned* hv) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        LkComp& K = C[c];
        const int h = K.y1 - K.y0 + 1;
        K.bstart = rstart[K.rowoff];
        K.nb = rstart[K.rowoff + h] - K.bstart;
        K.hoff = 2 * K.rowoff;
        K.hn = 0;
        if (K.flags & UNW_LINK_C_LINE) continue;
        unsigned* R = hv + K.hoff;
        unsigned* L = R + h;
        int nr = 0, nl = 0;
        for (int r = 0; r < h; r++) {
            const unsigned pr = pack_yx(K.y0 + r, xmax[K.rowoff + r]);
            while (nr >= 2 && crs_u(R[nr - 2], R[nr - 1], pr) <= 0) nr--;
            R[nr++] = pr;
            const unsigned pl = pack_yx(K.y0 + r, xmin[K.rowoff + r]);
            while (nl >= 2 && crs_u(L[nl - 2], L[nl - 1], pl) >= 0) nl--;
            L[nl++] = pl;
        }
        // polygon: R[0..nr) then L reversed; L lies at offset h >= nr
        for (int a = 0, b = nl - 1; a < b; a++, b--) { const unsigned t = L[a]; L[a] = L[b]; L[b] = t; }
        int m = nr;
        for (int k = 0; k < nl; k++) {
            const unsigned v = L[k];
            if (k == 0 && v == R[nr - 1]) continue;            // bottom row of one pixel
            if (k == nl - 1 && v == R[0]) continue;            // top row of one pixel
            R[m++] = v;
        }
        // remove vertices with a non-left turn until none remain
        bool changed = true;
        for (int guard = 0; changed && m >= 3 && guard < 2 * h + 4; guard++) {
            changed = false;
            int w = 0;
            for (int k = 0; k < m; k++) {
                const unsigned prev = w > 0 ? R[w - 1] : R[m - 1];
                const unsigned next = R[(k + 1) % m];
                if (crs_u(prev, R[k], next) > 0) R[w++] = R[k];
                else changed = true;
            }
            m = w;
        }
        K.hn = m;
    }
}

// ---------------------------------------------------------------------------- hull distances
__device__ bool separated(const unsigned* P, int m, const unsigned* Q, int n) {
    for (int k = 0; k < m; k++) {
        const unsigned a = P[k], b = P[k + 1 == m ? 0 : k + 1];
        bool all_out = true;
        for (int q = 0; q < n && all_out; q++) all_out = crs_u(a, b, Q[q]) < 0;
        if (all_out) return true;
    }
    return false;
}

__device__ double pseg(unsigned p, unsigned a, unsigned b) {
    const long long dx = px_(b) - px_(a), dy = py_(b) - py_(a);
    const long long ux = px_(p) - px_(a), uy = py_(p) - py_(a);
    const long long t = ux * dx + uy * dy;
    if (t <= 0) return sqrt((double)(ux * ux + uy * uy));
    const long long L2 = dx * dx + dy * dy;
    if (t >= L2) {
        const long long vx = px_(p) - px_(b), vy = py_(p) - py_(b);
        return sqrt((double)(vx * vx + vy * vy));
    }
    const long long cr = dx * uy - dy * ux;
    return fabs((double)cr) / sqrt((double)L2);
}

// Distance between two convex hulls P (m vertices) and Q (n vertices): 0 when no edge of either
// separates them, else the smallest distance from a vertex of one to an edge of the other.  The
// 32 lanes of a warp share the edge and vertex loops (all lanes call it with the same arguments
// and get the same result).
__device__ bool warp_separated(const unsigned* P, int m, const unsigned* Q, int n) {
    bool found = false;
    for (int k0 = 0; k0 < m && !found; k0 += 32) {
        const int k = k0 + (threadIdx.x & 31);
        bool all_out = k < m;
        if (all_out) {
            const unsigned a = P[k], b = P[k + 1 == m ? 0 : k + 1];
            for (int q = 0; q < n && all_out; q++) all_out = crs_u(a, b, Q[q]) < 0;
        }
        found = __any_sync(FULL, all_out);
    }
    return found;
}

__device__ double warp_hull_dist(const unsigned* P, int m, const unsigned* Q, int n) {
    if (!warp_separated(P, m, Q, n) && !warp_separated(Q, n, P, m)) return 0.0;
    double d = INFINITY;
    for (int i = threadIdx.x & 31; i < m; i += 32)
        for (int k = 0; k < n; k++) d = fmin(d, pseg(P[i], Q[k], Q[k + 1 == n ? 0 : k + 1]));
    for (int i = threadIdx.x & 31; i < n; i += 32)
        for (int k = 0; k < m; k++) d = fmin(d, pseg(Q[i], P[k], P[k + 1 == m ? 0 : k + 1]));
    for (int o = 16; o > 0; o >>= 1) d = fmin(d, __shfl_xor_sync(FULL, d, o));
    return d;
}

__device__ __forceinline__ bool key_less(double da, int ja, double db, int jb) {
    return da < db || (da == db && ja < jb);
}

// Insert (d, j) into a thread's ascending list of at most K keys.
__device__ __forceinline__ void topk_insert(double* md, int* mj, int& cnt, int K, double d, int j) {
    if (cnt == K && !key_less(d, j, md[K - 1], mj[K - 1])) return;
    int pos = cnt < K ? cnt++ : K - 1;
    while (pos > 0 && key_less(d, j, md[pos - 1], mj[pos - 1])) {
        md[pos] = md[pos - 1];
        mj[pos] = mj[pos - 1];
        pos--;
    }
    md[pos] = d;
    mj[pos] = j;
}

// K rounds of a block-wide argmin over the heads of the per-thread lists:
// res[r] = r-th smallest key's index (-1 past the end).  All threads call it.
__device__ void topk_merge(const double* md, const int* mj, int cnt, int K, int* res, double* resd,
                           double* bd, int* bj, int* bt) {
    int head = 0;
    for (int r = 0; r < K; r++) {
        double d = head < cnt ? md[head] : INFINITY;
        int j = head < cnt ? mj[head] : INT_MAX;
        int t = threadIdx.x;
        for (int o = 16; o > 0; o >>= 1) {
            const double od = __shfl_down_sync(FULL, d, o);
            const int oj = __shfl_down_sync(FULL, j, o);
            const int ot = __shfl_down_sync(FULL, t, o);
            if (key_less(od, oj, d, j)) { d = od; j = oj; t = ot; }
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        if (lane == 0) { bd[w] = d; bj[w] = j; bt[w] = t; }
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int k = 1; k < (int)(blockDim.x >> 5); k++)
                if (key_less(bd[k], bj[k], bd[0], bj[0])) { bd[0] = bd[k]; bj[0] = bj[k]; bt[0] = bt[k]; }
            res[r] = bj[0] == INT_MAX ? -1 : bj[0];
            resd[r] = bd[0];
        }
        __syncthreads();
        if (bj[0] != INT_MAX && bt[0] == (int)threadIdx.x) head++;
        __syncthreads();
    }
}

__device__ __forceinline__ double bbox_dist(const LkComp& a, const LkComp& b) {
    const long long dx = max(0, max(b.x0 - a.x1, a.x0 - b.x1));
    const long long dy = max(0, max(b.y0 - a.y1, a.y0 - b.y1));
    return sqrt((double)(dx * dx + dy * dy));
}

// One block per component in [c0, c1): the K nearest other components by
// (hull distance, index); -1 pads.  The bounding-box distance bounds the hull
// distance from below, so: the K components nearest by that bound give exact
// distances whose largest, T, bounds the K-th nearest from above; only
// components with bound <= T need their exact distance.
__global__ void k_lk_nbr(const LkComp* __restrict__ C, int n, int c0, int c1, const unsigned* __restrict__ hv, int K,
                         int* nbr) {
    extern __shared__ unsigned char smem[];
    double* sd = (double*)smem;
    int* sj = (int*)(sd + (size_t)blockDim.x * K);
    __shared__ double bd[32], resd[LK_MAX_K], thr;
    __shared__ int bj[32], bt[32], res[LK_MAX_K];
    for (int i = c0 + blockIdx.x; i < c1; i += gridDim.x) {
        const LkComp Ci = C[i];
        double* md = sd + (size_t)threadIdx.x * K;
        int* mj = sj + (size_t)threadIdx.x * K;
        int cnt = 0;
        const bool ok = Ci.hn >= 3;
        // 1. the K nearest by the bounding-box bound
        if (ok)
            for (int j = threadIdx.x; j < n; j += blockDim.x) {
                if (j == i || C[j].hn < 3) continue;
                topk_insert(md, mj, cnt, K, bbox_dist(Ci, C[j]), j);
            }
        topk_merge(md, mj, cnt, K, res, resd, bd, bj, bt);
        // 2. their exact distances (one warp per component): the threshold
        if (threadIdx.x == 0) thr = res[K - 1] < 0 ? INFINITY : 0.0;
        __syncthreads();
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int r = warp; r < K; r += nw) {
            const int j = res[r];
            if (j < 0) continue;
            const double d = warp_hull_dist(hv + Ci.hoff, Ci.hn, hv + C[j].hoff, C[j].hn);
            if (lane == 0 && thr != INFINITY) atomicMax((unsigned long long*)&thr, (unsigned long long)__double_as_longlong(d));
        }
        __syncthreads();
        const double T = thr;
        // 3. exact distances within the threshold, one warp per component, into lane 0's list
        cnt = 0;
        if (ok)
            for (int j = warp; j < n; j += nw) {
                if (j == i) continue;
                const LkComp Cj = C[j];
                if (Cj.hn < 3 || bbox_dist(Ci, Cj) > T) continue;
                const double d = warp_hull_dist(hv + Ci.hoff, Ci.hn, hv + Cj.hoff, Cj.hn);
                if (lane == 0) topk_insert(md, mj, cnt, K, d, j);
            }
        topk_merge(md, mj, cnt, K, res, resd, bd, bj, bt);
        int* out = nbr + (size_t)(i - c0) * K;
        for (int r = threadIdx.x; r < K; r += blockDim.x) out[r] = res[r];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------- candidate pairs
__device__ __forceinline__ long long bbox_d2(int y, int x, const LkComp& T) {
    const long long dy = y < T.y0 ? T.y0 - y : (y > T.y1 ? y - T.y1 : 0);
    const long long dx = x < T.x0 ? T.x0 - x : (x > T.x1 ? x - T.x1 : 0);
    return dy * dy + dx * dx;
}

// first index k in [lo, hi) with bpts[k] >= key (row segment sorted by x)
__device__ __forceinline__ int lower_bound_u(const unsigned* a, int lo, int hi, unsigned key) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ unsigned long long pair_key(bool swap, int yq, int xq, int yt, int xt) {
    // (y_i, x_i, y_j, x_j): the query belongs to comp j when swap
    const unsigned long long a = swap ? pack_yx(yt, xt) : pack_yx(yq, xq);
    const unsigned long long b = swap ? pack_yx(yq, xq) : pack_yx(yt, xt);
    return (a << 32) | b;
}

__global__ void k_lk_pairs(const LkComp* __restrict__ C, const int2* __restrict__ pin, int np,
                           const unsigned* __restrict__ bpts, const int* __restrict__ rstart,
                           const unsigned* __restrict__ hv, int ncomp, unw_link_pair* pout) {
    __shared__ unsigned long long best, key;
    __shared__ int blocked;
    for (int b = blockIdx.x; b < np; b += gridDim.x) {
        const int i = pin[b].x, j = pin[b].y;
        const LkComp Ci = C[i], Cj = C[j];
        const bool swap = Cj.nb < Ci.nb;
        const LkComp S = swap ? Cj : Ci;
        const LkComp T = swap ? Ci : Cj;
        if (threadIdx.x == 0) { best = ULLONG_MAX; key = ULLONG_MAX; blocked = 0; }
        __syncthreads();
        // Closest pair with ties broken by (y_i, x_i, y_j, x_j).  The pruning is non-strict
        // (a query or a row is skipped only when its bound exceeds the best squared distance),
        // so every pair at the final minimum is seen: its query is not pruned, its row is within
        // the bound, and its pixel is the nearest on its side of the row.
        unsigned long long bd2 = ULLONG_MAX, bkey = ULLONG_MAX;
        auto take = [&](unsigned long long d2, unsigned long long k2) {
            if (d2 < bd2 || (d2 == bd2 && k2 < bkey)) { bd2 = d2; bkey = k2; }
        };
        for (int q = threadIdx.x; q < S.nb; q += blockDim.x) {
            const unsigned pq = bpts[S.bstart + q];
            const int yq = py_(pq), xq = px_(pq);
            unsigned long long loc = min(*(volatile unsigned long long*)&best, bd2);
            if ((unsigned long long)bbox_d2(yq, xq, T) > loc) continue;
            const long long dy_lo = max(0LL, (long long)max(T.y0 - yq, yq - T.y1));
            for (long long dy = dy_lo;; dy++) {
                if ((unsigned long long)(dy * dy) > loc) break;
                const bool up = yq - dy >= T.y0 && yq - dy <= T.y1;
                const bool dn = dy > 0 && yq + dy >= T.y0 && yq + dy <= T.y1;
                if (!up && !dn && (yq - dy < T.y0 && yq + dy > T.y1)) break;
                for (int side = 0; side < 2; side++) {
                    if (side == 0 ? !up : !dn) continue;
                    const int y = side == 0 ? (int)(yq - dy) : (int)(yq + dy);
                    const int s = T.rowoff + (y - T.y0);
                    const int lo = rstart[s], hi = rstart[s + 1];
                    const int k = lower_bound_u(bpts, lo, hi, pack_yx(y, xq));
                    if (k < hi) {
                        const long long dx = px_(bpts[k]) - xq;
                        take((unsigned long long)(dx * dx + dy * dy), pair_key(swap, yq, xq, y, px_(bpts[k])));
                    }
                    if (k > lo) {
                        const long long dx = xq - px_(bpts[k - 1]);
                        take((unsigned long long)(dx * dx + dy * dy), pair_key(swap, yq, xq, y, px_(bpts[k - 1])));
                    }
                    loc = min(loc, bd2);
                }
            }
            atomicMin(&best, bd2);
        }
        __syncthreads();
        const unsigned long long dmin = best;
        if (bd2 == dmin) atomicMin(&key, bkey);
        __syncthreads();
        const unsigned long long kk = key;
        const unsigned pi = (unsigned)(kk >> 32), pj = (unsigned)kk;
        // blocking: the closed segment against the hulls of third components
        const int ax = px_(pi), ay = py_(pi), bx = px_(pj), by = py_(pj);
        const int sx0 = min(ax, bx), sx1 = max(ax, bx), sy0 = min(ay, by), sy1 = max(ay, by);
        for (int k = threadIdx.x; k < ncomp && !*(volatile int*)&blocked; k += blockDim.x) {
            if (k == i || k == j) continue;
            const LkComp Ck = C[k];
            if (Ck.hn < 3 || Ck.x1 < sx0 || Ck.x0 > sx1 || Ck.y1 < sy0 || Ck.y0 > sy1) continue;
            const unsigned* Hk = hv + Ck.hoff;
            const unsigned seg[2] = {pi, pj};
            if (separated(Hk, Ck.hn, seg, 2)) continue;
            bool pos = true, neg = true;
            for (int v = 0; v < Ck.hn; v++) {
                const long long cr = crs_u(pi, pj, Hk[v]);
                pos = pos && cr > 0;
                neg = neg && cr < 0;
            }
            if (!pos && !neg) blocked = 1;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unw_link_pair o{};
            o.comp_i = i; o.comp_j = j;
            o.yi = py_(pi); o.xi = px_(pi); o.yj = py_(pj); o.xj = px_(pj);
            o.d2 = (int64_t)dmin;
            o.blocked = blocked;
            pout[b] = o;
        }
        __syncthreads();
    }
}

// numpy's float32 pairwise sum (blocks of 8 accumulators up to 128 items,
// halves at a multiple of 8 above), which np.sum / np.nanmean use on a
// contiguous vector.  The halving is unrolled at compile time: a window of at
// most 31 x 31 = 961 values needs three levels above the 128-item leaf.
__device__ __forceinline__ float pairwise_leaf(const float* a, int n) {
    if (n < 8) {
        float r = 0.f;
        for (int i = 0; i < n; i++) r = __fadd_rn(r, a[i]);
        return r;
    }
    float r[8];
    for (int j = 0; j < 8; j++) r[j] = a[j];
    int i = 8;
    for (; i < n - (n % 8); i += 8)
        for (int j = 0; j < 8; j++) r[j] = __fadd_rn(r[j], a[i + j]);
    float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                          __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; i++) res = __fadd_rn(res, a[i]);
    return res;
}

template <int D>
__device__ __forceinline__ float pairwise_sum(const float* a, int n) {
    if (n <= 128) return pairwise_leaf(a, n);
    int n2 = n / 2;
    n2 -= n2 % 8;
    return __fadd_rn(pairwise_sum<D - 1>(a, n2), pairwise_sum<D - 1>(a + n2, n - n2));
}

template <>
__device__ __forceinline__ float pairwise_sum<0>(const float* a, int n) {
    return pairwise_leaf(a, n);   // n <= 128 here for n <= 1024 at the top
}

// One thread per (pair, side): the window of 2*half+1 pixels around the
// connection pixel, values of the side's component in raster order,
// np.nanmean of them (utils_unwrap2d.py:403-414).
__global__ void k_lk_window(const float* __restrict__ ph, long long pp, const int* __restrict__ cid, int H, int W,
                            int half, unw_link_pair* pout, int np) {
    float v[LK_MAX_WIN * LK_MAX_WIN];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * np; t += gridDim.x * blockDim.x) {
        unw_link_pair& o = pout[t >> 1];
        const bool side = t & 1;
        const int c = side ? o.comp_j : o.comp_i;
        const int cy = side ? o.yj : o.yi, cx = side ? o.xj : o.xi;
        const int y0 = max(0, cy - half), y1 = min(H, cy + half + 1);
        const int x0 = max(0, cx - half), x1 = min(W, cx + half + 1);
        int n = 0, nf = 0;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) {
                if (cid[(long long)y * W + x] != c) continue;
                const float val = ph[(long long)y * pp + x];
                if (isnan(val)) v[n++] = 0.f;
                else { v[n++] = val; nf++; }
            }
        const float mean = nf ? (float)((double)pairwise_sum<4>(v, n) / (double)nf) : __int_as_float(0x7fc00000);
        if (side) { o.n_j = n; o.nf_j = nf; o.mean_j = mean; }
        else { o.n_i = n; o.nf_i = nf; o.mean_i = mean; }
    }
}

// ---------------------------------------------------------------------------- apply
__global__ void k_lk_apply(const float* __restrict__ ph, long long pp, const int* __restrict__ cid, int H, int W,
                           const float* __restrict__ kf, float* out, long long op) {
    const long long N = (long long)H * W;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        const long long y = p / W, x = p % W;
        const int c = cid[p];
        float v = ph[y * pp + x];
        if (c == -2) v = __int_as_float(0x7fc00000);
        else if (c >= 0 && kf[c] != 0.f) v = __fadd_rn(v, kf[c]);
        out[y * op + x] = v;
    }
}

// ---------------------------------------------------------------------------- host
LkLayout lk_layout(long long H, long long W, int min_size) {
    LkLayout L{};
    L.N = H * W;
    L.RS = L.N;
    const long long nc = L.N / std::max(min_size, 1) + 1;
    L.NC = (int)std::min<long long>(nc, INT_MAX / 64);
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    size_t o = 0;
    L.cid = o; o = up(o + sizeof(int) * (size_t)L.N);
    L.par = o; o = up(o + sizeof(int) * (size_t)L.N);        // union-find parents, later the border lists
    L.rows = o; o = up(o + sizeof(int) * 4 * (size_t)(L.RS + 1));
    L.hv = o; o = up(o + sizeof(unsigned) * 2 * (size_t)L.RS);
    L.comps = o; o = up(o + sizeof(LkComp) * (size_t)L.NC);
    L.hist = o; o = up(o + sizeof(int) * LK_LABELS);
    L.map = o; o = up(o + sizeof(int) * LK_LABELS);
    L.roots = o; o = up(o + sizeof(int) * (size_t)L.NC);
    L.rsz = o; o = up(o + sizeof(int) * (size_t)L.NC);
    L.cnt = o; o = up(o + sizeof(int) * 16);
    L.scan = o; o = up(o + sizeof(int) * (size_t)scan_scratch(L.RS + 1));
    L.nbr = o; o = up(o + sizeof(int) * (size_t)LK_NBR_CHUNK);
    L.pin = o; o = up(o + sizeof(int2) * (size_t)LK_PAIR_CHUNK);
    L.pout = o; o = up(o + sizeof(unw_link_pair) * (size_t)LK_PAIR_CHUNK);
    L.kf = o; o = up(o + sizeof(float) * (size_t)L.NC);
    L.total = o + 256;
    return L;
}

#define LK_CK(x)                                                                            \
    do {                                                                                    \
        const cudaError_t e_ = (x);                                                         \
        if (e_ != cudaSuccess) return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e_));    \
    } while (0)

int grid_for(long long n, int threads) {
    const long long g = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(g, 148LL * 16));
}

char* lk_base(void* ws) { return (char*)(((size_t)ws + 255) / 256 * 256); }

}  // namespace

extern "C" {

size_t unw_link_workspace_bytes(int64_t H, int64_t W, int32_t min_size) {
    if (H <= 0 || W <= 0 || H > 65535 || W > 65535 || H * W > INT_MAX - 1) return 0;
    return lk_layout(H, W, std::max(min_size, 1)).total;
}

int unw_link_pairs_f32(const float* phase, int64_t phase_pitch, const uint16_t* labels, int64_t label_pitch,
                       int64_t H, int64_t W, const unw_link_params* prm, int64_t* comp_label, int64_t* comp_size,
                       int32_t* comp_flags, int32_t comp_cap, int32_t* n_comp, unw_link_pair* pairs,
                       int32_t pair_cap, int32_t* n_pairs, void* workspace, size_t workspace_bytes,
                       void* cuda_stream) {
    if (!phase || !prm || !n_comp || !n_pairs || !workspace) return unw_set_error(UNW_E_ARG, "link: null pointer");
    if (H <= 0 || W <= 0 || phase_pitch < W || (labels && label_pitch < W))
        return unw_set_error(UNW_E_ARG, "link: bad shape or pitch");
    if (H > 65535 || W > 65535 || H * W > INT_MAX - 1)
        return unw_set_error(UNW_E_UNSUPPORTED, "link: grid sides above 65535 or more than 2^31 pixels");
    const int min_size = std::max(prm->min_size, 1);
    const int K = prm->max_neighbors;
    if (K < 0 || prm->window < 0 || prm->window > LK_MAX_WIN)
        return unw_set_error(UNW_E_ARG, "link: max_neighbors >= 0 and window in [0, 31]");
    const LkLayout L = lk_layout(H, W, min_size);
    char* base = lk_base(workspace);
    if ((size_t)(base - (char*)workspace) + L.total - 256 > workspace_bytes)
        return unw_set_error(UNW_E_WORKSPACE, "link: workspace too small");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    int* cid = (int*)(base + L.cid);
    int* par = (int*)(base + L.par);
    unsigned* bpts = (unsigned*)(base + L.par);
    int* rxmin = (int*)(base + L.rows);
    int* rxmax = rxmin + (L.RS + 1);
    int* rcnt = rxmax + (L.RS + 1);
    int* rcur = rcnt + (L.RS + 1);
    unsigned* hv = (unsigned*)(base + L.hv);
    LkComp* C = (LkComp*)(base + L.comps);
    int* hist = (int*)(base + L.hist);
    int* map = (int*)(base + L.map);
    int* roots = (int*)(base + L.roots);
    int* rsz = (int*)(base + L.rsz);
    int* cnt = (int*)(base + L.cnt);
    int* scr = (int*)(base + L.scan);
    int* nbr = (int*)(base + L.nbr);
    int2* pin = (int2*)(base + L.pin);
    unw_link_pair* pout = (unw_link_pair*)(base + L.pout);
    const int Hi = (int)H, Wi = (int)W;
    const long long N = L.N;
    const int gpx = grid_for(N, 256);

    // 1. components
    int n = 0;
    std::vector<int64_t> hlabel, hsize;
    if (labels) {
        LK_CK(cudaMemsetAsync(hist, 0, sizeof(int) * LK_LABELS, s));
        k_lk_hist<<<gpx, 256, 0, s>>>(labels, label_pitch, Hi, Wi, hist);
        std::vector<int> h(LK_LABELS), m(LK_LABELS, -1);
        LK_CK(cudaMemcpyAsync(h.data(), hist, sizeof(int) * LK_LABELS, cudaMemcpyDeviceToHost, s));
        LK_CK(cudaStreamSynchronize(s));
        for (int lab = 1; lab < LK_LABELS; lab++) {
            if (h[lab] >= min_size) {
                m[lab] = n++;
                hlabel.push_back(lab);
                hsize.push_back(h[lab]);
            } else if (h[lab] > 0) {
                m[lab] = -2;
            }
        }
        if (n > L.NC) return unw_set_error(UNW_E_OVERFLOW, "link: component capacity");
        LK_CK(cudaMemcpyAsync(map, m.data(), sizeof(int) * LK_LABELS, cudaMemcpyHostToDevice, s));
        k_lk_comp_init<<<grid_for(std::max(n, 1), 256), 256, 0, s>>>(C, n);
        k_lk_cid_labels<<<gpx, 256, 0, s>>>(labels, label_pitch, Hi, Wi, map, cid, C);
    } else {
        k_lk_uf_init<<<gpx, 256, 0, s>>>(phase, phase_pitch, Hi, Wi, par);
        k_lk_uf_union<<<gpx, 256, 0, s>>>(Hi, Wi, par);
        LK_CK(cudaMemsetAsync(cid, 0, sizeof(int) * (size_t)N, s));
        k_lk_uf_flatten<<<gpx, 256, 0, s>>>(Hi, Wi, par, cid);
        LK_CK(cudaMemsetAsync(cnt, 0, sizeof(int) * 16, s));
        k_lk_roots<<<gpx, 256, 0, s>>>(Hi, Wi, par, cid, min_size, roots, rsz, cnt, L.NC);
        int nr = 0;
        LK_CK(cudaMemcpyAsync(&nr, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
        LK_CK(cudaStreamSynchronize(s));
        if (nr > L.NC) return unw_set_error(UNW_E_OVERFLOW, "link: component capacity");
        std::vector<int> r(nr), z(nr);
        if (nr) {
            LK_CK(cudaMemcpyAsync(r.data(), roots, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
            LK_CK(cudaMemcpyAsync(z.data(), rsz, sizeof(int) * nr, cudaMemcpyDeviceToHost, s));
            LK_CK(cudaStreamSynchronize(s));
        }
        std::vector<int> order(nr);
        for (int k = 0; k < nr; k++) order[k] = k;
        // size descending; equal sizes: the later first pixel (larger scipy label) first
        std::sort(order.begin(), order.end(), [&](int a, int b) { return z[a] != z[b] ? z[a] > z[b] : r[a] > r[b]; });
        std::vector<int> rs(nr);
        for (int k = 0; k < nr; k++) {
            rs[k] = r[order[k]];
            hlabel.push_back(r[order[k]]);
            hsize.push_back(z[order[k]]);
        }
        n = nr;
        k_lk_rootmark<<<gpx, 256, 0, s>>>(Hi, Wi, par, cid);
        if (n) {
            LK_CK(cudaMemcpyAsync(roots, rs.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
            k_lk_rootmap<<<grid_for(n, 256), 256, 0, s>>>(roots, n, cid);
        }
        k_lk_comp_init<<<grid_for(std::max(n, 1), 256), 256, 0, s>>>(C, n);
        k_lk_cid_mask<<<gpx, 256, 0, s>>>(Hi, Wi, par, cid, C);
    }
    LK_CK(cudaGetLastError());
    *n_comp = n;
    *n_pairs = 0;

    // 2. bounding boxes -> row slots
    std::vector<LkComp> hc(n);
    if (n) {
        LK_CK(cudaMemcpyAsync(hc.data(), C, sizeof(LkComp) * n, cudaMemcpyDeviceToHost, s));
        LK_CK(cudaStreamSynchronize(s));
    }
    long long RS = 0;
    int nvalid = 0;
    for (int c = 0; c < n; c++) {
        LkComp& K0 = hc[c];
        K0.size = (int)hsize[c];
        K0.rowoff = (int)RS;
        RS += K0.y1 - K0.y0 + 1;
        K0.flags = (K0.y0 == K0.y1 || K0.x0 == K0.x1) ? UNW_LINK_C_LINE : 0;
        if (!K0.flags) nvalid++;
    }
    if (RS > L.RS) return unw_set_error(UNW_E_OVERFLOW, "link: row slots");
    if (comp_cap < n) return unw_set_error(UNW_E_WORKSPACE, "link: component arrays too small (see n_comp)");
    for (int c = 0; c < n; c++) {
        if (comp_label) comp_label[c] = hlabel[c];
        if (comp_size) comp_size[c] = hsize[c];
        if (comp_flags) comp_flags[c] = hc[c].flags;
    }
    if (n < 2) return UNW_OK;
    LK_CK(cudaMemcpyAsync(C, hc.data(), sizeof(LkComp) * n, cudaMemcpyHostToDevice, s));

    // 3. border lists and hulls
    k_lk_rows_init<<<grid_for(RS + 1, 256), 256, 0, s>>>(rxmin, rxmax, rcnt, RS);
    const int grows = grid_for((long long)H * 32, 256);
    k_lk_rows<false><<<grows, 256, 0, s>>>(cid, Hi, Wi, C, rxmin, rxmax, rcnt, nullptr, nullptr);
    scan_levels(rcnt, RS + 1, scr, s);
    LK_CK(cudaMemcpyAsync(rcur, rcnt, sizeof(int) * (size_t)(RS + 1), cudaMemcpyDeviceToDevice, s));
    k_lk_rows<true><<<grows, 256, 0, s>>>(cid, Hi, Wi, C, rxmin, rxmax, rcnt, rcur, bpts);
    k_lk_hull<<<grid_for(n, 64), 64, 0, s>>>(C, n, rxmin, rxmax, rcnt, hv);
    LK_CK(cudaGetLastError());

    // 4. candidate pairs: each component with its K nearest (all when K >= nvalid - 1)
    std::vector<std::pair<int, int>> cand;
    if (K >= nvalid - 1) {
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                if (!hc[a].flags && !hc[b].flags) cand.emplace_back(a, b);
    } else if (K > 0) {
        if (K > LK_MAX_K) return unw_set_error(UNW_E_UNSUPPORTED, "link: max_neighbors above 256 with more components");
        int threads = 256;
        while (threads > 32 && (size_t)threads * K * 12 > 96 * 1024) threads >>= 1;
        const size_t smem = (size_t)threads * K * 12;
        LK_CK(unw_smem_limit((const void*)k_lk_nbr));
        const int rows = std::max(1, LK_NBR_CHUNK / K);
        std::vector<int> hn((size_t)rows * K);
        for (int c0 = 0; c0 < n; c0 += rows) {
            const int c1 = std::min(n, c0 + rows);
            k_lk_nbr<<<std::min(c1 - c0, 148 * 8), threads, smem, s>>>(C, n, c0, c1, hv, K, nbr);
            LK_CK(cudaGetLastError());
            LK_CK(cudaMemcpyAsync(hn.data(), nbr, sizeof(int) * (size_t)(c1 - c0) * K, cudaMemcpyDeviceToHost, s));
            LK_CK(cudaStreamSynchronize(s));
            for (int c = c0; c < c1; c++)
                for (int r = 0; r < K; r++) {
                    const int j = hn[(size_t)(c - c0) * K + r];
                    if (j >= 0) cand.emplace_back(std::min(c, j), std::max(c, j));
                }
        }
        std::sort(cand.begin(), cand.end());
        cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    }
    const long long P = (long long)cand.size();
    if (P > INT_MAX) return unw_set_error(UNW_E_OVERFLOW, "link: candidate pairs");
    *n_pairs = (int)P;
    if (pair_cap < P) return unw_set_error(UNW_E_WORKSPACE, "link: pair array too small (see n_pairs)");
    if (P && !pairs) return unw_set_error(UNW_E_ARG, "link: pairs is NULL");

    // 5. closest pixels, blocking and window means, chunk by chunk
    std::vector<int2> hp(std::min<long long>(P, LK_PAIR_CHUNK));
    for (long long p0 = 0; p0 < P; p0 += LK_PAIR_CHUNK) {
        const int m = (int)std::min<long long>(LK_PAIR_CHUNK, P - p0);
        for (int k = 0; k < m; k++) hp[k] = make_int2(cand[p0 + k].first, cand[p0 + k].second);
        LK_CK(cudaMemcpyAsync(pin, hp.data(), sizeof(int2) * m, cudaMemcpyHostToDevice, s));
        k_lk_pairs<<<std::min(m, 148 * 16), 256, 0, s>>>(C, pin, m, bpts, rcnt, hv, n, pout);
        k_lk_window<<<grid_for(2LL * m, 128), 128, 0, s>>>(phase, phase_pitch, cid, Hi, Wi, prm->window / 2, pout, m);
        LK_CK(cudaGetLastError());
        LK_CK(cudaMemcpyAsync(pairs + p0, pout, sizeof(unw_link_pair) * m, cudaMemcpyDeviceToHost, s));
    }
    LK_CK(cudaStreamSynchronize(s));
    return UNW_OK;
}

int unw_link_apply_f32(const float* phase, int64_t phase_pitch, int64_t H, int64_t W, const int32_t* k,
                       int32_t n_comp, float* out, int64_t out_pitch, void* workspace, size_t workspace_bytes,
                       int32_t min_size, void* cuda_stream) {
    if (!phase || !out || !workspace || (n_comp > 0 && !k)) return unw_set_error(UNW_E_ARG, "link apply: null pointer");
    if (H <= 0 || W <= 0 || phase_pitch < W || out_pitch < W || n_comp < 0)
        return unw_set_error(UNW_E_ARG, "link apply: bad shape or pitch");
    if (H > 65535 || W > 65535 || H * W > INT_MAX - 1)
        return unw_set_error(UNW_E_UNSUPPORTED, "link apply: grid too large");
    const LkLayout L = lk_layout(H, W, std::max(min_size, 1));
    char* base = lk_base(workspace);
    if ((size_t)(base - (char*)workspace) + L.total - 256 > workspace_bytes)
        return unw_set_error(UNW_E_WORKSPACE, "link apply: workspace too small");
    if (n_comp > L.NC) return unw_set_error(UNW_E_ARG, "link apply: n_comp above capacity");
    cudaStream_t s = (cudaStream_t)cuda_stream;
    float* kf = (float*)(base + L.kf);
    std::vector<float> h(std::max(n_comp, 1));
    // k * 2 * pi in float64, rounded once to float32 (a Python float added to float32 data)
    for (int c = 0; c < n_comp; c++) h[c] = (float)((double)(k[c] * 2) * 3.141592653589793);
    if (n_comp) LK_CK(cudaMemcpyAsync(kf, h.data(), sizeof(float) * n_comp, cudaMemcpyHostToDevice, s));
    k_lk_apply<<<grid_for(L.N, 256), 256, 0, s>>>(phase, phase_pitch, (const int*)(base + L.cid), (int)H, (int)W, kf,
                                                 out, out_pitch);
    LK_CK(cudaGetLastError());
    LK_CK(cudaStreamSynchronize(s));
    return UNW_OK;
}

}  // extern "C"
