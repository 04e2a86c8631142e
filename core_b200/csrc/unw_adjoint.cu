// Kernels of the frozen-weight adjoint (unw_adjoint_f32).
//
// The differentiated map: with the IRLS scale s = 1/sqrt(r^2 + eps^2) of the
// forward solution frozen (utils_unwrap2d.py:1560-1574), together with the
// valid mask, its components and the median 2-pi shift, the output is
//   out = u* + wrap(circmean(phase) - circmean(u*)) per component (- 2 pi k_med),
//   u*  = A(wI)^+ b,  A = -div(wI grad), b = -div(wI g),  wI = clip(wx s, 1e-6, 1e6),
// g the wrapped phase differences and wx the edge-averaged clipped coherence
// (utils_unwrap2d.py:1228-1290, :1367-1388, :1576-1581, :1667-1716).
// For dL/dout = G:
//   G'     = G - S_c (C_u cos u* + S_u sin u*) / (S_u^2 + C_u^2)     (through circmean(u*))
//   lambda = A^+ G'                                                  (PCG, same preconditioner)
//   dL/dphase  = A lambda + S_c (C_p cos phase + S_p sin phase) / (S_p^2 + C_p^2)
//   dL/dwI_e   = (D lambda)_e (g - D u*)_e,  dwI/dwx = wI / wx where wI is not clipped,
//   dL/dweight = sum over the pixel's valid edges of dL/dwx_e / 2, times the
//                derivative of clip(weight, 0.01, 1)
// with S_c the sum of G over the component and S/C the per-component sin/cos
// sums.
//
// Precision.  With u spanning many cycles, |sum exp(i u*)| is a small fraction rho of
// the component's pixel count (about 1% on a 1024^2 grid with +-40 rad of relief), and
// the alignment terms above are S_c / (rho N) times O(1): an error e in u* moves the
// gradient by about |mean G| e / rho, so a 1e-4 relative gradient needs u* to about
// 1e-7 rad.  Hence: u* is the float64 solution of the frozen system (iterative
// refinement, each residual formed in float64 with the phase differences in float64,
// each correction from the float32 PCG, accumulated in the float32 iterate pair), the
// sin/cos sums and per-pixel terms are float64 of the pair, and dL/dphase is formed in
// float64 without passing through a float32 intermediate.
#include "unw_kernels.h"
#include "unw_rowops.cuh"

#define UNW_ROWS_LOOP(G, local, nct)                     \
    for (int i = (local); i < (G).H; i += (nct))         \
        for (int j = threadIdx.x; j < (G).W; j += blockDim.x)

// u (forward output, NaN outside the valid pixels) -> iterate pair (U0, L0 = 0) on the crop, NaN -> 0;
// dL/dout -> z (unused by the solver), 0 at invalid pixels.
__global__ void k_adj_load(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const long long gi = (long long)(G.r0 + i), gj = (long long)(G.c0 + j);
        const float uv = G.a_u[gi * G.a_u_pitch + gj];
        const float gv = G.a_gu[gi * G.a_gu_pitch + gj];
        const bool v = G.valid[o] != 0;
        G.U0[o] = (v && isfinite(uv)) ? uv : 0.f;
        G.L0[o] = 0.f;
        G.z[o] = (v && isfinite(gv)) ? gv : 0.f;
    }
}

// wrapped difference of the NaN-filled phase in float64 (the differentiated map's g)
__device__ __forceinline__ double adj_ph(const GridDev& G, int i, int j) {
    const float p = G.phase[(long long)i * G.phase_pitch + j];
    return isnan(p) ? 0.0 : (double)p;
}
__device__ __forceinline__ double wrap_d(double d) {
    const double two_pi = 6.283185307179586;
    return d - two_pi * rint(d / two_pi);
}

__device__ __forceinline__ double dcircmean(double s, double c, double x) {
    const double d = s * s + c * c;
    double sn, cs;
    sincos(x, &sn, &cs);
    return d > 0.0 ? (c * cs + s * sn) / d : 0.0;
}

// r = b - A u* in float64 for the frozen weights, with the phase differences in float64:
// r_q = sum over the pixel's edges of +-wI_e (g_e - (D u*)_e), u* the pair (U1, L1) in
// float64.  WRITE 0 measures: ||r|| / ||b_64|| -> resid_rel, and the scale that brings
// ||r|| up to ||b_64|| -> refine_scale (the PCG's stop on a tiny r.z is absolute, so the
// correction solve runs on the scaled residual); a residual below 1e-13 of ||b_64||
// switches the instance off for the pass (the next REARM resets it).  WRITE 1 stores
// scale * r as the correction's right-hand side (b) and x0 = 0 in (U0, L0).
template <int WRITE>
__global__ void k_adj_refine(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!st->irls_active) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const long long npx = (long long)H * W;
    const double scale = WRITE ? st->refine_scale : 0.0;
    double acc[2] = {0.0, 0.0};
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        const size_t o = (size_t)i * P + j;
        const double x = pair_val(G.U1[o], G.L1[o]);
        const double ph = adj_ph(G, i, j);
        double r = 0.0, b = 0.0;
        if (j < W - 1) {
            const double e = wrap_d(adj_ph(G, i, j + 1) - ph), w = (double)G.wIx[o];
            r -= w * (e - (pair_val(G.U1[o + 1], G.L1[o + 1]) - x));
            b -= w * e;
        }
        if (j > 0) {
            const double e = wrap_d(ph - adj_ph(G, i, j - 1)), w = (double)G.wIx[o - 1];
            r += w * (e - (x - pair_val(G.U1[o - 1], G.L1[o - 1])));
            b += w * e;
        }
        if (i < H - 1) {
            const double e = wrap_d(adj_ph(G, i + 1, j) - ph), w = (double)G.wIy[o];
            r -= w * (e - (pair_val(G.U1[o + P], G.L1[o + P]) - x));
            b -= w * e;
        }
        if (i > 0) {
            const double e = wrap_d(ph - adj_ph(G, i - 1, j)), w = (double)G.wIy[o - P];
            r += w * (e - (x - pair_val(G.U1[o - P], G.L1[o - P])));
            b += w * e;
        }
        if (WRITE) {
            G.b[o] = (float)(r * scale);
            G.U0[o] = 0.f;
            G.L0[o] = 0.f;
        } else {
            acc[0] += r * r;
            acc[1] += b * b;
        }
    }
    if (WRITE) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) {
            const double rel = acc[1] > 0.0 ? sqrt(acc[0] / acc[1]) : sqrt(acc[0]);
            st->resid_rel = rel;
            st->refine_scale = acc[0] > 0.0 ? (acc[1] > 0.0 ? sqrt(acc[1] / acc[0]) : 1.0 / sqrt(acc[0])) : 1.0;
            if (!isfinite(rel) || !isfinite(st->refine_scale) || rel < 1e-13) st->irls_active = 0;
        }
    }
}

// u* += D / refine_scale (the correction solve's x - x0), in float64 into the pair
// (U1, L1); the pass's PCG iterations -> cg_log[2 + k]
__global__ void k_adj_addd(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n, int k) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!st->irls_active) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    if (local == 0 && threadIdx.x == 0 && 2 + k < UNW_MAX_LOG) st->cg_log[2 + k] = st->cg_iter;
    const double inv = 1.0 / st->refine_scale;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const float d = G.D[o];
        if (!isfinite(d)) continue;
        float hi, lo;
        split_pair(pair_val(G.U1[o], G.L1[o]) + (double)d * inv, hi, lo);
        G.U1[o] = hi;
        G.L1[o] = lo;
    }
}

// Per-component sums in float64 (parent[] holds the label after the post pipeline's
// accumulation): dL/dout -> adj[L]; sin/cos of the phase and of u* (the pair) -> csum
// (both zeroed by the host), replacing the forward alignment's float32-argument sums.
__global__ void k_adj_lsum(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int nlab = G.st->n_labels;
    const int W = G.W, P = G.P;
    const size_t cap = (size_t)G.lab_cap;
    const long long npx = (long long)G.H * W;
    for (long long q0 = (long long)local * blockDim.x; q0 < npx; q0 += (long long)nct * blockDim.x) {
        const long long q = q0 + threadIdx.x;
        int L = 0;
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (q < npx) {
            const int i = (int)(q / W), j = (int)(q - (long long)i * W);
            const size_t o = (size_t)i * P + j;
            if (G.valid[o]) {
                const int l = G.parent[q];
                if (l >= 1 && l <= nlab && l < G.lab_cap) {
                    L = l;
                    v[0] = (double)G.z[o];
                    sincos(adj_ph(G, i, j), &v[1], &v[2]);
                    sincos(pair_val(G.U1[o], G.L1[o]), &v[3], &v[4]);
                }
            }
        }
        const int L0 = __shfl_sync(0xffffffffu, L, 0);
        if (__all_sync(0xffffffffu, L == L0)) {
            if (L0 == 0) continue;
#pragma unroll
            for (int s = 16; s > 0; s >>= 1)
#pragma unroll
                for (int c = 0; c < 5; c++) v[c] += __shfl_down_sync(0xffffffffu, v[c], s);
            L = (threadIdx.x & 31) == 0 ? L0 : 0;
        }
        if (L > 0) {
            atomicAdd(&G.adj[L], v[0]);
            atomicAdd(&G.csum[L], v[1]);
            atomicAdd(&G.csum[cap + L], v[2]);
            atomicAdd(&G.csum[2 * cap + L], v[3]);
            atomicAdd(&G.csum[3 * cap + L], v[4]);
        }
    }
}

// right-hand side of the adjoint solve, b = G' (valid) / 0, and x0 = 0 in (U0, L0); the
// PCG then accumulates lambda = x - x0 in D
__global__ void k_adj_rhs(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const size_t cap = (size_t)G.lab_cap;
    const int nlab = G.st->n_labels;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        float v = 0.f;
        if (G.valid[o]) {
            const int L = G.parent[(long long)i * G.W + j];
            double gp = (double)G.z[o];
            if (L >= 1 && L <= nlab && L < G.lab_cap)
                gp -= G.adj[L] * dcircmean(G.csum[2 * cap + L], G.csum[3 * cap + L], pair_val(G.U1[o], G.L1[o]));
            v = (float)gp;
        }
        G.b[o] = v;
        G.U0[o] = 0.f;
        G.L0[o] = 0.f;
    }
}

// re-arms the solver state for the adjoint PCG (one thread per grid)
__global__ void k_adj_rearm(const GridDev* __restrict__ grids, int n) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n || grids[g].H == 0) return;
    InstState* st = grids[g].st;
    // no adjoint when the refinement reverted to a non-finite-free earlier iterate
    st->irls_active = (st->hist_ok && st->n_nonfinite == 0 && !(st->status & 2)) ? 1 : 0;
    st->cg_active = 0;
    st->cg_iter = 0;
}

// gradients into the caller's full grids (the crop region; the host zeroes the rest)
__global__ void k_adj_grad(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const size_t cap = (size_t)G.lab_cap;
    const int nlab = G.st->n_labels;
    const int H = G.H, W = G.W, P = G.P;
    float* __restrict__ gph = G.a_gph;
    float* __restrict__ gw = G.a_gw;
    const long long gpp = G.a_gph_pitch, gwp = G.a_gw_pitch;
    const float* __restrict__ lam = G.D;   // the adjoint PCG's x - x0 with x0 = 0
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * P + j;
        const long long gi = (long long)(G.r0 + i), gj = (long long)(G.c0 + j);
        float dph = 0.f, dw = 0.f;
        if (G.st->irls_active && G.valid[o]) {
            // through the solve: (d u*/d phase)^T G' = A lambda = A A^+ G' = G', because G'
            // sums to zero over every component (the alignment terms of a component sum to
            // its sum of dL/dout), so it lies in the range of A.  Formed here in float64
            // rather than by applying the stencil to the float32 lambda, whose
            // low-frequency part grows like the grid size squared.
            double d = (double)G.z[o];
            const int L = G.parent[(long long)i * W + j];
            if (L >= 1 && L <= nlab && L < G.lab_cap) {
                const double x = pair_val(G.U1[o], G.L1[o]);
                d -= G.adj[L] * dcircmean(G.csum[2 * cap + L], G.csum[3 * cap + L], x);
                d += G.adj[L] * dcircmean(G.csum[L], G.csum[cap + L], adj_ph(G, i, j));
            }
            dph = (float)d;
            if (gw) {
                const float wr = G.weight ? G.weight[(long long)i * G.weight_pitch + j] : 1.f;
                if (G.weight && isfinite(wr) && wr > 0.01f && wr < 1.0f) {
                    double a = 0.0;
                    // edge from pixel (ia, ja) at offset e to its neighbour at e + step, with
                    // its frozen weight wI and edge weight w; residual g - D u* in float64
                    auto edge = [&](size_t e, size_t step, int ia, int ja, int ib, int jb, const float* wI,
                                    const float* we) {
                        if (!G.valid[e] || !G.valid[e + step]) return;
                        const float wv = we[e], wi = wI[e];
                        if (!(wv > 0.f) || !(wi > 1e-6f) || !(wi < 1e6f)) return;
                        const double dl = (double)lam[e + step] - (double)lam[e];
                        const double t = wrap_d(adj_ph(G, ib, jb) - adj_ph(G, ia, ja));
                        const double r =
                            t - (pair_val(G.U1[e + step], G.L1[e + step]) - pair_val(G.U1[e], G.L1[e]));
                        a += 0.5 * dl * r * (double)wi / (double)wv;
                    };
                    if (j < W - 1) edge(o, 1, i, j, i, j + 1, G.wIx, G.wx);
                    if (j > 0) edge(o - 1, 1, i, j - 1, i, j, G.wIx, G.wx);
                    if (i < H - 1) edge(o, (size_t)P, i, j, i + 1, j, G.wIy, G.wy);
                    if (i > 0) edge(o - P, (size_t)P, i - 1, j, i, j, G.wIy, G.wy);
                    dw = (float)a;
                }
            }
        }
        gph[gi * gpp + gj] = dph;
        if (gw) gw[gi * gwp + gj] = dw;
    }
}

cudaError_t unw_launch_adj(int which, int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n, int k) {
    if (nblk <= 0) return cudaSuccess;
    switch (which) {
        case UNW_A_LOAD: k_adj_load<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_LSUM: k_adj_lsum<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_RHS: k_adj_rhs<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_REARM: k_adj_rearm<<<(n + 63) / 64, 64, 0, s>>>(gd, n); break;
        case UNW_A_GRAD: k_adj_grad<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_REFINE:
            if (k) k_adj_refine<1><<<nblk, 256, 0, s>>>(gd, starts, n);
            else k_adj_refine<0><<<nblk, 256, 0, s>>>(gd, starts, n);
            break;
        case UNW_A_ADDD: k_adj_addd<<<nblk, 256, 0, s>>>(gd, starts, n, k); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
