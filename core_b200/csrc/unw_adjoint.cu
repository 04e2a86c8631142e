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
// sums (the same float64 sums the forward alignment uses).
#include "unw_kernels.h"
#include "unw_rowops.cuh"

#define UNW_ROWS_LOOP(G, local, nct)                     \
    for (int i = (local); i < (G).H; i += (nct))         \
        for (int j = threadIdx.x; j < (G).W; j += blockDim.x)

// u (forward output, NaN outside the valid pixels) -> iterate pair (U0, L0 = 0) on the crop, NaN -> 0;
// dL/dout -> z (unused by the solver), 0 at invalid pixels.
__global__ void k_adj_load(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n,
                           const float* __restrict__ u, long long up, const float* __restrict__ gu, long long gp) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const long long gi = (long long)(G.r0 + i), gj = (long long)(G.c0 + j);
        const float uv = u[gi * up + gj];
        const float gv = gu[gi * gp + gj];
        const bool v = G.valid[o] != 0;
        G.U0[o] = (v && isfinite(uv)) ? uv : 0.f;
        G.L0[o] = 0.f;
        G.z[o] = (v && isfinite(gv)) ? gv : 0.f;
    }
}

// per-component sum of dL/dout (parent[] holds the label after the post pipeline's accumulation)
__global__ void k_adj_lsum(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int nlab = G.st->n_labels;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        if (!G.valid[o]) continue;
        const int L = G.parent[(long long)i * G.W + j];
        if (L >= 1 && L <= nlab && L < G.lab_cap) atomicAdd(&G.adj[L], (double)G.z[o]);
    }
}

__device__ __forceinline__ double dcircmean(double s, double c, float x) {
    const double d = s * s + c * c;
    return d > 0.0 ? (c * (double)cosf(x) + s * (double)sinf(x)) / d : 0.0;
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
    const float* __restrict__ us = G.U1;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        float v = 0.f;
        if (G.valid[o]) {
            const int L = G.parent[(long long)i * G.W + j];
            double gp = (double)G.z[o];
            if (L >= 1 && L <= nlab && L < G.lab_cap) gp -= G.adj[L] * dcircmean(G.csum[2 * cap + L], G.csum[3 * cap + L], us[o]);
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
__global__ void k_adj_grad(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n,
                           float* __restrict__ gph, long long gpp, float* __restrict__ gw, long long gwp) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const size_t cap = (size_t)G.lab_cap;
    const int nlab = G.st->n_labels;
    const int H = G.H, W = G.W, P = G.P;
    const float* __restrict__ lam = G.D;   // the adjoint PCG's x - x0 with x0 = 0
    const float* __restrict__ us = G.U1;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * P + j;
        const long long gi = (long long)(G.r0 + i), gj = (long long)(G.c0 + j);
        float dph = 0.f, dw = 0.f;
        if (G.st->irls_active && G.valid[o]) {
            const float ph = G.phase[(long long)i * G.phase_pitch + j];
            double d = (double)lap_at(lam, G.wIx, G.wIy, i, j, H, W, P);
            const int L = G.parent[(long long)i * W + j];
            if (L >= 1 && L <= nlab && L < G.lab_cap) d += G.adj[L] * dcircmean(G.csum[L], G.csum[cap + L], ph);
            dph = (float)d;
            if (gw) {
                const float wr = G.weight ? G.weight[(long long)i * G.weight_pitch + j] : 1.f;
                if (G.weight && isfinite(wr) && wr > 0.01f && wr < 1.0f) {
                    double a = 0.0;
                    // edge (o, o + step) with its frozen weight wI, edge weight w and target gradient t
                    auto edge = [&](size_t e, size_t step, const float* wI, const float* we, const float* t) {
                        if (!G.valid[e] || !G.valid[e + step]) return;
                        const float wv = we[e], wi = wI[e];
                        if (!(wv > 0.f) || !(wi > 1e-6f) || !(wi < 1e6f)) return;
                        const double dl = (double)lam[e + step] - (double)lam[e];
                        const double r = (double)t[e] - ((double)us[e + step] - (double)us[e]);
                        a += 0.5 * dl * r * (double)wi / (double)wv;
                    };
                    if (j < W - 1) edge(o, 1, G.wIx, G.wx, G.gx);
                    if (j > 0) edge(o - 1, 1, G.wIx, G.wx, G.gx);
                    if (i < H - 1) edge(o, (size_t)P, G.wIy, G.wy, G.gy);
                    if (i > 0) edge(o - P, (size_t)P, G.wIy, G.wy, G.gy);
                    dw = (float)a;
                }
            }
        }
        gph[gi * gpp + gj] = dph;
        if (gw) gw[gi * gwp + gj] = dw;
    }
}

cudaError_t unw_launch_adj(int which, int nblk, cudaStream_t s, const GridDev* gd, const int* starts, int n,
                           const float* a, long long ap, const float* b, long long bp, float* c, long long cp,
                           float* d, long long dp) {
    if (nblk <= 0) return cudaSuccess;
    switch (which) {
        case UNW_A_LOAD: k_adj_load<<<nblk, 256, 0, s>>>(gd, starts, n, a, ap, b, bp); break;
        case UNW_A_LSUM: k_adj_lsum<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_RHS: k_adj_rhs<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_A_REARM: k_adj_rearm<<<(n + 63) / 64, 64, 0, s>>>(gd, n); break;
        case UNW_A_GRAD: k_adj_grad<<<nblk, 256, 0, s>>>(gd, starts, n, c, cp, d, dp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
