// Solver kernels of the B200 DCT+IRLS unwrapper (sm_100a).
//
// One IRLS iteration (utils_unwrap2d.py:1533-1626) is the launch sequence
//   mean -> head -> copy_best -> row_fwd(R0) -> col -> row_inv(Z0)
//   -> cg_max_iter x [matvec -> row_fwd(UPD) -> col -> row_inv(Z)] -> rel
// Every kernel covers all grids of a batch and returns at once for grids whose
// IRLS or PCG has stopped; the stop decisions (the reference's Python `break`
// tests) are taken on the device by the last CTA of the reducing kernel, so
// no host synchronisation is needed inside an IRLS iteration.
//
// The DCT preconditioner (utils_unwrap2d.py:1390-1403) is three passes:
//   row_fwd: row DCT-II of a pair of rows through one complex FFT,
//   col:     column DCT-II -> scale by -1/lambda -> column DCT-III (fused),
//   row_inv: row DCT-III of a pair of rows through one complex FFT,
// each pass fused with the elementwise PCG work that reads or writes the
// same rows.  Float32 elementwise arithmetic follows the reference's
// operation order (one rounding per torch op); all inner products and norms
// accumulate in float64.
#include <climits>
#include "unw_fft.cuh"
#include "unw_rowops.cuh"
#include "unw_kernels.h"

// ============================================================ tables
// Twiddles, DCT weights and Bluestein chirps in float64, rounded once.
__global__ void k_tables(FftPlanDev f, DctPlanDev d, float* sv, int Ncos) {
    float2* tw = const_cast<float2*>(f.tw);
    float2* dw = const_cast<float2*>(d.dctw);
    float2* ch = const_cast<float2*>(d.chirp);
    const int n = f.n, N = d.N;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)m / (double)n, &s, &c);
        tw[m] = make_float2((float)c, (float)s);
    }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(-(double)k / (2.0 * (double)N), &s, &c);
        dw[k] = make_float2((float)c, (float)s);
        if (d.blue) {
            long long m2 = ((long long)k * (long long)k) % (2LL * N);
            sincospi((double)m2 / (double)N, &s, &c);
            ch[k] = make_float2((float)c, (float)s);
        }
    }
    // 4 sin^2(pi k / 2N) = 2 - 2 cos(pi k / N), eigenvalue part along this axis
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < Ncos; k += gridDim.x * blockDim.x) {
        const double sn = sinpi((double)k / (2.0 * (double)Ncos));
        sv[k] = (float)(4.0 * sn * sn);
    }
}

// Bluestein filter spectrum hspec = FFT_M(h) / M, h_j = chirp_|j| for |j| < N.
template <int T, int EMAX>
__global__ void __launch_bounds__(T) k_hspec(DctPlanDev d) {
    extern __shared__ float2 sm[];
    const int M = d.fft.n, N = d.N;
    for (int m = threadIdx.x; m < M; m += T) {
        float2 v = make_float2(0.f, 0.f);
        if (m < N) v = d.chirp[m];
        else if (M - m < N) v = d.chirp[M - m];
        sm[m] = v;
    }
    __syncthreads();
    fft_smem<T, EMAX>(sm, 1, M, d.fft);
    float2* hs = const_cast<float2*>(d.hspec);
    const float inv = 1.0f / (float)M;
    for (int m = threadIdx.x; m < M; m += T) hs[m] = make_float2(sm[m].x * inv, sm[m].y * inv);
}

// ============================================================ state / setup
__global__ void k_state_init(const GridDev* __restrict__ grids, int n, UnwScalars sc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    InstState* s = grids[g].st;
    s->rz = 0; s->pAp = 0; s->rnorm = 0; s->alpha = 0.f; s->beta = 0.f;
    s->cg_active = 0; s->cg_iter = 0;
    s->irls_active = sc.max_iter > 0; s->irls_iter = 0; s->max_iter = sc.max_iter;
    s->best_update = 0; s->revert = 0; s->u_index = 0; s->status = 0;
    s->vcount = 0; s->mean = 0; s->residual = 0; s->best_residual = INFINITY; s->rel_change = 0; s->resid_rel = 0;
    s->tol = sc.tol; s->cg_tol = sc.cg_tol; s->eps2 = sc.eps2; s->cg_max_iter = sc.cg_max_iter;
    s->cg_rel = sc.cg_rel;
    s->refine_scale = 1.0;
    s->cg_total = 0;
    for (int i = 0; i < UNW_MAX_LOG; i++) s->cg_log[i] = 0;
    s->n_nonfinite = 0; s->n_kneg = 0; s->n_kpos = 0; s->kmin = INT_MAX; s->kmax = INT_MIN; s->hist_ok = 1; s->kmed = 0.f; s->shift = 0.f;
    s->n_labels = 0;
    if (grids[g].H == 0) { s->irls_active = 0; s->hist_ok = 0; }
    *grids[g].counter = 0u;
}

// NaN fill, weight clipping, wrapped gradients and edge weights
// (utils_unwrap2d.py:1228-1241, :1254-1262, :1267-1275).  KS_ELEM shape.
__device__ __forceinline__ float wrap_f(float d) { return atan2f(sinf(d), cosf(d)); }

__device__ __forceinline__ void px_in(const GridDev& G, int i, int j, float& ph, float& w, bool& v) {
    const float p = G.phase[(long long)i * G.phase_pitch + j];
    v = !isnan(p);
    ph = v ? p : 0.f;
    if (G.weight) {
        float x = G.weight[(long long)i * G.weight_pitch + j];
        if (isnan(x) || !v) x = 0.f;
        w = fminf(fmaxf(x, 0.01f), 1.0f);
    } else {
        w = v ? 1.f : 0.f;
    }
}

__global__ void k_setup(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ double red[32 * 1];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const long long npx = (long long)H * W;
    double acc[1] = {0.0};
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        float ph, w, phr, wr, phd, wd;
        bool v, vr, vd;
        px_in(G, i, j, ph, w, v);
        float gxv = 0.f, wxv = 0.f, gyv = 0.f, wyv = 0.f;
        if (j < W - 1) {
            px_in(G, i, j + 1, phr, wr, vr);
            gxv = wrap_f(fsub(phr, ph));
            wxv = fmul(fdiv(fadd(w, wr), 2.0f), (v && vr) ? 1.f : 0.f);
        }
        if (i < H - 1) {
            px_in(G, i + 1, j, phd, wd, vd);
            gyv = wrap_f(fsub(phd, ph));
            wyv = fmul(fdiv(fadd(w, wd), 2.0f), (v && vd) ? 1.f : 0.f);
        }
        const size_t o = (size_t)i * P + j;
        G.gx[o] = gxv; G.gy[o] = gyv; G.wx[o] = wxv; G.wy[o] = wyv;
        G.valid[o] = v ? 1 : 0;
        acc[0] += v ? 1.0 : 0.0;
    }
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) G.st->vcount = acc[0];
    }
}

// ============================================================ row forward pass
// Generic lengths: row DCT-II of rows (i0, i0+1) of a source computed on the
// fly (modes in unw_rowops.cuh).  Output T[i][k] = DCT-II(row i)[k] (no 1/2).
template <int T, int EMAX, int MODE>
__global__ void __launch_bounds__(T) k_row_fwd(const GridDev* __restrict__ grids,
                                               const int* __restrict__ starts, int n, int it,
                                               int cgk) {
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowfwd_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    double acc[2] = {0.0, 0.0};
    float* U = rowfwd_x<MODE>(G, it);  // x0 of this IRLS iteration (U_nxt), or D in mode 2
    const float* Lo = rowfwd_lo(G, it);
    const float* pk = (MODE == 2) ? G.p0 : nullptr;
    const float alpha = (MODE == 2) ? st->alpha : 0.f;
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
    const int i0 = 2 * pair, i1 = i0 + 1;
    const bool has1 = i1 < H;
    __syncthreads();  // previous row pair's reads of sm are done
    for (int j = threadIdx.x; j < W; j += T) {
        const float a = rowfwd_value<MODE>(G, U, Lo, pk, alpha, i0, j, acc);
        const float b = has1 ? rowfwd_value<MODE>(G, U, Lo, pk, alpha, i1, j, acc) : 0.f;
        sm[mk_perm(j, W)] = make_float2(a, b);
    }
    __syncthreads();
    dft_n<T, EMAX>(sm, 1, G.prow);
    // Two real rows from one complex DFT, then X_k = Re(exp(-i pi k/2W) V_k).
    const float2* __restrict__ dw = G.prow.dctw;
    for (int k = threadIdx.x; k < W; k += T) {
        const float2 C = sm[k];
        const float2 Cm = sm[k == 0 ? 0 : W - k];
        const float2 Va = make_float2(C.x + Cm.x, C.y - Cm.y);
        const float2 Vb = make_float2(C.y + Cm.y, Cm.x - C.x);
        const float2 w = __ldg(&dw[k]);
        G.T[(size_t)i0 * P + k] = w.x * Va.x - w.y * Va.y;
        if (has1) G.T[(size_t)i1 * P + k] = w.x * Vb.x - w.y * Vb.y;
    }
    }
    if (MODE == 0 || MODE == 3) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowfwd_finalize<MODE>(st, acc);
    }
}

// ============================================================ column pass
// Column DCT-II -> scale by -1/(4 H W lambda) -> column DCT-III, in place on T.
// MODE 0: DCT initial solve (always runs); MODE 1 / 2: PCG (gated), also
// r.z by Parseval and its scalar step (col_finalize).
template <int T, int EMAX, int MODE>
__global__ void __launch_bounds__(T) k_col(const GridDev* __restrict__ grids,
                                           const int* __restrict__ starts, int n) {
    extern __shared__ float2 sm[];
    __shared__ double red[32];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (MODE >= 1 && !(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int nslab = (W + 2 * G.col_nseq - 1) / (2 * G.col_nseq);
    double acc[1] = {0.0};
    for (int slab = local; slab < nslab; slab += nct) {
    const int c0 = 2 * G.col_nseq * slab;
    const int nseq = min(G.col_nseq, (W - c0 + 1) >> 1);
    __syncthreads();  // previous slab's reads of sm are done
    const DctPlanDev& PC = G.pcol;
    const int sd = PC.stride;
    float* __restrict__ Tm = G.T;
    for (int q = threadIdx.x; q < nseq * H; q += T) {
        const int i = q / nseq, s = q - i * nseq;
        const int c = c0 + 2 * s;
        const float a = Tm[(size_t)i * P + c];
        const float b = (c + 1 < W) ? Tm[(size_t)i * P + c + 1] : 0.f;
        sm[s * sd + mk_perm(i, H)] = make_float2(a, b);
    }
    __syncthreads();
    dft_n<T, EMAX>(sm, nseq, PC);
    const float2* __restrict__ dw = PC.dctw;
    const float* __restrict__ sH = G.sH;
    const float* __restrict__ sW = G.sW;
    const float negs = -1.0f / (4.0f * (float)H * (float)W);
    const int nh = H / 2 + 1;
    for (int q = threadIdx.x; q < nseq * nh; q += T) {
        const int k = q / nseq, s = q - k * nseq;
        const int km = k == 0 ? 0 : H - k;
        if (k > km) continue;
        float2* base = sm + s * sd;
        const float2 C = base[k], Cm = base[km];
        const int ja = c0 + 2 * s;
        const bool hasb = ja + 1 < W;
        const float ca = sW[ja], cb = hasb ? sW[ja + 1] : 1.0f;
        const float2 wk = __ldg(&dw[k]), wm = __ldg(&dw[km]);
        float2 ok, om;
        col_spectral_pair<(MODE >= 1)>(C, Cm, k, km, wk, wm, sH[k], sH[km], ca, cb, ja == 0, hasb, negs, ok, om,
                                     acc[0]);
        if (km != k) base[km] = om;
        base[k] = ok;
    }
    __syncthreads();
    dft_n<T, EMAX>(sm, nseq, PC);
    for (int q = threadIdx.x; q < nseq * H; q += T) {
        const int i = q / nseq, s = q - i * nseq;
        const int c = c0 + 2 * s;
        const float2 v = sm[s * sd + mk_perm(i, H)];
        Tm[(size_t)i * P + c] = v.x;
        if (c + 1 < W) Tm[(size_t)i * P + c + 1] = -v.y;
    }
    }
    if (MODE == 0) return;
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) col_finalize<MODE>(st, acc[0]);
    }
}

// ============================================================ row inverse pass
// Generic lengths: row DCT-III of rows (i0, i0+1) of T with the epilogue of
// MODE (unw_rowops.cuh).
template <int T, int EMAX, int MODE>
__global__ void __launch_bounds__(T) k_row_inv(const GridDev* __restrict__ grids,
                                               const int* __restrict__ starts, int n) {
    extern __shared__ float2 sm[];
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!rowinv_gate<MODE>(st)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const float beta = MODE == 2 ? st->beta : 0.f;
    double acc[2] = {0.0, 0.0};
    for (int pair = local; pair < (H + 1) / 2; pair += nct) {
    const int i0 = 2 * pair, i1 = i0 + 1;
    const bool has1 = i1 < H;
    __syncthreads();  // previous row pair's reads of sm are done
    for (int k = threadIdx.x; k < W; k += T) {
        const float a = G.T[(size_t)i0 * P + k];
        const float b = has1 ? G.T[(size_t)i1 * P + k] : 0.f;
        sm[k] = make_float2(a, b);
    }
    __syncthreads();
    const float2* __restrict__ dw = G.prow.dctw;
    for (int k = threadIdx.x; k <= W / 2; k += T) {
        const int km = k == 0 ? 0 : W - k;
        if (k > km) continue;
        const float2 Yk = sm[k], Ym = sm[km];
        const float2 wk = __ldg(&dw[k]);
        const float mak = k == 0 ? 0.f : Ym.x, mbk = k == 0 ? 0.f : Ym.y;
        const float2 Pak = cmul(cconj(wk), make_float2(Yk.x, -mak));
        const float2 Pbk = cmul(cconj(wk), make_float2(Yk.y, -mbk));
        const float2 Ck = cconj(make_float2(Pak.x - Pbk.y, Pak.y + Pbk.x));
        if (km != k) {
            const float2 wm = __ldg(&dw[km]);
            const float2 Pam = cmul(cconj(wm), make_float2(Ym.x, -Yk.x));
            const float2 Pbm = cmul(cconj(wm), make_float2(Ym.y, -Yk.y));
            sm[km] = cconj(make_float2(Pam.x - Pbm.y, Pam.y + Pbm.x));
        }
        sm[k] = Ck;
    }
    __syncthreads();
    dft_n<T, EMAX>(sm, 1, G.prow);
    for (int j = threadIdx.x; j < W; j += T) {
        const float2 v = sm[mk_perm(j, W)];
        rowinv_store<MODE>(G, i0, j, v.x, beta, acc);
        if (has1) rowinv_store<MODE>(G, i1, j, -v.y, beta, acc);
    }
    }
    if (MODE != 0) return;
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) rowinv_finalize_initu(st, acc);
    }
}

// ============================================================ stencil kernels
// KS_STEN shape: a CTA is 8 warps; warp w of tile (tx, ty) covers columns
// [128 tx, 128 tx + 128) (4 per lane) and rows [(8 ty + w) R, (8 ty + w + 1) R),
// R = sten_rows, marching down the rows with the row above and below in registers.
struct F4 {
    float v[4];
};
__device__ __forceinline__ F4 ld4(const float* __restrict__ a, size_t o) {
    const float4 x = *reinterpret_cast<const float4*>(a + o);
    return F4{{x.x, x.y, x.z, x.w}};
}
__device__ __forceinline__ void st4(float* __restrict__ a, size_t o, const F4& x) {
    *reinterpret_cast<float4*>(a + o) = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
}

// p = z + beta p_old (reference: p.mul_(beta).add_(z)), p = z on the first PCG step
__device__ __forceinline__ F4 pnew4(const float* __restrict__ z, const float* __restrict__ po, size_t o,
                                    bool first, float beta) {
    F4 r = ld4(z, o);
    if (!first) {
        const F4 q = ld4(po, o);
#pragma unroll
        for (int c = 0; c < 4; c++) r.v[c] = fadd(fmul(q.v[c], beta), r.v[c]);
    }
    return r;
}
__device__ __forceinline__ float pnew1(const float* __restrict__ z, const float* __restrict__ po, size_t o,
                                       bool first, float beta) {
    return first ? z[o] : fadd(fmul(po[o], beta), z[o]);
}

// matvec: Ap = A p, pAp = p.Ap (utils_unwrap2d.py:1430-1436).  p is formed in
// place by the row-inverse pass, so this kernel only reads it.
// A CTA is 16 warps over a 128-column x 16-row tile; each warp computes one row
// (4 columns per lane) and issues all its loads (rows i-1, i, i+1 of p, the
// weights, the tile-edge scalars) before using any of them.  The neighbouring
// rows come back from L1/L2: DRAM traffic stays one pass per array.
__global__ void __launch_bounds__(512, 2) k_matvec(const GridDev* __restrict__ grids,
                                                   const int* __restrict__ starts, int n, int k) {
    __shared__ double red[32 * 1];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!(st->irls_active && st->cg_active)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const float* __restrict__ p = G.p0;
    double acc[1] = {0.0};
    const int ntiles = G.sten_tiles_x * ((H + 15) / 16);
    for (int tile = local; tile < ntiles; tile += nct) {
    // bottom rows first: the row-inverse pass that formed p ends at the bottom, so
    // its last rows are still in L2, and the row-forward pass that reads Ap next
    // starts at the top, where this pass ends
    const int tr = ntiles - 1 - tile;
    const int tx = tr % G.sten_tiles_x, ty = tr / G.sten_tiles_x;
    const int j0 = tx * 128 + lane * 4;
    const int i = ty * 16 + warp;
    // lanes past the last column load nothing (j0 < W implies j0 + 3 < P)
    const bool on = i < H && j0 < W;
    const bool hu = i > 0, hd = i < H - 1;
    const size_t o = (size_t)i * P + j0;
    F4 cur{}, up{}, dn{}, wx{}, wy{}, wyu{};
    float zl = 0.f, wl = 0.f, zr = 0.f;
    if (on) {
        cur = ld4(p, o);
        if (hu) up = ld4(p, o - P);
        if (hd) dn = ld4(p, o + P);
        wx = ld4(G.wIx, o);
        wy = ld4(G.wIy, o);
        if (hu) wyu = ld4(G.wIy, o - P);
        if (lane == 0 && j0 > 0) {
            zl = p[o - 1];
            wl = G.wIx[o - 1];
        }
        if (lane == 31 && j0 + 4 < W) zr = p[o + 4];
    }
    float pl = __shfl_up_sync(0xffffffffu, cur.v[3], 1);
    float wll = __shfl_up_sync(0xffffffffu, wx.v[3], 1);
    float pr = __shfl_down_sync(0xffffffffu, cur.v[0], 1);
    if (lane == 0) { pl = zl; wll = wl; }
    if (lane == 31) pr = zr;
    if (on) {
        F4 ap;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int j = j0 + c;
            const float pc = cur.v[c];
            const float pleft = c == 0 ? pl : cur.v[c - 1];
            const float pright = c == 3 ? pr : cur.v[c + 1];
            const float wleft = c == 0 ? wll : wx.v[c - 1];
            float res = 0.f;
            if (j > 0) res = fsub(res, fmul(fsub(pc, pleft), wleft));
            if (j < W - 1) res = fadd(res, fmul(fsub(pright, pc), wx.v[c]));
            if (hu) res = fsub(res, fmul(fsub(pc, up.v[c]), wyu.v[c]));
            if (hd) res = fadd(res, fmul(fsub(dn.v[c], pc), wy.v[c]));
            ap.v[c] = -res;
            if (j < W) acc[0] += (double)pc * (double)ap.v[c];
        }
        st4(G.Ap, o, ap);
    }
    }
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) matvec_finalize(st, acc[0]);
    }
}

// IRLS head (utils_unwrap2d.py:1536-1581): recentre, residual gradients,
// best-iterate test, IRLS weights and right-hand side.  Reads the iterate pair
// (U_cur, L_cur), writes the recentred pair to (U_nxt, L_nxt) (the current pair
// keeps u_prev for the convergence test).  The residual gradients take the
// neighbour differences of the pair (pair_diff; the mean cancels in them), the
// recentred pair is formed in float64, the weights and b are float32 in the
// reference's op order.
// One warp per row, 4 columns per lane; the weight of the left edge comes from
// the neighbouring lane, the weight of the upper edge is recomputed from the
// row above (the same operations, so it equals that row's own value).
__device__ __forceinline__ float irls_w(float w, float r, float eps2) {
    return clampf_nan(fdiv(w, __fsqrt_rn(fadd(fmul(r, r), eps2))), 1e-6f, 1e6f);
}

// Persistent: a CTA loops over 128 x 8 tiles and arrives once with its partial
// sums (one block reduction and one atomic per CTA, not per tile).  (Three resident
// CTAs per SM remove its few spilled registers but took 269 us instead of 214 us per
// launch at 4096^2.)
__global__ void __launch_bounds__(256, 4) k_head(const GridDev* __restrict__ grids,
                                                 const int* __restrict__ starts, int n, int it) {
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!st->irls_active) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double m = st->vcount > 0 ? st->mean : 0.0;
    const float eps2 = st->eps2;
    const float* __restrict__ uc = (it & 1) ? G.U1 : G.U0;
    const float* __restrict__ lc = (it & 1) ? G.L1 : G.L0;
    float* __restrict__ un = (it & 1) ? G.U0 : G.U1;
    float* __restrict__ ln = (it & 1) ? G.L0 : G.L1;
    double acc[2] = {0.0, 0.0};
    const int ntiles = G.sten_tiles_x * ((H + 8 * G.sten_rows - 1) / (8 * G.sten_rows));
    for (int tile = local; tile < ntiles; tile += nct) {
    const int tx = tile % G.sten_tiles_x, ty = tile / G.sten_tiles_x;
    const int j0 = tx * 128 + lane * 4;
    const int i = ty * 8 + warp;
    const bool on = i < H && j0 < W;
    const bool hu = i > 0, hd = i < H - 1;
    const size_t o = (size_t)i * P + j0;
    F4 u{}, l{}, ud{}, ld{}, uu{}, lu{}, gx{}, gy{}, gyu{}, wx{}, wy{}, wyu{};
    float ul = 0.f, ll = 0.f, ur = 0.f, lr = 0.f, gxl = 0.f, wxl = 0.f;
    if (on) {
        u = ld4(uc, o);
        l = ld4(lc, o);
        if (hd) { ud = ld4(uc, o + P); ld = ld4(lc, o + P); }
        if (hu) { uu = ld4(uc, o - P); lu = ld4(lc, o - P); gyu = ld4(G.gy, o - P); wyu = ld4(G.wy, o - P); }
        gx = ld4(G.gx, o);
        gy = ld4(G.gy, o);
        wx = ld4(G.wx, o);
        wy = ld4(G.wy, o);
        if (lane == 0 && j0 > 0) { ul = uc[o - 1]; ll = lc[o - 1]; gxl = G.gx[o - 1]; wxl = G.wx[o - 1]; }
        if (lane == 31 && j0 + 4 < W) { ur = uc[o + 4]; lr = lc[o + 4]; }
    }
    float rx[4], ry[4];
    F4 wix, wiy, bv;
    // the centre row's pairs as float64 values, converted once and shared (dpair_diff)
    double xv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) xv[q] = pair_val(u.v[q], l.v[q]);
    // right neighbour of column j0+3
    double xr = __shfl_down_sync(0xffffffffu, xv[0], 1);
    if (lane == 31) xr = pair_val(ur, lr);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = j0 + q;
        const double right = q == 3 ? xr : xv[q + 1];
        // r = grad(u) - g, last column / row: 0 - g
        rx[q] = (j < W - 1) ? fsub(dpair_diff(right, xv[q]), gx.v[q]) : fsub(0.f, gx.v[q]);
        ry[q] = hd ? fsub(dpair_diff(pair_val(ud.v[q], ld.v[q]), xv[q]), gy.v[q]) : fsub(0.f, gy.v[q]);
        wix.v[q] = irls_w(wx.v[q], rx[q], eps2);
        wiy.v[q] = irls_w(wy.v[q], ry[q], eps2);
    }
    float wl = __shfl_up_sync(0xffffffffu, wix.v[3], 1);
    float gl = __shfl_up_sync(0xffffffffu, gx.v[3], 1);
    if (lane == 0 && j0 > 0) {
        const float rxl = fsub(dpair_diff(xv[0], pair_val(ul, ll)), gxl);
        wl = irls_w(wxl, rxl, eps2);
        gl = gxl;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int j = j0 + q;
        float b = 0.f;
        if (j > 0) {
            const float wleft = q == 0 ? wl : wix.v[q - 1];
            const float gleft = q == 0 ? gl : gx.v[q - 1];
            b = fadd(b, fmul(wleft, gleft));
        }
        if (j < W - 1) b = fsub(b, fmul(wix.v[q], gx.v[q]));
        if (hu) {
            const float ryu = fsub(dpair_diff(xv[q], pair_val(uu.v[q], lu.v[q])), gyu.v[q]);
            b = fadd(b, fmul(irls_w(wyu.v[q], ryu, eps2), gyu.v[q]));
        }
        if (hd) b = fsub(b, fmul(wiy.v[q], gy.v[q]));
        bv.v[q] = b;
    }
    if (on) {
        F4 ch, cl4;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const double c = xv[q] - m;
            split_pair(c, ch.v[q], cl4.v[q]);
            if (j0 + q < W) {
                acc[0] += (double)fmul(rx[q], rx[q]) + (double)fmul(ry[q], ry[q]);
                acc[1] += isfinite(c) ? 0.0 : 1.0;
            }
        }
        st4(un, o, ch);
        st4(ln, o, cl4);
        st4(G.wIx, o, wix);
        st4(G.wIy, o, wiy);
        st4(G.b, o, bv);
    }
    }
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) {
            const double res = acc[0];
            st->residual = res;
            st->best_update = 0;
            if (res < st->best_residual && acc[1] == 0.0) {
                st->best_residual = res;
                st->best_update = 1;
            }
            st->cg_active = 1;
            st->cg_iter = 0;
        }
    }
}

// ============================================================ elementwise kernels (KS_ELEM)
// A CTA takes whole rows (grid-stride over rows), threads take float4 column
// groups; P is a multiple of 4, so a group starting below W stays in the row.
#define UNW_ROWS_LOOP(G, local, nct)                          \
    for (int i = (local); i < (G).H; i += (nct))              \
        for (int j = 4 * threadIdx.x; j < (G).W; j += 4 * blockDim.x)

// sum over all pixels of u * valid (utils_unwrap2d.py:1539-1541), u = U + L in float64
__global__ void k_mean(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n, int it) {
    __shared__ double red[32 * 1];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!st->irls_active) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const float* __restrict__ uc = (it & 1) ? G.U1 : G.U0;
    const float* __restrict__ lc = (it & 1) ? G.L1 : G.L0;
    double acc[1] = {0.0};
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const F4 u = ld4(uc, o), l = ld4(lc, o);
        const uchar4 v = *reinterpret_cast<const uchar4*>(G.valid + o);
        const unsigned char vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (j + q < G.W) acc[0] += pair_val(u.v[q], l.v[q]) * (vv[q] ? 1.0 : 0.0);
    }
    if (arrive<1>(G, local, nct, acc, red)) {
        finish_sum<1>(G, nct, acc, red);
        if (threadIdx.x == 0) st->mean = st->vcount > 0 ? acc[0] / st->vcount : 0.0;
    }
}

// After the DCT initial solve: u -= mean_valid(u); u_best = u (utils_unwrap2d.py:1509-1531),
// in float64 into the iterate pair (U0, L0) and the best pair (Ub, Lb).
__global__ void k_init_recentre(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const double m = st->vcount > 0 ? st->mean : 0.0;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const F4 u = ld4(G.U0, o);
        F4 hi, lo;
#pragma unroll
        for (int q = 0; q < 4; q++) split_pair((double)u.v[q] - m, hi.v[q], lo.v[q]);
        st4(G.U0, o, hi);
        st4(G.L0, o, lo);
        st4(G.Ub, o, hi);
        st4(G.Lb, o, lo);
    }
}

// u_best = u_rc when the head found a smaller residual (utils_unwrap2d.py:1555-1558)
__global__ void k_copy_best(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n, int it) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const InstState* st = G.st;
    if (!(st->irls_active && st->best_update)) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const float* __restrict__ un = (it & 1) ? G.U0 : G.U1;
    const float* __restrict__ ln = (it & 1) ? G.L0 : G.L1;
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        st4(G.Ub, o, ld4(un, o));
        st4(G.Lb, o, ld4(ln, o));
    }
}

// IRLS tail (utils_unwrap2d.py:1599-1626): u = x0 + D (the PCG result, formed in
// float64 into the iterate pair); non-finite -> revert to u_best and stop;
// rel_change = |u_prev - u| / (|u| + 1e-10) over the full grid.
__global__ void k_rel(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n, int it) {
    __shared__ double red[32 * 3];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (!st->irls_active) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const float* __restrict__ up = (it & 1) ? G.U1 : G.U0;
    const float* __restrict__ lp = (it & 1) ? G.L1 : G.L0;
    float* __restrict__ un = (it & 1) ? G.U0 : G.U1;
    float* __restrict__ ln = (it & 1) ? G.L0 : G.L1;
    double acc[3] = {0.0, 0.0, 0.0};
    UNW_ROWS_LOOP(G, local, nct) {
        const size_t o = (size_t)i * G.P + j;
        const F4 uh = ld4(un, o), ul = ld4(ln, o), dd = ld4(G.D, o), vh = ld4(up, o), vl = ld4(lp, o);
        F4 nh, nl;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const double u = pair_val(uh.v[q], ul.v[q]) + (double)dd.v[q];
            split_pair(u, nh.v[q], nl.v[q]);
            if (j + q >= G.W) continue;
            const double d = pair_val(vh.v[q], vl.v[q]) - u;
            acc[0] += d * d;
            acc[1] += u * u;
            acc[2] += isfinite(u) ? 0.0 : 1.0;
        }
        st4(un, o, nh);
        st4(ln, o, nl);
    }
    if (arrive<3>(G, local, nct, acc, red)) {
        finish_sum<3>(G, nct, acc, red);
        if (threadIdx.x == 0) {
            const int t = st->irls_iter;
            if (t < UNW_MAX_LOG) st->cg_log[t] = st->cg_iter;
            st->cg_total += st->cg_iter;
            st->irls_iter = t + 1;
            if (acc[2] != 0.0) {
                st->u_index = 2;             // u_best holds the result
                st->status |= 2;             // UNW_S_REVERTED
                st->irls_active = 0;
            } else {
                st->u_index = (it & 1) ? 0 : 1;
                const double rel = sqrt(acc[0]) / (sqrt(acc[1]) + 1e-10);
                st->rel_change = rel;
                if (rel < (double)st->tol || st->irls_iter >= st->max_iter) st->irls_active = 0;
            }
        }
    }
}

// ||b - A u|| / ||b|| in float64 for the final iterate pair (u_index) and the weights
// and right-hand side of the last IRLS head: how far the result is from an exact
// solve of the last weighted Poisson system (utils_unwrap2d.py:1576-1593).
__global__ void k_resid(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    __shared__ double red[32 * 2];
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    InstState* st = G.st;
    if (st->irls_iter == 0) return;
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const float* U = st->u_index == 2 ? G.Ub : (st->u_index == 1 ? G.U1 : G.U0);
    const float* L = st->u_index == 2 ? G.Lb : (st->u_index == 1 ? G.L1 : G.L0);
    const long long npx = (long long)H * W;
    double acc[2] = {0.0, 0.0};
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        const double b = (double)G.b[(size_t)i * P + j];
        const double r = b - lap_at_pair(U, L, G.wIx, G.wIy, i, j, H, W, P);
        acc[0] += r * r;
        acc[1] += b * b;
    }
    if (arrive<2>(G, local, nct, acc, red)) {
        finish_sum<2>(G, nct, acc, red);
        if (threadIdx.x == 0) st->resid_rel = acc[1] > 0.0 ? sqrt(acc[0] / acc[1]) : sqrt(acc[0]);
    }
}

// Ax for a whole grid (operator entry point unw_apply_laplacian), x = G.r, Ax -> G.Ap.
__global__ void k_lap_apply(const GridDev* __restrict__ grids, const int* __restrict__ starts, int n) {
    const int g = find_grid(starts, n, blockIdx.x);
    const GridDev& G = grids[g];
    const int local = blockIdx.x - starts[g];
    const int nct = starts[g + 1] - starts[g];
    const int H = G.H, W = G.W, P = G.P;
    const long long npx = (long long)H * W;
    for (long long q = (long long)local * blockDim.x + threadIdx.x; q < npx; q += (long long)nct * blockDim.x) {
        const int i = (int)(q / W), j = (int)(q - (long long)i * W);
        G.Ap[(size_t)i * P + j] = lap_at(G.r, G.wIx, G.wIy, i, j, H, W, P);
    }
}

// ============================================================ launchers
template <int MODE>
static cudaError_t launch_row_fwd_t(int T, int emax, dim3 grid, size_t smem, cudaStream_t s,
                                    const GridDev* gd, const int* st, int n, int it, int cgk) {
#define UNW_RF(TT, EE)                                                                      \
    if (T == TT && emax == EE) {                                                            \
        auto kfn = k_row_fwd<TT, EE, MODE>;                                                 \
        unw_smem_limit((const void*)kfn);                                                   \
        kfn<<<grid, TT, smem, s>>>(gd, st, n, it, cgk);                                     \
        return cudaGetLastError();                                                          \
    }
    UNW_RF(128, 16) UNW_RF(256, 16) UNW_RF(512, 16) UNW_RF(1024, 16) UNW_RF(1024, 32)
#undef UNW_RF
    return cudaErrorInvalidConfiguration;
}

cudaError_t unw_launch_row_fwd(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                               const GridDev* gd, const int* starts, int n, int it, int cgk) {
    if (nblk <= 0) return cudaSuccess;
    dim3 grid(nblk);
    switch (mode) {
        case 0: return launch_row_fwd_t<0>(T, emax, grid, smem, s, gd, starts, n, it, cgk);
        case 1: return launch_row_fwd_t<1>(T, emax, grid, smem, s, gd, starts, n, it, cgk);
        case 2: return launch_row_fwd_t<2>(T, emax, grid, smem, s, gd, starts, n, it, cgk);
        default: return launch_row_fwd_t<3>(T, emax, grid, smem, s, gd, starts, n, it, cgk);
    }
}

template <int MODE>
static cudaError_t launch_row_inv_t(int T, int emax, dim3 grid, size_t smem, cudaStream_t s,
                                    const GridDev* gd, const int* st, int n) {
#define UNW_RI(TT, EE)                                                                      \
    if (T == TT && emax == EE) {                                                            \
        auto kfn = k_row_inv<TT, EE, MODE>;                                                 \
        unw_smem_limit((const void*)kfn);                                                   \
        kfn<<<grid, TT, smem, s>>>(gd, st, n);                                              \
        return cudaGetLastError();                                                          \
    }
    UNW_RI(128, 16) UNW_RI(256, 16) UNW_RI(512, 16) UNW_RI(1024, 16) UNW_RI(1024, 32)
#undef UNW_RI
    return cudaErrorInvalidConfiguration;
}

cudaError_t unw_launch_row_inv(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                               const GridDev* gd, const int* starts, int n) {
    if (nblk <= 0) return cudaSuccess;
    dim3 grid(nblk);
    switch (mode) {
        case 0: return launch_row_inv_t<0>(T, emax, grid, smem, s, gd, starts, n);
        case 1: return launch_row_inv_t<1>(T, emax, grid, smem, s, gd, starts, n);
        case 2: return launch_row_inv_t<2>(T, emax, grid, smem, s, gd, starts, n);
        default: return launch_row_inv_t<3>(T, emax, grid, smem, s, gd, starts, n);
    }
}

template <int MODE>
static cudaError_t launch_col_t(int T, int emax, dim3 grid, size_t smem, cudaStream_t s,
                                const GridDev* gd, const int* st, int n) {
#define UNW_CL(TT, EE)                                                                      \
    if (T == TT && emax == EE) {                                                            \
        auto kfn = k_col<TT, EE, MODE>;                                                     \
        unw_smem_limit((const void*)kfn);                                                   \
        kfn<<<grid, TT, smem, s>>>(gd, st, n);                                              \
        return cudaGetLastError();                                                          \
    }
    UNW_CL(128, 16) UNW_CL(256, 16) UNW_CL(512, 16) UNW_CL(1024, 16) UNW_CL(1024, 32)
#undef UNW_CL
    return cudaErrorInvalidConfiguration;
}

cudaError_t unw_launch_col(int mode, int T, int emax, int nblk, size_t smem, cudaStream_t s,
                           const GridDev* gd, const int* starts, int n) {
    if (nblk <= 0) return cudaSuccess;
    dim3 grid(nblk);
    switch (mode) {
        case 0: return launch_col_t<0>(T, emax, grid, smem, s, gd, starts, n);
        case 1: return launch_col_t<1>(T, emax, grid, smem, s, gd, starts, n);
        default: return launch_col_t<2>(T, emax, grid, smem, s, gd, starts, n);
    }
}

cudaError_t unw_launch_tables(const FftPlanDev& f, const DctPlanDev& d, float* sv, int Ncos,
                              cudaStream_t s) {
    int m = f.n > d.N ? f.n : d.N;
    m = m > Ncos ? m : Ncos;
    int nb = (m + 255) / 256;
    nb = nb > 64 ? 64 : nb;
    k_tables<<<nb, 256, 0, s>>>(f, d, sv, Ncos);
    return cudaGetLastError();
}

cudaError_t unw_launch_hspec(int T, int emax, const DctPlanDev& d, cudaStream_t s) {
    const size_t smem = (size_t)d.fft.n * sizeof(float2);
#define UNW_HS(TT, EE)                                                                      \
    if (T == TT && emax == EE) {                                                            \
        auto kfn = k_hspec<TT, EE>;                                                         \
        unw_smem_limit((const void*)kfn);                                                   \
        kfn<<<1, TT, smem, s>>>(d);                                                         \
        return cudaGetLastError();                                                          \
    }
    UNW_HS(128, 16) UNW_HS(256, 16) UNW_HS(512, 16) UNW_HS(1024, 16) UNW_HS(1024, 32)
#undef UNW_HS
    return cudaErrorInvalidConfiguration;
}

cudaError_t unw_launch_simple(int which, int nblk, cudaStream_t s, const GridDev* gd,
                              const int* starts, int n, int it, UnwScalars sc) {
    if (nblk <= 0) return cudaSuccess;
    switch (which) {
        case UNW_K_STATE_INIT: k_state_init<<<(n + 63) / 64, 64, 0, s>>>(gd, n, sc); break;
        case UNW_K_SETUP: k_setup<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_K_MATVEC: k_matvec<<<nblk, 512, 0, s>>>(gd, starts, n, it); break;
        case UNW_K_HEAD: k_head<<<nblk, 256, 0, s>>>(gd, starts, n, it); break;
        case UNW_K_MEAN: k_mean<<<nblk, 256, 0, s>>>(gd, starts, n, it); break;
        case UNW_K_INIT_RECENTRE: k_init_recentre<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_K_COPY_BEST: k_copy_best<<<nblk, 256, 0, s>>>(gd, starts, n, it); break;
        case UNW_K_REL: k_rel<<<nblk, 256, 0, s>>>(gd, starts, n, it); break;
        case UNW_K_LAP_APPLY: k_lap_apply<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        case UNW_K_RESID: k_resid<<<nblk, 256, 0, s>>>(gd, starts, n); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}
