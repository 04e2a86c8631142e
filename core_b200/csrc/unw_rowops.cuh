// Elementwise work fused into the DCT row passes, shared by the generic and
// the power-of-two kernels: the value a row-forward pass transforms, what a
// row-inverse pass does with the transformed value, and the scalar decisions
// the last CTA of each pass takes (the reference's PCG `break` tests).
#pragma once
#include "unw_internal.cuh"

// A x at (i, j): -div(w grad x) in the reference's op order (utils_unwrap2d.py:1367-1388):
// res = 0; res -= dx[j-1]; res += dx[j]; res -= dy[i-1]; res += dy[i]; Ax = -res.
__device__ __forceinline__ float lap_at(const float* __restrict__ x, const float* __restrict__ wx,
                                        const float* __restrict__ wy, int i, int j, int H, int W, int P) {
    const size_t o = (size_t)i * P + j;
    const float xc = x[o];
    float res = 0.f;
    if (j > 0) res = fsub(res, fmul(fsub(xc, x[o - 1]), wx[o - 1]));
    if (j < W - 1) res = fadd(res, fmul(fsub(x[o + 1], xc), wx[o]));
    if (i > 0) res = fsub(res, fmul(fsub(xc, x[o - P]), wy[o - P]));
    if (i < H - 1) res = fadd(res, fmul(fsub(x[o + P], xc), wy[o]));
    return -res;
}

// Difference a - b of two iterate values held as float32 pairs: exact in float64,
// rounded once to float32.  (A float32 form, fl(fl(ah - bh) + fl(al - bl)), is within a
// few ulps of the difference too; on the 4096^2 fault grid, whose IRLS stop test is
// decided by rel_change within about 1% of tol at the 29th iteration, that form ended
// after 29 iterations where the reference's FP64 run takes 30, and this one takes 30.)
__device__ __forceinline__ float pair_diff(float ah, float al, float bh, float bl) {
    return __double2float_rn(((double)ah - (double)bh) + ((double)al - (double)bl));
}
// The same from the pairs' float64 values (hi + lo is exact in float64, and so is each of
// the two differences above; both forms round the exact difference once): each pixel's
// pair is converted once and shared by the differences it takes part in.
__device__ __forceinline__ float dpair_diff(double a, double b) { return __double2float_rn(a - b); }

// A x at (i, j) for the iterate x = U + L held as a float32 pair: the reference's op
// order (lap_at), each neighbour difference formed from the pair by pair_diff.
__device__ __forceinline__ float lap_at_pair(const float* __restrict__ U, const float* __restrict__ L,
                                             const float* __restrict__ wx, const float* __restrict__ wy, int i, int j,
                                             int H, int W, int P) {
    const size_t o = (size_t)i * P + j;
    const double xc = pair_val(U[o], L[o]);
    float res = 0.f;
    if (j > 0) res = fsub(res, fmul(dpair_diff(xc, pair_val(U[o - 1], L[o - 1])), wx[o - 1]));
    if (j < W - 1) res = fadd(res, fmul(dpair_diff(pair_val(U[o + 1], L[o + 1]), xc), wx[o]));
    if (i > 0) res = fsub(res, fmul(dpair_diff(xc, pair_val(U[o - P], L[o - P])), wy[o - P]));
    if (i < H - 1) res = fadd(res, fmul(dpair_diff(pair_val(U[o + P], L[o + P]), xc), wy[o]));
    return -res;
}

// Row-forward modes:
//  0 RHO  rho = -div(w g), the DCT initial solve (utils_unwrap2d.py:1478-1483)
//  1 R0   r = b - A x0, PCG start (utils_unwrap2d.py:1413-1419), with the neighbour
//         differences of x0 formed from the iterate pair; D (the PCG correction) = 0
//  2 UPD  x += alpha p; r -= alpha Ap (utils_unwrap2d.py:1445-1459); x is the
//         correction D = x - x0, added to the iterate pair at the IRLS tail
//  3 COPY r as given (operator entry point)
template <int MODE>
__device__ __forceinline__ bool rowfwd_gate(const InstState* s) {
    if (MODE == 0 || MODE == 3) return true;
    if (MODE == 1) return s->irls_active != 0;
    return s->irls_active != 0 && s->cg_active != 0;
}

// The iterate pointers of a row-forward pass at IRLS iteration `it`: mode 1 reads the
// current pair (U, L); mode 2 updates D.
template <int MODE>
__device__ __forceinline__ float* rowfwd_x(const GridDev& G, int it) {
    return MODE == 2 ? G.D : ((it & 1) ? G.U0 : G.U1);
}
__device__ __forceinline__ const float* rowfwd_lo(const GridDev& G, int it) { return (it & 1) ? G.L0 : G.L1; }

template <int MODE>
__device__ __forceinline__ float rowfwd_value(const GridDev& G, float* __restrict__ U, const float* __restrict__ Lo,
                                              const float* __restrict__ pk, float alpha, int i, int j,
                                              double (&acc)[2]) {
    const int H = G.H, W = G.W, P = G.P;
    const size_t o = (size_t)i * P + j;
    if (MODE == 0) {
        float rr = 0.f;
        if (j > 0) rr = fadd(rr, fmul(G.wx[o - 1], G.gx[o - 1]));
        if (j < W - 1) rr = fsub(rr, fmul(G.wx[o], G.gx[o]));
        if (i > 0) rr = fadd(rr, fmul(G.wy[o - P], G.gy[o - P]));
        if (i < H - 1) rr = fsub(rr, fmul(G.wy[o], G.gy[o]));
        return rr;
    } else if (MODE == 3) {
        return G.r[o];
    } else if (MODE == 1) {
        const float ax = lap_at_pair(U, Lo, G.wIx, G.wIy, i, j, H, W, P);
        const float val = fsub(G.b[o], ax);
        G.r[o] = val;
        G.D[o] = 0.f;
        acc[0] += isfinite(val) ? 0.0 : 1.0;
        acc[1] += (double)val * (double)val;
        return val;
    } else {
        const float xn = fmaf(alpha, pk[o], U[o]);
        const float rn = fmaf(-alpha, G.Ap[o], G.r[o]);
        U[o] = xn;
        G.r[o] = rn;
        acc[0] += (double)rn * (double)rn;
        acc[1] += isfinite(xn) ? 0.0 : 1.0;
        return rn;
    }
}

template <int MODE>
__device__ __forceinline__ void rowfwd_finalize(InstState* st, const double (&acc)[2]) {
    if (MODE == 1) {
        // non-finite initial residual: CG returns x0 (utils_unwrap2d.py:1418-1419)
        st->cg_active = acc[0] == 0.0 ? 1 : 0;
        if (st->cg_rel > 0.f) st->cg_tol = (float)((double)st->cg_rel * sqrt(acc[1]));
    } else if (MODE == 2) {
        const double rn = sqrt(acc[0]);
        st->rnorm = rn;
        if (acc[1] != 0.0 || !(rn >= (double)st->cg_tol) || !isfinite(rn)) st->cg_active = 0;
    }
}

// Last CTA of the matvec: pAp and its scalar step (utils_unwrap2d.py:1433-1442): stop on a tiny
// or non-finite pAp, else alpha = rz / pAp clamped to [-1e6, 1e6].
__device__ __forceinline__ void matvec_finalize(InstState* st, double pAp) {
    st->pAp = pAp;
    st->cg_iter += 1;
    if (fabs(pAp) < 1e-15 || !isfinite(pAp)) {
        st->cg_active = 0;
    } else {
        double a = st->rz / pAp;
        a = a < -1e6 ? -1e6 : (a > 1e6 ? 1e6 : a);
        st->alpha = (float)a;
    }
}

// Row-inverse modes:
//  0 INITU u = nan_to_num(z) (utils_unwrap2d.py:1498-1502), sum of u * valid
//  1 P0    p = z = M^-1 r                     (utils_unwrap2d.py:1421-1424)
//  2 P     p = z + beta p, z = M^-1 r         (utils_unwrap2d.py:1461-1473)
//  3 COPY  z as computed (operator entry point)
// r.z and beta come from the column pass (Parseval, col_finalize), so modes 1
// and 2 write p in place and never store z.
template <int MODE>
__device__ __forceinline__ bool rowinv_gate(const InstState* s) {
    if (MODE == 0 || MODE == 3) return true;
    return s->irls_active != 0 && s->cg_active != 0;
}

template <int MODE>
__device__ __forceinline__ void rowinv_store(const GridDev& G, int i, int j, float zv, float beta,
                                             double (&acc)[2]) {
    const size_t o = (size_t)i * G.P + j;
    if (MODE == 3) {
        G.z[o] = zv;
    } else if (MODE == 0) {
        const float u = isfinite(zv) ? zv : 0.f;
        acc[1] += isfinite(zv) ? 0.0 : 1.0;
        G.U0[o] = u;
        // (u * valid_float).sum(): an invalid pixel contributes u * 0
        acc[0] += (double)(u * (G.valid[o] ? 1.f : 0.f));
    } else if (MODE == 1) {
        G.p0[o] = zv;
    } else {
        // _cg_p.mul_(beta).add_(_cg_z): one rounding per operation
        G.p0[o] = fadd(fmul(G.p0[o], beta), zv);
    }
}

__device__ __forceinline__ void rowinv_finalize_initu(InstState* st, const double (&acc)[2]) {
    if (acc[1] != 0.0) st->status |= 1;  // UNW_S_DCT_INIT_NONFINITE
    st->mean = st->vcount > 0 ? acc[0] / st->vcount : 0.0;
}

// Last CTA of a PCG column pass: r.z of the new preconditioned residual.
// MODE 1 starts the recurrence (utils_unwrap2d.py:1427); MODE 2 applies the
// reference's test on the previous r.z, then beta (utils_unwrap2d.py:1464-1473).
template <int MODE>
__device__ __forceinline__ void col_finalize(InstState* st, double rzn) {
    if (MODE == 1) {
        st->rz = rzn;
    } else if (MODE == 2) {
        if (fabs(st->rz) < 1e-15) {
            st->cg_active = 0;
        } else {
            double be = rzn / st->rz;
            be = be < -1e6 ? -1e6 : (be > 1e6 ? 1e6 : be);
            st->beta = (float)be;
            st->rz = rzn;
        }
    }
}

// Both outputs of the column-pass spectral step for the frequency pair
// (k, km = H-k): the DCT-II extraction and the eigenvalue scaling are shared,
// only the DCT-III pre-twiddles differ.  For k = 0 (km = 0) or k = km the
// second output equals the first and is not used.
//
// RZ adds this pair's share of r.z to `rz` by Parseval's identity for the
// unnormalised DCT-II / DCT-III pair: with X the 2-D DCT-II of r and Y the
// scaled spectrum that the DCT-III turns into z,
//     r.z = sum_{k,l} e_k e_l X_kl Y_kl,   e_0 = 1/2, e_{k>0} = 1,
// so the preconditioned inner product needs no extra pass over r and z.
template <bool RZ>
__device__ __forceinline__ void col_spectral_pair(float2 C, float2 Cm, int k, int km, float2 wk, float2 wm,
                                                  float ck, float cm, float ca, float cb, bool ja0, bool hasb,
                                                  float negs, float2& ok, float2& om, double& rz) {
    const float2 Vak = make_float2(C.x + Cm.x, C.y - Cm.y);
    const float2 Vbk = make_float2(C.y + Cm.y, Cm.x - C.x);
    const float2 Vam = make_float2(Vak.x, -Vak.y);   // conj: the pair's extraction is symmetric
    const float2 Vbm = make_float2(Vbk.x, -Vbk.y);
    const float xak = wk.x * Vak.x - wk.y * Vak.y, xbk = wk.x * Vbk.x - wk.y * Vbk.y;
    const float xam = wm.x * Vam.x - wm.y * Vam.y, xbm = wm.x * Vbm.x - wm.y * Vbm.y;
    // X * (negs / lambda), lambda = -(sH + sW) in (-8, 0): a fast division (2 ulp),
    // well inside the preconditioner's tolerance
    const float Xak = (k == 0 && ja0) ? 0.f : xak * __fdividef(negs, -(ck + ca));
    const float Xam = (km == 0 && ja0) ? 0.f : xam * __fdividef(negs, -(cm + ca));
    const float Xbk = hasb ? xbk * __fdividef(negs, -(ck + cb)) : 0.f;
    const float Xbm = hasb ? xbm * __fdividef(negs, -(cm + cb)) : 0.f;
    if (RZ) {
        const float ea = ja0 ? 0.5f : 1.0f;
        float tk = fmaf(xak * ea, Xak, xbk * Xbk);
        if (k == 0) tk *= 0.5f;
        const float tm = km != k ? fmaf(xam * ea, Xam, xbm * Xbm) : 0.f;
        rz += (double)tk + (double)tm;
    }
    // DCT-III pre-twiddle V'_k = conj(w_k) (Y_k - i Y_{H-k}) with Y_H = 0
    const float mak = k == 0 ? 0.f : Xam, mbk = k == 0 ? 0.f : Xbm;
    const float2 Pak = cmul(cconj(wk), make_float2(Xak, -mak));
    const float2 Pbk = cmul(cconj(wk), make_float2(Xbk, -mbk));
    ok = cconj(make_float2(Pak.x - Pbk.y, Pak.y + Pbk.x));
    const float2 Pam = cmul(cconj(wm), make_float2(Xam, -Xak));
    const float2 Pbm = cmul(cconj(wm), make_float2(Xbm, -Xbk));
    om = cconj(make_float2(Pam.x - Pbm.y, Pam.y + Pbm.x));
}
