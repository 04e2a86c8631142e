// Allocation-free DCT preconditioner: z = IDCT2(-DCT2(r)/lambda), DC zeroed,
// the same operator and kernels as unw_apply_preconditioner, with every byte
// of scratch (plan tables, grid descriptor, the spectral work array) taken
// from one file-scope device array instead of a caller-provided workspace.
//
// Why: some callers cannot allocate device memory at the point where they
// need the operator -- plain C or Fortran codes that have no device allocator
// of their own, and real-time loops that must not allocate after start-up
// (an allocation can fail under memory pressure in the middle of a run, and
// releasing one with cudaFree synchronises the whole device).  They pass only inputs and outputs.
//
// Limits and rules:
//  * the array holds UNW_NOALLOC_BYTES (16 MiB) per GPU that loads the
//    library, for the life of the process;
//  * a grid must fit: H * W <= UNW_NOALLOC_MAX_PX float32 work values and
//    each transform length within the usual limits; larger grids are
//    rejected with UNW_E_UNSUPPORTED and a message;
//  * r and z must be 16-byte aligned device pointers (the row kernels move
//    four floats per access); others are rejected with UNW_E_ARG;
//  * every call on a device uses the same array, so calls that overlap on
//    the GPU (different streams, or threads without ordering) race; calls on
//    one stream are ordered and safe;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it for the
//    life of the process; after cudaDeviceReset that cached address is stale,
//    so a process that resets a device must not call this entry point again;
//  * each call uploads the grid descriptor from host memory with
//    cudaMemcpyAsync on the caller's stream;
//  * nothing in this path calls cudaMalloc, cudaFree or any allocating
//    library routine, and no host heap memory is used.
#include <cuda_runtime.h>
#include <cstring>
#include <mutex>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

#define UNW_NOALLOC_BYTES (16u << 20)
#define UNW_NOALLOC_HEADER (1u << 20)  // descriptor, CTA prefixes, plan tables
#define UNW_NOALLOC_MAX_PX ((UNW_NOALLOC_BYTES - UNW_NOALLOC_HEADER) / 4)
#define UNW_NOALLOC_MAX_DEV 64

static __device__ __align__(256) unsigned char g_unw_scratch[UNW_NOALLOC_BYTES];

namespace {

std::mutex g_mu;
void* g_dev_ptr[UNW_NOALLOC_MAX_DEV];  // device address of g_unw_scratch per device

// Device address of the scratch array on the current device (looked up once).
int scratch_ptr(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= UNW_NOALLOC_MAX_DEV)
        return unw_set_error(UNW_E_CUDA, "no current CUDA device for the allocation-free preconditioner");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_unw_scratch);
        if (e != cudaSuccess || !p) return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
        g_dev_ptr[dev] = p;
    }
    *out = (unsigned char*)g_dev_ptr[dev];
    return UNW_OK;
}

// ---- plan arithmetic on fixed arrays (same rules as the allocating path)
bool smooth7(long long n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}
long long next_smooth(long long x) {
    while (!smooth7(x)) x++;
    return x;
}
struct LeanPlan {
    int N, n, blue, npass, cap;
    int rad[UNW_MAX_PASSES];
};
bool make_plan(int N, LeanPlan& p) {
    p.N = N;
    p.blue = smooth7(N) ? 0 : 1;
    p.n = p.blue ? (int)next_smooth(2LL * N - 1) : N;
    int m = p.n, k = 0, tmp[UNW_MAX_PASSES + 8];
    int twos = 0;
    for (int q : {7, 5, 3})
        while (m % q == 0) { if (k >= UNW_MAX_PASSES) return false; tmp[k++] = q; m /= q; }
    while (m % 2 == 0) { twos++; m /= 2; }
    int pre[8], np = 0;
    while (twos >= 4) { pre[np++] = 16; twos -= 4; if (np >= 8) return false; }
    if (twos) pre[np++] = 1 << twos;
    // radix-16 (and the small power of two) first, then 7, 5, 3 -- the order of the allocating path
    p.npass = 0;
    for (int i = np - 1; i >= 0; i--) {  // the allocating path inserts at the front: small radix first
        if (p.npass >= UNW_MAX_PASSES) return false;
        p.rad[p.npass++] = pre[i];
    }
    for (int i = 0; i < k; i++) {
        if (p.npass >= UNW_MAX_PASSES) return false;
        p.rad[p.npass++] = tmp[i];
    }
    if (p.n == 1) p.npass = 0;
    p.cap = 16;
    for (int i = 0; i < p.npass; i++) p.cap = p.cap < (16 / p.rad[i]) * p.rad[i] ? p.cap : (16 / p.rad[i]) * p.rad[i];
    return true;
}
int pick_threads(long long elems, int cap) {
    for (int T : {128, 256, 512, 1024})
        if ((long long)T * cap >= elems) return T;
    return 0;
}
size_t up(size_t x, size_t a) { return (x + a - 1) / a * a; }
bool pow2_ok(int n) { return n >= 256 && n <= 16384 && (n & (n - 1)) == 0; }

}  // namespace

extern "C" int unw_apply_preconditioner_noalloc(const float* r, int64_t H, int64_t W, float* z,
                                                void* cuda_stream) {
    if (!r || !z) return unw_set_error(UNW_E_ARG, "null pointer");
    if (((uintptr_t)r | (uintptr_t)z) & 15)
        return unw_set_error(UNW_E_ARG, "r and z must be 16-byte aligned device pointers");
    if (H <= 0 || W <= 0) return unw_set_error(UNW_E_ARG, "bad shape");
    if (H * W > (int64_t)UNW_NOALLOC_MAX_PX)
        return unw_set_error(UNW_E_UNSUPPORTED,
                             "grid too large for the allocation-free preconditioner: H*W must be <= 3932160");
    LeanPlan pr, pc;
    if (!make_plan((int)W, pr) || !make_plan((int)H, pc) || pr.n > 16384 || pc.n > 16384)
        return unw_set_error(UNW_E_UNSUPPORTED, "transform length beyond 16384");
    unsigned char* base = nullptr;
    int rc = scratch_ptr(&base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)cuda_stream;

    // header layout inside the first UNW_NOALLOC_HEADER bytes
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t at = o; o = up(o + bytes, 256); return at; };
    const size_t o_g = take(sizeof(GridDev));
    const size_t o_st = take(sizeof(int) * 8 * (KS_NKIND + 1));
    const size_t o_state = take(sizeof(InstState));
    const size_t o_cnt = take(sizeof(unsigned) * 4);
    const size_t o_twr = take(sizeof(float2) * pr.n), o_hsr = take(sizeof(float2) * pr.n);
    const size_t o_dwr = take(sizeof(float2) * pr.N), o_chr = take(sizeof(float2) * pr.N);
    const size_t o_sw = take(sizeof(float) * pr.N);
    const size_t o_twc = take(sizeof(float2) * pc.n), o_hsc = take(sizeof(float2) * pc.n);
    const size_t o_dwc = take(sizeof(float2) * pc.N), o_chc = take(sizeof(float2) * pc.N);
    const size_t o_sh = take(sizeof(float) * pc.N);
    if (o > UNW_NOALLOC_HEADER)
        return unw_set_error(UNW_E_UNSUPPORTED, "plan tables exceed the allocation-free header");

    GridDev G;
    memset(&G, 0, sizeof(G));
    G.H = (int)H;
    G.W = (int)W;
    G.P = (int)W;  // r and z are dense; the spectral array T uses the same pitch
    G.H0 = G.H;
    G.W0 = G.W;
    G.r = const_cast<float*>(r);
    G.z = z;
    G.T = (float*)(base + UNW_NOALLOC_HEADER);
    G.st = (InstState*)(base + o_state);
    G.counter = (unsigned*)(base + o_cnt);
    G.sW = (const float*)(base + o_sw);
    G.sH = (const float*)(base + o_sh);
    const LeanPlan* lp[2] = {&pr, &pc};
    DctPlanDev* dp[2] = {&G.prow, &G.pcol};
    const size_t tw[2] = {o_twr, o_twc}, hs[2] = {o_hsr, o_hsc}, dw[2] = {o_dwr, o_dwc}, ch[2] = {o_chr, o_chc};
    for (int d = 0; d < 2; d++) {
        DctPlanDev& D = *dp[d];
        D.N = lp[d]->N;
        D.blue = lp[d]->blue;
        D.stride = lp[d]->n;
        D.fft.n = lp[d]->n;
        D.fft.npass = lp[d]->npass;
        for (int i = 0; i < lp[d]->npass; i++) D.fft.radix[i] = lp[d]->rad[i];
        D.fft.tw = (const float2*)(base + tw[d]);
        D.dctw = (const float2*)(base + dw[d]);
        D.chirp = (const float2*)(base + ch[d]);
        D.hspec = (const float2*)(base + hs[d]);
    }
    // launch shapes: the power-of-two register-FFT kernels or the generic ones
    const int row_p2 = pow2_ok(G.W) ? G.W : 0;
    const int col_p2 = pow2_ok(G.H) ? G.H : 0;
    const int rT = pick_threads(pr.n, pr.cap);
    int nseq = (int)(96 * 1024 / ((size_t)pc.n * sizeof(float2)));
    nseq = nseq < 1 ? 1 : (nseq > 8 ? 8 : nseq);
    nseq = nseq < (G.W + 1) / 2 ? nseq : (G.W + 1) / 2;
    int cT = 0;
    while (nseq >= 1 && !(cT = pick_threads((long long)nseq * pc.n, pc.cap))) nseq--;
    if (!rT || !cT) return unw_set_error(UNW_E_UNSUPPORTED, "no launch shape");
    G.col_nseq = col_p2 ? unw_p2_col_nseq(col_p2) : nseq;
    const int cthreads = col_p2 ? col_p2 / 16 * G.col_nseq : cT;
    int per_sm = 2048 / cthreads;
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    G.col_ctas = 148 * per_sm;
    const int n_row = (G.H + 1) / 2 < 148 * 4 ? (G.H + 1) / 2 : 148 * 4;
    const int nslab = (G.W + 2 * G.col_nseq - 1) / (2 * G.col_nseq);
    const int n_col = nslab < G.col_ctas ? nslab : G.col_ctas;
    int starts[2 * (KS_NKIND + 1)];
    memset(starts, 0, sizeof(starts));
    starts[2 * KS_ROWPAIR + 1] = n_row;
    starts[2 * KS_COL + 1] = n_col;
    GridDev* dG = (GridDev*)(base + o_g);
    int* dS = (int*)(base + o_st);
    cudaError_t e;
    if ((e = cudaMemcpyAsync(dG, &G, sizeof(G), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(dS, starts, sizeof(starts), cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    if ((e = unw_launch_tables(G.prow.fft, G.prow, const_cast<float*>(G.sW), G.W, s)) != cudaSuccess ||
        (e = unw_launch_tables(G.pcol.fft, G.pcol, const_cast<float*>(G.sH), G.H, s)) != cudaSuccess)
        return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    if (G.prow.blue && (e = unw_launch_hspec(pick_threads(pr.n, pr.cap), 16, G.prow, s)) != cudaSuccess)
        return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    if (G.pcol.blue && (e = unw_launch_hspec(pick_threads(pc.n, pc.cap), 16, G.pcol, s)) != cudaSuccess)
        return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    const size_t row_smem = (size_t)pr.n * sizeof(float2), col_smem = (size_t)nseq * pc.n * sizeof(float2);
    e = row_p2 ? unw_launch_rowf_p2(row_p2, 3, n_row, s, dG, dS + 2 * KS_ROWPAIR, 1, 0, 0)
               : unw_launch_row_fwd(3, rT, 16, n_row, row_smem, s, dG, dS + 2 * KS_ROWPAIR, 1, 0, 0);
    if (e == cudaSuccess)
        e = col_p2 ? unw_launch_col_p2(col_p2, 0, n_col, s, dG, dS + 2 * KS_COL, 1)
                   : unw_launch_col(0, cT, 16, n_col, col_smem, s, dG, dS + 2 * KS_COL, 1);
    if (e == cudaSuccess)
        e = row_p2 ? unw_launch_rowi_p2(row_p2, 3, n_row, s, dG, dS + 2 * KS_ROWPAIR, 1)
                   : unw_launch_row_inv(3, rT, 16, n_row, row_smem, s, dG, dS + 2 * KS_ROWPAIR, 1);
    if (e != cudaSuccess) return unw_set_error(UNW_E_CUDA, cudaGetErrorString(e));
    return UNW_OK;
}
