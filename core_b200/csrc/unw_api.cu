// Host orchestration and C ABI of the B200 unwrapper.
//
// A solve is: bounding box of valid pixels (one device->host read), per-grid
// FFT plans and tables, setup + DCT initial solve, the IRLS loop (enqueued
// `check_every` iterations at a time, then one small device->host read of the
// per-grid state to see whether any grid is still iterating), and the device
// post-processing.  All device memory comes from the caller's workspace; the
// layout is computed by one function for both sizing and carving.
#include <cuda_runtime.h>
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <thread>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

namespace {

thread_local char g_err[512];
thread_local cudaStream_t g_worker_stream = nullptr;  // a launch-group worker thread's own stream

int set_err(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return set_err(UNW_E_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

// a kernel launch of family `fam`, timed when profiling is on
#define PL(fam, call)              \
    do {                           \
        S.prof.begin((fam), S.s);  \
        CK(call);                  \
        S.prof.end(S.s);           \
    } while (0)

constexpr int EMAX = 16;
constexpr size_t ALIGN = 256;
constexpr int HIST_CAP = 65536;
constexpr int ELEM_MAX_CTAS = 1184;      // 8 x 148 SMs
constexpr size_t COL_SMEM_BUDGET = 96 * 1024;
constexpr int MAX_FFT = 16384;           // longest register FFT (1024 threads x 16)
// longest transform of the shared-memory FFT (1024 threads x up to 32 elements,
// one 8-byte slot per element within the 227 KB of shared memory a CTA can have)
constexpr int MAX_GEN = 28672;
// CTAs of the persistent PCG kernels (148 SMs x resident CTAs per SM)
constexpr int NUM_SMS = 148;
constexpr int CTAS_ROW = NUM_SMS * 4;
constexpr int CTAS_MATVEC = NUM_SMS * 2;
constexpr int CTAS_HEAD = NUM_SMS * 4;

size_t up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// ------------------------------------------------------------ FFT plans
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
int fft_len(int N) { return smooth7(N) ? N : (int)next_smooth(2LL * N - 1); }
long long next_pow2(long long x) {
    long long p = 1;
    while (p < x) p <<= 1;
    return p;
}
// Bluestein length M >= 2N - 1 of the register-FFT path for a DCT length N that
// is not a power of two: the shorter of the power of two (>= 256) and three
// times a power of two (>= 768) that fit; 0 where the path is not used (powers
// of two have their own kernels; very short axes stay on the generic
// shared-memory FFT; N > 8192 would need M > 16384).
int bl_len(int N) {
    if (N <= 64 || 2LL * N - 1 > MAX_FFT || (N & (N - 1)) == 0) return 0;
    const long long need = 2LL * N - 1;
    const long long m2 = std::max<long long>(256, next_pow2(need));
    const long long m3 = 3 * std::max<long long>(256, next_pow2((need + 2) / 3));
    return (int)std::min(m2, m3);
}

std::vector<int> factor(int n) {
    std::vector<int> r;
    int m = n;
    for (int p : {7, 5, 3})
        while (m % p == 0) { r.push_back(p); m /= p; }
    int twos = 0;
    while (m % 2 == 0) { twos++; m /= 2; }
    while (twos >= 4) { r.insert(r.begin(), 16); twos -= 4; }
    if (twos == 3) r.insert(r.begin(), 8);
    if (twos == 2) r.insert(r.begin(), 4);
    if (twos == 1) r.insert(r.begin(), 2);
    return r;
}
// elements per thread of the shared-memory FFT: 16, or 32 for lengths a
// 1024-thread CTA cannot cover with 16
int emax_of(long long n) { return n > 16384 ? 32 : EMAX; }
// complex elements one thread can hold per pass, over the radices of a plan
int plan_cap(const std::vector<int>& rad, int emax) {
    int c = emax;
    for (int R : rad) c = std::min(c, (emax / R) * R);
    return c;
}
int pick_threads(long long elems, int cap) {
    for (int T : {128, 256, 512, 1024})
        if ((long long)T * cap >= elems) return T;
    return 0;
}

struct HostPlan {
    int N = 0, n = 0, blue = 0, cap = 0, emax = 16;
    std::vector<int> rad;
};
HostPlan make_plan(int N) {
    HostPlan p;
    p.N = N;
    const int M = bl_len(N);
    p.blue = (M || !smooth7(N)) ? 1 : 0;
    p.n = M ? M : fft_len(N);
    p.rad = p.n > 1 ? factor(p.n) : std::vector<int>{};
    p.emax = emax_of(p.n);
    p.cap = plan_cap(p.rad, p.emax);
    return p;
}

// ------------------------------------------------------------ layout
struct GridLayout {
    size_t st, counter, part, tw_r, dw_r, ch_r, hs_r, cos_r, tw_c, dw_c, ch_c, hs_c, cos_c;
    size_t arr[20];          // gx gy wx wy | wIx wIy b r z p0 p1 Ap T | U0 U1 Ub | L0 L1 Lb D
    size_t valid, hist, tilecnt;
    size_t tc;               // split DCT matrices of the tensor-core column pass (H0 <= UNW_TC_MAX_H), else 0
    size_t post_parent, post_lab, post_csum, post_ccount, post_remap, post_adj;
    size_t end;
    long long P0, max_ctas, lab_cap, ntiles_max;
    int fr_cap, fc_cap;      // capacities of the FFT tables (row / column)
};

struct BatchLayout {
    size_t rowany, colany, bbox, gdev, starts;
    size_t tcmaps;           // UNW_MAPS_PER_GRID 128-byte tensor maps per grid (TMA-staged passes)
    std::vector<size_t> base;
    std::vector<GridLayout> g;
    size_t total;
};

GridLayout grid_layout(long long H0, long long W0) {
    GridLayout L{};
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o = up(o + bytes, ALIGN); return r; };
    L.P0 = (long long)up((size_t)W0, 32);
    const size_t A = (size_t)H0 * (size_t)L.P0 * sizeof(float);
    L.max_ctas = std::max<long long>({(H0 + 1) / 2, (W0 + 1) / 2, ((W0 + 127) / 128) * ((H0 + 7) / 8),
                                      ELEM_MAX_CTAS});
    // room for the longest transform of any crop: Bluestein lengths (smooth or
    // power of two, see bl_len) and direct lengths
    auto cap = [](long long N0) {
        long long c = std::max<long long>(next_smooth(2 * N0 - 1), N0);
        return std::max<long long>(c, std::min<long long>(MAX_FFT, std::max<long long>(256, next_pow2(2 * N0 - 1))));
    };
    L.fr_cap = (int)cap(W0);
    L.fc_cap = (int)cap(H0);
    L.st = take(sizeof(InstState));
    L.counter = take(sizeof(unsigned) * 4);
    L.part = take((size_t)L.max_ctas * UNW_NPART * sizeof(double));
    L.tw_r = take(sizeof(float2) * L.fr_cap);
    L.hs_r = take(sizeof(float2) * L.fr_cap);
    L.dw_r = take(sizeof(float2) * W0);
    L.ch_r = take(sizeof(float2) * W0);
    L.cos_r = take(sizeof(float) * W0);
    L.tw_c = take(sizeof(float2) * L.fc_cap);
    L.hs_c = take(sizeof(float2) * L.fc_cap);
    L.dw_c = take(sizeof(float2) * H0);
    L.ch_c = take(sizeof(float2) * H0);
    L.cos_c = take(sizeof(float) * H0);
    for (int a = 0; a < 20; a++) L.arr[a] = take(A);
    L.valid = take((size_t)H0 * L.P0);
    L.tc = H0 <= UNW_TC_MAX_H ? take(unw_tc_table_bytes((int)H0)) : 0;
    L.hist = take(sizeof(int) * HIST_CAP);
    L.ntiles_max = (H0 * W0 + 4095) / 4096;
    L.tilecnt = take(sizeof(int) * (size_t)L.ntiles_max);
    // post-processing scratch overlays the PCG arrays wIx..T (dead after the solve)
    const long long npx = H0 * W0;
    L.lab_cap = npx / 2 + 2;
    size_t po = L.arr[4];
    auto ptake = [&](size_t bytes) { size_t r = po; po = up(po + bytes, ALIGN); return r; };
    L.post_parent = ptake(sizeof(int) * (size_t)npx);
    L.post_lab = ptake(sizeof(int) * (size_t)npx);
    L.post_csum = ptake(sizeof(double) * 4 * (size_t)L.lab_cap);
    L.post_adj = ptake(sizeof(double) * (size_t)L.lab_cap);
    L.post_ccount = ptake(sizeof(int) * (size_t)L.lab_cap);
    L.post_remap = ptake(sizeof(int) * (size_t)L.lab_cap);
    L.end = std::max(o, po);
    return L;
}

BatchLayout batch_layout(int n, const long long* H, const long long* W) {
    BatchLayout B;
    size_t o = 0;
    auto take = [&](size_t bytes) { size_t r = o; o = up(o + bytes, ALIGN); return r; };
    long long sh = 0, sw = 0;
    for (int g = 0; g < n; g++) { sh += H[g]; sw += W[g]; }
    B.rowany = take(sizeof(int) * (size_t)std::max(1LL, sh));
    B.colany = take(sizeof(int) * (size_t)std::max(1LL, sw));
    B.bbox = take(sizeof(int) * 4 * (size_t)n);
    B.gdev = take(sizeof(GridDev) * (size_t)n);
    B.starts = take(sizeof(int) * (size_t)(KS_NKIND + 1) * (2 * (size_t)n + 1));
    B.tcmaps = take(UNW_MAP_BYTES * (size_t)n);
    for (int g = 0; g < n; g++) {
        GridLayout L = grid_layout(H[g], W[g]);
        B.base.push_back(o);
        B.g.push_back(L);
        o = up(o + L.end, ALIGN);
    }
    B.total = o + ALIGN;  // slack for aligning the caller's base pointer
    return B;
}

// ------------------------------------------------------------ launch shapes
struct Shape {
    int row_T = 0, col_T = 0;
    int row_emax = 16, col_emax = 16;   // elements per thread of the shared-memory FFT
    size_t row_smem = 0, col_smem = 0;
    int row_p2 = 0, col_p2 = 0;   // power-of-two register-FFT paths (length), 0 = generic
    int row_bl = 0, col_bl = 0;   // Bluestein register-FFT paths (FFT length M), 0 = not used
    int col_tc = 0;               // tensor-core column pass (mixed precision), chosen by the autotuner
    int col_p2_tma = 0;           // power-of-two column pass with the slab moved by TMA (H 2048 / 4096)
    int mv_tma = 0;               // matvec on TMA-staged halo tiles
};

int elem_ctas(long long npx) {
    long long c = (npx + 2047) / 2048;
    return (int)std::max<long long>(1, std::min<long long>(c, ELEM_MAX_CTAS));
}

// Optional per-launch CUDA-event timing (UNW_F_PROFILE): an event pair brackets
// each kernel launch on the solve stream; times are summed per kernel family.
struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<std::pair<int, size_t>> marks;  // (family, index of the start event)
    size_t next = 0;
    int fam = 0;
    size_t cur = 0;
    cudaEvent_t get() {
        if (next == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[next++];
    }
    void begin(int f, cudaStream_t s) {
        if (!on) return;
        fam = f;
        cur = next;
        cudaEventRecord(get(), s);
    }
    void end(cudaStream_t s) {
        if (!on) return;
        cudaEventRecord(get(), s);
        marks.push_back({fam, cur});
    }
    void collect(float* ms, int* cnt) {
        if (!on) return;
        for (auto& m : marks) {
            float t = 0.f;
            if (cudaEventSynchronize(pool[m.second + 1]) == cudaSuccess &&
                cudaEventElapsedTime(&t, pool[m.second], pool[m.second + 1]) == cudaSuccess) {
                ms[m.first] += t;
                cnt[m.first] += 1;
            }
        }
    }
    ~Prof() {
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct TuneResult {
    int tc = 0;
    float ms_fft = 0.f, ms_tc = 0.f;   // per launch of each column pass
};

struct Solver {
    int n = 0;
    Prof prof;
    cudaStream_t s = nullptr;
    std::vector<GridDev> hg;     // host copies
    std::vector<int> starts;     // [KS_NKIND + 1][n + 1]  (last row: post tiles)
    std::vector<int> total;      // CTAs per kind
    GridDev* dg = nullptr;
    int* dstarts = nullptr;
    Shape sh;
    TcMaps maps;                 // tensor maps of the split DCT matrices (col_tc)
    void* bmaps = nullptr;       // device: per-grid tensor maps of the TMA-staged passes
    std::vector<unsigned char> hmaps;  // their host image (UNW_MAP_BYTES per grid, 64-byte aligned)
    unsigned char* host_maps(int ngrids) {
        if (hmaps.size() < UNW_MAP_BYTES * (size_t)ngrids + 64) hmaps.assign(UNW_MAP_BYTES * (size_t)ngrids + 64, 0);
        return (unsigned char*)(((size_t)hmaps.data() + 63) & ~(size_t)63);
    }
    TuneResult tune;             // autotuner timings of the column pass (mixed precision)
    UnwScalars sc{};
    const int* ds(int kind) const { return dstarts + (size_t)kind * (n + 1); }
};

int kind_ctas(const GridDev& G, int kind) {
    if (G.H == 0) return 0;
    const long long npx = (long long)G.H * G.W;
    switch (kind) {
        // persistent kinds: at most a few CTAs per SM, each loops over its units
        case KS_ROWPAIR: return std::min((G.H + 1) / 2, CTAS_ROW);
        case KS_COL: return std::min((G.W + 2 * G.col_nseq - 1) / (2 * G.col_nseq), G.col_ctas);
        case KS_STEN: return std::min(G.sten_tiles_x * ((G.H + 8 * G.sten_rows - 1) / (8 * G.sten_rows)), CTAS_HEAD);
        case KS_MATVEC: return std::min(G.sten_tiles_x * ((G.H + 15) / 16), CTAS_MATVEC);
        case KS_ELEM: return elem_ctas(npx);
        case KS_ONE: return 1;
        default: return (int)((npx + 4095) / 4096);  // post tiles
    }
}

// DCT pass launchers: power-of-two register-FFT kernels or the generic ones
cudaError_t L_rowf(Solver& S, int mode, int it, int cgk) {
    if (S.sh.row_p2)
        return unw_launch_rowf_p2(S.sh.row_p2, mode, S.total[KS_ROWPAIR], S.s, S.dg, S.ds(KS_ROWPAIR), S.n, it, cgk);
    if (S.sh.row_bl)
        return unw_launch_rowf_bl(S.sh.row_bl, mode, S.total[KS_ROWPAIR], S.s, S.dg, S.ds(KS_ROWPAIR), S.n, it, cgk);
    return unw_launch_row_fwd(mode, S.sh.row_T, S.sh.row_emax, S.total[KS_ROWPAIR], S.sh.row_smem, S.s, S.dg,
                              S.ds(KS_ROWPAIR), S.n, it, cgk);
}
cudaError_t L_rowi(Solver& S, int mode) {
    if (S.sh.row_p2) return unw_launch_rowi_p2(S.sh.row_p2, mode, S.total[KS_ROWPAIR], S.s, S.dg, S.ds(KS_ROWPAIR), S.n);
    if (S.sh.row_bl) return unw_launch_rowi_bl(S.sh.row_bl, mode, S.total[KS_ROWPAIR], S.s, S.dg, S.ds(KS_ROWPAIR), S.n);
    return unw_launch_row_inv(mode, S.sh.row_T, S.sh.row_emax, S.total[KS_ROWPAIR], S.sh.row_smem, S.s, S.dg,
                              S.ds(KS_ROWPAIR), S.n);
}
cudaError_t L_col(Solver& S, int mode) {
    if (S.sh.col_tc) return unw_launch_col_tc(mode, S.total[KS_TC], S.s, S.dg, S.ds(KS_TC), S.n, &S.maps, S.bmaps);
    if (S.sh.col_p2_tma)
        return unw_launch_col_p2_tma(S.sh.col_p2, mode, S.total[KS_COL], S.s, S.dg, S.ds(KS_COL), S.n, S.bmaps);
    if (S.sh.col_p2) return unw_launch_col_p2(S.sh.col_p2, mode, S.total[KS_COL], S.s, S.dg, S.ds(KS_COL), S.n);
    if (S.sh.col_bl) return unw_launch_col_bl(S.sh.col_bl, mode, S.total[KS_COL], S.s, S.dg, S.ds(KS_COL), S.n);
    return unw_launch_col(mode, S.sh.col_T, S.sh.col_emax, S.total[KS_COL], S.sh.col_smem, S.s, S.dg, S.ds(KS_COL),
                          S.n);
}

// ------------------------------------------------------------ IRLS enqueue
int enqueue_pcg(Solver& S, int t, int k0, int k1);

// The PCG of a single-instance solver after its start pass, in chunks of `chunk` iterations
// until the instance's PCG has stopped or cg_max_iter is reached: a solve that stops after k
// iterations costs about k launches of each kernel instead of cg_max_iter gated ones.
int pcg_chunked(Solver& S, int t, int chunk) {
    const int n = S.n;
    std::vector<int> flags(2 * (size_t)n);  // cg_active, irls_active per instance
    for (int k0 = 0; k0 < S.sc.cg_max_iter; k0 += chunk) {
        const int rc = enqueue_pcg(S, t, k0, std::min(S.sc.cg_max_iter, k0 + chunk));
        if (rc) return rc;
        for (int g = 0; g < n; g++) {
            const InstState* d = S.hg[g].st;
            CK(cudaMemcpyAsync(&flags[2 * g], &d->cg_active, sizeof(int), cudaMemcpyDeviceToHost, S.s));
            CK(cudaMemcpyAsync(&flags[2 * g + 1], &d->irls_active, sizeof(int), cudaMemcpyDeviceToHost, S.s));
        }
        CK(cudaStreamSynchronize(S.s));
        bool any = false;
        for (int g = 0; g < n; g++) any |= S.hg[g].H > 0 && flags[2 * g] && flags[2 * g + 1];
        if (!any) break;
    }
    return UNW_OK;
}

// PCG iterations k0 .. k1-1 of IRLS iteration t (each kernel returns at once for an
// instance whose PCG has stopped)
int enqueue_pcg(Solver& S, int t, int k0, int k1) {
    const int n = S.n;
    cudaStream_t s = S.s;
    for (int k = k0; k < k1; k++) {
        PL(UNW_PROF_MATVEC, S.sh.mv_tma ? unw_launch_matvec_tma(S.total[KS_MATVEC], s, S.dg, S.ds(KS_MATVEC), n, S.bmaps)
                                        : unw_launch_simple(UNW_K_MATVEC, S.total[KS_MATVEC], s, S.dg, S.ds(KS_MATVEC),
                                                            n, k, S.sc));
        PL(UNW_PROF_ROW_UPD, L_rowf(S, 2, t, k));
        PL(UNW_PROF_COL, L_col(S, 2));
        PL(UNW_PROF_ROW_INV, L_rowi(S, 2));
    }
    return UNW_OK;
}

// One IRLS iteration; with chunk > 0 the PCG runs in chunks of that many iterations with a
// read of the instance's state between chunks (single-instance solvers with a large PCG cap:
// the adjoint), else all cg_max_iter iterations are enqueued (graph capture).
int enqueue_iteration(Solver& S, int t, int chunk = 0) {
    const int n = S.n;
    cudaStream_t s = S.s;
    PL(UNW_PROF_ELEM, unw_launch_simple(UNW_K_MEAN, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, t, S.sc));
    PL(UNW_PROF_HEAD, unw_launch_simple(UNW_K_HEAD, S.total[KS_STEN], s, S.dg, S.ds(KS_STEN), n, t, S.sc));
    PL(UNW_PROF_ELEM, unw_launch_simple(UNW_K_COPY_BEST, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, t, S.sc));
    PL(UNW_PROF_ROW_R0, L_rowf(S, 1, t, 0));
    PL(UNW_PROF_COL, L_col(S, 1));
    PL(UNW_PROF_ROW_INV, L_rowi(S, 1));
    const int rc = chunk > 0 ? pcg_chunked(S, t, chunk) : enqueue_pcg(S, t, 0, S.sc.cg_max_iter);
    if (rc) return rc;
    PL(UNW_PROF_ELEM, unw_launch_simple(UNW_K_REL, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, t, S.sc));
    return UNW_OK;
}

// One IRLS iteration as a CUDA graph.  Kernels only use the parity of the
// iteration index (which U buffer is current), so two executable graphs cover
// a whole solve.  Capture runs on a private non-blocking stream of this thread
// (the caller's stream may be the legacy default stream, which cannot be
// captured); the graphs are then launched on the caller's stream.
struct IterGraphs {
    cudaGraphExec_t ex[2] = {nullptr, nullptr};
    ~IterGraphs() {
        for (auto e : ex)
            if (e) cudaGraphExecDestroy(e);
    }
};

cudaStream_t capture_stream() {
    thread_local std::map<int, cudaStream_t> streams;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    auto it = streams.find(dev);
    if (it != streams.end()) return it->second;
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    streams[dev] = cs;
    return cs;
}

// Returns UNW_OK with both graphs built, or an error code; a failed capture
// leaves no graph and no stream in capture mode.
int build_iteration_graphs(Solver& S, IterGraphs& G) {
    // a launch-group worker captures on its own stream; otherwise capture runs on this
    // thread's private stream (the caller's stream may be the legacy default stream,
    // which cannot be captured, or be shared with other work)
    cudaStream_t cs = (S.s && S.s == g_worker_stream) ? S.s : capture_stream();
    if (!cs) return set_err(UNW_E_CUDA, "no capture stream");
    cudaStream_t user = S.s;
    for (int par = 0; par < 2; par++) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
        S.s = cs;
        const int rc = enqueue_iteration(S, par);
        S.s = user;
        const cudaError_t e = cudaStreamEndCapture(cs, &g);
        if (rc != UNW_OK || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return rc != UNW_OK ? rc : set_err(UNW_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
        }
        const cudaError_t ei = cudaGraphInstantiate(&G.ex[par], g, 0);
        cudaGraphDestroy(g);
        CK(ei);
    }
    return UNW_OK;
}

int read_states(Solver& S, std::vector<InstState>& out) {
    out.resize(S.n);
    for (int g = 0; g < S.n; g++)
        CK(cudaMemcpyAsync(&out[g], S.hg[g].st, sizeof(InstState), cudaMemcpyDeviceToHost, S.s));
    CK(cudaStreamSynchronize(S.s));
    return UNW_OK;
}

int validate_params(const unw_params* p) {
    if (!p) return set_err(UNW_E_ARG, "params is NULL");
    if (p->max_iter < 0 || p->cg_max_iter < 0) return set_err(UNW_E_ARG, "negative iteration count");
    return UNW_OK;
}

// column pairs per generic column CTA under the shared-memory budget
int col_nseq_generic(int nfft, int W) {
    int nseq = (int)std::max<size_t>(1, std::min<size_t>(8, COL_SMEM_BUDGET / ((size_t)nfft * sizeof(float2))));
    return std::min(nseq, (W + 1) / 2);
}

// Launch-group key of a cropped H x W grid: grids with equal keys share every
// kernel configuration (power-of-two length, or generic thread count) per axis.
std::array<int, 4> group_key(int H, int W) {
    if (H <= 0 || W <= 0) return {-1, 0, -1, 0};
    auto p2 = [](int n) { return n >= 256 && n <= MAX_FFT && (n & (n - 1)) == 0; };
    std::array<int, 4> k{};
    if (p2(W)) { k[0] = 1; k[1] = W; }
    else if (bl_len(W)) { k[0] = 2; k[1] = bl_len(W); }
    else { const HostPlan hp = make_plan(W); k[0] = 0; k[1] = pick_threads(hp.n, hp.cap) * 64 + hp.emax; }
    if (p2(H)) { k[2] = 1; k[3] = H; }
    else if (bl_len(H)) { k[2] = 2; k[3] = bl_len(H); }
    else {
        const HostPlan hp = make_plan(H);
        int nseq = col_nseq_generic(hp.n, W), cT = 0;
        while (nseq >= 1 && !(cT = pick_threads((long long)nseq * hp.n, hp.cap))) nseq--;
        k[2] = 0; k[3] = cT * 64 + hp.emax;
    }
    return k;
}

// Autotuner of the power-of-two column pass at H = 2048 / 4096: times the pass with the
// slab moved by TMA against the plain-load pass on the group's own buffers (DCT
// initial-solve mode; two warm-up and three timed launches of each on the solve stream)
// and returns 1 when TMA is faster.  Both give the same bits, so the choice changes only
// the time.  Cached per device, H and the group's total width for the life of the
// process; it runs before any graph capture.
int autotune_tma(Solver& S, int H, int Wsum) {
    static std::mutex mu;
    static std::map<std::array<int, 3>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const std::array<int, 3> key{dev, H, Wsum};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    cudaEvent_t e[4];
    for (auto& x : e) cudaEventCreate(&x);
    bool ok = true;
    for (int tma = 0; tma < 2; tma++) {
        S.sh.col_p2_tma = tma;
        for (int r = 0; r < 2; r++) ok &= L_col(S, 0) == cudaSuccess;
        cudaEventRecord(e[2 * tma], S.s);
        for (int r = 0; r < 3; r++) ok &= L_col(S, 0) == cudaSuccess;
        cudaEventRecord(e[2 * tma + 1], S.s);
    }
    float t_plain = 0.f, t_tma = 0.f;
    int res = 1;
    if (ok && cudaEventSynchronize(e[3]) == cudaSuccess && cudaEventElapsedTime(&t_plain, e[0], e[1]) == cudaSuccess &&
        cudaEventElapsedTime(&t_tma, e[2], e[3]) == cudaSuccess)
        res = t_tma < t_plain ? 1 : 0;
    cudaGetLastError();
    for (auto& x : e) cudaEventDestroy(x);
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = res;
    return res;
}

// Autotuner of the mixed-precision form: times the FFT column pass against the
// tensor-core one on the group's own buffers (DCT initial-solve mode, which has no
// PCG gate; two warm-up and three timed launches of each on the solve stream) and
// returns 1 when the tensor cores are faster.  The choice is cached per device and
// (H, max W) for the life of the process; it runs before any graph capture.
TuneResult autotune_col(Solver& S, int H, int W) {
    static std::mutex mu;
    static std::map<std::array<int, 3>, TuneResult> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const std::array<int, 3> key{dev, H, W};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    cudaEvent_t e[4];
    for (auto& x : e) cudaEventCreate(&x);
    bool ok = true;
    for (int tc = 0; tc < 2; tc++) {
        S.sh.col_tc = tc;
        for (int r = 0; r < 2; r++) ok &= L_col(S, 0) == cudaSuccess;
        cudaEventRecord(e[2 * tc], S.s);
        for (int r = 0; r < 3; r++) ok &= L_col(S, 0) == cudaSuccess;
        cudaEventRecord(e[2 * tc + 1], S.s);
    }
    S.sh.col_tc = 0;
    TuneResult res;
    float t_fft = 0.f, t_tc = 0.f;
    if (ok && cudaEventSynchronize(e[3]) == cudaSuccess && cudaEventElapsedTime(&t_fft, e[0], e[1]) == cudaSuccess &&
        cudaEventElapsedTime(&t_tc, e[2], e[3]) == cudaSuccess) {
        res.ms_fft = t_fft / 3.f;
        res.ms_tc = t_tc / 3.f;
        res.tc = t_tc < t_fft ? 1 : 0;
    }
    cudaGetLastError();
    for (auto& x : e) cudaEventDestroy(x);
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = res;
    return res;
}

// Per-grid descriptors, FFT plans, launch shapes, CTA prefix arrays and
// tables for grids cropped to bbox (r0, r1, c0, c1 per grid).
int prepare(Solver& S, const std::vector<int>& idx, const unw_grid* grids, const std::vector<int>& bbox,
            const unw_params* prm, char* base, const BatchLayout& B, cudaStream_t s, bool dense, int slot,
            int soff) {
    const int n = (int)idx.size();
    S.n = n;
    S.s = s;
    S.hg.resize(n);
    S.sc.max_iter = prm->max_iter;
    S.sc.cg_max_iter = prm->cg_max_iter;
    const bool fixed = (prm->flags & UNW_F_FIXED_ITERS) != 0;
    S.sc.tol = fixed ? 0.f : prm->tol;        // rel_change < 0 never holds
    S.sc.cg_tol = fixed ? 0.f : prm->cg_tol;  // ||r|| < 0 never holds
    S.sc.eps2 = (float)((double)prm->epsilon * (double)prm->epsilon);
    S.sc.conncomp_size = prm->conncomp_size;
    std::vector<HostPlan> prow(n), pcol(n);
    for (int gi = 0; gi < n; gi++) {
        const int g = idx[gi];
        const unw_grid& q = grids[g];
        const GridLayout& L = B.g[g];
        char* gb = base + B.base[g];
        GridDev& G = S.hg[gi];
        memset(&G, 0, sizeof(G));
        const int r0 = bbox[4 * g], r1 = bbox[4 * g + 1], c0 = bbox[4 * g + 2], c1 = bbox[4 * g + 3];
        G.H0 = (int)q.H;
        G.W0 = (int)q.W;
        G.H = r1 - r0;
        G.W = c1 - c0;
        G.r0 = r0;
        G.c0 = c0;
        G.P = dense ? G.W : (int)up((size_t)std::max(G.W, 1), 32);
        G.phase = q.phase + (long long)r0 * q.phase_pitch + c0;
        G.phase_pitch = q.phase_pitch;
        G.weight = q.weight ? q.weight + (long long)r0 * q.weight_pitch + c0 : nullptr;
        G.weight_pitch = q.weight_pitch;
        G.out_u = q.out_u;
        G.out_u_pitch = q.out_u_pitch;
        G.out_cc = q.out_cc;
        G.out_cc_pitch = q.out_cc_pitch;
        G.congruent = (prm->flags & UNW_F_CONGRUENT) ? 1 : 0;
        G.st = (InstState*)(gb + L.st);
        G.counter = (unsigned*)(gb + L.counter);
        G.part = (double*)(gb + L.part);
        float** arrs[20] = {&G.gx, &G.gy, &G.wx, &G.wy, &G.wIx, &G.wIy, &G.b, &G.r,
                            &G.z, &G.p0, &G.p1, &G.Ap, &G.T, &G.U0, &G.U1, &G.Ub,
                            &G.L0, &G.L1, &G.Lb, &G.D};
        for (int a = 0; a < 20; a++) *arrs[a] = (float*)(gb + L.arr[a]);
        G.valid = (uint8_t*)(gb + L.valid);
        G.sH = (const float*)(gb + L.cos_c);
        G.sW = (const float*)(gb + L.cos_r);
        G.hist = (int*)(gb + L.hist);
        G.hist_cap = HIST_CAP;
        G.tilecnt = (int*)(gb + L.tilecnt);
        G.parent = (int*)(gb + L.post_parent);
        G.lab = (int*)(gb + L.post_lab);
        G.csum = (double*)(gb + L.post_csum);
        G.adj = (double*)(gb + L.post_adj);
        G.ccount = (int*)(gb + L.post_ccount);
        G.remap = (int*)(gb + L.post_remap);
        G.lab_cap = (int)std::min<long long>(L.lab_cap, (long long)G.H * G.W / 2 + 2);
        G.ntiles = (int)(((long long)G.H * G.W + 4095) / 4096);
        if (G.H == 0) continue;
        prow[gi] = make_plan(G.W);
        pcol[gi] = make_plan(G.H);
        const HostPlan* pl[2] = {&prow[gi], &pcol[gi]};
        DctPlanDev* dp[2] = {&G.prow, &G.pcol};
        size_t tw[2] = {L.tw_r, L.tw_c}, hs[2] = {L.hs_r, L.hs_c}, dw[2] = {L.dw_r, L.dw_c},
               ch[2] = {L.ch_r, L.ch_c};
        int capn[2] = {L.fr_cap, L.fc_cap};
        for (int d = 0; d < 2; d++) {
            const HostPlan& hp = *pl[d];
            if (hp.n > MAX_GEN || hp.n > capn[d] || (int)hp.rad.size() > UNW_MAX_PASSES)
                return set_err(UNW_E_UNSUPPORTED, "grid %d: transform length %d (from %d) exceeds %d", g, hp.n,
                               hp.N, MAX_GEN);
            DctPlanDev& D = *dp[d];
            D.N = hp.N;
            D.blue = hp.blue;
            D.stride = hp.n;
            D.fft.n = hp.n;
            D.fft.npass = (int)hp.rad.size();
            for (size_t i = 0; i < hp.rad.size(); i++) D.fft.radix[i] = hp.rad[i];
            D.fft.tw = (const float2*)(gb + tw[d]);
            D.dctw = (const float2*)(gb + dw[d]);
            D.chirp = (const float2*)(gb + ch[d]);
            D.hspec = (const float2*)(gb + hs[d]);
        }
        // row kernel: one complex sequence (two rows) of fft_len(W)
        const int rT = pick_threads(prow[gi].n, prow[gi].cap);
        // column kernel: nseq column pairs of fft_len(H) under the shared-memory budget
        int nseq = col_nseq_generic(pcol[gi].n, G.W);
        int cT = 0;
        while (nseq >= 1 && !(cT = pick_threads((long long)nseq * pcol[gi].n, pcol[gi].cap))) nseq--;
        if (!rT || !cT) return set_err(UNW_E_UNSUPPORTED, "grid %d: no launch shape", g);
        G.col_nseq = nseq;
        S.sh.row_T = std::max(S.sh.row_T, rT);
        S.sh.col_T = std::max(S.sh.col_T, cT);
        S.sh.row_emax = std::max(S.sh.row_emax, prow[gi].emax);
        S.sh.col_emax = std::max(S.sh.col_emax, pcol[gi].emax);
        S.sh.row_smem = std::max(S.sh.row_smem, (size_t)prow[gi].n * sizeof(float2));
        S.sh.col_smem = std::max(S.sh.col_smem, (size_t)nseq * pcol[gi].n * sizeof(float2));
        G.sten_tiles_x = (G.W + 127) / 128;
        G.sten_rows = 1;
    }
    // power-of-two register-FFT paths when every grid shares the dimension
    {
        int w = -1, h = -1;
        bool wsame = true, hsame = true;
        for (int g = 0; g < n; g++) {
            const GridDev& G = S.hg[g];
            if (G.H == 0) continue;
            if (w < 0) w = G.W; else wsame &= (w == G.W);
            if (h < 0) h = G.H; else hsame &= (h == G.H);
        }
        if (w > 0 && wsame && unw_p2_col_nseq(w) > 0 && (w & (w - 1)) == 0) S.sh.row_p2 = w;
        if (h > 0 && hsame && unw_p2_col_nseq(h) > 0 && (h & (h - 1)) == 0) {
            S.sh.col_p2 = h;
            for (int g = 0; g < n; g++) S.hg[g].col_nseq = unw_p2_col_nseq(h);
        }
        // Bluestein register-FFT paths when every grid has the same M along the axis
        int mw = -1, mh = -1;
        bool mwsame = true, mhsame = true;
        for (int g = 0; g < n; g++) {
            const GridDev& G = S.hg[g];
            if (G.H == 0) continue;
            const int a = bl_len(G.W), b = bl_len(G.H);
            if (mw < 0) mw = a; else mwsame &= (mw == a);
            if (mh < 0) mh = b; else mhsame &= (mh == b);
        }
        if (!S.sh.row_p2 && mw > 0 && mwsame) S.sh.row_bl = mw;
        if (!S.sh.col_p2 && mh > 0 && mhsame) {
            S.sh.col_bl = mh;
            for (int g = 0; g < n; g++) S.hg[g].col_nseq = unw_bl_col_nseq(mh);
        }
        // persistent column pass: 148 x min(4, 2048 / threads) CTAs.  This is more than the
        // register limit lets reside at once (2 per SM at 512 threads), so a second wave starts
        // as first-wave CTAs finish; measured at 4096^2 that beats sizing the grid to the
        // resident count (102 us vs 113 us per launch), as the late CTAs fill the tail
        const int cthreads = S.sh.col_p2 ? S.sh.col_p2 / 16 * unw_p2_col_nseq(S.sh.col_p2)
                             : S.sh.col_bl ? S.sh.col_bl / 16 * unw_bl_col_nseq(S.sh.col_bl)
                                           : S.sh.col_T;
        const int per_sm = std::max(1, std::min(4, 2048 / std::max(cthreads, 1)));
        for (int g = 0; g < n; g++) S.hg[g].col_ctas = NUM_SMS * per_sm;
    }
    // tensor-core column pass (mixed precision): every grid of the group has the same
    // H <= UNW_TC_MAX_H (one pair of DCT matrices for the launch)
    int tc_h = 0;
    if (prm->flags & UNW_F_MIXED) {
        for (int g = 0; g < n; g++) {
            const int h = S.hg[g].H;
            if (h == 0) continue;
            if (tc_h == 0) tc_h = h;
            else if (tc_h != h) { tc_h = -1; break; }
        }
        if (tc_h < 16 || tc_h > UNW_TC_MAX_H || (prm->flags & UNW_F_COL_FFT)) tc_h = 0;
        for (int g = 0; g < n && tc_h > 0; g++)
            if (S.hg[g].H > 0 && (S.hg[g].P & 3)) tc_h = 0;  // the pass moves float4 groups of rows
    }
    // CTA prefix arrays
    S.starts.assign((size_t)(KS_NKIND + 1) * (n + 1), 0);
    S.total.assign(KS_NKIND + 1, 0);
    for (int k = 0; k <= KS_NKIND; k++) {
        int acc = 0;
        for (int g = 0; g < n; g++) {
            S.starts[(size_t)k * (n + 1) + g] = acc;
            if (k == KS_TC) acc += (tc_h > 0 && S.hg[g].H > 0) ? unw_tc_ctas(S.hg[g].H, S.hg[g].W) : 0;
            else acc += kind_ctas(S.hg[g], k);
        }
        S.starts[(size_t)k * (n + 1) + n] = acc;
        S.total[k] = acc;
    }
    S.dg = (GridDev*)(base + B.gdev) + slot;
    S.dstarts = (int*)(base + B.starts) + soff;
    CK(cudaMemcpyAsync(S.dg, S.hg.data(), sizeof(GridDev) * n, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(S.dstarts, S.starts.data(), sizeof(int) * S.starts.size(), cudaMemcpyHostToDevice, s));

    // tables
    for (int g = 0; g < n; g++) {
        GridDev& G = S.hg[g];
        if (G.H == 0) continue;
        CK(unw_launch_tables(G.prow.fft, G.prow, const_cast<float*>(G.sW), G.W, s));
        CK(unw_launch_tables(G.pcol.fft, G.pcol, const_cast<float*>(G.sH), G.H, s));
        if (G.prow.blue) CK(unw_launch_hspec(pick_threads(prow[g].n, prow[g].cap), prow[g].emax, G.prow, s));
        if (G.pcol.blue) CK(unw_launch_hspec(pick_threads(pcol[g].n, pcol[g].cap), pcol[g].emax, G.pcol, s));
        CK(cudaMemsetAsync(G.hist, 0, sizeof(int) * HIST_CAP, s));
    }
    if (tc_h > 0) {
        char* tab = base + B.base[idx[0]] + B.g[idx[0]].tc;
        cudaError_t te = B.g[idx[0]].tc ? unw_tc_prepare(tc_h, tab, &S.maps, s) : cudaErrorInvalidValue;
        if (te == cudaSuccess) {
            // per-grid tensor maps of T and p1 (the pass's float32 sources), 64-byte aligned
            unsigned char* h = S.host_maps(n);
            for (int g = 0; g < n && te == cudaSuccess; g++) {
                const GridDev& G = S.hg[g];
                if (G.H > 0 && !unw_tc_data_maps(G.T, G.p1, G.H, G.W, G.P, h + UNW_MAP_BYTES * (size_t)g))
                    te = cudaErrorNotSupported;
            }
            S.bmaps = base + B.tcmaps + UNW_MAP_BYTES * (size_t)slot;
            if (te == cudaSuccess) te = cudaMemcpyAsync(S.bmaps, h, UNW_MAP_BYTES * (size_t)n, cudaMemcpyHostToDevice, s);
        }
        if (te == cudaSuccess) {
            if (prm->flags & UNW_F_COL_TC) {
                S.sh.col_tc = 1;
            } else {
                int W0 = 0;
                for (int g = 0; g < n; g++) W0 = std::max(W0, S.hg[g].W);
                S.tune = autotune_col(S, tc_h, W0);
                S.sh.col_tc = S.tune.tc;
            }
        }
        cudaGetLastError();
    }
    // power-of-two column pass with the slab moved by TMA: per-grid tensor maps of T (even and
    // odd rows) in the grid's 256-byte map slot (the tensor-core pass, which uses the same slots,
    // covers H <= 1024 only)
    S.sh.col_p2_tma = 0;
    if (!S.sh.col_tc && S.sh.col_p2 && unw_p2_tma_nseq(S.sh.col_p2) > 0 && !(prm->flags & UNW_F_COL_NO_TMA)) {
        unsigned char* h = S.host_maps(n);
        bool ok = true;
        for (int g = 0; g < n && ok; g++) {
            const GridDev& G = S.hg[g];
            if (G.H > 0)
                ok = G.col_nseq == unw_p2_tma_nseq(S.sh.col_p2) &&
                     unw_p2_tma_maps(G.T, G.H, G.W, G.P, G.col_nseq,
                                     h + UNW_MAP_BYTES * (size_t)g + 128 * UNW_MAP_COL);
        }
        if (ok) {
            S.bmaps = base + B.tcmaps + UNW_MAP_BYTES * (size_t)slot;
            CK(cudaMemcpyAsync(S.bmaps, h, UNW_MAP_BYTES * (size_t)n, cudaMemcpyHostToDevice, s));
            S.sh.col_p2_tma = 1;
            if (!(prm->flags & UNW_F_COL_TMA)) {
                int Wsum = 0;
                for (int g = 0; g < n; g++) Wsum += S.hg[g].W;
                S.sh.col_p2_tma = autotune_tma(S, S.sh.col_p2, Wsum);
            }
        }
    }
    // matvec on TMA-staged halo tiles: per-grid maps of p, wIx and wIy in the grid's map slot
    S.sh.mv_tma = 0;
    if (!(prm->flags & UNW_F_MV_NO_TMA)) {
        unsigned char* h = S.host_maps(n);
        bool ok = true;
        for (int g = 0; g < n && ok; g++) {
            const GridDev& G = S.hg[g];
            if (G.H > 0)
                ok = unw_mv_tma_maps(G.p0, G.wIx, G.wIy, G.H, G.W, G.P,
                                     h + UNW_MAP_BYTES * (size_t)g + 128 * UNW_MAP_MV);
        }
        if (ok) {
            S.bmaps = base + B.tcmaps + UNW_MAP_BYTES * (size_t)slot;
            CK(cudaMemcpyAsync(S.bmaps, h, UNW_MAP_BYTES * (size_t)n, cudaMemcpyHostToDevice, s));
            S.sh.mv_tma = 1;
        }
    }
    bool any_grid = false;
    for (int g = 0; g < n; g++) any_grid |= S.hg[g].H > 0;
    if ((prm->flags & UNW_F_MIXED) && (prm->flags & UNW_F_COL_TC) && !S.sh.col_tc && any_grid) {
        return set_err(UNW_E_UNSUPPORTED, "tensor-core column pass requested but unavailable for this grid "
                                          "(all grids need the same H <= %d rows and a pitch of whole float4 groups)",
                       UNW_TC_MAX_H);
    }
    return UNW_OK;
}

// One launch group: every kernel covers the group's grids with shapes sized for
// them; each grid stops on its own convergence test.
int solve_group(const std::vector<int>& idx, const unw_grid* grids, const std::vector<int>& bbox,
                const unw_params* prm, char* base, const BatchLayout& B, unw_stats* stats, cudaStream_t s,
                int slot, int soff) {
    const int n = (int)idx.size();
    int rc;
    Solver S;
    S.prof.on = (prm->flags & UNW_F_PROFILE) != 0;
    rc = prepare(S, idx, grids, bbox, prm, base, B, s, false, slot, soff);
    if (rc) return rc;

    // 4. setup and DCT initial solve (utils_unwrap2d.py:1228-1513)
    const int tot_active = S.total[KS_ROWPAIR];
    PL(UNW_PROF_SETUP, unw_launch_simple(UNW_K_STATE_INIT, 1, s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));
    if (tot_active > 0) {
        PL(UNW_PROF_SETUP, unw_launch_simple(UNW_K_SETUP, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));
        PL(UNW_PROF_ROW_RHO, L_rowf(S, 0, 0, 0));
        PL(UNW_PROF_COL, L_col(S, 0));
        PL(UNW_PROF_ROW_INV, L_rowi(S, 0));
        PL(UNW_PROF_ELEM, unw_launch_simple(UNW_K_INIT_RECENTRE, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));

        // 5. IRLS loop (utils_unwrap2d.py:1533-1626)
        const int every = std::max(1, prm->check_every);
        std::vector<InstState> hs;
        IterGraphs graphs;
        const bool use_graph = !S.prof.on && !(prm->flags & UNW_F_NO_GRAPH) && prm->max_iter >= 2;
        if (use_graph) {
            rc = build_iteration_graphs(S, graphs);
            if (rc) return rc;
        }
        for (int t = 0; t < prm->max_iter; t++) {
            if (use_graph) {
                CK(cudaGraphLaunch(graphs.ex[t & 1], s));
            } else {
                rc = enqueue_iteration(S, t);
                if (rc) return rc;
            }
            if ((t + 1) % every == 0 || t + 1 == prm->max_iter) {
                rc = read_states(S, hs);
                if (rc) return rc;
                bool any = false;
                for (int g = 0; g < n; g++) any |= (S.hg[g].H > 0 && hs[g].irls_active);
                if (!any) break;
            }
        }

        // float64 residual of the final system (mixed-precision form), before the
        // post-processing scratch overlays the weights
        if (prm->flags & UNW_F_MIXED)
            PL(UNW_PROF_ELEM, unw_launch_simple(UNW_K_RESID, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));

        // 6. post-processing (utils_unwrap2d.py:1659-1757)
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_KSTATS, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_HIST, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_MEDIAN, n, s, S.dg, nullptr, n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_SHIFT_CCINIT, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_UNION, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_FLATTEN, S.total[KS_NKIND], s, S.dg, S.ds(KS_NKIND), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_TILESCAN, n, s, S.dg, nullptr, n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_LABEL, S.total[KS_NKIND], s, S.dg, S.ds(KS_NKIND), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_ACCUM, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_ADJUST, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
        // size-ranked relabel (utils_unwrap2d.py:1722-1746): sizes to the host, sorted there
        rc = read_states(S, hs);
        if (rc) return rc;
        for (int g = 0; g < n; g++) {
            const GridDev& G = S.hg[g];
            if (G.H == 0 || hs[g].n_nonfinite || !hs[g].hist_ok) continue;
            const int nl = hs[g].n_labels;
            std::vector<int> cnt(nl + 1);
            CK(cudaMemcpyAsync(cnt.data(), G.ccount, sizeof(int) * (nl + 1), cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            std::vector<int> order(nl);
            std::iota(order.begin(), order.end(), 1);
            std::sort(order.begin(), order.end(), [&](int a, int b) {
                return cnt[a] != cnt[b] ? cnt[a] > cnt[b] : a > b;  // size desc; ties larger label first
            });
            std::vector<int> remap(nl + 1, 0);
            int nw = 1;
            for (int L : order)
                if (cnt[L] >= prm->conncomp_size) remap[L] = nw++;
            if (nw - 1 > 65535)
                return set_err(UNW_E_OVERFLOW, "grid %d: %d components do not fit uint16 labels", idx[g], nw - 1);
            CK(cudaMemcpyAsync(G.remap, remap.data(), sizeof(int) * (nl + 1), cudaMemcpyHostToDevice, s));
            if (stats) stats[idx[g]].n_components = nw - 1;
        }
        PL(UNW_PROF_POST, unw_launch_post(UNW_P_WRITE, S.total[KS_ELEM], s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
    }
    PL(UNW_PROF_POST, unw_launch_post(UNW_P_FILL, 0, s, S.dg, nullptr, n, S.sc, S.hg.data()));
    std::vector<InstState> fin;
    rc = read_states(S, fin);
    if (rc) return rc;
    int ret = UNW_OK;
    for (int g = 0; g < n; g++) {
        const GridDev& G = S.hg[g];
        const InstState& st = fin[g];
        int status = 0;
        if (G.H == 0) status |= UNW_S_ALL_NAN;
        else {
            status = st.status;
            if (status & UNW_S_TC_TIMEOUT)
                return set_err(UNW_E_CUDA, "grid %d: a TMA-staged column pass gave up waiting on its copies",
                               idx[g]);
            if (st.n_nonfinite) { status |= UNW_S_NONFINITE_OUT; ret = UNW_W_NUMERIC; }
            else if (!st.hist_ok) return set_err(UNW_E_UNSUPPORTED, "grid %d: post-processing limits exceeded", idx[g]);
        }
        if (stats) {
            // stats were zeroed by solve_batch; n_components was set by the relabel
            // step, the profile sums (grid 0) accumulate over groups
            unw_stats& o = stats[idx[g]];
            if (!(G.H > 0 && !st.n_nonfinite)) o.n_components = 0;
            o.irls_iters = G.H ? st.irls_iter : 0;
            o.cg_iters_total = G.H ? st.cg_total : 0;
            o.cg_iters_last = (G.H && st.irls_iter > 0 && st.irls_iter <= UNW_MAX_LOG) ? st.cg_log[st.irls_iter - 1] : 0;
            o.n_labels = G.H ? st.n_labels : 0;
            o.status = status;
            const int og = idx[g];
            o.bbox[0] = bbox[4 * og]; o.bbox[1] = bbox[4 * og + 1]; o.bbox[2] = bbox[4 * og + 2]; o.bbox[3] = bbox[4 * og + 3];
            o.rel_change = st.rel_change;
            o.best_residual = st.best_residual;
            o.k_median = st.kmed;
            for (int i = 0; i < 64 && i < UNW_MAX_LOG; i++) o.cg_iters[i] = G.H ? st.cg_log[i] : 0;
            o.col_path = S.sh.col_tc;
            o.col_tma = S.sh.col_p2_tma;
            o.tune_ms[0] = S.tune.ms_fft;
            o.tune_ms[1] = S.tune.ms_tc;
            o.resid_rel = st.resid_rel;
        }
    }
    if (stats && S.prof.on) S.prof.collect(stats[0].prof_ms, stats[0].prof_launches);
    return ret;
}

// ------------------------------------------------------------ batch solve
int solve_batch(int n, const unw_grid* grids, const unw_params* prm, void* ws, size_t ws_bytes,
                unw_stats* stats, cudaStream_t s) {
    if (n <= 0 || !grids) return set_err(UNW_E_ARG, "empty batch");
    int rc = validate_params(prm);
    if (rc) return rc;
    std::vector<long long> H0(n), W0(n);
    for (int g = 0; g < n; g++) {
        const unw_grid& q = grids[g];
        if (!q.phase || !q.out_u || !q.out_cc) return set_err(UNW_E_ARG, "grid %d: null pointer", g);
        if (q.H <= 0 || q.W <= 0) return set_err(UNW_E_ARG, "grid %d: bad shape %lld x %lld", g, q.H, q.W);
        if (q.H * q.W >= (1LL << 31)) return set_err(UNW_E_UNSUPPORTED, "grid %d: too many pixels", g);
        if (q.phase_pitch < q.W || q.out_u_pitch < q.W || q.out_cc_pitch < q.W ||
            (q.weight && q.weight_pitch < q.W))
            return set_err(UNW_E_ARG, "grid %d: pitch smaller than width", g);
        H0[g] = q.H;
        W0[g] = q.W;
    }
    BatchLayout B = batch_layout(n, H0.data(), W0.data());
    if (!ws) return set_err(UNW_E_ARG, "workspace is NULL");
    char* base = (char*)up((size_t)ws, ALIGN);
    if ((size_t)(base - (char*)ws) + B.total - ALIGN > ws_bytes)
        return set_err(UNW_E_WORKSPACE, "workspace %zu bytes < %zu needed", ws_bytes, B.total);

    // 1. bounding boxes
    int* rowany = (int*)(base + B.rowany);
    int* colany = (int*)(base + B.colany);
    int* dbbox = (int*)(base + B.bbox);
    {
        long long ro = 0, co = 0;
        for (int g = 0; g < n; g++) {
            CK(unw_launch_bbox(grids[g].phase, grids[g].phase_pitch, (int)H0[g], (int)W0[g], rowany + ro,
                               colany + co, dbbox + 4 * g, s));
            ro += H0[g];
            co += W0[g];
        }
    }
    std::vector<int> bbox(4 * n);
    CK(cudaMemcpyAsync(bbox.data(), dbbox, sizeof(int) * 4 * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));

    // 2. launch groups (kernel configuration per axis).  Several groups run at the same
    // time, each from its own host thread on its own non-blocking stream, so the GPU
    // overlaps their kernels and one group's convergence reads do not stall the others;
    // every input is ready (the bounding-box read above synchronised the caller's
    // stream) and every output is complete when the call returns (each group ends
    // with a synchronising state read).  Under UNW_F_PROFILE the groups run one after
    // another on the caller's stream, so that the per-launch timings stay serial.
    std::map<std::array<int, 4>, std::vector<int>> groups;
    for (int g = 0; g < n; g++)
        groups[group_key(bbox[4 * g + 1] - bbox[4 * g], bbox[4 * g + 3] - bbox[4 * g + 2])].push_back(g);
    if (stats)
        for (int g = 0; g < n; g++) memset(&stats[g], 0, sizeof(unw_stats));
    struct Job {
        const std::vector<int>* idx;
        int slot, soff, rc = UNW_OK;
        std::string err;
    };
    std::vector<Job> jobs;
    {
        int slot = 0, soff = 0;
        for (auto& kv : groups) {
            Job j;
            j.idx = &kv.second;
            j.slot = slot;
            j.soff = soff;
            jobs.push_back(j);
            slot += (int)kv.second.size();
            soff += (KS_NKIND + 1) * ((int)kv.second.size() + 1);
        }
    }
    const bool concurrent = jobs.size() > 1 && !(prm->flags & UNW_F_PROFILE);
    if (!concurrent) {
        for (Job& j : jobs) {
            j.rc = solve_group(*j.idx, grids, bbox, prm, base, B, stats, s, j.slot, j.soff);
            if (j.rc < 0) return j.rc;
        }
    } else {
        int dev = 0;
        CK(cudaGetDevice(&dev));
        std::vector<std::thread> th;
        for (Job& j : jobs) {
            th.emplace_back([&, dev, jp = &j] {
                cudaStream_t gs = nullptr;
                if (cudaSetDevice(dev) != cudaSuccess ||
                    cudaStreamCreateWithFlags(&gs, cudaStreamNonBlocking) != cudaSuccess) {
                    jp->rc = set_err(UNW_E_CUDA, "no stream for a launch group");
                } else {
                    g_worker_stream = gs;
                    jp->rc = solve_group(*jp->idx, grids, bbox, prm, base, B, stats, gs, jp->slot, jp->soff);
                    cudaStreamSynchronize(gs);
                    cudaStreamDestroy(gs);
                }
                if (jp->rc < 0) jp->err = g_err;
            });
        }
        for (auto& t : th) t.join();
        for (Job& j : jobs)
            if (j.rc < 0) return set_err(j.rc, "%s", j.err.c_str());
    }
    int ret = UNW_OK;
    for (Job& j : jobs)
        if (j.rc == UNW_W_NUMERIC) ret = j.rc;
    return ret;
}

// ------------------------------------------------------------ adjoint
// Workspace of the adjoint: the solver layout of the batch plus a separate
// post-processing region per grid, since the component labels and sums must live
// next to the frozen weights (which the forward solve lets them overlay).
struct AdjLayout {
    BatchLayout B;
    std::vector<size_t> parent, lab, csum, adj, ccount, remap;
    size_t total;
};

AdjLayout adjoint_layout(int n, const long long* H, const long long* W) {
    AdjLayout A;
    A.B = batch_layout(n, H, W);
    size_t o = up(A.B.total - ALIGN, ALIGN);
    auto take = [&](size_t bytes) { size_t r = o; o = up(o + bytes, ALIGN); return r; };
    for (int g = 0; g < n; g++) {
        const long long cap = A.B.g[g].lab_cap;
        A.parent.push_back(take(sizeof(int) * (size_t)(H[g] * W[g])));
        A.lab.push_back(take(sizeof(int) * (size_t)(H[g] * W[g])));
        A.csum.push_back(take(sizeof(double) * 4 * (size_t)cap));
        A.adj.push_back(take(sizeof(double) * (size_t)cap));
        A.ccount.push_back(take(sizeof(int) * (size_t)cap));
        A.remap.push_back(take(sizeof(int) * (size_t)cap));
    }
    A.total = o + ALIGN;
    return A;
}

// One launch group of the adjoint: every kernel covers the group's grids; each grid's
// PCG solves stop on their own tolerance.
int adjoint_group(const std::vector<int>& idx, const unw_adj_grid* grids, const std::vector<unw_grid>& q,
                  const std::vector<int>& bbox, const unw_params* prm, char* base, const AdjLayout& A,
                  unw_stats* stats, cudaStream_t s, int slot, int soff) {
    unw_params pa = *prm;
    pa.max_iter = 1;
    pa.flags = 0;
    Solver S;
    int rc = prepare(S, idx, q.data(), bbox, &pa, base, A.B, s, false, slot, soff);
    if (rc) return rc;
    S.sc.cg_tol = 0.f;            // replaced by cg_rel * ||r0|| at each PCG start
    S.sc.cg_rel = prm->cg_tol;
    const int n = (int)idx.size();
    for (int g = 0; g < n; g++) {
        GridDev& G = S.hg[g];
        const int j = idx[g];
        G.parent = (int*)(base + A.parent[j]);
        G.lab = (int*)(base + A.lab[j]);
        G.csum = (double*)(base + A.csum[j]);
        G.adj = (double*)(base + A.adj[j]);
        G.ccount = (int*)(base + A.ccount[j]);
        G.remap = (int*)(base + A.remap[j]);
        G.a_u = grids[j].u;
        G.a_u_pitch = grids[j].u_pitch;
        G.a_gu = grids[j].grad_u;
        G.a_gu_pitch = grids[j].grad_u_pitch;
        G.a_gph = grids[j].grad_phase;
        G.a_gph_pitch = grids[j].grad_phase_pitch;
        G.a_gw = grids[j].grad_weight;
        G.a_gw_pitch = grids[j].grad_weight_pitch;
    }
    CK(cudaMemcpyAsync(S.dg, S.hg.data(), sizeof(GridDev) * (size_t)n, cudaMemcpyHostToDevice, s));
    const int ne = S.total[KS_ELEM];
    CK(unw_launch_simple(UNW_K_STATE_INIT, 1, s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));
    CK(unw_launch_simple(UNW_K_SETUP, ne, s, S.dg, S.ds(KS_ELEM), n, 0, S.sc));
    CK(unw_launch_adj(UNW_A_LOAD, ne, s, S.dg, S.ds(KS_ELEM), n));
    // 1. the frozen-weight system at u (IRLS weights and right-hand side from u), solved to
    //    the relative tolerance from u: u* in U1
    rc = enqueue_iteration(S, 0, UNW_ADJ_CHUNK);
    if (rc) return rc;
    // 2. iterative refinement of u* on the frozen system: residual in float64 (phase
    //    differences in float64), correction by the PCG from x0 = 0, added to the pair; the
    //    last REFINE only measures the residual of the final u*.  Before the post pipeline,
    //    which sets u* to NaN outside the valid pixels (its shift is 0 here: no median ran)
    for (int k = 0; k <= UNW_ADJ_REFINE; k++) {
        CK(unw_launch_adj(UNW_A_REARM, 1, s, S.dg, nullptr, n));
        CK(unw_launch_adj(UNW_A_REFINE, ne, s, S.dg, S.ds(KS_ELEM), n, 0));
        if (k == UNW_ADJ_REFINE) break;
        CK(unw_launch_adj(UNW_A_REFINE, ne, s, S.dg, S.ds(KS_ELEM), n, 1));
        CK(L_rowf(S, 1, 1, 0));
        CK(L_col(S, 1));
        CK(L_rowi(S, 1));
        rc = pcg_chunked(S, 1, UNW_ADJ_CHUNK);
        if (rc) return rc;
        CK(unw_launch_adj(UNW_A_ADDD, ne, s, S.dg, S.ds(KS_ELEM), n, k));
    }
    // 3. components of the valid mask
    const int nt = S.total[KS_NKIND];
    CK(unw_launch_post(UNW_P_SHIFT_CCINIT, ne, s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
    CK(unw_launch_post(UNW_P_UNION, ne, s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
    CK(unw_launch_post(UNW_P_FLATTEN, nt, s, S.dg, S.ds(KS_NKIND), n, S.sc, S.hg.data()));
    CK(unw_launch_post(UNW_P_TILESCAN, n, s, S.dg, nullptr, n, S.sc, S.hg.data()));
    CK(unw_launch_post(UNW_P_LABEL, nt, s, S.dg, S.ds(KS_NKIND), n, S.sc, S.hg.data()));
    CK(unw_launch_post(UNW_P_ACCUM, ne, s, S.dg, S.ds(KS_ELEM), n, S.sc, S.hg.data()));
    // 4. adjoint right-hand side through the alignment, then lambda = A^+ G' (x0 = 0 in U0/L0,
    //    lambda accumulated in D)
    for (int g = 0; g < n; g++) {
        CK(cudaMemsetAsync(S.hg[g].adj, 0, sizeof(double) * (size_t)S.hg[g].lab_cap, s));
        CK(cudaMemsetAsync(S.hg[g].csum, 0, sizeof(double) * 4 * (size_t)S.hg[g].lab_cap, s));
    }
    CK(unw_launch_adj(UNW_A_LSUM, ne, s, S.dg, S.ds(KS_ELEM), n));
    CK(unw_launch_adj(UNW_A_RHS, ne, s, S.dg, S.ds(KS_ELEM), n));
    CK(unw_launch_adj(UNW_A_REARM, 1, s, S.dg, nullptr, n));
    CK(L_rowf(S, 1, 1, 0));
    CK(L_col(S, 1));
    CK(L_rowi(S, 1));
    rc = pcg_chunked(S, 1, UNW_ADJ_CHUNK);
    if (rc) return rc;
    // 5. gradients
    CK(unw_launch_adj(UNW_A_GRAD, ne, s, S.dg, S.ds(KS_ELEM), n));
    std::vector<InstState> hs;
    rc = read_states(S, hs);
    if (rc) return rc;
    int ret = UNW_OK;
    for (int g = 0; g < n; g++) {
        const InstState& st = hs[g];
        if (st.status & UNW_S_TC_TIMEOUT)
            return set_err(UNW_E_CUDA, "grid %d: a TMA-staged column pass gave up waiting on its copies", idx[g]);
        if (stats) {
            unw_stats& o = stats[idx[g]];
            o.irls_iters = 1;
            o.cg_iters[0] = st.cg_log[0];
            o.cg_iters[1] = st.cg_iter;
            o.cg_iters_last = st.cg_iter;
            o.cg_iters_total = st.cg_log[0] + st.cg_iter;
            for (int k = 0; k < UNW_ADJ_REFINE; k++) {
                o.cg_iters[2 + k] = st.cg_log[2 + k];
                o.cg_iters_total += st.cg_log[2 + k];
            }
            o.resid_rel = st.resid_rel;
            o.n_labels = st.n_labels;
            o.status = st.status;
            // relative residual of the adjoint solve (cg_tol = cg_rel * ||r0||)
            o.rel_change = st.cg_tol > 0.f ? st.rnorm * (double)prm->cg_tol / (double)st.cg_tol : 0.0;
            for (int k = 0; k < 4; k++) o.bbox[k] = bbox[4 * idx[g] + k];
        }
        if (!st.irls_active) ret = UNW_W_NUMERIC;  // non-finite refinement: this grid's gradients are zero
    }
    return ret;
}

int adjoint_batch(int n, const unw_adj_grid* grids, const unw_params* prm, void* ws, size_t ws_bytes,
                  unw_stats* stats, cudaStream_t s) {
    if (n <= 0 || !grids) return set_err(UNW_E_ARG, "empty batch");
    int rc = validate_params(prm);
    if (rc) return rc;
    if (prm->cg_max_iter < 1 || !(prm->cg_tol > 0.f))
        return set_err(UNW_E_ARG, "adjoint needs cg_max_iter >= 1 and a relative cg_tol > 0");
    std::vector<long long> H0(n), W0(n);
    std::vector<unw_grid> q(n);
    for (int g = 0; g < n; g++) {
        const unw_adj_grid& a = grids[g];
        if (!a.phase || !a.u || !a.grad_u || !a.grad_phase) return set_err(UNW_E_ARG, "grid %d: null pointer", g);
        if (a.H <= 0 || a.W <= 0) return set_err(UNW_E_ARG, "grid %d: bad shape %lld x %lld", g, a.H, a.W);
        if (a.H * a.W >= (1LL << 31)) return set_err(UNW_E_UNSUPPORTED, "grid %d: too many pixels", g);
        if (a.phase_pitch < a.W || a.u_pitch < a.W || a.grad_u_pitch < a.W || a.grad_phase_pitch < a.W ||
            (a.weight && a.weight_pitch < a.W) || (a.grad_weight && a.grad_weight_pitch < a.W))
            return set_err(UNW_E_ARG, "grid %d: pitch smaller than width", g);
        if (a.grad_weight && !a.weight) return set_err(UNW_E_ARG, "grid %d: grad_weight needs weight", g);
        H0[g] = a.H;
        W0[g] = a.W;
        unw_grid& x = q[g];
        memset(&x, 0, sizeof(x));
        x.phase = a.phase;
        x.phase_pitch = a.phase_pitch;
        x.weight = a.weight;
        x.weight_pitch = a.weight_pitch;
        x.H = a.H;
        x.W = a.W;
    }
    if (!ws) return set_err(UNW_E_ARG, "workspace is NULL");
    const AdjLayout A = adjoint_layout(n, H0.data(), W0.data());
    char* base = (char*)up((size_t)ws, ALIGN);
    if ((size_t)(base - (char*)ws) + A.total - ALIGN > ws_bytes)
        return set_err(UNW_E_WORKSPACE, "workspace %zu bytes < %zu needed", ws_bytes, A.total);
    if (stats)
        for (int g = 0; g < n; g++) memset(&stats[g], 0, sizeof(unw_stats));
    for (int g = 0; g < n; g++) {
        const unw_adj_grid& a = grids[g];
        CK(cudaMemset2DAsync(a.grad_phase, sizeof(float) * a.grad_phase_pitch, 0, sizeof(float) * a.W, a.H, s));
        if (a.grad_weight)
            CK(cudaMemset2DAsync(a.grad_weight, sizeof(float) * a.grad_weight_pitch, 0, sizeof(float) * a.W, a.H, s));
    }
    // bounding boxes of the valid pixels, as in the forward solve
    const BatchLayout& B = A.B;
    int* rowany = (int*)(base + B.rowany);
    int* colany = (int*)(base + B.colany);
    int* dbbox = (int*)(base + B.bbox);
    {
        long long ro = 0, co = 0;
        for (int g = 0; g < n; g++) {
            CK(unw_launch_bbox(grids[g].phase, grids[g].phase_pitch, (int)H0[g], (int)W0[g], rowany + ro,
                               colany + co, dbbox + 4 * g, s));
            ro += H0[g];
            co += W0[g];
        }
    }
    std::vector<int> bbox(4 * n);
    CK(cudaMemcpyAsync(bbox.data(), dbbox, sizeof(int) * 4 * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // launch groups of the non-empty grids (an all-NaN grid has zero gradients), one after another
    std::map<std::array<int, 4>, std::vector<int>> groups;
    for (int g = 0; g < n; g++) {
        const int h = bbox[4 * g + 1] - bbox[4 * g], w = bbox[4 * g + 3] - bbox[4 * g + 2];
        if (h > 0 && w > 0) groups[group_key(h, w)].push_back(g);
    }
    int ret = UNW_OK, slot = 0, soff = 0;
    for (auto& kv : groups) {
        rc = adjoint_group(kv.second, grids, q, bbox, prm, base, A, stats, s, slot, soff);
        if (rc < 0) return rc;
        if (rc == UNW_W_NUMERIC) ret = rc;
        slot += (int)kv.second.size();
        soff += (KS_NKIND + 1) * ((int)kv.second.size() + 1);
    }
    return ret;
}

// Full-grid, dense-pitch descriptor over caller arrays for the operator entry points.
int op_prepare(Solver& S, int64_t H, int64_t W, void* ws, size_t wsb, cudaStream_t s, const float* phase,
               const float* weight) {
    if (H <= 0 || W <= 0) return set_err(UNW_E_ARG, "bad shape %lld x %lld", (long long)H, (long long)W);
    if (!ws) return set_err(UNW_E_ARG, "workspace is NULL");
    long long h = H, w = W;
    BatchLayout B = batch_layout(1, &h, &w);
    char* base = (char*)up((size_t)ws, ALIGN);
    if ((size_t)(base - (char*)ws) + B.total - ALIGN > wsb)
        return set_err(UNW_E_WORKSPACE, "workspace %zu bytes < %zu needed", wsb, B.total);
    unw_grid q{};
    q.phase = phase;
    q.phase_pitch = W;
    q.weight = weight;
    q.weight_pitch = W;
    q.H = H;
    q.W = W;
    unw_params prm{};
    prm.epsilon = 1e-2f;
    std::vector<int> bbox = {0, (int)H, 0, (int)W};
    return prepare(S, std::vector<int>{0}, &q, bbox, &prm, base, B, s, true, 0, 0);
}

int op_upload(Solver& S) {
    CK(cudaMemcpyAsync(S.dg, S.hg.data(), sizeof(GridDev), cudaMemcpyHostToDevice, S.s));
    return UNW_OK;
}

}  // namespace

// error text setter shared with the other host translation units
int unw_set_error(int code, const char* msg) { return set_err(code, "%s", msg); }

// ================================================================== C ABI
extern "C" {

int unw_abi_version(void) { return UNW_ABI_VERSION; }

const char* unw_last_error(void) { return g_err; }

size_t unw_batch_workspace_bytes(int32_t n, const int64_t* H, const int64_t* W) {
    if (n <= 0 || !H || !W) return 0;
    std::vector<long long> h(n), w(n);
    for (int g = 0; g < n; g++) {
        if (H[g] <= 0 || W[g] <= 0) return 0;
        h[g] = H[g];
        w[g] = W[g];
    }
    return batch_layout(n, h.data(), w.data()).total;
}

size_t unw_workspace_bytes(int64_t H, int64_t W) { return unw_batch_workspace_bytes(1, &H, &W); }

int unw_solve_f32(const float* phase, int64_t phase_pitch, const float* weight, int64_t weight_pitch,
                  int64_t H, int64_t W, const unw_params* params, float* out_u, int64_t out_u_pitch,
                  uint16_t* out_cc, int64_t out_cc_pitch, void* workspace, size_t workspace_bytes,
                  unw_stats* stats, void* cuda_stream) {
    unw_grid g;
    g.phase = phase;
    g.phase_pitch = phase_pitch;
    g.weight = weight;
    g.weight_pitch = weight_pitch;
    g.H = H;
    g.W = W;
    g.out_u = out_u;
    g.out_u_pitch = out_u_pitch;
    g.out_cc = out_cc;
    g.out_cc_pitch = out_cc_pitch;
    return solve_batch(1, &g, params, workspace, workspace_bytes, stats, (cudaStream_t)cuda_stream);
}

int unw_solve_batch(int32_t n, const unw_grid* grids, const unw_params* params, void* workspace,
                    size_t workspace_bytes, unw_stats* stats, void* cuda_stream) {
    return solve_batch(n, grids, params, workspace, workspace_bytes, stats, (cudaStream_t)cuda_stream);
}

size_t unw_adjoint_batch_workspace_bytes(int32_t n, const int64_t* H, const int64_t* W) {
    if (n <= 0 || !H || !W) return 0;
    std::vector<long long> h(n), w(n);
    for (int g = 0; g < n; g++) {
        if (H[g] <= 0 || W[g] <= 0) return 0;
        h[g] = H[g];
        w[g] = W[g];
    }
    return adjoint_layout(n, h.data(), w.data()).total;
}

size_t unw_adjoint_workspace_bytes(int64_t H, int64_t W) { return unw_adjoint_batch_workspace_bytes(1, &H, &W); }

int unw_adjoint_batch(int32_t n, const unw_adj_grid* grids, const unw_params* params, void* workspace,
                      size_t workspace_bytes, unw_stats* stats, void* cuda_stream) {
    return adjoint_batch(n, grids, params, workspace, workspace_bytes, stats, (cudaStream_t)cuda_stream);
}

int unw_adjoint_f32(const float* phase, int64_t phase_pitch, const float* weight, int64_t weight_pitch, int64_t H,
                    int64_t W, const unw_params* params, const float* u, int64_t u_pitch, const float* grad_u,
                    int64_t grad_u_pitch, float* grad_phase, int64_t grad_phase_pitch, float* grad_weight,
                    int64_t grad_weight_pitch, void* workspace, size_t workspace_bytes, unw_stats* stats,
                    void* cuda_stream) {
    unw_adj_grid g;
    g.phase = phase;
    g.phase_pitch = phase_pitch;
    g.weight = weight;
    g.weight_pitch = weight_pitch;
    g.H = H;
    g.W = W;
    g.u = u;
    g.u_pitch = u_pitch;
    g.grad_u = grad_u;
    g.grad_u_pitch = grad_u_pitch;
    g.grad_phase = grad_phase;
    g.grad_phase_pitch = grad_phase_pitch;
    g.grad_weight = grad_weight;
    g.grad_weight_pitch = grad_weight_pitch;
    return adjoint_batch(1, &g, params, workspace, workspace_bytes, stats, (cudaStream_t)cuda_stream);
}

int unw_setup_gradients(const float* phase, const float* weight, int64_t H, int64_t W, float* gx, float* gy,
                        float* wx, float* wy, uint8_t* valid, void* workspace, size_t workspace_bytes,
                        void* cuda_stream) {
    if (!phase || !gx || !gy || !wx || !wy || !valid) return set_err(UNW_E_ARG, "null pointer");
    Solver S;
    int rc = op_prepare(S, H, W, workspace, workspace_bytes, (cudaStream_t)cuda_stream, phase, weight);
    if (rc) return rc;
    GridDev& G = S.hg[0];
    G.gx = gx; G.gy = gy; G.wx = wx; G.wy = wy; G.valid = valid;
    rc = op_upload(S);
    if (rc) return rc;
    CK(unw_launch_simple(UNW_K_STATE_INIT, 1, S.s, S.dg, S.ds(KS_ELEM), 1, 0, S.sc));
    CK(unw_launch_simple(UNW_K_SETUP, S.total[KS_ELEM], S.s, S.dg, S.ds(KS_ELEM), 1, 0, S.sc));
    return UNW_OK;
}

int unw_apply_laplacian(const float* x, const float* wx, const float* wy, int64_t H, int64_t W, float* Ax,
                        void* workspace, size_t workspace_bytes, void* cuda_stream) {
    if (!x || !wx || !wy || !Ax) return set_err(UNW_E_ARG, "null pointer");
    Solver S;
    int rc = op_prepare(S, H, W, workspace, workspace_bytes, (cudaStream_t)cuda_stream, nullptr, nullptr);
    if (rc) return rc;
    GridDev& G = S.hg[0];
    G.r = const_cast<float*>(x); G.wIx = const_cast<float*>(wx); G.wIy = const_cast<float*>(wy); G.Ap = Ax;
    rc = op_upload(S);
    if (rc) return rc;
    CK(unw_launch_simple(UNW_K_LAP_APPLY, S.total[KS_ELEM], S.s, S.dg, S.ds(KS_ELEM), 1, 0, S.sc));
    return UNW_OK;
}

int unw_apply_preconditioner(const float* r, int64_t H, int64_t W, float* z, void* workspace,
                             size_t workspace_bytes, void* cuda_stream) {
    if (!r || !z) return set_err(UNW_E_ARG, "null pointer");
    Solver S;
    int rc = op_prepare(S, H, W, workspace, workspace_bytes, (cudaStream_t)cuda_stream, nullptr, nullptr);
    if (rc) return rc;
    GridDev& G = S.hg[0];
    G.r = const_cast<float*>(r); G.z = z;
    rc = op_upload(S);
    if (rc) return rc;
    CK(L_rowf(S, 3, 0, 0));
    CK(L_col(S, 0));
    CK(L_rowi(S, 3));
    return UNW_OK;
}

int unw_apply_preconditioner_mixed(const float* r, int64_t H, int64_t W, float* z, int32_t col_path,
                                   void* workspace, size_t workspace_bytes, void* cuda_stream) {
    if (!r || !z) return set_err(UNW_E_ARG, "null pointer");
    if (col_path < -1 || col_path > 1) return set_err(UNW_E_ARG, "col_path must be -1, 0 or 1");
    if (H <= 0 || W <= 0) return set_err(UNW_E_ARG, "bad shape %lld x %lld", (long long)H, (long long)W);
    if (!workspace) return set_err(UNW_E_ARG, "workspace is NULL");
    long long h = H, w = W;
    BatchLayout B = batch_layout(1, &h, &w);
    char* base = (char*)up((size_t)workspace, ALIGN);
    if ((size_t)(base - (char*)workspace) + B.total - ALIGN > workspace_bytes)
        return set_err(UNW_E_WORKSPACE, "workspace %zu bytes < %zu needed", workspace_bytes, B.total);
    unw_grid q{};
    q.phase_pitch = W;
    q.weight_pitch = W;
    q.H = H;
    q.W = W;
    unw_params prm{};
    prm.epsilon = 1e-2f;
    prm.flags = UNW_F_MIXED | (col_path == 1 ? UNW_F_COL_TC : 0) | (col_path == 0 ? UNW_F_COL_FFT : 0);
    std::vector<int> bbox = {0, (int)H, 0, (int)W};
    Solver S;
    int rc = prepare(S, std::vector<int>{0}, &q, bbox, &prm, base, B, (cudaStream_t)cuda_stream, true, 0, 0);
    if (rc) return rc;
    GridDev& G = S.hg[0];
    G.r = const_cast<float*>(r); G.z = z;
    rc = op_upload(S);
    if (rc) return rc;
    CK(L_rowf(S, 3, 0, 0));
    CK(L_col(S, 0));
    CK(L_rowi(S, 3));
    return S.sh.col_tc ? 1 : 0;
}

}  // extern "C"
