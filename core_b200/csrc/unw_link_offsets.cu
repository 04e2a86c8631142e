// Integer 2-pi offsets per component for component linking: the program
// connect_components_ilp_fast gives to CP-SAT (insardev/insardev/
// utils_unwrap2d.py:933-970),
//     minimise  sum_e w_e |s (k_i - k_j) - o_e|,  k_0 = 0,  k in [-100, 100],
//               |s (k_i - k_j) - o_e| <= 200,
// with, among the optimal assignments, the least sum_i |k_i|.  Host code only.
//
// Both criteria go into one integer objective F = B * primary + sum |k| with
// B = 100 n + 1 (so the second never outweighs one unit of the first).  F is
// L-natural convex (sums of convex functions of k_i - k_j and of k_i), so it is
// minimised by steepest descent over unit moves k +/- chi_S (Murota, Discrete
// Convex Analysis, 2003, section 10.3): a point from which no such move lowers
// F is a global minimum.  The best move for each sign is a minimum cut: unit
// moves change each pair term by a submodular table (the term is convex in the
// difference), which is graph-representable (Kolmogorov & Zabih, 2004).  Cuts
// are found with Dinic's max-flow, in int64 when every finite capacity fits and
// in 128-bit integers otherwise (B * w * |d| exceeds int64 for large
// instances); the moved set is the smallest
// minimiser (the nodes that still reach the sink in the residual graph), so the
// result is deterministic.
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <queue>
#include <thread>
#include <vector>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

namespace {

using Wide = __int128;

// Dinic's max-flow on a graph built once per move: arcs in one array, the
// arcs of a node contiguous (counted, then filled), an array queue.
template <class Cap>
struct Flow {
    struct Arc { int to; int rev; Cap cap; };
    int n = 0;
    std::vector<int> start, level, it, queue, path;
    std::vector<Arc> arcs;
    std::vector<int> eu, ev;
    std::vector<Cap> ec;
    void reset(int nodes) { n = nodes; eu.clear(); ev.clear(); ec.clear(); }
    void add(int u, int v, Cap c) {
        if (c <= 0) return;
        eu.push_back(u); ev.push_back(v); ec.push_back(c);
    }
    void build() {
        start.assign(n + 1, 0);
        for (size_t e = 0; e < eu.size(); e++) { start[eu[e] + 1]++; start[ev[e] + 1]++; }
        for (int v = 0; v < n; v++) start[v + 1] += start[v];
        arcs.resize(start[n]);
        std::vector<int> fill(start.begin(), start.end() - 1);
        for (size_t e = 0; e < eu.size(); e++) {
            const int a = fill[eu[e]]++, b = fill[ev[e]]++;
            arcs[a] = {ev[e], b, ec[e]};
            arcs[b] = {eu[e], a, 0};
        }
        level.resize(n); it.resize(n); queue.resize(n);
    }
    bool bfs(int s, int t) {
        std::fill(level.begin(), level.end(), -1);
        int qh = 0, qt = 0;
        level[s] = 0; queue[qt++] = s;
        while (qh < qt) {
            const int u = queue[qh++];
            for (int a = start[u]; a < start[u + 1]; a++)
                if (arcs[a].cap > 0 && level[arcs[a].to] < 0) { level[arcs[a].to] = level[u] + 1; queue[qt++] = arcs[a].to; }
        }
        return level[t] >= 0;
    }
    // one augmenting path in the level graph (explicit stack: paths can be long)
    bool augment(int s, int t) {
        path.clear();
        int u = s;
        while (true) {
            if (u == t) {
                Cap f = arcs[path[0]].cap;
                for (int a : path) f = std::min(f, arcs[a].cap);
                for (int a : path) { arcs[a].cap -= f; arcs[arcs[a].rev].cap += f; }
                return true;
            }
            bool adv = false;
            for (int& a = it[u]; a < start[u + 1]; a++) {
                if (arcs[a].cap > 0 && level[arcs[a].to] == level[u] + 1) {
                    path.push_back(a);
                    u = arcs[a].to;
                    adv = true;
                    break;
                }
            }
            if (!adv) {
                if (path.empty()) return false;
                level[u] = -1;                      // dead end
                const int a = path.back();
                path.pop_back();
                u = arcs[arcs[a].rev].to;
                it[u]++;
            }
        }
    }
    void run(int s, int t) {
        while (bfs(s, t)) {
            for (int v = 0; v < n; v++) it[v] = start[v];
            while (augment(s, t)) {}
        }
    }
    // nodes that reach t in the residual graph (the smallest sink side)
    std::vector<char> reach_sink(int t) {
        std::vector<char> r(n, 0);
        int qt = 0;
        r[t] = 1; queue[qt++] = t;
        for (int qh = 0; qh < qt; qh++) {
            const int v = queue[qh];
            for (int a = start[v]; a < start[v + 1]; a++) {
                const int u = arcs[a].to;          // arc v -> u; its reverse u -> v
                if (!r[u] && arcs[arcs[a].rev].cap > 0) { r[u] = 1; queue[qt++] = u; }
            }
        }
        return r;
    }
};

constexpr Wide HARD = (Wide)1 << 100;      // a forbidden move (outside the bounds)
constexpr int64_t HARD64 = (int64_t)1 << 62;

struct Program {
    int n, m;
    const int32_t *ei, *ej, *off;
    const int64_t* w;
    int s;
    Wide B;
    bool narrow;                            // every finite capacity fits int64 with room
    Flow<int64_t> f64[2];                   // one graph per move direction
    Flow<Wide> f128[2];
    Wide objective(const std::vector<int>& k) const {
        Wide f = 0;
        for (int e = 0; e < m; e++) f += B * (Wide)w[e] * (Wide)std::llabs((int64_t)s * (k[ei[e]] - k[ej[e]]) - off[e]);
        for (int i = 0; i < n; i++) f += std::llabs((int64_t)k[i]);
        return f;
    }
    // the smallest best set S for k + dir * chi_S (empty if no move lowers F)
    template <class Cap>
    std::vector<char> best_move(Flow<Cap>& g, const std::vector<int>& k, int dir, Cap hard) {
        const int S = n, T = n + 1;
        g.reset(n + 2);
        std::vector<Wide> unary(n, 0);           // cost of x_v = 1 (moved) over x_v = 0
        for (int e = 0; e < m; e++) {
            const int i = ei[e], j = ej[e];
            const int64_t d = (int64_t)s * (k[i] - k[j]) - off[e];
            const int64_t step = (int64_t)s * dir;       // change of d when only i moves
            auto term = [&](int64_t dd) -> Wide { return std::llabs(dd) > 200 ? HARD : B * (Wide)w[e] * (Wide)std::llabs(dd); };
            // E(x_i, x_j) = A + (C-A) x_i + (D-C) x_j + (B+C-A-D)(1-x_i) x_j
            const Wide A = term(d), Bc = term(d - step), Cc = term(d + step), D = A;
            unary[i] += Cc - A;
            unary[j] += D - Cc;
            g.add(i, j, (Cap)(Bc + Cc - A - D));
        }
        for (int v = 0; v < n; v++) {
            const int nk = k[v] + dir;
            if (v == 0 || nk < -100 || nk > 100) unary[v] += HARD;
            else unary[v] += (Wide)(std::llabs((int64_t)nk) - std::llabs((int64_t)k[v]));
        }
        for (int v = 0; v < n; v++) {
            // paid when moved.  On the int64 path a forbidden node's unary is HARD plus a small
            // term (no pair term is forbidden there), so it maps to the int64 HARD; the 128-bit
            // path keeps exact values (its pair terms may carry +HARD / -HARD that must cancel)
            if (unary[v] > 0) g.add(S, v, (sizeof(Cap) == 8 && unary[v] >= HARD / 2) ? hard : (Cap)unary[v]);
            else if (unary[v] < 0) g.add(v, T, (Cap)(-unary[v]));
        }
        g.build();
        g.run(S, T);
        std::vector<char> r = g.reach_sink(T);
        r.resize(n);
        return r;
    }
    std::vector<char> move(const std::vector<int>& k, int dir) {
        // int64 is exact while no edge is at the +-200 bound (no forbidden pair terms) and
        // every finite capacity fits (the caller checked the total)
        bool edge_ok = true;
        for (int e = 0; e < m && edge_ok; e++)
            edge_ok = std::llabs((int64_t)s * (k[ei[e]] - k[ej[e]]) - off[e]) < 200;
        const int slot = dir > 0 ? 0 : 1;
        if (narrow && edge_ok) return best_move<int64_t>(f64[slot], k, dir, HARD64);
        return best_move<Wide>(f128[slot], k, dir, HARD);
    }
};

// Starting point: every edge of a maximum-weight spanning forest satisfied
// exactly (k_0 = 0, the first node of every other tree at 0).  Only shortens the
// descent; the descent then reaches the minimum from here.  Falls back to zero
// when the start leaves the bounds.
std::vector<int> spanning_start(const Program& P) {
    const int n = P.n, m = P.m;
    std::vector<int> order(m);
    for (int e = 0; e < m; e++) order[e] = e;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return P.w[a] > P.w[b]; });
    std::vector<int> root(n);
    for (int v = 0; v < n; v++) root[v] = v;
    auto find = [&](int v) { while (root[v] != v) v = root[v] = root[root[v]]; return v; };
    std::vector<std::vector<std::pair<int, int>>> adj(n);   // (neighbour, edge)
    for (int e : order) {
        const int a = find(P.ei[e]), b = find(P.ej[e]);
        if (a == b) continue;
        root[std::max(a, b)] = std::min(a, b);
        adj[P.ei[e]].push_back({P.ej[e], e});
        adj[P.ej[e]].push_back({P.ei[e], e});
    }
    std::vector<int> k(n, 0);
    std::vector<char> seen(n, 0);
    for (int r = 0; r < n; r++) {
        if (seen[r]) continue;
        seen[r] = 1;
        std::vector<int> st{r};
        while (!st.empty()) {
            const int u = st.back(); st.pop_back();
            for (auto [v, e] : adj[u]) {
                if (seen[v]) continue;
                seen[v] = 1;
                // s (k_i - k_j) = off[e]
                if (P.ei[e] == u) k[v] = k[u] - P.s * P.off[e];
                else k[v] = k[u] + P.s * P.off[e];
                st.push_back(v);
            }
        }
    }
    for (int v = 0; v < n; v++)
        if (k[v] < -100 || k[v] > 100) return std::vector<int>(n, 0);
    for (int e = 0; e < m; e++)
        if (std::llabs((int64_t)P.s * (k[P.ei[e]] - k[P.ej[e]]) - P.off[e]) > 200) return std::vector<int>(n, 0);
    return k;
}

}  // namespace

extern "C" int unw_link_offsets(int32_t n, int32_t m, const int32_t* ei, const int32_t* ej, const int32_t* off,
                                const int64_t* w, int32_t sign, int32_t* k_out) {
    if (n < 0 || m < 0 || (n > 0 && !k_out) || (m > 0 && (!ei || !ej || !off || !w)))
        return unw_set_error(UNW_E_ARG, "link offsets: null pointer or negative size");
    for (int e = 0; e < m; e++) {
        if (ei[e] < 0 || ei[e] >= n || ej[e] < 0 || ej[e] >= n || w[e] < 0 || w[e] > ((int64_t)1 << 31) ||
            off[e] < -200 || off[e] > 200)
            return unw_set_error(UNW_E_ARG, "link offsets: edge out of range");
    }
    if (n > (1 << 22)) return unw_set_error(UNW_E_UNSUPPORTED, "link offsets: too many components");
    std::vector<int> k(n, 0);
    if (n >= 2 && m > 0) {
        Program P{n, m, ei, ej, off, w, sign >= 0 ? 1 : -1, (Wide)100 * n + 1, false, {}, {}};
        Wide total = 0;                          // bound on the sum of finite capacities
        for (int e = 0; e < m; e++) total += P.B * (Wide)w[e] * 4;
        total += (Wide)4 * n;
        P.narrow = total < ((Wide)1 << 60);
        k = spanning_start(P);
        Wide f = P.objective(k);
        for (int iter = 0; iter < 1000; iter++) {
            Wide best = f;
            std::vector<int> kb;
            // the two directions are independent cuts: the -1 move on a second thread
            std::vector<char> Sdir[2];
            std::thread down([&] { Sdir[1] = P.move(k, -1); });
            Sdir[0] = P.move(k, 1);
            down.join();
            for (int dir = 1; dir >= -1; dir -= 2) {
                const std::vector<char>& S = Sdir[dir > 0 ? 0 : 1];
                std::vector<int> kn = k;
                bool any = false;
                for (int v = 0; v < n; v++)
                    if (S[v]) { kn[v] += dir; any = true; }
                if (!any) continue;
                const Wide fn = P.objective(kn);
                if (fn < best) { best = fn; kb = kn; }
            }
            if (kb.empty()) break;
            k = kb;
            f = best;
        }
    }
    for (int i = 0; i < n; i++) k_out[i] = k[i];
    return UNW_OK;
}
