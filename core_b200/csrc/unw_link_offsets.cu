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
// are found with Dinic's max-flow in 128-bit integers (B * w * |d| exceeds
// int64 for large instances); the moved set is the smallest
// minimiser (the nodes that still reach the sink in the residual graph), so the
// result is deterministic.
#include <stdint.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <queue>
#include <vector>

#include "../../include/unwrap_b200.h"
#include "unw_kernels.h"

namespace {

using Cap = __int128;
constexpr Cap CAP_MAX = (Cap)1 << 120;
constexpr Cap HARD = (Cap)1 << 100;      // a forbidden move (outside the bounds)

struct Dinic {
    struct Arc { int to; Cap cap; };
    std::vector<Arc> arcs;
    std::vector<std::vector<int>> adj;
    std::vector<int> level, it, path;
    explicit Dinic(int n) : adj(n), level(n), it(n) {}
    void add(int u, int v, Cap c) {
        if (c <= 0) return;
        adj[u].push_back((int)arcs.size()); arcs.push_back({v, c});
        adj[v].push_back((int)arcs.size()); arcs.push_back({u, 0});
    }
    bool bfs(int s, int t) {
        std::fill(level.begin(), level.end(), -1);
        std::queue<int> q;
        level[s] = 0; q.push(s);
        while (!q.empty()) {
            const int u = q.front(); q.pop();
            for (int a : adj[u])
                if (arcs[a].cap > 0 && level[arcs[a].to] < 0) { level[arcs[a].to] = level[u] + 1; q.push(arcs[a].to); }
        }
        return level[t] >= 0;
    }
    // one augmenting path in the level graph (explicit stack: paths can be long)
    Cap augment(int s, int t) {
        path.clear();
        int u = s;
        while (true) {
            if (u == t) {
                Cap f = CAP_MAX;
                for (int a : path) f = std::min(f, arcs[a].cap);
                for (int a : path) { arcs[a].cap -= f; arcs[a ^ 1].cap += f; }
                return f;
            }
            bool adv = false;
            for (int& i = it[u]; i < (int)adj[u].size(); i++) {
                const int a = adj[u][i];
                if (arcs[a].cap > 0 && level[arcs[a].to] == level[u] + 1) {
                    path.push_back(a);
                    u = arcs[a].to;
                    adv = true;
                    break;
                }
            }
            if (!adv) {
                if (path.empty()) return 0;
                level[u] = -1;                      // dead end
                const int a = path.back();
                path.pop_back();
                u = arcs[a ^ 1].to;
                it[u]++;
            }
        }
    }
    void run(int s, int t) {
        while (bfs(s, t)) {
            std::fill(it.begin(), it.end(), 0);
            while (augment(s, t) > 0) {}
        }
    }
    // nodes that reach t in the residual graph (the smallest sink side)
    std::vector<char> reach_sink(int t) {
        std::vector<char> r(adj.size(), 0);
        std::vector<int> st{t};
        r[t] = 1;
        while (!st.empty()) {
            const int v = st.back(); st.pop_back();
            for (int a : adj[v]) {
                const int u = arcs[a].to;          // arc a: v -> u; its pair a^1: u -> v
                if (!r[u] && arcs[a ^ 1].cap > 0) { r[u] = 1; st.push_back(u); }
            }
        }
        return r;
    }
};

struct Program {
    int n, m;
    const int32_t *ei, *ej, *off;
    const int64_t* w;
    int s;
    Cap B;
    Cap objective(const std::vector<int>& k) const {
        Cap f = 0;
        for (int e = 0; e < m; e++) f += B * (Cap)w[e] * (Cap)std::llabs((int64_t)s * (k[ei[e]] - k[ej[e]]) - off[e]);
        for (int i = 0; i < n; i++) f += std::llabs((int64_t)k[i]);
        return f;
    }
    // the best set S for k + dir * chi_S (empty if none lowers F)
    std::vector<char> best_move(const std::vector<int>& k, int dir) const {
        const int S = n, T = n + 1;
        Dinic g(n + 2);
        std::vector<Cap> unary(n, 0);            // cost of x_v = 1 (moved) over x_v = 0
        auto pair_term = [&](int u, int v, Cap A, Cap Bc, Cap Cc, Cap D) {
            // E(x_u, x_v) = A + (C-A) x_u + (D-C) x_v + (B+C-A-D)(1-x_u) x_v
            unary[u] += Cc - A;
            unary[v] += D - Cc;
            g.add(u, v, Bc + Cc - A - D);
        };
        for (int e = 0; e < m; e++) {
            const int i = ei[e], j = ej[e];
            const int64_t d = (int64_t)s * (k[i] - k[j]) - off[e];
            const int64_t step = (int64_t)s * dir;       // change of d when only i moves
            auto term = [&](int64_t dd) -> Cap { return std::llabs(dd) > 200 ? HARD : B * (Cap)w[e] * (Cap)std::llabs(dd); };
            pair_term(i, j, term(d), term(d - step), term(d + step), term(d));
        }
        for (int v = 0; v < n; v++) {
            const int nk = k[v] + dir;
            if (v == 0 || nk < -100 || nk > 100) unary[v] += HARD;
            else unary[v] += (Cap)(std::llabs((int64_t)nk) - std::llabs((int64_t)k[v]));
        }
        for (int v = 0; v < n; v++) {
            if (unary[v] > 0) g.add(S, v, unary[v]);    // paid when v is on the sink side (moved)
            else if (unary[v] < 0) g.add(v, T, -unary[v]);
        }
        g.run(S, T);
        std::vector<char> r = g.reach_sink(T);
        std::vector<char> moved(n);
        for (int v = 0; v < n; v++) moved[v] = r[v];
        return moved;
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
        Program P{n, m, ei, ej, off, w, sign >= 0 ? 1 : -1, (Cap)100 * n + 1};
        k = spanning_start(P);
        Cap f = P.objective(k);
        for (int iter = 0; iter < 1000; iter++) {
            Cap best = f;
            std::vector<int> kb;
            for (int dir = 1; dir >= -1; dir -= 2) {
                const std::vector<char> S = P.best_move(k, dir);
                std::vector<int> kn = k;
                bool any = false;
                for (int v = 0; v < n; v++)
                    if (S[v]) { kn[v] += dir; any = true; }
                if (!any) continue;
                const Cap fn = P.objective(kn);
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
