// The coarsening of the stage-2 multigrid (host code): one level of
// build_coarse_level (oracle/tpe_stage2_oracle.py:816-937).
//
// Vertices of degree other than 2 and pinned vertices are anchors. Every chain
// between anchors is walked from the anchors in ascending order and colored
// alternately, the anchors and the even positions black (and the vertex before
// a chain's closing anchor black when it was left white); closed cycles with no
// anchor are colored from their smallest vertex, the last vertex of an odd
// cycle black. Black vertices become the coarse vertices (ascending fine
// index); a white vertex is prolonged from its first two black neighbours with
// weights 1/2 (from its one black neighbour with weight 1). Coarse edges join
// black vertices along the fine paths between them, once per pair, and carry
// the original fine edges of those paths. The walks, their order and every tie
// follow the oracle, so the levels are the oracle's levels.
#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <set>
#include <utility>
#include <vector>

#include "tpe_internal.h"

namespace tpe {
namespace {

struct CoarseLevel {
    std::vector<int32_t> black;                 // fine vertex of each coarse vertex
    std::vector<int32_t> p_idx;                 // 2 per fine vertex: coarse indices (-1: none)
    std::vector<double> p_w;                    // 2 per fine vertex: weights
    std::vector<int32_t> edges;                 // 2 per coarse edge
    std::vector<int32_t> path_off, path_edges;  // original fine edges of each coarse edge
};

// Returns false when the oracle returns None (no coarser level).
bool coarsen(int32_t n, const int32_t* edges, int32_t E, const int32_t* orig,
             const std::set<int32_t>& pinned_orig, const int32_t* path_off,
             const int32_t* path_edges, int32_t min_vertices, CoarseLevel& out) {
    if (n <= min_vertices) return false;
    std::vector<std::vector<std::pair<int32_t, int32_t>>> adj((size_t)n);
    for (int32_t ei = 0; ei < E; ei++) {
        const int32_t a = edges[2 * ei], b = edges[2 * ei + 1];
        adj[a].push_back({b, ei});
        adj[b].push_back({a, ei});
    }
    std::vector<int32_t> deg((size_t)n);
    for (int32_t i = 0; i < n; i++) deg[i] = (int32_t)adj[i].size();
    std::vector<char> anchor((size_t)n, 0), black((size_t)n, 0), vis((size_t)E, 0);
    for (int32_t i = 0; i < n; i++)
        if (deg[i] != 2 || pinned_orig.count(orig[i])) anchor[i] = 1;
    for (int32_t i = 0; i < n; i++)
        if (anchor[i]) black[i] = 1;
    // the first neighbour other than prev, in adjacency order
    auto next = [&](int32_t cur, int32_t prev, int32_t& nxt, int32_t& eidx) {
        for (const auto& pr : adj[cur])
            if (pr.first != prev) {
                nxt = pr.first;
                eidx = pr.second;
                return true;
            }
        return false;
    };
    for (int32_t a = 0; a < n; a++) {
        if (!anchor[a]) continue;
        for (const auto& first : adj[a]) {
            if (vis[first.second]) continue;
            std::vector<int32_t> path{a, first.first};
            int32_t prev = a, cur = first.first;
            vis[first.second] = 1;
            while (!anchor[cur] && deg[cur] == 2) {
                int32_t nxt, eidx;
                if (!next(cur, prev, nxt, eidx)) break;
                if (vis[eidx]) break;
                path.push_back(nxt);
                vis[eidx] = 1;
                prev = cur;
                cur = nxt;
            }
            for (size_t pos = 0; pos < path.size(); pos++)
                if (pos % 2 == 0 || anchor[path[pos]]) black[path[pos]] = 1;
            if (anchor[path.back()]) {
                black[path.back()] = 1;
                if (path.size() >= 2 && !black[path[path.size() - 2]]) black[path[path.size() - 2]] = 1;
            }
        }
    }
    // closed cycles without anchors (and anything left unvisited)
    for (int32_t start = 0; start < n; start++) {
        for (const auto& first : adj[start]) {
            if (vis[first.second]) continue;
            std::vector<int32_t> cycle{start};
            int32_t prev = start, cur = first.first;
            vis[first.second] = 1;
            while (cur != start) {
                cycle.push_back(cur);
                int32_t nxt, eidx;
                if (!next(cur, prev, nxt, eidx)) break;
                if (vis[eidx] && nxt != start) break;
                if (!vis[eidx]) vis[eidx] = 1;
                prev = cur;
                cur = nxt;
            }
            for (size_t pos = 0; pos < cycle.size(); pos += 2) black[cycle[pos]] = 1;
            if (cycle.size() % 2 == 1 && cycle.size() > 1) black[cycle.back()] = 1;
        }
    }
    out.black.clear();
    std::vector<int32_t> cidx((size_t)n, -1);
    for (int32_t v = 0; v < n; v++)
        if (black[v]) {
            cidx[v] = (int32_t)out.black.size();
            out.black.push_back(v);
        }
    if ((int32_t)out.black.size() == n) return false;
    out.p_idx.assign(2 * (size_t)n, -1);
    out.p_w.assign(2 * (size_t)n, 0.0);
    for (int32_t v = 0; v < n; v++) {
        if (cidx[v] >= 0) {
            out.p_idx[2 * v] = cidx[v];
            out.p_w[2 * v] = 1.0;
            continue;
        }
        std::vector<int32_t> bn;
        for (const auto& pr : adj[v])
            if (cidx[pr.first] >= 0) bn.push_back(pr.first);
        if (bn.size() >= 2) {
            // (the oracle assigns P[v, b] = 0.5 twice when both neighbours are one vertex)
            out.p_idx[2 * v] = cidx[bn[0]];
            out.p_w[2 * v] = 0.5;
            if (bn[1] != bn[0]) {
                out.p_idx[2 * v + 1] = cidx[bn[1]];
                out.p_w[2 * v + 1] = 0.5;
            }
        } else if (bn.size() == 1) {
            out.p_idx[2 * v] = cidx[bn[0]];
            out.p_w[2 * v] = 1.0;
        } else {
            return false;  // the oracle's pathological case
        }
    }
    // coarse edges along the fine paths between black vertices
    std::vector<char> visf((size_t)E, 0);
    std::set<std::pair<int32_t, int32_t>> seen;
    out.edges.clear();
    out.path_off.assign(1, 0);
    out.path_edges.clear();
    for (int32_t bi : out.black) {
        for (const auto& first : adj[bi]) {
            if (visf[first.second]) continue;
            std::vector<int32_t> pe{first.second};
            int32_t prev = bi, cur = first.first;
            visf[first.second] = 1;
            while (cidx[cur] < 0) {
                int32_t nxt, eidx;
                if (!next(cur, prev, nxt, eidx)) break;
                if (visf[eidx]) break;
                pe.push_back(eidx);
                visf[eidx] = 1;
                prev = cur;
                cur = nxt;
            }
            if (cidx[cur] >= 0 && cur != bi) {
                const int32_t a = cidx[bi], b = cidx[cur];
                const std::pair<int32_t, int32_t> key{std::min(a, b), std::max(a, b)};
                if (!seen.count(key)) {
                    seen.insert(key);
                    out.edges.push_back(a);
                    out.edges.push_back(b);
                    for (int32_t f : pe)
                        for (int32_t q = path_off[f]; q < path_off[f + 1]; q++)
                            out.path_edges.push_back(path_edges[q]);
                    out.path_off.push_back((int32_t)out.path_edges.size());
                }
            }
        }
    }
    return !out.edges.empty();
}

}  // namespace
}  // namespace tpe

// One coarsening step of the stage-2 multigrid hierarchy (build_coarse_level,
// oracle/tpe_stage2_oracle.py:816-937), on the host. Inputs: the level's V
// vertices and E edges, orig[V] (the original vertex of each), the original
// fine edges of each level edge (path_edges with offsets path_off[E + 1]), the
// pinned original vertices. Outputs (caller-allocated at the sizes the level
// bounds them by): black[Vc] (the level vertex of each coarse vertex), p_idx[2V]
// and p_w[2V] (the prolongation: up to two coarse vertices per level vertex,
// -1 where none), cedges[2 Ec], the coarse edges' original edges
// (cpath_edges with offsets cpath_off[Ec + 1]; at most the level's path_off[E]
// entries), and *Vc, *Ec. *Vc = 0 when the oracle would return no coarser level.
extern "C" int32_t tpe_mg_coarsen(int32_t V, const int32_t* edges, int32_t E, const int32_t* orig,
                                  const int32_t* path_off, const int32_t* path_edges,
                                  const int32_t* pinned, int32_t npinned, int32_t min_vertices,
                                  int32_t* black, int32_t* p_idx, double* p_w, int32_t* cedges,
                                  int32_t* cpath_off, int32_t* cpath_edges, int32_t* Vc,
                                  int32_t* Ec) {
    try {
        if (V < 0 || E < 0 || !orig || !path_off || !Vc || !Ec || (E > 0 && (!edges || !path_edges)) ||
            npinned < 0 || (npinned > 0 && !pinned) || !black || !p_idx || !p_w || !cedges ||
            !cpath_off || !cpath_edges)
            return TPE_ERR_BAD_ARG;
        for (int64_t q = 0; q < 2 * (int64_t)E; q++)
            if (edges[q] < 0 || edges[q] >= V) return TPE_ERR_BAD_ARG;
        std::set<int32_t> pin(pinned, pinned + npinned);
        tpe::CoarseLevel cl;
        *Vc = 0;
        *Ec = 0;
        if (!tpe::coarsen(V, edges, E, orig, pin, path_off, path_edges, min_vertices, cl)) return TPE_OK;
        *Vc = (int32_t)cl.black.size();
        *Ec = (int32_t)(cl.edges.size() / 2);
        std::memcpy(black, cl.black.data(), sizeof(int32_t) * cl.black.size());
        std::memcpy(p_idx, cl.p_idx.data(), sizeof(int32_t) * cl.p_idx.size());
        std::memcpy(p_w, cl.p_w.data(), sizeof(double) * cl.p_w.size());
        std::memcpy(cedges, cl.edges.data(), sizeof(int32_t) * cl.edges.size());
        std::memcpy(cpath_off, cl.path_off.data(), sizeof(int32_t) * cl.path_off.size());
        std::memcpy(cpath_edges, cl.path_edges.data(), sizeof(int32_t) * cl.path_edges.size());
        return TPE_OK;
    } catch (const std::bad_alloc&) {
        return TPE_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return TPE_ERR_INTERNAL;
    }
}
