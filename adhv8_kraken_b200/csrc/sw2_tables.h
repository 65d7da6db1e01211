// sw2_tables.h -- the mesh tables of a context, host only: the BCSR block pattern and the
// reference-order gather lists with which the assembly kernels sum element contributions
// without atomics, in the order fe_sw2_resid (src/fe/sw2/fe_sw2_resid.c:74-160) and
// fe_sw2_load's global assembly (src/fe/fe_assemble_matrix.c:166-224) add them.
//
// Slots: block (a, b) of triangle e is slot 9 e + 3 a + b and block (a, b) of boundary edge j is
// slot 9 T + 4 j + 2 a + b; vertex i's residual of triangle e is residual slot 3 e + i and of
// edge j residual slot 3 T + 2 j + i.  Elements come first, then edges, as in the reference.
//
// build_tables() makes the tables of a mesh from scratch; update_tables() makes the tables of
// an adapted mesh from those of the mesh before (the adaption keeps node and element numbers,
// changes some triangles' nodes, appends nodes and triangles, may drop trailing triangles and
// changes the boundary edges): only the pattern rows of nodes that a changed, new or removed
// element or edge touches are rebuilt, every other row is copied; the gather lists follow in
// one linear pass.  Both give identical tables for the same mesh.  Also here: the node orders
// of the banded exact solve (reverse Cuthill-McKee) and of the block D-ILU solve (colouring).
#pragma once
#include <algorithm>
#include <cstdlib>
#include <functional>
#include <queue>
#include <vector>

namespace sw2 {

struct MeshTables {
    int V = 0, T = 0, E = 0;
    std::vector<int> rp, col;             // BCSR pattern: sorted unique columns of every node row
    std::vector<int> blk_row, dpos;       // row of every block; diagonal block of every row
    std::vector<int> blk_ptr, blk_src;    // block k <- slots blk_src[blk_ptr[k] .. blk_ptr[k+1]-1], ascending
    std::vector<int> slot_ptr, slot_idx;  // node n <- residual slots slot_idx[slot_ptr[n] ..], ascending
};

// The gather lists and per-block rows from a finished pattern.  Returns 0, or 1 + n when node n
// belongs to no element (no diagonal block).
inline int finish_tables(const int* tri, const int* edg, MeshTables& t) {
    const int V = t.V, T = t.T, E = t.E;
    const int nnzb = (int)t.col.size();
    t.blk_row.assign(nnzb, 0);
    t.dpos.assign(V, -1);
    for (int n = 0; n < V; n++)
        for (int k = t.rp[n]; k < t.rp[n + 1]; k++) {
            t.blk_row[k] = n;
            if (t.col[k] == n) t.dpos[n] = k;
        }
    for (int n = 0; n < V; n++)
        if (t.dpos[n] < 0) return 1 + n;
    auto find_blk = [&](int i, int j) {
        const auto b = t.col.begin() + t.rp[i], e = t.col.begin() + t.rp[i + 1];
        return (int)(std::lower_bound(b, e, j) - t.col.begin());
    };
    const size_t nsrc = 9ull * T + 4ull * E;
    std::vector<int> src_blk(nsrc);
    for (int e = 0; e < T; e++)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) src_blk[9ull * e + 3 * a + b] = find_blk(tri[3 * e + a], tri[3 * e + b]);
    for (int j = 0; j < E; j++)
        for (int a = 0; a < 2; a++)
            for (int b = 0; b < 2; b++) src_blk[9ull * T + 4 * j + 2 * a + b] = find_blk(edg[2 * j + a], edg[2 * j + b]);
    t.blk_ptr.assign(nnzb + 1, 0);
    t.blk_src.assign(nsrc, 0);
    for (size_t q = 0; q < nsrc; q++) t.blk_ptr[src_blk[q] + 1]++;
    for (int k = 0; k < nnzb; k++) t.blk_ptr[k + 1] += t.blk_ptr[k];
    {
        std::vector<int> f(t.blk_ptr.begin(), t.blk_ptr.end() - 1);
        for (size_t q = 0; q < nsrc; q++) t.blk_src[f[src_blk[q]]++] = (int)q;   // q ascending = reference order
    }
    const size_t nslot = 3ull * T + 2ull * E;
    t.slot_ptr.assign(V + 1, 0);
    t.slot_idx.assign(nslot, 0);
    for (int e = 0; e < T; e++)
        for (int i = 0; i < 3; i++) t.slot_ptr[tri[3 * e + i] + 1]++;
    for (int j = 0; j < E; j++)
        for (int i = 0; i < 2; i++) t.slot_ptr[edg[2 * j + i] + 1]++;
    for (int n = 0; n < V; n++) t.slot_ptr[n + 1] += t.slot_ptr[n];
    {
        std::vector<int> f(t.slot_ptr.begin(), t.slot_ptr.end() - 1);
        for (int e = 0; e < T; e++)
            for (int i = 0; i < 3; i++) t.slot_idx[f[tri[3 * e + i]]++] = 3 * e + i;
        for (int j = 0; j < E; j++)
            for (int i = 0; i < 2; i++) t.slot_idx[f[edg[2 * j + i]]++] = 3 * T + 2 * j + i;
    }
    return 0;
}

// Pattern rows of the nodes marked in `want` (others left empty): the sorted unique nodes of
// the triangles and edges that contain each node.  rows[n] receives node n's columns.
inline void pattern_rows(int V, int T, int E, const int* tri, const int* edg, const std::vector<char>& want,
                         std::vector<std::vector<int>>& rows) {
    rows.assign(V, std::vector<int>());
    for (int e = 0; e < T; e++)
        for (int i = 0; i < 3; i++) {
            const int a = tri[3 * e + i];
            if (want[a]) rows[a].insert(rows[a].end(), tri + 3 * e, tri + 3 * e + 3);
        }
    for (int j = 0; j < E; j++)
        for (int i = 0; i < 2; i++) {
            const int a = edg[2 * j + i];
            if (want[a]) rows[a].insert(rows[a].end(), edg + 2 * j, edg + 2 * j + 2);
        }
    for (int n = 0; n < V; n++)
        if (want[n]) {
            std::sort(rows[n].begin(), rows[n].end());
            rows[n].erase(std::unique(rows[n].begin(), rows[n].end()), rows[n].end());
        }
}

// Tables of a mesh from scratch.  Returns 0, or 1 + n when node n belongs to no element.
inline int build_tables(int V, int T, int E, const int* tri, const int* edg, MeshTables& t) {
    t.V = V;
    t.T = T;
    t.E = E;
    std::vector<char> all(V, 1);
    std::vector<std::vector<int>> rows;
    pattern_rows(V, T, E, tri, edg, all, rows);
    t.rp.assign(V + 1, 0);
    t.col.clear();
    for (int n = 0; n < V; n++) {
        t.col.insert(t.col.end(), rows[n].begin(), rows[n].end());
        t.rp[n + 1] = (int)t.col.size();
    }
    return finish_tables(tri, edg, t);
}

// Tables of an adapted mesh from those of the mesh before (o, with its triangles tri_old and
// edges edg_old): node and triangle numbers kept, nodes appended (V >= o.V).  `rebuilt`, when
// given, receives the number of pattern rows rebuilt.  Returns as build_tables(), or -1 when
// the mesh lost nodes (build from scratch then).
inline int update_tables(const MeshTables& o, const int* tri_old, const int* edg_old, int V, int T, int E,
                         const int* tri, const int* edg, MeshTables& t, int* rebuilt = nullptr) {
    if (V < o.V) return -1;
    std::vector<char> touched(V, 0);
    for (int n = o.V; n < V; n++) touched[n] = 1;
    const int Tc = std::min(T, o.T);
    for (int e = 0; e < Tc; e++)
        if (tri[3 * e] != tri_old[3 * e] || tri[3 * e + 1] != tri_old[3 * e + 1] || tri[3 * e + 2] != tri_old[3 * e + 2])
            for (int i = 0; i < 3; i++) touched[tri[3 * e + i]] = touched[tri_old[3 * e + i]] = 1;
    for (int e = Tc; e < T; e++)
        for (int i = 0; i < 3; i++) touched[tri[3 * e + i]] = 1;
    for (int e = Tc; e < o.T; e++)
        for (int i = 0; i < 3; i++) touched[tri_old[3 * e + i]] = 1;
    for (int j = 0; j < std::max(E, o.E); j++) {
        const bool same = j < E && j < o.E && edg[2 * j] == edg_old[2 * j] && edg[2 * j + 1] == edg_old[2 * j + 1];
        if (same) continue;
        if (j < E) touched[edg[2 * j]] = touched[edg[2 * j + 1]] = 1;
        if (j < o.E) touched[edg_old[2 * j]] = touched[edg_old[2 * j + 1]] = 1;
    }
    std::vector<std::vector<int>> rows;
    pattern_rows(V, T, E, tri, edg, touched, rows);
    t.V = V;
    t.T = T;
    t.E = E;
    t.rp.assign(V + 1, 0);
    t.col.clear();
    t.col.reserve(o.col.size() + 9ull * (V - o.V));
    int nre = 0;
    for (int n = 0; n < V; n++) {
        if (touched[n]) {
            t.col.insert(t.col.end(), rows[n].begin(), rows[n].end());
            nre++;
        } else {
            t.col.insert(t.col.end(), o.col.begin() + o.rp[n], o.col.begin() + o.rp[n + 1]);
        }
        t.rp[n + 1] = (int)t.col.size();
    }
    if (rebuilt) *rebuilt = nre;
    return finish_tables(tri, edg, t);
}

// Reverse Cuthill-McKee order of the nodes (the banded exact solve): breadth-first from a node
// of least degree in every connected part, each node's unvisited neighbours taken by increasing
// degree, the whole sequence reversed.  perm[i] = new position of node i; returns the
// half-bandwidth in nodes.
inline int rcm_order(const std::vector<int>& rp, const std::vector<int>& col, int V, std::vector<int>& perm) {
    std::vector<int> deg(V), start(V), order;
    order.reserve(V);
    for (int i = 0; i < V; i++) {
        deg[i] = rp[i + 1] - rp[i];
        start[i] = i;
    }
    std::stable_sort(start.begin(), start.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    std::vector<char> seen(V, 0);
    size_t head = 0;
    for (int s0 : start) {
        if (seen[s0]) continue;
        seen[s0] = 1;
        order.push_back(s0);
        while (head < order.size()) {
            const int a = order[head++];
            const size_t n0 = order.size();
            for (int k = rp[a]; k < rp[a + 1]; k++)
                if (!seen[col[k]]) {
                    seen[col[k]] = 1;
                    order.push_back(col[k]);
                }
            std::stable_sort(order.begin() + n0, order.end(), [&](int a2, int b2) { return deg[a2] < deg[b2]; });
        }
    }
    perm.assign(V, 0);
    for (int i = 0; i < V; i++) perm[order[V - 1 - i]] = i;
    int bw = 0;
    for (int i = 0; i < V; i++)
        for (int k = rp[i]; k < rp[i + 1]; k++) bw = std::max(bw, std::abs(perm[i] - perm[col[k]]));
    return bw;
}

// Greedy colouring of the node graph for the block D-ILU order: nodes in smallest-last order
// (repeatedly take out a node of least remaining degree, the lowest index among equals, and
// colour in the reverse of that order), each node taking the lowest colour none of its
// neighbours has.  Needs few colours on planar meshes (5 on the benchmark basins, where
// largest-degree-first needs 6).  colour[n] in 0 .. ncol-1; returns ncol, or -1 when more than
// maxcol (at most 32) colours would be needed.
inline int smallest_last_colouring(const std::vector<int>& rp, const std::vector<int>& col, int V, int maxcol,
                                   std::vector<int>& colour) {
    std::vector<int> order;
    order.reserve(V);
    {
        std::vector<int> deg(V);
        std::vector<char> gone(V, 0);
        std::priority_queue<std::pair<int, int>, std::vector<std::pair<int, int>>, std::greater<std::pair<int, int>>> pq;
        for (int n = 0; n < V; n++) {
            deg[n] = rp[n + 1] - rp[n] - 1;
            pq.push({deg[n], n});
        }
        while (!pq.empty()) {
            const auto top = pq.top();
            pq.pop();
            const int n = top.second;
            if (gone[n] || top.first != deg[n]) continue;
            gone[n] = 1;
            order.push_back(n);
            for (int k = rp[n]; k < rp[n + 1]; k++) {
                const int j = col[k];
                if (j != n && !gone[j]) pq.push({--deg[j], j});
            }
        }
        std::reverse(order.begin(), order.end());
    }
    colour.assign(V, -1);
    int ncol = 0;
    for (int n : order) {
        unsigned used = 0;
        for (int k = rp[n]; k < rp[n + 1]; k++) {
            const int j = col[k];
            if (j != n && colour[j] >= 0) used |= 1u << colour[j];
        }
        int cc = 0;
        while (cc < maxcol && ((used >> cc) & 1u)) cc++;
        if (cc >= maxcol) return -1;
        colour[n] = cc;
        ncol = std::max(ncol, cc + 1);
    }
    return ncol;
}

}  // namespace sw2
