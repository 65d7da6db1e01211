"""Mesh tables and node orders (adhv8_kraken_b200/csrc/sw2_tables.h, compiled for the host).

After an adaption:
the incremental update that sw2gpu_remesh uses -- rebuilding only the pattern rows of nodes a
changed, new or removed element or edge touches -- gives exactly the tables of a build from
scratch (BCSR pattern, per-block rows and diagonal positions, the reference-order element-slot
gather lists and the node residual-slot lists), on refinements, edge flips, dropped trailing
triangles and changed boundary edges; a mesh that lost nodes is reported for a full build.  The
node orders of the solvers: the block D-ILU colouring is proper, the banded solve's reverse
Cuthill-McKee order a permutation with a narrow band."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import basin_model, centroid_refine, channel_model

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "adhv8_kraken_b200", "csrc")

SHIM = r'''
#include "sw2_tables.h"
extern "C" int tables_compare(int Vo, int To, int Eo, const int* tri_o, const int* edg_o,
                              int V, int T, int E, const int* tri, const int* edg, int* rebuilt) {
    sw2::MeshTables o, a, b;
    if (sw2::build_tables(Vo, To, Eo, tri_o, edg_o, o)) return 10;
    const int ra = sw2::update_tables(o, tri_o, edg_o, V, T, E, tri, edg, a, rebuilt);
    if (ra == -1) return 20;
    const int rb = sw2::build_tables(V, T, E, tri, edg, b);
    if (ra != rb) return 30;
    if (ra) return 40;
    if (a.rp != b.rp || a.col != b.col || a.blk_row != b.blk_row || a.dpos != b.dpos || a.blk_ptr != b.blk_ptr ||
        a.blk_src != b.blk_src || a.slot_ptr != b.slot_ptr || a.slot_idx != b.slot_idx)
        return 1;
    return 0;
}
// the D-ILU colouring: 0 when no block of the pattern joins two nodes of one colour
extern "C" int colour_check(int V, int T, int E, const int* tri, const int* edg, int* ncol) {
    sw2::MeshTables t;
    if (sw2::build_tables(V, T, E, tri, edg, t)) return 10;
    std::vector<int> colour;
    *ncol = sw2::smallest_last_colouring(t.rp, t.col, V, 16, colour);
    if (*ncol < 0) return 20;
    for (int n = 0; n < V; n++)
        for (int k = t.rp[n]; k < t.rp[n + 1]; k++)
            if (t.col[k] != n && colour[t.col[k]] == colour[n]) return 1;
    return 0;
}
// the banded solve's reverse Cuthill-McKee order: its half-bandwidth, -1 if perm is not a permutation
extern "C" int rcm_check(int V, int T, int E, const int* tri, const int* edg) {
    sw2::MeshTables t;
    if (sw2::build_tables(V, T, E, tri, edg, t)) return -2;
    std::vector<int> perm;
    const int bw = sw2::rcm_order(t.rp, t.col, V, perm);
    std::vector<char> seen(V, 0);
    for (int p : perm) {
        if (p < 0 || p >= V || seen[p]) return -1;
        seen[p] = 1;
    }
    return bw;
}
'''


@pytest.fixture(scope="module")
def tables():
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    work = os.path.join(ROOT, "_build", "mesh_tables")   # git-ignored scratch inside the tree
    os.makedirs(work, exist_ok=True)
    src, lib = os.path.join(work, "shim.cpp"), os.path.join(work, "libtables.so")
    with open(src, "w") as fh:
        fh.write(SHIM)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", CSRC, "-o", lib, src],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    yield C.CDLL(lib)
    shutil.rmtree(work, ignore_errors=True)
    try:
        os.rmdir(os.path.dirname(work))
    except OSError:
        pass


def _ip(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(C.POINTER(C.c_int))


def _compare(L, m0, tri, edges, V):
    tri0, e0 = np.ascontiguousarray(m0.tri, np.int32), np.ascontiguousarray(m0.edges, np.int32).reshape(-1, 2)
    tri, edges = np.ascontiguousarray(tri, np.int32), np.ascontiguousarray(edges, np.int32).reshape(-1, 2)
    nre = C.c_int(-1)
    rc = L.tables_compare(m0.nnodes, len(tri0), len(e0), _ip(tri0), _ip(e0), V, len(tri), len(edges), _ip(tri),
                          _ip(edges), C.byref(nre))
    return rc, nre.value


def _flip(tri, rng, tries=200):
    """Flips the shared edge of a random pair of neighbouring triangles (numbers kept)."""
    tri = tri.copy()
    owner = {}
    for e, t in enumerate(tri):
        for i in range(3):
            owner.setdefault((int(t[(i + 1) % 3]), int(t[i])), e)   # the neighbour sees the edge reversed
    for _ in range(tries):
        e = int(rng.integers(len(tri)))
        i = int(rng.integers(3))
        a, b, c = (int(tri[e][(i + k) % 3]) for k in range(3))
        f = owner.get((a, b))
        if f is None or f == e:
            continue
        d = next(int(q) for q in tri[f] if q not in (a, b))
        tri[e] = (c, a, d)
        tri[f] = (d, b, c)
        return tri
    return tri


@pytest.mark.parametrize("make", [channel_model, basin_model])
def test_incremental_tables_equal_a_full_build(tables, make):
    m0 = make()
    rng = np.random.Generator(np.random.PCG64(11))
    T = m0.nelems2d
    # refinement of 40 triangles: nodes and triangles appended
    m1 = centroid_refine(m0, sorted(rng.choice(T, 40, replace=False).tolist()))
    rc, nre = _compare(tables, m0, m1.tri, m1.edges, m1.nnodes)
    assert rc == 0 and 0 < nre < m1.nnodes // 2, (rc, nre)
    # edge flips: same nodes, two triangles changed each
    tri = m0.tri
    for _ in range(5):
        tri = _flip(tri, rng)
    rc, nre = _compare(tables, m0, tri, m0.edges, m0.nnodes)
    assert rc == 0 and 0 < nre < 60, (rc, nre)
    # refinement, then the last two appended triangles dropped again with their parent restored
    m2 = centroid_refine(m0, [5, 17])
    tri2 = m2.tri[:-2].copy()
    tri2[17] = m0.tri[17]
    rc, nre = _compare(tables, m0, tri2, m2.edges, m2.nnodes)
    assert rc == 40   # the dropped triangles' node belongs to no element: both builds report it
    rc, nre = _compare(tables, m0, m1.tri, m1.edges[:-3], m1.nnodes)   # boundary edges removed
    assert rc == 0
    shuffled = m1.edges[rng.permutation(len(m1.edges))]                # edges renumbered
    rc, nre = _compare(tables, m0, m1.tri, shuffled, m1.nnodes)
    assert rc == 0


def test_mesh_that_lost_nodes_is_rebuilt_from_scratch(tables):
    m0 = centroid_refine(channel_model(), [3])
    m1 = channel_model()
    rc, _ = _compare(tables, m0, m1.tri, m1.edges, m1.nnodes)
    assert rc == 20


def test_dilu_colouring_is_proper_and_needs_five_colours(tables):
    """Smallest-last greedy colouring (block D-ILU order): no two neighbours share a colour; the
    benchmark generator's basin needs 5 colours."""
    import math
    from adhv8_kraken_b200 import meshgen
    for m in (channel_model(), basin_model(),
              meshgen.bumpy_basin(10000, seed=2024, size=20000.0 * math.sqrt(10000 / 5e5), nsteps=1, dt=5.0, name="b")):
        tri, e = np.ascontiguousarray(m.tri, np.int32), np.ascontiguousarray(m.edges, np.int32).reshape(-1, 2)
        n = C.c_int(0)
        assert tables.colour_check(m.nnodes, len(tri), len(e), _ip(tri), _ip(e), C.byref(n)) == 0
        assert 3 <= n.value <= 6, (m.name, n.value)
    assert n.value == 5


def test_rcm_order_is_a_permutation_with_a_narrow_band(tables):
    """Reverse Cuthill-McKee order of the banded exact solve: a permutation whose half-bandwidth
    is within 10 % of scipy's reverse Cuthill-McKee on the same graph."""
    import scipy.sparse as sp
    from scipy.sparse.csgraph import reverse_cuthill_mckee
    for m in (channel_model(), basin_model()):
        tri, e = np.ascontiguousarray(m.tri, np.int32), np.ascontiguousarray(m.edges, np.int32).reshape(-1, 2)
        bw = tables.rcm_check(m.nnodes, len(tri), len(e), _ip(tri), _ip(e))
        assert bw > 0
        r = np.concatenate([tri[:, a] for a in range(3) for b in range(3)])
        c = np.concatenate([tri[:, b] for a in range(3) for b in range(3)])
        G = sp.csr_matrix((np.ones(len(r)), (r, c)), shape=(m.nnodes, m.nnodes))
        order = reverse_cuthill_mckee(G, symmetric_mode=True)
        pos = np.empty(m.nnodes, int)
        pos[order] = np.arange(m.nnodes)
        coo = G.tocoo()
        ref = int(np.abs(pos[coo.row] - pos[coo.col]).max())
        assert bw <= 1.1 * ref + 1, (m.name, bw, ref)
