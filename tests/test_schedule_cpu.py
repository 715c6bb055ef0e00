"""CPU checks of the work queue that the fused element loop + CSR assembly runs (csrc/schedule.cpp).

The planner is compiled here with g++ from the library's own source, with its flat test entry point
(ceos_test_plan_schedule).  For structured, plate-shaped and randomly numbered meshes, one and four
host slabs and small staging buffers (many conversion items), the tests check:
- the queue holds every tile and every conversion item once, slab by slab, and every item's rows
  belong to nodes the slabs up to its own have finished;
- every wait targets an earlier queue position: an item after all tiles containing its nodes, a
  tile after the items that held its ring slots before;
- ring safety: for every node-pair block b that a tile reduces into, the block b - R that used the
  same slot before is converted by an item the tile waits for;
- the queue drains under the kernel's protocol (P workers take tickets in order, each holds its
  current and its next ticket, a ticket starts once its waits are met), simulated with random
  durations.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from ceos_b200 import meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "ceos-eems_b200", "csrc", "schedule.cpp")
TILE = 32


@pytest.fixture(scope="module")
def planner(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("sched") / "libsched_test.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-DCEOS_SCHEDULE_TEST", SRC, "-o", so])
    L = C.CDLL(so)
    f = L.ceos_test_plan_schedule
    f.restype = C.c_int
    return f


def pattern(n_nodes, conn0):
    """Upper neighbours per node, CSR row starts rs (row 3n) and node-pair block ranks per element pair."""
    up = [set() for _ in range(n_nodes)]
    for el in conn0:
        for a in el:
            for b in el:
                if b > a:
                    up[a].add(b)
    nup = np.array([len(u) for u in up], np.int32)
    rs = np.zeros(n_nodes, np.int64)
    rs[1:] = np.cumsum(6 + 9 * nup.astype(np.int64))[:-1]
    up_sorted = [sorted(u) for u in up]
    nnz = int(6 * n_nodes + 9 * nup.sum())
    n_blocks = n_nodes + (nnz - 6 * n_nodes) // 9
    return rs, nup, up_sorted, n_blocks


def slabs(n_elem, conn0, n_nodes, ns):
    se = [0] + [n_elem * c // ns // TILE * TILE for c in range(1, ns)] + [n_elem]
    last = np.zeros(n_nodes, np.int64)
    for c in range(ns):
        last[conn0[se[c]:se[c + 1]].ravel()] = c
    sn, run, n = [], 0, 0
    for c in range(ns):
        while n < n_nodes and max(run, last[n]) <= c:
            run = max(run, last[n])
            n += 1
        sn.append(n)
    sn[-1] = n_nodes
    return np.array(se, np.int32), np.array(sn, np.int32)


def plan(f, X, conn, ns=1, slack=296, stage_max=7294, max_nodes=256):
    conn0 = np.ascontiguousarray(conn - 1, np.int32)
    N, E = X.shape[0], conn0.shape[0]
    rs, nup, up, n_blocks = pattern(N, conn0)
    se, sn = slabs(E, conn0, N, ns)
    T = (E + TILE - 1) // TILE
    queue = np.zeros(T + N + 1, np.int32)
    conv = np.zeros(4 * N, np.int32)
    wait = np.zeros(2 * T, np.int32)
    slab_q = np.zeros(ns + 1, np.int32)
    counts = np.zeros(3, np.int32)
    ring = C.c_longlong(0)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = f(N, E, p(conn0), p(rs), p(nup), C.c_longlong(n_blocks), ns, p(se), p(sn), TILE, slack,
           C.c_longlong(stage_max), max_nodes, p(queue), p(conv), p(wait), p(slab_q), p(counts), C.byref(ring))
    assert rc == 0
    nq, nc = counts[0], counts[1]
    return {"queue": queue[:nq], "conv": conv[:4 * nc].reshape(nc, 4), "wait": wait.reshape(T, 2), "slab_q": slab_q,
            "R": ring.value, "conn0": conn0, "rs": rs, "nup": nup, "up": up, "n_blocks": n_blocks, "se": se, "sn": sn,
            "T": T, "N": N, "E": E, "stage_max": stage_max, "max_nodes": max_nodes}


def tile_blocks(P, t):
    """The node-pair blocks tile t reduces into."""
    conn0, rs, up = P["conn0"], P["rs"], P["up"]
    bb = lambda n: n + (rs[n] - 6 * n) // 9
    out = set()
    for el in conn0[t * TILE:(t + 1) * TILE]:
        for i in range(8):
            for j in range(i, 8):
                A, B = int(el[i]), int(el[j])
                lo, hi = min(A, B), max(A, B)
                out.add(bb(lo) if A == B else bb(lo) + 1 + up[lo].index(hi))
    return out


def check_plan(P, seed=0):
    q, conv, T = P["queue"], P["conv"], P["T"]
    J = conv.shape[0]
    pos_tile = np.full(T, -1)
    pos_item = np.full(J, -1)
    for k, v in enumerate(q):
        if v >= 0:
            assert pos_tile[v] < 0
            pos_tile[v] = k
        else:
            assert pos_item[-v - 1] < 0
            pos_item[-v - 1] = k
    assert (pos_tile >= 0).all() and (pos_item >= 0).all()
    # items: contiguous node runs covering every node, rows within the staging buffer, nodes within
    # the item's node table
    assert conv[0, 0] == 0 and conv[-1, 1] == P["N"] and (conv[1:, 0] == conv[:-1, 1]).all()
    rs, nup = P["rs"], P["nup"]
    for n0, n1, t0, t1 in conv:
        L = (rs[n1 - 1] + 6 + 9 * nup[n1 - 1]) - rs[n0]
        assert L <= P["stage_max"] - 1
        assert 1 <= n1 - n0 <= P["max_nodes"]
    # tiles containing each node
    node_tiles = [[] for _ in range(P["N"])]
    for e, el in enumerate(P["conn0"]):
        for n in el:
            node_tiles[n].append(e // TILE)
    for j, (n0, n1, t0, t1) in enumerate(conv):
        ts = [t for n in range(n0, n1) for t in node_tiles[n]]
        assert min(ts) >= t0 and max(ts) <= t1
        assert pos_tile[t1] < pos_item[j]
    # slabs: tiles of slab c and the items finishing its node prefix lie in its queue range
    se, sn, sq = P["se"], P["sn"], P["slab_q"]
    for c in range(len(sn)):
        for t in range(se[c] // TILE, (se[c + 1] + TILE - 1) // TILE):
            assert sq[c] <= pos_tile[t] < sq[c + 1]
        for j, (n0, n1, _, _) in enumerate(conv):
            if n1 <= sn[c]:
                assert pos_item[j] < sq[c + 1]
    # ring safety and waits targeting earlier positions
    R = P["R"]
    assert R & (R - 1) == 0
    item_b0 = np.array([n0 + (rs[n0] - 6 * n0) // 9 for n0 in conv[:, 0]])
    for t in range(T):
        x, y = P["wait"][t]
        for j in range(x, y):
            assert pos_item[j] < pos_tile[t]
        for b in tile_blocks(P, t):
            if b - R >= 0:
                j = int(np.searchsorted(item_b0, b - R, side="right") - 1)
                assert x <= j < y, (t, b, j, x, y)
    # the queue drains under the kernel's protocol
    simulate(P, pos_tile, pos_item, workers=37, seed=seed)


def simulate(P, pos_tile, pos_item, workers, seed):
    q, conv, wait = P["queue"], P["conv"], P["wait"]
    rng = np.random.default_rng(seed)
    done = np.zeros(len(q), bool)
    deps = []
    for v in q:
        if v >= 0:
            x, y = wait[v]
            deps.append([pos_item[j] for j in range(x, y)])
        else:
            n0, n1, t0, t1 = conv[-v - 1]
            deps.append([pos_tile[t] for t in range(t0, t1 + 1)])
    ticket = 0
    held = []                                   # per worker: [cur, next, finish time or None]
    for _ in range(workers):
        cur = ticket if ticket < len(q) else None
        ticket += 1
        nxt = ticket if ticket < len(q) else None
        ticket += 1
        held.append([cur, nxt, None])
    now, steps = 0.0, 0
    while not done.all():
        steps += 1
        assert steps < 50 * len(q), "queue does not drain"
        progressed = False
        for w in held:
            if w[0] is not None and w[2] is None and all(done[d] for d in deps[w[0]]):
                w[2] = now + rng.uniform(0.5, 2.0)
                progressed = True
        running = [w for w in held if w[2] is not None]
        if not running:
            assert progressed, "every worker waits: deadlock"
            continue
        w = min(running, key=lambda r: r[2])
        now = w[2]
        done[w[0]] = True
        w[0], w[2] = w[1], None
        w[1] = ticket if ticket < len(q) else None
        ticket += 1


@pytest.mark.parametrize("case", ["cube", "plate", "shuffled"])
@pytest.mark.parametrize("ns", [1, 4])
def test_schedule_waits_ring_and_drain(planner, case, ns):
    if case == "cube":
        X, conn = meshgen.structured_box(12, 12, 12, jitter=0.05, seed=0)
    elif case == "plate":
        X, conn = meshgen.structured_box(16, 16, 8, lx=2.0, ly=2.0, jitter=0.05, seed=0)
    else:
        X, conn = meshgen.structured_box(9, 8, 7, jitter=0.05, seed=1)
        rng = np.random.default_rng(3)
        perm = rng.permutation(X.shape[0])
        Xn = np.empty_like(X)
        Xn[perm] = X
        X, conn = Xn, (perm[conn - 1] + 1)[rng.permutation(conn.shape[0])].astype(np.int32)
    # a small staging buffer (many conversion items) and a short slack (a small ring)
    P = plan(planner, X, conn, ns=ns, slack=3, stage_max=600, max_nodes=24)
    check_plan(P, seed=ns)


def test_schedule_ring_stays_small_on_a_swept_mesh(planner):
    """On a mesh numbered along a sweep, the ring holds a few layers of node rows, not the mesh."""
    X, conn = meshgen.structured_box(24, 24, 24, jitter=0.05, seed=0)
    P = plan(planner, X, conn, ns=1, slack=8)
    assert P["R"] < P["n_blocks"] / 2
    check_plan(P)


# ---- banded two-pass assembly (plan_bands) ----

@pytest.fixture(scope="module")
def band_planner(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("bands") / "libbands_test.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-DCEOS_SCHEDULE_TEST", SRC, "-o", so])
    f = C.CDLL(so).ceos_test_plan_bands
    f.restype = C.c_int
    return f


def plan_bands(f, X, conn, band_elems, depth=2, stage_max=7294, max_nodes=256):
    conn0 = np.ascontiguousarray(conn - 1, np.int32)
    N, E = X.shape[0], conn0.shape[0]
    rs, nup, up, n_blocks = pattern(N, conn0)
    nb_max = E // band_elems + 2
    band_e = np.zeros(nb_max, np.int32)
    node_end = np.zeros(nb_max, np.int32)
    conv = np.zeros(4 * N, np.int32)
    band_conv = np.zeros(nb_max, np.int32)
    counts = np.zeros(2, np.int32)
    ring = np.zeros(2, np.int64)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = f(N, E, p(conn0), p(rs), p(nup), C.c_longlong(n_blocks), band_elems, TILE, C.c_longlong(stage_max), max_nodes,
           depth, p(band_e), p(node_end), p(conv), p(band_conv), p(counts), p(ring))
    assert rc == 0
    nb, nc = counts
    return {"band_e": band_e[:nb + 1], "node_end": node_end[:nb], "conv": conv[:4 * nc].reshape(nc, 4),
            "band_conv": band_conv[:nb + 1], "R": int(ring[0]), "span": int(ring[1]), "conn0": conn0, "rs": rs,
            "nup": nup, "n_blocks": n_blocks, "N": N, "E": E, "depth": depth, "stage_max": stage_max,
            "max_nodes": max_nodes}


def check_bands(P):
    """Items cover every row once, band by band, with rows final after their band; at every moment of
    the pipeline (element bands c and c + 1 running, conversions done up to band c - depth) the blocks
    of the live rows occupy distinct ring slots."""
    be, ne, conv, bc = P["band_e"], P["node_end"], P["conv"], P["band_conv"]
    nb = len(ne)
    assert be[0] == 0 and be[-1] == P["E"] and all(b % TILE == 0 for b in be[:-1])
    assert (np.diff(ne) >= 0).all() and ne[-1] == P["N"]
    rs, nup, conn0 = P["rs"], P["nup"], P["conn0"]
    first, last = np.full(P["N"], nb), np.full(P["N"], -1)
    for c in range(nb):
        nodes = np.unique(conn0[be[c]:be[c + 1]])
        first[nodes] = np.minimum(first[nodes], c)
        last[nodes] = np.maximum(last[nodes], c)
    lo = 0
    for c in range(nb):
        items = conv[bc[c]:bc[c + 1]]
        if len(items):
            assert items[0, 0] == lo and items[-1, 1] == ne[c] and (items[1:, 0] == items[:-1, 1]).all()
        for n0, n1, _, _ in items:
            assert 1 <= n1 - n0 <= P["max_nodes"]
            assert rs[n1 - 1] + 6 + 9 * nup[n1 - 1] - rs[n0] <= P["stage_max"] - 1
            assert last[n0:n1].max() <= c  # no later band touches these rows
        lo = ne[c]
    R = P["R"]
    assert R & (R - 1) == 0
    bb = np.arange(P["N"]) + (rs - 6 * np.arange(P["N"])) // 9
    for c in range(nb):
        low = ne[c - P["depth"]] if c - P["depth"] >= 0 else 0
        live = [n for n in range(low, P["N"]) if first[n] <= min(c + 1, nb - 1)]
        blocks = np.concatenate([np.arange(bb[n], bb[n] + 1 + nup[n]) for n in live]) if live else np.zeros(0, int)
        slots = blocks % R
        assert len(np.unique(slots)) == len(slots), c


@pytest.mark.parametrize("depth", [2, 3])
@pytest.mark.parametrize("case,band_elems", [("cube", 128), ("plate", 256), ("plate", 64), ("shuffled", 96)])
def test_band_plan_items_and_ring(band_planner, case, band_elems, depth):
    if case == "cube":
        X, conn = meshgen.structured_box(12, 12, 12, jitter=0.05, seed=0)
    elif case == "plate":
        X, conn = meshgen.structured_box(16, 16, 8, lx=2.0, ly=2.0, jitter=0.05, seed=0)
    else:
        X, conn = meshgen.structured_box(9, 8, 7, jitter=0.05, seed=1)
        rng = np.random.default_rng(3)
        perm = rng.permutation(X.shape[0])
        Xn = np.empty_like(X)
        Xn[perm] = X
        X, conn = Xn, (perm[conn - 1] + 1)[rng.permutation(conn.shape[0])].astype(np.int32)
    P = plan_bands(band_planner, X, conn, band_elems, depth=depth, stage_max=600, max_nodes=24)
    check_bands(P)


def test_band_ring_stays_small_on_a_swept_mesh(band_planner):
    """On a mesh numbered along a sweep the band ring holds a few bands of node rows, not the mesh
    (the live span; the ring is that span rounded up to a power of two)."""
    X, conn = meshgen.structured_box(24, 24, 24, jitter=0.05, seed=0)
    P = plan_bands(band_planner, X, conn, band_elems=24 * 24 * 2, depth=3)
    rmax = 1 << int(np.ceil(np.log2(P["n_blocks"])))
    assert P["span"] <= P["n_blocks"] / 2 and P["R"] < rmax
    check_bands(P)


# ---- item bounds of the bulk-copy conversion pass (csr_convert_kernel) ----

def _bulk_limits():
    """kBulkNodes, kBulkStage and kBulkBlocks as the kernel header defines them."""
    import re
    src = open(os.path.join(ROOT, "ceos-eems_b200", "csrc", "element_kernel.cuh")).read()
    nodes = int(re.search(r"constexpr int kBulkNodes = (\d+);", src).group(1))
    stage = int(re.search(r"constexpr int kBulkStage = (\d+);", src).group(1))
    assert "constexpr int kBulkBlocks = kBulkNodes + kBulkStage / 9 + 1;" in src
    return nodes, stage, nodes + stage // 9 + 1


def _check_bulk_items(P, nodes_max, stage_max, blocks_max):
    rs, nup = P["rs"], P["nup"]
    bb = np.arange(P["N"]) + (rs - 6 * np.arange(P["N"])) // 9
    for n0, n1, _, _ in P["conv"]:
        nval = rs[n1 - 1] + 6 + 9 * nup[n1 - 1] - rs[n0]
        nblk = bb[n1 - 1] + 1 + nup[n1 - 1] - bb[n0]
        assert 1 <= n1 - n0 <= nodes_max
        assert nval <= stage_max - 1  # the staging holds the values and one alignment slot
        assert nblk <= blocks_max     # one block buffer holds the item's blocks
        assert nblk * 48 % 16 == 0


@pytest.mark.parametrize("case", ["cube", "plate", "shuffled"])
def test_conversion_items_fit_the_bulk_buffers(planner, band_planner, case):
    """Items planned with the conversion kernel's limits (two-pass items from plan_schedule, banded
    items from plan_bands) fit its shared-memory buffers: at most kBulkNodes nodes, kBulkStage - 1 K
    values and kBulkBlocks node-pair blocks, the bounds the kernel checks before each bulk copy."""
    nodes_max, stage_max, blocks_max = _bulk_limits()
    if case == "cube":
        X, conn = meshgen.structured_box(14, 14, 14, jitter=0.05, seed=0)
    elif case == "plate":
        X, conn = meshgen.structured_box(24, 24, 6, lx=2.0, ly=2.0, jitter=0.05, seed=0)
    else:
        X, conn = meshgen.structured_box(9, 8, 7, jitter=0.05, seed=1)
        rng = np.random.default_rng(5)
        perm = rng.permutation(X.shape[0])
        Xn = np.empty_like(X)
        Xn[perm] = X
        X, conn = Xn, (perm[conn - 1] + 1)[rng.permutation(conn.shape[0])].astype(np.int32)
    P = plan(planner, X, conn, ns=2, stage_max=stage_max, max_nodes=nodes_max)
    _check_bulk_items(P, nodes_max, stage_max, blocks_max)
    B = plan_bands(band_planner, X, conn, band_elems=128, depth=3, stage_max=stage_max, max_nodes=nodes_max)
    _check_bulk_items(B, nodes_max, stage_max, blocks_max)
