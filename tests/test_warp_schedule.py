"""The per-warp schedule of row groups (scl_gpu_warp_schedule) that the SpMM
plan kinds 9, 10, 12 and 14 follow on a reordered graph. Host only, so these
run without a GPU: the lists are checked against a NumPy/heapq restatement of
the dealing rule, for coverage, list order and the greedy balance bound. The
GPU parity tests check that a scheduled SpMM returns the same bits as the
oracle."""
import ctypes
import heapq

import numpy as np
import pytest

import scl.gpu as G
from scl._bindings._loader import get_library


def restated(indptr, R, nw):
    """Groups over eight times the mean row length first (longest first, stable),
    each to the least-loaded warp (ties: lowest warp), then the others in index
    order; cost = longest row + 8. Lists hold long groups first, then the rest."""
    ip = np.asarray(indptr, np.int64)
    n = ip.size - 1
    ng = (n + R - 1) // R
    lens = np.diff(ip)
    glen = [int(lens[g * R:min(n, g * R + R)].max()) if n else 0 for g in range(ng)]
    mean = max(1, (int(ip[n] - ip[0]) + n - 1) // max(n, 1))
    thr = 8 * mean
    hubs = sorted([g for g in range(ng) if glen[g] > thr], key=lambda g: -glen[g])
    heap = [(0, w) for w in range(nw)]
    heapq.heapify(heap)
    owner = [0] * ng
    load = [0] * nw

    def deal(g):
        t, w = heapq.heappop(heap)
        owner[g] = w
        load[w] = t + glen[g] + 8
        heapq.heappush(heap, (load[w], w))

    hubset = set(hubs)
    for g in hubs:
        deal(g)
    for g in range(ng):
        if g not in hubset:
            deal(g)
    lists = [[] for _ in range(nw)]
    for g in hubs:
        lists[owner[g]].append(g)
    for g in range(ng):
        if g not in hubset:
            lists[owner[g]].append(g)
    offs = np.zeros(nw + 1, np.int64)
    offs[1:] = np.cumsum([len(x) for x in lists])
    flat = np.array([g for x in lists for g in x], np.int64)
    return offs, flat, glen, hubset, load


def heavy_tailed(n, seed):
    rng = np.random.default_rng(seed)
    lens = rng.poisson(40, n)
    hub = rng.choice(n, max(1, n // 200), replace=False)
    lens[hub] = rng.integers(400, 3000, hub.size)  # a few long rows, as in a kNN union graph
    lens[rng.choice(n, n // 50, replace=False)] = 0  # and some empty ones
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)


@pytest.mark.parametrize("n,R,nw,seed", [(20000, 2, 2368, 1), (20000, 1, 296, 2), (9999, 4, 148, 3),
                                         (5000, 2, 64, 4), (7, 4, 16, 5), (1, 1, 1, 6)])
def test_schedule_matches_restatement_and_covers_every_group(n, R, nw, seed):
    ip = heavy_tailed(n, seed)
    offs, groups = G.warp_schedule(ip, R, nw)
    want_offs, want_groups, glen, hubs, load = restated(ip, R, nw)
    assert np.array_equal(offs, want_offs)
    assert np.array_equal(groups, want_groups)
    ng = (n + R - 1) // R
    assert offs[0] == 0 and offs[-1] == ng and np.all(np.diff(offs) >= 0)
    assert np.array_equal(np.sort(groups), np.arange(ng))  # every group exactly once
    for w in range(nw):
        lst = groups[offs[w]:offs[w + 1]].tolist()
        k = sum(1 for g in lst if g in hubs)
        assert all(g in hubs for g in lst[:k])  # long groups first ...
        assert [glen[g] for g in lst[:k]] == sorted((glen[g] for g in lst[:k]), reverse=True)
        assert lst[k:] == sorted(lst[k:])  # ... then the others by index
    # greedy list scheduling: no warp ends more than one group's cost above the mean
    cost = np.array(glen) + 8
    assert max(load) <= cost.sum() / nw + cost.max()


def test_schedule_spreads_the_long_groups():
    ip = heavy_tailed(40000, 7)
    nw = 512
    offs, groups = G.warp_schedule(ip, 2, nw)
    _, _, glen, hubs, _ = restated(ip, 2, nw)
    assert len(hubs) > 0
    first = [groups[offs[w]] for w in range(nw) if offs[w + 1] > offs[w]]
    # with fewer long groups than warps, each long group leads its own warp's list
    assert len(hubs) < nw and sorted(g for g in first if g in hubs) == sorted(hubs)


def test_empty_graph_and_more_warps_than_groups():
    offs, groups = G.warp_schedule(np.zeros(1, np.int64), 2, 8)
    assert np.array_equal(offs, np.zeros(9)) and groups.size == 0
    ip = np.array([0, 5, 9, 9], np.int64)
    offs, groups = G.warp_schedule(ip, 1, 10)
    assert offs[-1] == 3 and sorted(groups.tolist()) == [0, 1, 2]


def test_schedule_errors():
    lib = get_library("f32_i32")
    ip = np.array([0, 3, 5], np.int64)
    out = np.empty(2 + 1 + 2, np.int32)
    p = ctypes.c_void_p
    args = lambda R=1, nw=2, ln=out.size, ipa=ip: (p(ipa.ctypes.data), 2, R, nw, p(out.ctypes.data), ln)
    assert lib.scl_gpu_warp_schedule(*args()) == 0
    assert lib.scl_gpu_warp_schedule(*args(R=3)) != 0  # groups of 1, 2 or 4 rows
    assert lib.scl_gpu_warp_schedule(*args(nw=0)) != 0
    assert lib.scl_gpu_warp_schedule(*args(ln=out.size - 1)) != 0  # wrong output length
    assert lib.scl_gpu_warp_schedule(*args(ipa=np.array([0, 3, 1], np.int64))) != 0  # decreasing offsets
    assert lib.scl_gpu_warp_schedule(None, 2, 1, 2, p(out.ctypes.data), out.size) != 0
    assert lib.scl_gpu_warp_schedule(p(ip.ctypes.data), 2, 1, 2, None, out.size) != 0
