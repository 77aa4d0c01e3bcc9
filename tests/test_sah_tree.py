"""The surface-area inner tree: host build invariants and edge cases (CPU),
and the device build at scene upload against the host build, bit for bit
(GPU).

The tree is rebuilt over the leaves of the reference's BVH (BVH::createBinary,
Src/bvh.cpp:283-314, flattened by Src/meshmapping.cpp:62-125); what makes a
traversal's results independent of it is covered by the traversal parity
tests.  Here: every leaf appears once with its own box and triangle count,
every inner box is the union of its children, the depth is the deepest leaf,
and the device's records equal the host's.
"""
import numpy as np
import pytest

from fornos_b200 import api
from tests import cases


def flat_nodes(lo, hi, tris):
    """Flattened skip-pointer node array (Src/meshmapping.cpp:62-125 layout)
    of a balanced binary tree over leaf boxes lo / hi (n x 3), leaves in the
    given order, leaf i holding tris[i] triangles."""
    lo = np.asarray(lo, np.float32)
    hi = np.asarray(hi, np.float32)
    n = len(lo)
    out = np.zeros(2 * n - 1, api.NODE_DTYPE)
    state = {"node": 0, "corner": 0}

    def emit(a, b):
        i = state["node"]
        state["node"] += 1
        if b - a == 1:
            s = state["corner"]
            state["corner"] += 3 * int(tris[a])
            out[i] = (lo[a], hi[a], s, state["corner"], i + 1)
            return
        m = (a + b) // 2
        emit(a, m)
        emit(m, b)
        out[i] = (lo[a:b].min(0), hi[a:b].max(0), 0, 0, state["node"])

    emit(0, n)
    return out, state["corner"]


def random_leaves(rng, n, spread=100.0, size=1.0):
    c = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    e = rng.uniform(0.01, size, (n, 3)).astype(np.float32)
    return c - e, c + e, rng.integers(1, 9, n)


def check_tree(nodes, rec, depth):
    """Structural invariants of a 2-wide record array over the leaves of
    `nodes`; returns the number of leaves reached."""
    leaf_idx = np.nonzero(nodes["jump"] == np.arange(1, len(nodes) + 1))[0]
    ints = rec.view(np.int32)
    seen_leaf = np.zeros(len(nodes), np.int64)
    seen_rec = np.zeros(len(rec), np.int64)

    def child(r, s):
        lo = np.array([rec[r, 4 * s + 0], rec[r, 4 * s + 2], rec[r, 8 + 2 * s]], np.float32)
        hi = np.array([rec[r, 4 * s + 1], rec[r, 4 * s + 3], rec[r, 9 + 2 * s]], np.float32)
        return lo, hi, int(ints[r, 12 + s]), int(ints[r, 14 + s])

    deepest = 0
    stack = [(0, 1)]
    while stack:
        r, level = stack.pop()
        seen_rec[r] += 1
        for s in (0, 1):
            lo, hi, ref, cnt = child(r, s)
            if ref < 0:
                f = -ref - 1
                seen_leaf[f] += 1
                nd = nodes[f]
                assert np.array_equal(lo.view(np.uint32), nd["lo"].view(np.uint32))
                assert np.array_equal(hi.view(np.uint32), nd["hi"].view(np.uint32))
                assert cnt == (nd["end"] - nd["start"]) // 3
                deepest = max(deepest, level + 1)
            else:
                assert cnt == 0 and 0 < ref < len(rec)
                l0, h0, _, _ = child(ref, 0)
                l1, h1, _, _ = child(ref, 1)
                assert np.array_equal(lo, np.minimum(l0, l1)) and np.array_equal(hi, np.maximum(h0, h1))
                stack.append((ref, level + 1))
    assert np.all(seen_rec == 1)
    assert np.array_equal(np.nonzero(seen_leaf)[0], leaf_idx) and np.all(seen_leaf[leaf_idx] == 1)
    assert deepest == depth
    return len(leaf_idx)


# ------------------------------------------------------------------ host (CPU)
@pytest.mark.parametrize("name", ["sphere", "plane", "icosphere"])
def test_host_tree_invariants_on_cases(lib, name):
    c = getattr(cases, name)()
    rec, depth = api.sah_tree_host(c.nodes)
    leaves = check_tree(c.nodes, rec, depth)
    assert len(rec) == leaves - 1 and 2 <= depth <= 48


def test_host_tree_invariants_random(lib):
    rng = np.random.default_rng(11)
    lo, hi, tris = random_leaves(rng, 3000)
    nodes, _ = flat_nodes(lo, hi, tris)
    rec, depth = api.sah_tree_host(nodes)
    assert check_tree(nodes, rec, depth) == 3000


def test_host_tree_no_plane_splits_in_flat_order(lib):
    # identical boxes: no candidate plane, every node takes its first half
    n = 11
    lo = np.zeros((n, 3), np.float32)
    hi = np.ones((n, 3), np.float32)
    nodes, _ = flat_nodes(lo, hi, np.full(n, 2))
    rec, depth = api.sah_tree_host(nodes)
    check_tree(nodes, rec, depth)
    ints = rec.view(np.int32)
    leaves = [int(-r - 1) for r in ints[:, 12:14].ravel() if r < 0]
    # the root's left subtree holds the first n // 2 leaves in flattened order
    first = []
    stack = [int(ints[0, 12])]
    while stack:
        r = stack.pop()
        if r < 0:
            first.append(-r - 1)
        else:
            stack += [int(ints[r, 12]), int(ints[r, 13])]
    leaf_idx = np.nonzero(nodes["jump"] == np.arange(1, len(nodes) + 1))[0]
    assert sorted(first) == list(leaf_idx[: n // 2])
    assert sorted(leaves) == list(leaf_idx)


def test_host_tree_signed_zero_merges_to_the_lower(lib):
    lo = np.array([[0.0, 0, 0], [-0.0, 0, 0], [5, 5, 5]], np.float32)
    hi = np.array([[1.0, 1, 1], [1, 1, 1], [6, 6, 6]], np.float32)
    lo[0, 0] = 0.0
    lo[1, 0] = -0.0
    nodes, _ = flat_nodes(lo, hi, [1, 1, 1])
    rec, depth = api.sah_tree_host(nodes)
    check_tree(nodes, rec, depth)
    ints = rec.view(np.int32)
    # the two boxes at the origin share a subtree; its x lower bound is -0
    side = 0 if ints[0, 12] >= 0 else 1
    assert ints[0, 12 + side] > 0
    assert np.signbit(rec[0, 4 * side]) and rec[0, 4 * side] == 0.0


@pytest.mark.parametrize("bad", [np.nan, np.inf, 1e30, -2e30])
def test_host_tree_out_of_range_boxes_get_no_tree(lib, bad):
    rng = np.random.default_rng(5)
    lo, hi, tris = random_leaves(rng, 20)
    lo[7, 1] = bad
    nodes, _ = flat_nodes(lo, hi, tris)
    rec, depth = api.sah_tree_host(nodes)
    assert len(rec) == 0 and depth == 0


def test_host_tree_single_leaf(lib):
    nodes, _ = flat_nodes([[0, 0, 0]], [[1, 1, 1]], [3])
    rec, depth = api.sah_tree_host(nodes)
    assert len(rec) == 0 and depth == 1


@pytest.mark.parametrize("kind", ["deep_chain", "deep_chain_large"])
def test_host_tree_deep_chains_exceed_the_ordered_depth(lib, kind):
    lo, hi, tris = _synthetic(kind, None)
    nodes, _ = flat_nodes(lo, hi, tris)
    rec, depth = api.sah_tree_host(nodes)
    assert depth > 48 and check_tree(nodes, rec, depth) == len(lo)


def test_host_tree_rejects_malformed(lib):
    nodes, _ = flat_nodes([[0, 0, 0], [1, 1, 1]], [[1, 1, 1], [2, 2, 2]], [1, 1])
    nodes["jump"][1] = 0
    with pytest.raises(api.FornosError):
        api.sah_tree_host(nodes)


# ------------------------------------------------------------------ device (GPU)
def _scene_from(ctx, nodes, corners, rng):
    pos4 = np.zeros((corners, 4), np.float32)
    pos4[:, :3] = rng.uniform(-1, 1, (corners, 3))
    nrm4 = np.zeros((corners, 4), np.float32)
    nrm4[:, 2] = 1.0
    return api.Scene(ctx, nodes, pos4, nrm4)


def _same_tree(ctx, scene, nodes):
    dev, ddepth = scene.tree(api.TREE_SAH)
    host, hdepth = api.sah_tree_host(nodes)
    if hdepth > 48:
        assert len(dev) == 0
        return
    assert ddepth == hdepth
    assert dev.shape == host.shape
    assert np.array_equal(dev.view(np.uint32), host.view(np.uint32))


def _synthetic(kind, rng):
    if kind == "random_small":
        return random_leaves(rng, 200)
    if kind == "random_large":
        return random_leaves(rng, 60000)
    if kind == "clustered":
        lo, hi, t = random_leaves(rng, 20000, spread=1.0, size=0.01)
        lo[::7] *= 1000
        hi[::7] *= 1000
        return np.minimum(lo, hi), np.maximum(lo, hi), t
    if kind == "identical_large":
        n = 5000
        return np.zeros((n, 3), np.float32), np.ones((n, 3), np.float32), np.full(n, 4)
    if kind == "flat_plane":
        # zero-extent boxes in z: surface-area candidates with zero area
        lo, hi, t = random_leaves(rng, 4000)
        lo[:, 2] = 0.0
        hi[:, 2] = 0.0
        return lo, hi, t
    if kind == "points":
        # zero-volume boxes: no candidate has a non-zero cost, every split is the fallback
        lo, _, t = random_leaves(rng, 1000)
        return lo, lo.copy(), t
    if kind == "signed_zero":
        lo, hi, t = random_leaves(rng, 3000, spread=1.0)
        lo[::3, 0] = -0.0
        lo[1::3, 0] = 0.0
        return lo, np.maximum(hi, lo), t
    if kind in ("deep_chain", "deep_chain_large"):
        # centres +-32^e (the bin count as ratio): each split isolates one
        # extreme, so the tree is deeper than the ordered traversals accept
        # (58 levels over 86 leaves; 61 over 688, the level passes reaching
        # level 48 with more than 256 leaves left)
        reps = 1 if kind == "deep_chain" else 8
        e = np.arange(-24, 19).astype(np.float64)
        c = np.repeat(np.concatenate([32.0 ** e, -(32.0 ** e)]), reps)
        h = np.abs(c) * 0.01
        lo = np.repeat((c - h)[:, None], 3, 1).astype(np.float32)
        hi = np.repeat((c + h)[:, None], 3, 1).astype(np.float32)
        return lo, hi, np.ones(len(c), np.int64)
    raise KeyError(kind)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["sphere", "plane", "icosphere"])
def test_device_tree_equals_host_on_cases(ctx, name):
    c = getattr(cases, name)()
    scene = api.Scene(ctx, c.nodes, c.pos4, c.nrm4)
    _same_tree(ctx, scene, c.nodes)


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["random_small", "random_large", "clustered", "identical_large", "flat_plane",
                                  "points", "signed_zero", "deep_chain", "deep_chain_large"])
def test_device_tree_equals_host_synthetic(ctx, kind):
    rng = np.random.default_rng(sum(map(ord, kind)))
    lo, hi, tris = _synthetic(kind, rng)
    nodes, corners = flat_nodes(lo, hi, tris)
    scene = _scene_from(ctx, nodes, corners, rng)
    _same_tree(ctx, scene, nodes)


@pytest.mark.gpu
def test_device_tree_out_of_range_falls_back_to_reference(ctx):
    rng = np.random.default_rng(3)
    lo, hi, tris = random_leaves(rng, 500)
    hi[17, 0] = 1e31
    nodes, corners = flat_nodes(lo, hi, tris)
    scene = _scene_from(ctx, nodes, corners, rng)
    rec, _ = scene.tree(api.TREE_SAH)
    assert len(rec) == 0
    ref, _ = scene.tree(api.TREE_REFERENCE)
    assert len(ref) == 499
    with pytest.raises(api.FornosError):
        scene.set_tree(api.TREE_SAH)
