"""IsolatedLandscape's landscape decompositions (CPU): the backend's
necsim_subdomain_ranks against an independent Python restatement of
decomposition/{modulo,radial,equal/{mod,weight}}.rs, and the properties the
reference's own equal/test.rs asserts."""
import math
import random

import numpy as np
import pytest

M32 = 0xFFFFFFFF


def lineages(points):
    from importlib import import_module
    nb = import_module("necsim-rust_b200")
    a = np.zeros(len(points), dtype=nb.LINEAGE_DTYPE)
    for j, (x, y) in enumerate(points):
        a[j]["x"], a[j]["y"] = x, y
    return a


def modulo_rank(x, y, width, size):
    return (y * width + x) % size


def radial_rank(x, y, size):
    half = 1 << 31
    fraction = math.atan2(float(y - half), float(x - half)) * float("0.318309886183790671537767526745028724") \
        * 0.5 + 0.5
    return min(int(math.floor(size * fraction)), size - 1)


def morton(mx, my, dx, dy):
    m, both = 0, min(mx, my)
    for b in range(both):
        m |= (dx & 1) << (b * 2)
        dx >>= 1
        m |= (dy & 1) << (b * 2 + 1)
        dy >>= 1
    mx, my = mx - both, my - both
    if mx > 0:
        m |= dx << (both * 2)
    if my > 0:
        m |= dy << (both * 2 + mx)
    return m


def next_log2(n):
    return int(math.ceil(math.log(float(n)) / float("0.693147180559945309417232121458176568"))) if n > 1 else 0


def equal_weight(habitat, size):
    """EqualDecomposition::weight: (rank of each habitable cell, exact)."""
    h, w = habitat.shape
    mx, my = next_log2(w), next_log2(h)
    cells = sorted((morton(mx, my, x, y), int(habitat[y, x])) for y in range(h) for x in range(w) if habitat[y, x])
    total = sum(c[1] for c in cells)
    cum, last, idx = 0, 0, []
    for m, hv in cells:
        nxt = cum * size // total
        cum += hv
        if nxt != last:
            last = nxt
            idx.append(m)

    def rank(x, y):
        import bisect
        m = morton(mx, my, x, y)
        i = bisect.bisect_left(idx, m)
        return i + 1 if i < len(idx) and idx[i] == m else i
    return rank, len(idx) + 1 == size


def test_modulo_and_radial_match_restatement(nb):
    rnd = random.Random(5)
    pts = [(rnd.randrange(1 << 32), rnd.randrange(1 << 32)) for _ in range(3000)]
    pts += [(0, 0), (M32, M32), (1 << 31, 1 << 31), ((1 << 31) - 1, 1 << 31), (0, M32)]
    lin = lineages(pts)
    for size in (1, 2, 3, 7, 64, 1000):
        si = nb.SpatiallyImplicit((4, 4), 2, (8, 8), 1, 0.1)
        ranks, exact = nb.subdomain_ranks(si, size, lin)
        assert exact and ranks.tolist() == [modulo_rank(x, y, 1 << 32, size) for x, y in pts]
        for sample in (nb.Circle(5), nb.Rectangle((0, 0), 3, 3)):
            ai = nb.AlmostInfinite(sample, nb.Normal(2.0))
            ranks, _ = nb.subdomain_ranks(ai, size, lin)
            assert ranks.tolist() == [radial_rank(x, y, size) for x, y in pts]
        wn = nb.WrappingNoise(0, 0.5, 0.07, 0.5, 2, nb.Rectangle((0, 0), 2, 2), 1.0)
        assert nb.subdomain_ranks(wn, size, lin)[0].tolist() == [radial_rank(x, y, size) for x, y in pts]
    ns_pts = [(x, y) for y in range(7) for x in range(13)]
    ranks, _ = nb.subdomain_ranks(nb.NonSpatial((13, 7), 3), 5, lineages(ns_pts))
    assert ranks.tolist() == [modulo_rank(x, y, 13, 5) for x, y in ns_pts]


@pytest.mark.parametrize("w,h", [(1, 1), (5, 3), (8, 8), (13, 7), (33, 17)])
def test_equal_weight_matches_restatement(nb, w, h):
    rnd = np.random.default_rng(w * 100 + h)
    habitat = rnd.integers(0, 5, size=(h, w)).astype(np.uint32)
    habitat[0, 0] = 1
    se = nb.SpatiallyExplicit(habitat, np.ones((w * h, w * h)))  # the decomposition reads no dispersal
    pts = [(x, y) for y in range(h) for x in range(w) if habitat[y, x]]
    for size in (1, 2, 3, 6, 17, int(habitat.sum()) + 1):
        ranks, exact = nb.subdomain_ranks(se, size, lineages(pts))
        rank, ok = equal_weight(habitat, size)
        assert exact == ok and ranks.tolist() == [rank(x, y) for x, y in pts], size


@pytest.mark.parametrize("w", range(1, 9))
@pytest.mark.parametrize("h", range(1, 9))
def test_equal_area_properties(nb, w, h):
    """equal/test.rs:19-95 test_equal_area_decomposition on habitat 1 everywhere
    (weight == area): exactly `partition` ranks when it succeeds, else one
    rank per cell; every rank in [0, n) used; frequencies differ by <= 1."""
    habitat = np.ones((h, w), dtype=np.uint32)
    se = nb.SpatiallyExplicit(habitat, np.ones((w * h, w * h)))
    lin = lineages([(x, y) for y in range(h) for x in range(w)])
    for partition in range(1, w * h + 2):
        ranks, exact = nb.subdomain_ranks(se, partition, lin)
        freq = np.bincount(ranks)
        n = len(freq)
        if exact:
            assert n == partition
        else:
            assert 0 < n < partition and n == w * h
        assert (freq > 0).all()
        assert freq.max() - freq.min() <= 1


@pytest.mark.parametrize("local", [1, 3, 8])
@pytest.mark.parametrize("meta", [1, 2, 8])
def test_equal_weight_properties(nb, local, meta):
    """equal/test.rs:97-175 test_equal_weight_decomposition's properties on an
    8 x 2 map whose rows hold `local` and `meta` individuals per cell."""
    habitat = np.array([[local] * 8, [meta] * 8], dtype=np.uint32)
    se = nb.SpatiallyExplicit(habitat, np.ones((16, 16)))
    pts = [(x, y) for y in range(2) for x in range(8)]
    lin = lineages(pts)
    for partition in range(1, local * 8 + meta * 8 + 2):
        ranks, exact = nb.subdomain_ranks(se, partition, lin)
        weight = np.bincount(ranks, weights=[habitat[y, x] for x, y in pts])
        n = len(weight)
        if exact:
            assert n == partition
        else:
            assert 0 < n < partition
        assert (weight > 0).all()
        assert weight.max() - weight.min() <= max(local, meta) * 2


def test_invalid_size_is_rejected(nb):
    with pytest.raises(nb.NecsimError):
        nb.subdomain_ranks(nb.NonSpatial((3, 3), 1), 0, lineages([(0, 0)]))
