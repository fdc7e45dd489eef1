"""Friends-of-friends groups (tg_find_groups, tg_group_catalog) against the
oracle: the oracle's fast partition is pinned to the literal restatement of
the reference's label propagation (src/part_vect.cpp:85-124) on the CPU; the
GPU partition must equal the oracle's exactly (group ids included), and the
catalogue must agree within rounding."""
import numpy as np
import pytest

import fof as ofof


def _planted(n, seed, periodic=True):
    """Uniform particles plus planted cases: a duplicate pair (separation 0, never
    friends of each other), a pair at d2 = (L-1)^2 (friends) and one at exactly
    L2 (not), a chain through the x = +-1/2 face, and four dense clumps of 40."""
    rng = np.random.default_rng(seed)
    x = rng.integers(-2 ** 31, 2 ** 31, size=(n, 3), dtype=np.int64)
    L, L2 = ofof.link_int(n, 0.2)
    x[:6] //= 2  # away from the faces
    x[1] = x[0]
    x[3] = x[2]
    x[3, 0] += L - 1
    x[5] = x[4]
    x[5, 1] += L
    if periodic:
        x[6] = [2 ** 31 - L // 3, 0, 0]
        x[7] = [-2 ** 31 + L // 3, 0, 0]
        x[8] = [-2 ** 31 + L, 0, 0]
    for c in range(4):
        base = np.array([-2 ** 30 + c * 2 ** 29, c * 2 ** 28, -c * 2 ** 28])
        k = slice(16 + 40 * c, 16 + 40 * (c + 1))
        x[k] = base + rng.integers(-L // 2, L // 2, size=(40, 3))
    return ((x + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_partition_matches_literal_propagation(periodic, seed):
    x = _planted(400, seed, periodic)
    lit = ofof.propagate_labels(x, 0.2, periodic)
    fast = ofof.groups(x, 0.2, periodic)
    assert np.array_equal(lit, fast)
    L, L2 = ofof.link_int(len(x), 0.2)
    assert ofof._d2(x[2], x[3], periodic) < L2 and ofof._d2(x[4], x[5], periodic) == L2
    assert ofof._d2(x[0], x[1], periodic) == 0
    assert fast[2] == fast[3] == 2
    if periodic:
        assert fast[6] == fast[7] == fast[8] == 6
    sizes = np.bincount(fast[fast >= 0])
    assert (sizes >= 40).sum() == 4


def test_oracle_catalog_small():
    x = _planted(400, 3)
    g = ofof.groups(x, 0.2)
    v = np.random.default_rng(5).standard_normal((400, 3)).astype(np.float32)
    c = ofof.catalog(x, v, g, a=0.5)
    assert (np.diff(c["id"]) > 0).all() and c["N"].sum() == (g >= 0).sum()
    assert ((c["x"] >= 0) & (c["x"] <= 1)).all() and (c["rc"] <= c["rmax"]).all()


# ---------------------------------------------------------------- GPU -------


def _solver(n, ewald=True, leaf_max=None):
    from tigergrav_b200.solver import GravitySolver
    kw = {} if leaf_max is None else dict(leaf_max=leaf_max)
    return GravitySolver(n, theta=0.7, ewald=ewald, **kw)


@pytest.mark.gpu
@pytest.mark.parametrize("periodic", [True, False])
def test_fof_planted_matches_oracle(periodic):
    x = _planted(4096, 7, periodic)
    ref = ofof.groups(x, 0.2, periodic)
    with _solver(len(x), ewald=periodic) as s:
        s.set_particles(x)
        g = s.find_groups(0.2)
    assert np.array_equal(g, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("link", [0.1, 0.2, 0.28])
def test_fof_clustered_matches_oracle(link):
    from tigergrav_b200 import ics
    x = ics.halos(32 ** 3)
    ref = ofof.groups(x, link)
    with _solver(len(x)) as s:
        s.set_particles(x).solve_gravity()  # groups on the tree the force solve built
        g = s.find_groups(link)
    assert (ref >= 0).sum() > 3000
    assert np.array_equal(g, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("leaf_max", [1, 8, 64])
def test_fof_leaf_sizes(leaf_max):
    from tigergrav_b200 import ics
    x = ics.halos(16 ** 3, seed=9)
    ref = ofof.groups(x, 0.2)
    with _solver(len(x), leaf_max=leaf_max) as s:
        s.set_particles(x)
        assert np.array_equal(s.find_groups(0.2), ref)


@pytest.mark.gpu
def test_fof_catalog_matches_oracle():
    from tigergrav_b200 import ics
    x = ics.halos(32 ** 3, seed=4)
    v = np.random.default_rng(11).standard_normal((len(x), 3)).astype(np.float32)
    a = 0.25
    g_ref = ofof.groups(x, 0.2)
    ref = ofof.catalog(x, v, g_ref, a=a)
    from tigergrav_b200.solver import GravitySolver
    with GravitySolver(len(x), theta=0.7) as s:
        s.set_particles(x, v)
        g = s.find_groups(0.2)
        c = s.group_catalog(a)
    assert np.array_equal(g, g_ref)
    assert np.array_equal(c["id"], ref["id"]) and np.array_equal(c["N"], ref["N"])
    dx = np.abs(c["x"] - ref["x"])
    dx = np.minimum(dx, 1.0 - dx)
    assert dx.max() < 1e-9
    assert np.allclose(c["v"], ref["v"], rtol=1e-5, atol=1e-6)
    assert np.allclose(c["dv"], ref["dv"], rtol=1e-5, atol=1e-6)
    assert np.allclose(c["rmax"], ref["rmax"], rtol=1e-5, atol=1e-9)
    assert np.allclose(c["rc"], ref["rc"], rtol=1e-5, atol=1e-9)


@pytest.mark.gpu
def test_fof_edges(tmp_path):
    from tigergrav_b200 import _lib
    from tigergrav_b200.solver import GravitySolver
    # one particle: no friends, no groups
    with GravitySolver(1, theta=0.7) as s:
        s.set_particles(np.zeros((1, 3), np.int32))
        assert s.find_groups(0.2).tolist() == [-1]
        assert len(s.group_catalog()["id"]) == 0
    # every particle on one point: separation 0 links nobody
    with GravitySolver(64, theta=0.7, leaf_max=64) as s:
        s.set_particles(np.full((64, 3), 12345, np.int32))
        assert (s.find_groups(0.2) == -1).all()
        # linking length of half the box or more is refused
        with pytest.raises(_lib.TGError):
            s.find_groups(2.0)
        # the catalogue belongs to the tree it was found on
        s.drift(0.0)
        with pytest.raises(_lib.TGError):
            s.group_catalog()
    x = _planted(2048, 12)
    with GravitySolver(len(x), theta=0.7) as s:
        s.set_particles(x)
        s.find_groups(0.2)
        k = s.groups_output(tmp_path / "groups.0.0.dat", min_size=10)
        lines = (tmp_path / "groups.0.0.dat").read_text().splitlines()
    assert k == 4 and len(lines) == 4 and int(lines[0].split()[1]) >= 10


@pytest.mark.gpu
def test_fof_full_size_partition_and_catalog():
    """128^3 particles (the bench's size): the partition equals the oracle's;
    the catalogue covers every grouped particle once, ids ascending."""
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.halos(128 ** 3)
    ref = ofof.groups(x, 0.2)
    with GravitySolver(len(x), theta=0.7) as s:
        s.set_particles(x)
        g = s.find_groups(0.2)
        c = s.group_catalog(1.0)
    assert np.array_equal(g, ref)
    ids, cnt = np.unique(ref[ref >= 0], return_counts=True)
    assert np.array_equal(c["id"], ids) and np.array_equal(c["N"], cnt)
    assert (c["rc"] <= c["rmax"]).all() and (c["rc"] >= 0).all()


@pytest.mark.gpu
def test_fof_catalog_64cubed_matches_oracle():
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import GravitySolver
    x = ics.halos(64 ** 3, seed=6)
    v = np.random.default_rng(2).standard_normal((len(x), 3)).astype(np.float32)
    g_ref = ofof.groups(x, 0.2)
    ref = ofof.catalog(x, v, g_ref, a=0.5)
    with GravitySolver(len(x), theta=0.7) as s:
        s.set_particles(x, v)
        assert np.array_equal(s.find_groups(0.2), g_ref)
        c = s.group_catalog(0.5)
    assert np.array_equal(c["id"], ref["id"]) and np.array_equal(c["N"], ref["N"])
    dx = np.abs(c["x"] - ref["x"])
    assert np.minimum(dx, 1.0 - dx).max() < 1e-9
    assert np.allclose(c["dv"], ref["dv"], rtol=1e-5, atol=1e-6)
    assert np.allclose(c["rmax"], ref["rmax"], rtol=1e-5, atol=1e-9)
    assert np.allclose(c["rc"], ref["rc"], rtol=1e-5, atol=1e-9)


# ---- the partition against the reference's own find_groups -----------------
# (src/tree.cpp + src/part_vect.cpp + src/groups.cpp compiled into
# oracle/_ref/libtg_reftree.so; skipped where it was not built)

def _canon(label):
    """group id = the smallest caller index in the group, -1 alone"""
    out = np.full(len(label), -1, np.int64)
    for g in np.unique(label[label >= 0]):
        m = np.nonzero(label == g)[0]
        out[m] = m.min()
    return out


def _distinct_planted(n, seed):
    """uniform particles, four clumps of 40 inside the box and a chain of
    three through the x = +-1/2 face; all positions distinct"""
    rng = np.random.default_rng(seed)
    x = rng.integers(-2 ** 31, 2 ** 31, size=(n, 3), dtype=np.int64)
    L, _ = ofof.link_int(n, 0.2)
    x[6] = [2 ** 31 - L // 3, 0, 0]
    x[7] = [-2 ** 31 + L // 3, 0, 0]
    x[8] = [-2 ** 31 + L, 0, 0]
    for c in range(4):
        base = np.array([-2 ** 30 + c * 2 ** 29, c * 2 ** 28, -c * 2 ** 28])
        k = slice(16 + 40 * c, 16 + 40 * (c + 1))
        x[k] = base + rng.integers(-L // 2, L // 2, size=(40, 3))
    x = ((x + 2 ** 31) % 2 ** 32 - 2 ** 31).astype(np.int32)
    assert len(np.unique(x, axis=0)) == n
    return x


@pytest.mark.parametrize("case", ["planted400", "planted3000", "uniform4096_l03", "uniform4096_l04_leaf16"])
def test_partition_matches_reference_find_groups(case):
    """The reference's own group finder (tree::find_groups at theta 0.99 and
    part_vect_find_groups until nothing changes) gives the oracle's partition
    without the friends that only the periodic wrap makes: the reference's
    tree search tests box intersection without the wrap, so it never pairs
    particles across the box boundary.  The CUDA path and the oracle keep
    those links (the partition of the periodic friend relation); the two
    partitions differ exactly there."""
    import ref_tree
    if not ref_tree.available():
        pytest.skip("oracle/_ref/libtg_reftree.so not built")
    from tigergrav_b200 import ics
    leaf = 64
    if case.startswith("planted"):
        x, ll = _distinct_planted(int(case[7:]), 3), 0.2
    else:
        x, ll = ics.uniform(4096, 1), 0.3 if "l03" in case else 0.4
        leaf = 16 if "leaf16" in case else 64
    ref = _canon(ref_tree.fof(x, ll, leaf))
    np.testing.assert_array_equal(ref, _canon(ofof.groups(x, ll, True, across_boundary=False)))
    full = _canon(ofof.groups(x, ll, True))
    diff = np.nonzero(full != ref)[0]
    if len(diff):  # only groups that a boundary-crossing link joins or creates
        wrap = ofof.friend_pairs(x, ll, True)
        wrap = wrap[ofof._d2(x[wrap[:, 0]], x[wrap[:, 1]], False) != ofof._d2(x[wrap[:, 0]], x[wrap[:, 1]], True)]
        touched = set(full[np.unique(wrap)])
        assert set(full[diff]) <= touched
    if case.startswith("planted"):
        # the chain through the face: one group here, 7-8 and a lone 6 in the reference
        assert full[6] == full[7] == full[8] >= 0
        assert ref[6] == -1 and ref[7] == ref[8] >= 0


def test_catalog_matches_reference_groups():
    """The oracle's catalogue against groups.cpp itself (fed by the
    reference's output kick), on the reference's partition: the same groups
    and sizes, centres and radii equal, mean velocity and dispersion within the
    rounding of the reference's float sums (the oracle sums in double)."""
    import ref_tree
    if not ref_tree.available():
        pytest.skip("oracle/_ref/libtg_reftree.so not built")
    x = _distinct_planted(3000, 3)
    v = (np.random.default_rng(2).standard_normal((3000, 3)) * 0.1).astype(np.float32)
    label, cat = ref_tree.fof_catalog(x, v, 0.2)
    first = {}
    for i, g in enumerate(label):
        if g >= 0:
            first.setdefault(g, i)
    gid = np.array([first[g] for g in cat["id"]])
    order = np.argsort(gid)
    mine = ofof.catalog(x, v, _canon(ofof.groups(x, 0.2, True, across_boundary=False)), a=1.0)
    np.testing.assert_array_equal(gid[order], mine["id"])
    assert len(gid) >= 40
    np.testing.assert_array_equal(cat["N"][order], mine["N"])
    np.testing.assert_allclose(cat["x"][order], mine["x"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(cat["rmax"][order], mine["rmax"], rtol=1e-6)
    np.testing.assert_allclose(cat["rc"][order], mine["rc"], rtol=1e-6)
    np.testing.assert_allclose(cat["v"][order], mine["v"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(cat["dv"][order], mine["dv"], rtol=0, atol=1e-7)
