"""The oracle's tree and walk against the reference's own (src/tree.cpp run on
the host through oracle/_ref/libtg_reftree.so): node and leaf counts, the
interaction statistics, every list of every node in content and order (as
the reference's walk hands them to its kernels), and the forces of a whole
solve with the reference's kernels.  The CUDA path's trees and lists are
bit-identical to the oracle's (tests/test_gpu_path.py,
tests/test_parity_config1.py), so these pin them to the reference's code.

Needs the reference sources at build time (oracle/Makefile `reftree`);
skipped where the library was not built.
"""
import numpy as np
import pytest

import ref_tree

pytestmark = pytest.mark.skipif(not ref_tree.available(), reason="oracle/_ref/libtg_reftree.so not built")

CASES = {
    "clustered16_free_t07": dict(kind="clustered", nside=16, theta=0.7, ewald=False, leaf=64),
    "clustered16_free_t03_leaf16": dict(kind="clustered", nside=16, theta=0.3, ewald=False, leaf=16),
    "uniform2048_ewald_t05": dict(kind="uniform", n=2048, theta=0.5, ewald=True, leaf=64),
    "clustered12_ewald_t07_leaf24": dict(kind="clustered", nside=12, theta=0.7, ewald=True, leaf=24),
}

_solved = {}


def _case(name, oracle_mod):
    if name not in _solved:
        from tigergrav_b200 import ics
        c = CASES[name]
        x = ics.clustered(c["nside"], 3) if c["kind"] == "clustered" else ics.uniform(c["n"], 1)
        r = ref_tree.solve(x, c["theta"], c["ewald"], c["leaf"], record=True)
        o = oracle_mod.Oracle(theta=c["theta"], ewald=c["ewald"], leaf_max=c["leaf"]).set_particles(x)
        o.build().multipoles().walk()
        _solved[name] = (x, r, o)
    return _solved[name]


def _oracle_calls(x, o):
    """the lists of o (the oracle, or the CUDA path's GravitySolver: the same
    introspection) in the form the reference's walk calls its kernels"""
    nd = o.nodes()
    xs = x[o.perm()]
    out = []
    for name in ref_tree.KIND_NAMES:
        off, ids = o.list(name)
        for i in range(o.num_nodes):
            lst = ids[off[i]:off[i + 1]]
            if len(lst) == 0:
                continue
            pb, pe = nd["pbegin"][i], nd["pend"][i]
            if name in ("PC_D", "PP_D", "PC_E", "PP_E"):
                sink, ns = tuple(int(v) for v in xs[pb]), int(pe - pb)
            else:
                sink, ns = tuple(int(v) for v in nd["x"][i]), 1
            if name in ("CC_D", "CC_E", "PC_D", "PC_E"):
                src = nd["x"][lst]
            else:
                src = np.concatenate([xs[nd["pbegin"][j]:nd["pend"][j]] for j in lst])
            if len(src):
                out.append((name, sink, ns, src.astype(np.int32)))
    return out


def _key(c):
    return (c[0], c[1], c[2], c[3].tobytes())


@pytest.mark.parametrize("name", list(CASES))
def test_tree_counts_and_stats_match_reference(name, oracle_mod):
    x, r, o = _case(name, oracle_mod)
    nd = o.nodes()
    assert r["nodes"] == o.num_nodes
    assert r["leaves"] == int((nd["child0"] < 0).sum())
    ref_stats, _, _ = o.stats()
    assert r["stats"] == ref_stats


@pytest.mark.parametrize("name", list(CASES))
def test_lists_match_reference_walk(name, oracle_mod):
    """every kernel call of the reference's kick_fmm that has sources is one
    of the oracle's lists (same sink, same sources in the same order), and
    the other way round"""
    x, r, o = _case(name, oracle_mod)
    ref = sorted(_key(c) for c in r["calls"] if len(c[3]))
    mine = sorted(_key(c) for c in _oracle_calls(x, o))
    assert len(ref) == len(mine)
    assert ref == mine


@pytest.mark.parametrize("name", list(CASES))
def test_forces_match_reference_solve(name, oracle_mod, has_ref):
    """the whole solve: the oracle's lists through the reference's kernels
    against the reference's own run, to the last bits of FP32 (the expansion
    arithmetic of L2L / L2P is restated in the oracle, and the reference's
    build contracts it into FMAs)"""
    if not has_ref:
        pytest.skip("reference kernels not built")
    x, r, o = _case(name, oracle_mod)
    o.evaluate(use_ref=True)
    phi, g = o.forces()
    gn = np.linalg.norm(g, axis=1)
    eg = np.linalg.norm(r["g"].astype(np.float64) - g, axis=1) / gn
    ep = np.abs(r["phi"].astype(np.float64) - phi) / np.abs(phi).max()
    assert eg.max() <= 1e-6, eg.max()
    assert ep.max() <= 1e-6, ep.max()
    assert np.median(eg) <= 1e-7


def _canonical(x, s, ref_calls):
    """Both walks in a form that does not depend on the order of particles
    inside a leaf (the CUDA path sorts the particles of a leaf by Morton key,
    the reference by its midpoint partition; the leaves and their sets are the
    same): a leaf sink is named by the node of s that holds its first
    particle, and particle sources are cut into s's source leaves, each taken
    as a set.  Returns (reference calls, s's calls) as sorted lists."""
    nd = s.nodes()
    perm = s.perm()
    xs = x[perm]
    leaf_of = np.full(len(x), -1, np.int64)  # caller index -> leaf of s
    for i in np.nonzero(nd["child0"] < 0)[0]:
        leaf_of[perm[nd["pbegin"][i]:nd["pend"][i]]] = i
    index_of = {tuple(int(v) for v in p): k for k, p in enumerate(x)}
    mine, cuts = [], {}
    for name in ref_tree.KIND_NAMES:
        off, ids = s.list(name)
        for i in range(s.num_nodes):
            lst = ids[off[i]:off[i + 1]]
            if len(lst) == 0:
                continue
            leafk = name in ("PC_D", "PP_D", "PC_E", "PP_E")
            sink = int(i) if leafk else tuple(int(v) for v in nd["x"][i])
            ns = int(nd["pend"][i] - nd["pbegin"][i]) if leafk else 1
            if name in ("CC_D", "CC_E", "PC_D", "PC_E"):
                src = tuple(tuple(int(v) for v in c) for c in nd["x"][lst])
            else:
                sizes = [int(nd["pend"][j] - nd["pbegin"][j]) for j in lst]
                cuts[(name, sink)] = sizes
                src = tuple(tuple(sorted(tuple(int(v) for v in p) for p in xs[nd["pbegin"][j]:nd["pend"][j]]))
                            for j in lst)
            if len(src):
                mine.append((name, sink, ns, src))
    ref = []
    for name, first, ns, src in ref_calls:
        if len(src) == 0:
            continue
        leafk = name in ("PC_D", "PP_D", "PC_E", "PP_E")
        sink = int(leaf_of[index_of[first]]) if leafk else first
        pts = [tuple(int(v) for v in p) for p in src]
        if name in ("CC_D", "CC_E", "PC_D", "PC_E"):
            can = tuple(pts)
        else:
            sizes = cuts.get((name, sink), [len(pts)])
            if sum(sizes) != len(pts):
                sizes = [len(pts)]
            can, k = [], 0
            for n in sizes:
                can.append(tuple(sorted(pts[k:k + n])))
                k += n
            can = tuple(can)
        ref.append((name, sink, ns, can))
    return sorted(ref), sorted(mine)


@pytest.mark.parametrize("name", ["clustered12_ewald_t07_leaf24"])
def test_canonical_form_ignores_the_order_inside_leaves(name, oracle_mod):
    """the comparison the GPU test below makes, on the oracle with the
    particles of every leaf put in another order: it still matches, and a
    changed list does not"""
    x, r, o = _case(name, oracle_mod)

    class Shuffled:
        num_nodes = o.num_nodes

        def __init__(self):
            self.nd = o.nodes()
            p = o.perm().copy()
            rng = np.random.default_rng(5)
            for i in np.nonzero(self.nd["child0"] < 0)[0]:
                b, e = self.nd["pbegin"][i], self.nd["pend"][i]
                p[b:e] = p[b:e][rng.permutation(e - b)]
            self.p = p

        def nodes(self):
            return self.nd

        def perm(self):
            return self.p

        def list(self, kind):
            return o.list(kind)

    ref, mine = _canonical(x, Shuffled(), r["calls"])
    assert ref == mine
    bad = [c for c in r["calls"] if c[0] == "PP_D" and len(c[3]) > 1][0]
    calls = [c for c in r["calls"] if c is not bad] + [(bad[0], bad[1], bad[2], bad[3][:-1])]
    ref2, _ = _canonical(x, Shuffled(), calls)
    assert ref2 != mine


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["clustered16_free_t07", "uniform2048_ewald_t05", "clustered12_ewald_t07_leaf24"])
def test_gpu_walk_matches_reference_walk(name, oracle_mod):
    """the CUDA path's tree counts, statistics and lists against the
    reference's own walk directly (the lists' sources in order, the particles
    of each leaf as a set)"""
    import tigergrav_b200 as tg
    x, r, _ = _case(name, oracle_mod)
    c = CASES[name]
    with tg.GravitySolver(len(x), theta=c["theta"], ewald=c["ewald"], leaf_max=c["leaf"]) as s:
        s.set_particles(x).solve_gravity()
        st = s.stats()
        assert st["nodes"] == r["nodes"]
        assert st["ref_stats"] == r["stats"]
        ref, mine = _canonical(x, s, r["calls"])
    assert len(ref) == len(mine)
    assert ref == mine


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["clustered16_free_t07", "clustered12_ewald_t07_leaf24"])
def test_gpu_forces_match_reference_solve(name, oracle_mod):
    """the CUDA path's FP32 forces against the reference's own whole solve
    (its tree, walk and kernels), per particle: no further from the FP64
    evaluation of the same lists than the reference's run is, plus 1e-5 of
    the force (the bound of tests/helpers.py)"""
    import tigergrav_b200 as tg
    from helpers import arbiter_excess
    x, r, o = _case(name, oracle_mod)
    c = CASES[name]
    with tg.GravitySolver(len(x), theta=c["theta"], ewald=c["ewald"], leaf_max=c["leaf"]) as s:
        s.set_particles(x).solve_gravity()
        phi, g = s.get_forces()
    o.evaluate(fp64=True)
    phi64, g64 = o.forces()
    fx, px = arbiter_excess(g, r["g"].astype(np.float64), g64, phi, r["phi"].astype(np.float64), phi64)
    assert fx <= 0.0, fx
    assert px <= 0.0, px
