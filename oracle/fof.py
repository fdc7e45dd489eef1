"""Oracle (test infrastructure only): friends-of-friends groups and the group
catalogue of the reference, restated on the CPU.

* link_int           -- the integer linking length of part_vect_find_groups
                        (src/part_vect.cpp:87-88).
* propagate_labels   -- a literal restatement of the reference's min-label
                        propagation (part_vect_find_groups,
                        src/part_vect.cpp:85-124, repeated until nothing
                        changes as groups_execute_finders drives it,
                        src/main.cpp:41-46), all pairs: small n only.
* groups             -- the same partition through a k-d tree candidate search
                        plus the exact integer friend test and connected
                        components (scipy), for tens of thousands of particles;
                        pinned against propagate_labels by the tests.
* catalog            -- groups_add_particle1 / groups_finish1 /
                        groups_add_particle2 / groups_finish2
                        (src/groups.cpp:124-226): the running nearest-image
                        mean centre, mean v/a, velocity dispersion, rmax and
                        the median radius radii[N/2].

Group ids are the smallest index in the group (the reference labels with its
own storage index; here storage order is the caller's order), -1 for a
particle without friends (DEFAULT_GROUP).
"""
import numpy as np

DEFAULT = -1


def link_int(n, link_len):
    """(uint64)(n^(-1/3) link_len (2^32 - 1)) and its square (src/part_vect.cpp:87-88)."""
    L = int((float(n) ** (-1.0 / 3.0) * link_len) * 4294967295.0)
    return L, np.uint64(L * L)


def _d2(xi, xj, periodic):
    d = xi.astype(np.int64) - xj.astype(np.int64)
    if periodic:  # int32 difference, as pos_type arithmetic wraps
        d = (d + 2 ** 31) % 2 ** 32 - 2 ** 31
    # |d| >= 2^31 already means d2 >= 2^62 > L2: clamp so the uint64 sum cannot wrap
    a = np.minimum(np.abs(d), 2 ** 31).astype(np.uint64)
    return (a * a).sum(axis=-1, dtype=np.uint64)


def propagate_labels(x, link_len, periodic=True):
    """Literal min-label propagation over all pairs (small n)."""
    x = np.asarray(x, np.int32)
    n = len(x)
    _, L2 = link_int(n, link_len)
    group = [DEFAULT] * n
    changed = True
    while changed:
        changed = False
        others = list(group)  # part_vect_read_group: a copy of the current labels
        for i in range(n):
            d2 = _d2(x[i][None, :], x, periodic)
            for j in np.nonzero((d2 < L2) & (d2 != 0))[0]:
                this_id = group[i]
                if this_id == DEFAULT:
                    this_id = i
                    group[i] = i
                    changed = True
                oid = others[j]
                if oid != DEFAULT and oid != this_id:
                    g = min(this_id, oid)
                    if group[i] != g:
                        changed = True
                    group[i] = g
                    this_id = g
    return np.array(group, np.int64)


def friend_pairs(x, link_len, periodic=True, across_boundary=True):
    """All friend pairs (i < j) by the exact integer test; candidates from a k-d tree.
    across_boundary=False drops the pairs that are friends only through the
    periodic wrap, which the reference's search never pairs: tree::find_groups
    (src/tree.cpp:661-662, 701-702) rejects a node, and pairs a leaf, only
    where the boxes intersect without the wrap (ranges_intersect), although
    part_vect_find_groups measures the pair itself with the int32 wrap."""
    from scipy.spatial import cKDTree
    x = np.asarray(x, np.int32)
    n = len(x)
    L, L2 = link_int(n, link_len)
    xd = x.astype(np.float64) / 2.0 ** 32 + 0.5
    r = L / 2.0 ** 32 * (1.0 + 1e-9) + 1e-12
    tree = cKDTree(xd, boxsize=1.0 if periodic else None)
    pairs = tree.query_pairs(r, output_type="ndarray")
    if len(pairs) == 0:
        return pairs.reshape(0, 2)
    d2 = _d2(x[pairs[:, 0]], x[pairs[:, 1]], periodic)
    keep = (d2 < L2) & (d2 != 0)
    if periodic and not across_boundary:
        keep &= _d2(x[pairs[:, 0]], x[pairs[:, 1]], False) == d2
    return pairs[keep]


def groups(x, link_len, periodic=True, across_boundary=True):
    """Group id per particle (smallest index in its group) or -1
    (across_boundary: see friend_pairs)."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import connected_components
    n = len(x)
    p = friend_pairs(x, link_len, periodic, across_boundary)
    out = np.full(n, DEFAULT, np.int64)
    if len(p) == 0:
        return out
    A = coo_matrix((np.ones(len(p)), (p[:, 0], p[:, 1])), shape=(n, n))
    _, comp = connected_components(A, directed=False)
    first = np.full(comp.max() + 1, n, np.int64)
    np.minimum.at(first, comp, np.arange(n))
    has = np.zeros(n, bool)
    has[p.ravel()] = True
    out[has] = first[comp[has]]
    return out


def catalog(x, v, group, a=1.0, periodic=True):
    """Group statistics, ids ascending: dict of id, N, x, v, dv, rmax, rc."""
    x = np.asarray(x, np.int32)
    v = np.asarray(v, np.float32)
    ainv = 1.0 / a
    ids = np.unique(group[group >= 0])
    cat = {k: [] for k in ("id", "N", "x", "v", "dv", "rmax", "rc")}
    xd = x.astype(np.float64) / 2.0 ** 32 + 0.5
    for gid in ids:
        mem = np.nonzero(group == gid)[0]
        # groups_add_particle1: running sum of positions kept near the first member
        gx = xd[mem[0]].copy()
        N = 1
        gv = np.zeros(3)
        gv += v[mem[0]] * ainv
        for i in mem[1:]:
            dx = xd[i] - gx / N
            if periodic:
                ad = np.abs(dx)
                dx = np.copysign(np.minimum(ad, 1.0 - ad), dx * (0.5 - ad))
            gx += dx + gx / N
            N += 1
            if periodic:
                for d in range(3):
                    while gx[d] < 0.0:
                        gx[d] += N
                    while gx[d] > N:
                        gx[d] -= N
            gv += v[i] * ainv
        cen = gx / N  # groups_finish1
        vm = gv / N
        # groups_add_particle2 / groups_finish2
        dv = ((v[mem] * ainv - vm) ** 2).sum(axis=0)
        dxr = np.abs(xd[mem] - cen)
        if periodic:
            dxr = np.minimum(dxr, 1.0 - dxr)
        radii = np.sort((a * np.sqrt((dxr ** 2).sum(axis=1))).astype(np.float32))
        cat["id"].append(gid)
        cat["N"].append(len(mem))
        cat["x"].append(cen)
        cat["v"].append(vm)
        cat["dv"].append(np.sqrt(dv / len(mem)))
        cat["rmax"].append(radii[-1])
        cat["rc"].append(radii[len(radii) // 2])
    return {k: np.array(val) for k, val in cat.items()}
