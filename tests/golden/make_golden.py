"""Generate golden vectors from the reference's own gravity kernels.

Runs the reference kernels (src/gravity.cpp, compiled from the reference
sources by `make -C oracle ref` into oracle/_ref/libtg_ref.so) on seeded
inputs that cover the cases the kernels distinguish: empty source lists,
source counts around the 16-lane padding, coincident particles (r = 0),
separations inside h/2 and h (the three softening branches), separations
below the Ewald cut (1e-6), minimum-image wrap at the box edge, and a small
full force evaluation (oracle walk + reference kernels).

The reference freezes its options on the first kernel call
(src/gravity.cpp:176-187), so each parameter set runs in its own process:
    python tests/golden/make_golden.py            # writes tests/golden/*.npz
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

PARAMS = {
    # name: (n_nominal, ewald, theta)
    "ewald": (2000, 1, 0.7),
    "free": (2000, 0, 0.7),
}


def _pos(a):
    from tigergrav_b200.ics import double_to_pos
    return double_to_pos(np.mod(a, 1.0))


def sink_source_sets(rng, h):
    """(sinks, sources) arrays covering the kernels' branches."""
    c = rng.random(3)
    sinks = c + (rng.random((40, 3)) - 0.5) * 0.02
    parts = [c + (rng.random((30, 3)) - 0.5) * 0.05,                       # near field
             c + (rng.random((10, 3)) - 0.5) * 0.6,                        # far (and wrapped) field
             sinks[:3] + (rng.random((3, 3)) - 0.5) * 0.6 * h,             # inside h/2 .. h
             sinks[3:5] + (rng.random((2, 3)) - 0.5) * 1.6 * h,
             sinks[5:7]]                                                    # coincident (r = 0)
    src = np.concatenate(parts)
    return _pos(sinks), _pos(src)


def edge_set():
    """sinks / sources straddling the periodic boundary (fixed point -2^31 and 2^31-1)"""
    x = np.array([[-2 ** 31, 0, 5], [2 ** 31 - 1, -7, 2 ** 31 - 1]], np.int64).astype(np.int32)
    y = np.array([[2 ** 31 - 1, 3, 0], [-2 ** 31, 2 ** 31 - 1, -2 ** 31], [-2 ** 31 + 1000, 0, 0],
                  [0, 0, 0]], np.int64).astype(np.int32)
    return x, y


def multipoles(rng, n, scale):
    m = np.zeros((n, 17), np.float32)
    m[:, 0] = rng.uniform(0.5, 2.0, n) * 1e-3
    m[:, 1:7] = (m[:, :1] * rng.normal(size=(n, 6)) * scale ** 2).astype(np.float32)
    m[:, 7:] = (m[:, :1] * rng.normal(size=(n, 10)) * scale ** 3).astype(np.float32)
    return m


def run(name):
    import oracle as O
    from tigergrav_b200 import ics
    n, ewald, theta = PARAMS[name]
    h = 0.02 * n ** (-1.0 / 3.0)
    m = 1.0 / n
    R = O.ref_lib()
    assert R is not None, "build the reference kernels first: make -C oracle ref"
    assert R.ref_init(theta, h, 1.0, n, ewald, 1.0) == 0
    p = O.params(theta=theta, soft_len=h, m=m, ewald=bool(ewald))
    rng = np.random.Generator(np.random.PCG64(20240 + ewald))
    out = dict(n=n, ewald=ewald, theta=theta, h=h, m=m)
    kinds = ["direct", "ewald"] if ewald else ["direct"]
    # PP
    cases = [sink_source_sets(rng, h) for _ in range(2)] + [edge_set()]
    for ci, (x, y) in enumerate(cases):
        for ny in sorted({0, 1, 15, 16, 17, len(y)}):
            if ny > len(y):
                continue
            for kind in kinds:
                f = rng.normal(size=(len(x), 4))  # accumulated into
                out[f"pp_{kind}_{ci}_{ny}_x"] = x
                out[f"pp_{kind}_{ci}_{ny}_y"] = y[:ny]
                out[f"pp_{kind}_{ci}_{ny}_f0"] = f.copy()
                fl = O.pp(kind, p, f, x, y[:ny], do_phi=True, use_ref=True)
                out[f"pp_{kind}_{ci}_{ny}_f"] = f
                out[f"pp_{kind}_{ci}_{ny}_flops"] = fl
    # PC / CC / CP
    for ci in range(2):
        c = rng.random(3)
        x = _pos(c + (rng.random((24, 3)) - 0.5) * 0.01)
        yx = _pos(c + (rng.random((37, 3)) - 0.5) * 0.7)
        ym = multipoles(rng, 37, 0.01)
        yp = _pos(c + (rng.random((29, 3)) - 0.5) * 0.7)
        for kind in kinds:
            f = rng.normal(size=(len(x), 4))
            out[f"pc_{kind}_{ci}_f0"] = f.copy()
            out[f"pc_{kind}_{ci}_flops"] = O.pc(kind, p, f, x, ym, yx, use_ref=True)
            out[f"pc_{kind}_{ci}_f"] = f
            L = rng.normal(size=35)
            out[f"cc_{kind}_{ci}_L0"] = L.copy()
            out[f"cc_{kind}_{ci}_flops"] = O.cc(kind, p, L, x[0], ym, yx, use_ref=True)
            out[f"cc_{kind}_{ci}_L"] = L
            L = rng.normal(size=35)
            out[f"cp_{kind}_{ci}_L0"] = L.copy()
            out[f"cp_{kind}_{ci}_flops"] = O.cp(kind, p, L, x[0], yp, use_ref=True)
            out[f"cp_{kind}_{ci}_L"] = L
        out[f"pc_{ci}_x"], out[f"pc_{ci}_ym"], out[f"pc_{ci}_yx"], out[f"pc_{ci}_yp"] = x, ym, yx, yp
    if ewald:
        # Green's functions and expansion algebra
        dxs = np.concatenate([rng.uniform(-0.5, 0.5, (40, 3)), [[0, 0, 0], [1e-7, 0, 0], [0.3, -0.2, 1e-3]]])
        dxs = dxs.astype(np.float32)
        out["green_dx"] = dxs
        out["green_direct"] = np.array([O.green("direct", d, use_ref=True) for d in dxs])
        out["green_ewald"] = np.array([O.green("ewald", d, use_ref=True) for d in dxs])
        Ls = rng.normal(size=(10, 35))
        ds = rng.uniform(-0.05, 0.05, (10, 3))
        out["alg_L"], out["alg_dx"] = Ls, ds
        out["l2l"] = np.array([O.l2l(Ls[i], ds[i], use_ref=True) for i in range(10)])
        out["l2p"] = np.array([O.l2p(Ls[i], ds[i], use_ref=True) for i in range(10)])
        Ms = multipoles(rng, 10, 0.05)
        out["alg_M"] = Ms
        out["m2m"] = np.array([O.m2m(Ms[i], ds[i].astype(np.float32), use_ref=True) for i in range(10)])
        # a full force evaluation: oracle walk + reference kernels
        x = ics.uniform(n, 77)
        o = O.Oracle(theta=theta, ewald=True, leaf_max=64).set_particles(x)
        o.build().multipoles().walk().evaluate(use_ref=True)
        phi, g = o.forces()
        out["solve_x"], out["solve_phi"], out["solve_g"] = x, phi, g
        ref, clean, fl = o.stats()
        out["solve_stats"] = np.array([ref[k] for k in ("PP_direct", "PP_ewald", "CC_direct", "CC_ewald",
                                                        "CP_direct", "CP_ewald")], np.uint64)
        out["solve_flops"] = fl
    np.savez_compressed(os.path.join(HERE, f"kernels_{name}.npz"), **out)
    print("wrote", name, len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        run(sys.argv[1])
    else:
        for name in PARAMS:
            subprocess.check_call([sys.executable, os.path.abspath(__file__), name])
