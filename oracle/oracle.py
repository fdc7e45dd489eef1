"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is the checker: a serial CPU restatement of TigerGrav's periodic
gravity evaluation (oracle/tg_oracle.cpp) plus, where the reference tree is
present at build time, the reference's own kernels compiled from its sources
(oracle/_ref/libtg_ref.so, see oracle/ref_driver.cpp).  Only the test suite,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline / reference arm
use this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtg_oracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libtg_ref.so")

KINDS = {"CC_D": 0, "CP_D": 1, "CC_E": 2, "CP_E": 3, "PC_D": 4, "PP_D": 5, "PC_E": 6, "PP_E": 7}


class Params(C.Structure):
    _fields_ = [("theta", C.c_double), ("soft_len", C.c_double), ("m", C.c_double), ("G", C.c_double),
                ("ewald", C.c_int), ("leaf_max", C.c_int)]


def build(with_ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree exists, its kernels)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "libtg_oracle.so"])
    if with_ref:
        extra = ["REF=" + os.environ["TG_REFERENCE"]] if os.environ.get("TG_REFERENCE") else []
        subprocess.check_call(["make", "-s", "-C", HERE, "ref-if-present"] + extra)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_ref=False)
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        L.tgo_create.restype = vp
        L.tgo_create.argtypes = [P(Params)]
        L.tgo_destroy.argtypes = [vp]
        L.tgo_set_particles.argtypes = [vp, vp, vp, i64]
        for f in ("tgo_build", "tgo_multipoles", "tgo_walk"):
            getattr(L, f).argtypes = [vp]
        L.tgo_walk_mt.argtypes = [vp, i32]
        L.tgo_evaluate.argtypes = [vp, i32, i32, vp, i64]
        L.tgo_load_reference.argtypes = [vp, C.c_char_p]
        L.tgo_num_nodes.restype = i64
        L.tgo_num_nodes.argtypes = [vp]
        L.tgo_num_particles.restype = i64
        L.tgo_num_particles.argtypes = [vp]
        L.tgo_get_nodes.argtypes = [vp] + [vp] * 10
        L.tgo_get_perm.argtypes = [vp, vp]
        L.tgo_list_size.restype = i64
        L.tgo_list_size.argtypes = [vp, i32]
        L.tgo_get_list.argtypes = [vp, i32, vp, vp]
        L.tgo_get_forces.argtypes = [vp, vp, vp]
        L.tgo_get_expansions.argtypes = [vp, vp]
        L.tgo_get_stats.argtypes = [vp, vp, vp, vp]
        L.tgo_kind_costs.argtypes = [vp, i32, i32, C.c_double, C.c_uint64, vp, vp]
        L.tgo_kick.argtypes = [vp, C.c_double]
        L.tgo_drift.argtypes = [vp, C.c_double, vp]
        L.tgo_get_particles.argtypes = [vp, vp, vp]
        L.tgo_energy.argtypes = [vp, vp]
        L.tgo_truth.argtypes = [vp, i64, vp, i64, C.c_double, C.c_double, C.c_double, i32, vp, vp]
        L.tgo_ewald_corr_f64.argtypes = [vp, vp]
        for f in ("tgo_green_ewald", "tgo_green_direct"):
            getattr(L, f).argtypes = [vp, vp]
        L.tgo_L2L.argtypes = [vp, vp]
        L.tgo_L2P.argtypes = [vp, vp, vp]
        L.tgo_M2M.argtypes = [vp, vp]
        for f in ("tgo_PP_direct", "tgo_PP_ewald"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [P(Params), vp, vp, i32, vp, i32, i32]
        for f in ("tgo_PC_direct", "tgo_PC_ewald"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [P(Params), vp, vp, i32, vp, vp, i32]
        for f in ("tgo_CC_direct", "tgo_CC_ewald"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [P(Params), vp, vp, vp, vp, i32]
        for f in ("tgo_CP_direct", "tgo_CP_ewald"):
            getattr(L, f).restype = C.c_uint64
            getattr(L, f).argtypes = [P(Params), vp, vp, vp, i32]
        _lib = L
    return _lib


_ref = None


def ref_lib():
    """The reference's own kernels (None when oracle/_ref was not built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        R = C.CDLL(REF_PATH)
        vp, i32 = C.c_void_p, C.c_int
        R.ref_init.restype = i32
        R.ref_init.argtypes = [C.c_double, C.c_double, C.c_double, C.c_uint64, i32, C.c_double]
        for f in ("ref_PP_direct", "ref_PP_ewald"):
            getattr(R, f).restype = C.c_uint64
            getattr(R, f).argtypes = [vp, vp, vp, i32, vp, i32, i32]
        for f in ("ref_PC_direct", "ref_PC_ewald"):
            getattr(R, f).restype = C.c_uint64
            getattr(R, f).argtypes = [vp, vp, vp, i32, vp, vp, i32]
        for f in ("ref_CC_direct", "ref_CC_ewald"):
            getattr(R, f).restype = C.c_uint64
            getattr(R, f).argtypes = [vp, vp, vp, vp, vp, i32]
        for f in ("ref_CP_direct", "ref_CP_ewald"):
            getattr(R, f).restype = C.c_uint64
            getattr(R, f).argtypes = [vp, vp, vp, vp, i32]
        for f in ("ref_green_ewald", "ref_green_direct"):
            getattr(R, f).argtypes = [vp, vp]
        R.ref_L2L.argtypes = [vp, vp]
        R.ref_L2P.argtypes = [vp, vp, vp]
        R.ref_M2M.argtypes = [vp, vp]
        _ref = R
    return _ref


_ref_copies = {}
_ref_tmpdir = None


def ref_path_for(theta, soft_len, m_tot, n, ewald, G) -> str:
    """Path of a copy of the reference's kernel library to load for these
    options.  The reference's kernels keep the options of their first call in
    function-local statics (src/gravity.cpp:176-187, 307-312, 375-378), so
    one loaded library serves one parameter set per process: every further
    parameter set gets its own copy of the file, loaded separately."""
    global _ref_tmpdir
    key = (float(theta), float(soft_len), float(m_tot), int(n), int(ewald), float(G))
    if key not in _ref_copies:
        if not _ref_copies:
            _ref_copies[key] = REF_PATH
        else:
            import atexit
            import shutil
            import tempfile
            if _ref_tmpdir is None:
                _ref_tmpdir = tempfile.mkdtemp(prefix="tg_ref_")
                atexit.register(shutil.rmtree, _ref_tmpdir, True)
            path = os.path.join(_ref_tmpdir, "libtg_ref_%d.so" % len(_ref_copies))
            shutil.copyfile(REF_PATH, path)
            _ref_copies[key] = path
    return _ref_copies[key]


def _p(a):
    return None if a is None else a.ctypes.data


def params(theta=0.7, soft_len=0.02 / 32, m=1.0 / 32768, G=1.0, ewald=True, leaf_max=64) -> Params:
    return Params(theta, soft_len, m, G, int(bool(ewald)), leaf_max)


def _kernel(prefix: str, name: str, p: Params, *arrays, n=None, ints=()):
    """Call tgo_<name> (prefix 'tgo') or ref_<name> (prefix 'ref')."""
    L = lib() if prefix == "tgo" else ref_lib()
    fn = getattr(L, prefix + "_" + name)
    return fn(C.byref(p), *arrays)


def pp(kind: str, p: Params, f: np.ndarray, x: np.ndarray, y: np.ndarray, do_phi=True, use_ref=False):
    """gravity_PP_<kind>: f (nx,4) float64 accumulated in place."""
    x = np.ascontiguousarray(x, np.int32)
    y = np.ascontiguousarray(y, np.int32)
    assert f.dtype == np.float64 and f.flags.c_contiguous
    if use_ref:
        return getattr(ref_lib(), "ref_PP_" + kind)(None, _p(f), _p(x), len(x), _p(y) if len(y) else None,
                                                     len(y), int(do_phi))
    return getattr(lib(), "tgo_PP_" + kind)(C.byref(p), _p(f), _p(x), len(x), _p(y) if len(y) else None,
                                            len(y), int(do_phi))


def pc(kind: str, p: Params, f: np.ndarray, x: np.ndarray, ym: np.ndarray, yx: np.ndarray, use_ref=False):
    x = np.ascontiguousarray(x, np.int32)
    ym = np.ascontiguousarray(ym, np.float32)
    yx = np.ascontiguousarray(yx, np.int32)
    if use_ref:
        return getattr(ref_lib(), "ref_PC_" + kind)(None, _p(f), _p(x), len(x), _p(ym), _p(yx), len(yx))
    return getattr(lib(), "tgo_PC_" + kind)(C.byref(p), _p(f), _p(x), len(x), _p(ym), _p(yx), len(yx))


def cc(kind: str, p: Params, L: np.ndarray, x: np.ndarray, ym: np.ndarray, yx: np.ndarray, use_ref=False):
    x = np.ascontiguousarray(x, np.int32)
    ym = np.ascontiguousarray(ym, np.float32)
    yx = np.ascontiguousarray(yx, np.int32)
    if use_ref:
        return getattr(ref_lib(), "ref_CC_" + kind)(None, _p(L), _p(x), _p(ym), _p(yx), len(yx))
    return getattr(lib(), "tgo_CC_" + kind)(C.byref(p), _p(L), _p(x), _p(ym), _p(yx), len(yx))


def cp(kind: str, p: Params, L: np.ndarray, x: np.ndarray, y: np.ndarray, use_ref=False):
    x = np.ascontiguousarray(x, np.int32)
    y = np.ascontiguousarray(y, np.int32)
    if use_ref:
        return getattr(ref_lib(), "ref_CP_" + kind)(None, _p(L), _p(x), _p(y), len(y))
    return getattr(lib(), "tgo_CP_" + kind)(C.byref(p), _p(L), _p(x), _p(y), len(y))


def green(kind: str, dx, use_ref=False) -> np.ndarray:
    dx = np.ascontiguousarray(dx, np.float32)
    D = np.zeros(35, np.float32)
    L = ref_lib() if use_ref else lib()
    getattr(L, ("ref_green_" if use_ref else "tgo_green_") + kind)(_p(dx), _p(D))
    return D


def l2l(Lexp, dx, use_ref=False):
    Lexp = np.array(Lexp, np.float64)
    dx = np.ascontiguousarray(dx, np.float64)
    (ref_lib().ref_L2L if use_ref else lib().tgo_L2L)(_p(Lexp), _p(dx))
    return Lexp


def l2p(Lexp, dx, use_ref=False):
    Lexp = np.ascontiguousarray(Lexp, np.float64)
    dx = np.ascontiguousarray(dx, np.float64)
    out = np.zeros(4)
    (ref_lib().ref_L2P if use_ref else lib().tgo_L2P)(_p(Lexp), _p(dx), _p(out))
    return out


def m2m(M, dx, use_ref=False):
    M = np.array(M, np.float32)
    dx = np.ascontiguousarray(dx, np.float32)
    (ref_lib().ref_M2M if use_ref else lib().tgo_M2M)(_p(M), _p(dx))
    return M


def ewald_corr_f64(dx) -> np.ndarray:
    dx = np.ascontiguousarray(dx, np.float64)
    out = np.zeros(4)
    lib().tgo_ewald_corr_f64(_p(dx), _p(out))
    return out


def truth(x: np.ndarray, samples: np.ndarray, m: float, h: float, alpha: float = 6.0, nthreads: int = 0):
    """FP64 direct Ewald sum at the sample particles: (phi[ns], g[ns,3])."""
    x = np.ascontiguousarray(x, np.int32)
    samples = np.ascontiguousarray(samples, np.int64)
    phi = np.zeros(len(samples))
    g = np.zeros((len(samples), 3))
    nt = nthreads or os.cpu_count() or 1
    rc = lib().tgo_truth(_p(x), len(x), _p(samples), len(samples), m, h, alpha, nt, _p(phi), _p(g))
    if rc != 0:
        raise RuntimeError("tgo_truth failed: %d" % rc)
    return phi, g


class Oracle:
    """Serial restatement of refine / compute_multipoles / kick_fmm."""

    def __init__(self, theta=0.7, soft_len=None, m=None, G=1.0, ewald=True, leaf_max=64):
        self._args = dict(theta=theta, soft_len=soft_len, m=m, G=G, ewald=ewald, leaf_max=leaf_max)
        self.h = None

    def set_particles(self, x: np.ndarray, v: np.ndarray | None = None):
        n = len(x)
        a = dict(self._args)
        if a["soft_len"] is None:
            a["soft_len"] = 0.02 * n ** (-1.0 / 3.0)
        if a["m"] is None:
            a["m"] = 1.0 / n
        self.p = params(**a)
        if self.h is not None:
            lib().tgo_destroy(self.h)
        self.h = lib().tgo_create(C.byref(self.p))
        self.x = np.ascontiguousarray(x, np.int32)
        self.v = np.zeros((n, 3), np.float32) if v is None else np.ascontiguousarray(v, np.float32)
        self.n = n
        rc = lib().tgo_set_particles(self.h, _p(self.x), _p(self.v), n)
        assert rc == 0
        return self

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.tgo_destroy(self.h)
            self.h = None

    def build(self):
        rc = lib().tgo_build(self.h)
        if rc != 0:
            raise RuntimeError("tgo_build: %d" % rc)
        return self

    def multipoles(self):
        assert lib().tgo_multipoles(self.h) == 0
        return self

    def walk(self, nthreads=1):
        """kick_fmm list generation; nthreads > 1 walks subtrees concurrently (same lists)."""
        assert (lib().tgo_walk(self.h) if nthreads <= 1 else lib().tgo_walk_mt(self.h, int(nthreads))) == 0
        return self

    def _ref_path(self):
        p = self.p
        return ref_path_for(p.theta, p.soft_len, p.m * self.n, self.n, p.ewald, p.G)

    def evaluate(self, use_ref=False, nthreads=0, leaf_subset=None, fp64=False):
        """use_ref: the reference's own kernels; fp64: the restated kernels in double."""
        if use_ref:
            if ref_lib() is None:
                raise RuntimeError("reference kernels not built (oracle/_ref)")
            rc = lib().tgo_load_reference(self.h, self._ref_path().encode())
            if rc != 0:
                raise RuntimeError("tgo_load_reference: %d" % rc)
        nt = nthreads or os.cpu_count() or 1
        sub = None if leaf_subset is None else np.ascontiguousarray(leaf_subset, np.int32)
        mode = 1 if use_ref else (2 if fp64 else 0)
        rc = lib().tgo_evaluate(self.h, mode, nt, _p(sub), 0 if sub is None else len(sub))
        if rc != 0:
            raise RuntimeError("tgo_evaluate: %d" % rc)
        return self

    def solve(self, use_ref=False, nthreads=0):
        return self.build().multipoles().walk().evaluate(use_ref=use_ref, nthreads=nthreads)

    @property
    def num_nodes(self):
        return lib().tgo_num_nodes(self.h)

    def nodes(self) -> dict:
        nn = self.num_nodes
        d = dict(boxid=np.zeros(nn, np.uint64), level=np.zeros(nn, np.int32), pbegin=np.zeros(nn, np.int64),
                 pend=np.zeros(nn, np.int64), child0=np.zeros(nn, np.int32), parent=np.zeros(nn, np.int32),
                 x=np.zeros((nn, 3), np.int32), r=np.zeros(nn, np.float32), rmax=np.zeros(nn, np.float32),
                 m=np.zeros((nn, 17), np.float32))
        lib().tgo_get_nodes(self.h, *[_p(d[k]) for k in
                                      ("boxid", "level", "pbegin", "pend", "child0", "parent", "x", "r", "rmax", "m")])
        return d

    def perm(self) -> np.ndarray:
        p = np.zeros(self.n, np.int64)
        lib().tgo_get_perm(self.h, _p(p))
        return p

    def list(self, kind: str):
        k = KINDS[kind]
        tot = lib().tgo_list_size(self.h, k)
        off = np.zeros(self.num_nodes + 1, np.int64)
        ids = np.zeros(max(tot, 1), np.int32)
        lib().tgo_get_list(self.h, k, _p(off), _p(ids))
        return off, ids[:tot]

    def forces(self):
        phi = np.zeros(self.n)
        g = np.zeros((self.n, 3))
        assert lib().tgo_get_forces(self.h, _p(phi), _p(g)) == 0
        return phi, g

    def expansions(self):
        L = np.zeros((self.num_nodes, 35))
        lib().tgo_get_expansions(self.h, _p(L))
        return L

    def stats(self):
        rs = np.zeros(6, np.uint64)
        cnt = np.zeros(8, np.uint64)
        fl = np.zeros(1, np.uint64)
        lib().tgo_get_stats(self.h, _p(rs), _p(cnt), _p(fl))
        ref = dict(zip(("PP_direct", "PP_ewald", "CC_direct", "CC_ewald", "CP_direct", "CP_ewald"), map(int, rs)))
        clean = dict(zip(("PP_D", "PP_E", "PC_D", "PC_E", "CC_D", "CC_E", "CP_D", "CP_E"), map(int, cnt)))
        return ref, clean, int(fl[0])

    def kind_costs(self, use_ref=True, nthreads=0, budget_s=1.0, seed=1):
        """Host throughput per interaction kind: {kind: (ns per interaction, interactions sampled)}
        (each kind's kernel alone over random sinks for at most budget_s seconds; after walk())."""
        if use_ref:
            if ref_lib() is None:
                raise RuntimeError("reference kernels not built (oracle/_ref)")
            rc = lib().tgo_load_reference(self.h, self._ref_path().encode())
            if rc != 0:
                raise RuntimeError("tgo_load_reference: %d" % rc)
        ns = np.zeros(8)
        done = np.zeros(8, np.uint64)
        nt = nthreads or os.cpu_count() or 1
        rc = lib().tgo_kind_costs(self.h, 1 if use_ref else 0, nt, float(budget_s), int(seed), _p(ns), _p(done))
        if rc != 0:
            raise RuntimeError("tgo_kind_costs: %d" % rc)
        return {k: (float(ns[v]), int(done[v])) for k, v in KINDS.items()}

    def kick(self, dt):
        assert lib().tgo_kick(self.h, dt) == 0

    def drift(self, dt):
        ek = np.zeros(1)
        assert lib().tgo_drift(self.h, dt, _p(ek)) == 0
        return float(ek[0])

    def particles(self):
        x = np.zeros((self.n, 3), np.int32)
        v = np.zeros((self.n, 3), np.float32)
        lib().tgo_get_particles(self.h, _p(x), _p(v))
        return x, v

    def energy(self):
        out = np.zeros(5)
        lib().tgo_energy(self.h, _p(out))
        return out
