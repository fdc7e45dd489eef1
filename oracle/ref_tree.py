"""The reference's own tree build and walk, run on the host (TEST
INFRASTRUCTURE ONLY).

oracle/_ref/libtg_reftree.so is src/tree.cpp, src/part_vect.cpp,
src/gravity.cpp, src/cosmo.cpp and src/range.cpp of the reference, compiled
where they lie by oracle/Makefile (target `reftree`) against the serial HPX
stand-in oracle/hpx_shim, with the driver oracle/ref_tree.cpp: one call is the
reference's solve_gravity (src/main.cpp:31-73) on a tree refined as its main
loop refines it (src/main.cpp:201-207).  It gives the FP32 phi and g of every
particle (the kick's output records), the interaction statistics of kick_fmm,
the node and leaf counts of refine, and every kernel call of the walk with its
sink and sources in call order, for checking the oracle's restated tree and
walk (and through them the CUDA path) against the reference's code; and the
reference's cosmology (src/cosmo.cpp) for the oracle's restatement of it.

The reference caches options in function-local statics (src/gravity.cpp:
176-187, src/tree.cpp), so one loaded library serves one parameter set per
process; further parameter sets load their own copies of the file.
"""
from __future__ import annotations

import atexit
import ctypes as C
import os
import shutil
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libtg_reftree.so")
KIND_NAMES = ("CC_D", "CP_D", "CC_E", "CP_E", "PC_D", "PP_D", "PC_E", "PP_E")

_libs: dict = {}
_tmp = None


def available() -> bool:
    return os.path.exists(PATH)


def _lib(key):
    global _tmp
    if key not in _libs:
        path = PATH
        if _libs:
            if _tmp is None:
                _tmp = tempfile.mkdtemp(prefix="tg_reftree_")
                atexit.register(shutil.rmtree, _tmp, True)
            path = os.path.join(_tmp, "libtg_reftree_%d.so" % len(_libs))
            shutil.copyfile(PATH, path)
        L = C.CDLL(path)
        L.reftree_solve.restype = C.c_int
        L.reftree_solve.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.reftree_num_calls.restype = C.c_int64
        L.reftree_call_size.restype = C.c_int64
        L.reftree_call_size.argtypes = [C.c_int64]
        L.reftree_get_call.restype = C.c_int
        L.reftree_get_call.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.reftree_cosmos_advance.restype = None
        L.reftree_cosmos_advance.argtypes = [C.c_double] * 7 + [C.c_void_p]
        L.reftree_kick.restype = C.c_int
        L.reftree_kick.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int, C.c_int] + [C.c_double] * 4 + \
            [C.c_void_p] * 3
        L.reftree_drift.restype = C.c_int
        L.reftree_drift.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
        L.reftree_load_gadget1.restype = C.c_int
        L.reftree_load_gadget1.argtypes = [C.c_char_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p]
        L.reftree_fof_catalog.restype = C.c_int
        L.reftree_fof_catalog.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_int, C.c_void_p,
                                          C.c_int64, C.c_void_p, C.c_void_p]
        L.reftree_fof.restype = C.c_int
        L.reftree_fof.argtypes = [C.c_void_p, C.c_int64, C.c_double, C.c_int, C.c_void_p]
        L.reftree_cosmo_steps.restype = C.c_int
        L.reftree_cosmo_steps.argtypes = [C.c_double] * 5 + [C.c_void_p, C.c_int, C.c_void_p]
        _libs[key] = L
    return _libs[key]


def solve(x: np.ndarray, theta: float, ewald: bool, leaf_max: int = 64, soft_len: float | None = None,
          G: float = 1.0, record: bool = False) -> dict:
    """The reference's solve of int32 fixed-point positions x (n x 3), m = 1/n,
    soft_len 0.02 n^-1/3 unless given.  Returns phi (n, FP32), g (n x 3,
    FP32), stats (the six interaction_stats counters), nodes, leaves and, with
    record, calls: (kind, sink, nsink, sources) per kernel call with sources,
    sink = the first sink particle (leaf kinds) or the node centre, sources =
    positions or multipole centres as an (m x 3) int32 array."""
    x = np.ascontiguousarray(x, np.int32)
    n = len(x)
    if soft_len is None:
        soft_len = 0.02 * n ** (-1.0 / 3.0)
    key = (float(theta), int(bool(ewald)), int(leaf_max), float(soft_len), float(G), int(n))
    L = _lib(key)
    phi = np.zeros(n, np.float32)
    g = np.zeros((n, 3), np.float32)
    st = np.zeros(6, np.uint64)
    tc = np.zeros(2, np.int64)
    rc = L.reftree_solve(x.ctypes.data, n, float(theta), int(bool(ewald)), int(leaf_max), float(soft_len), float(G),
                         int(bool(record)), phi.ctypes.data, g.ctypes.data, st.ctypes.data, tc.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_solve: %d" % rc)
    out = dict(phi=phi, g=g, nodes=int(tc[0]), leaves=int(tc[1]),
               stats=dict(zip(("PP_direct", "PP_ewald", "CC_direct", "CC_ewald", "CP_direct", "CP_ewald"),
                              map(int, st))))
    if record:
        calls = []
        kind = np.zeros(1, np.int32)
        sink = np.zeros(3, np.int32)
        ns = np.zeros(1, np.int64)
        for k in range(L.reftree_num_calls()):
            m = L.reftree_call_size(k)
            src = np.zeros((max(m, 1), 3), np.int32)
            L.reftree_get_call(k, kind.ctypes.data, sink.ctypes.data, ns.ctypes.data, src.ctypes.data)
            calls.append((KIND_NAMES[int(kind[0])], tuple(int(v) for v in sink), int(ns[0]), src[:m].copy()))
        out["calls"] = calls
    return out


RUNG_MAX = 30


def cosmos_advance(state, t0, H0, omega_m, omega_lambda):
    """The reference's cosmos::advance_to_time (src/cosmo.cpp:50-106) from
    state = (a, adot, tau): returns ([a, adot, tau], drift_dt, kick_dt)."""
    out = np.zeros(5)
    _lib("cosmo").reftree_cosmos_advance(float(state[0]), float(state[1]), float(state[2]), float(t0), float(H0),
                                         float(omega_m), float(omega_lambda), out.ctypes.data)
    return [out[0], out[1], out[2]], out[3], out[4]


def cosmo_steps(a0, adot0, dts, H0, omega_m, omega_lambda) -> list:
    """The reference's cosmo_init(a0, adot0) and one cosmo_advance per dt
    (src/cosmo.cpp:187-232, t_max = 1): per step a dict of a_last, a, the
    float time, tau, drift, kick1 and kick2 (RUNG_MAX + 1 each)."""
    dts = np.ascontiguousarray(dts, np.float64)
    W = 5 + 2 * (RUNG_MAX + 1)
    out = np.zeros((len(dts), W))
    rc = _lib("cosmo").reftree_cosmo_steps(float(a0), float(adot0), float(H0), float(omega_m), float(omega_lambda),
                                          dts.ctypes.data, len(dts), out.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_cosmo_steps: %d" % rc)
    return [dict(a_last=o[0], a=o[1], time=o[2], tau=o[3], drift=o[4], kick1=o[5:5 + RUNG_MAX + 1],
                 kick2=o[5 + RUNG_MAX + 1:]) for o in out]


def kick(x, v, rung, g, min_rung, do_out, dt_max, eta, soft_len, G=1.0):
    """The reference's part_vect_kick (src/part_vect.cpp:341-436) on these
    particles with accelerations g (float32, per unit G) for the ones it takes:
    returns (v, rung, largest new rung).  t_max = 1, no cosmology, Ewald off."""
    x = np.ascontiguousarray(x, np.int32)
    v = np.ascontiguousarray(v, np.float32)
    rung = np.ascontiguousarray(rung, np.int8)
    g = np.ascontiguousarray(g, np.float32)
    n = len(x)
    vo = np.zeros((n, 3), np.float32)
    ro = np.zeros(n, np.int8)
    mr = np.zeros(1, np.int32)
    key = ("kick", float(dt_max), float(eta), float(soft_len), float(G))
    rc = _lib(key).reftree_kick(x.ctypes.data, v.ctypes.data, rung.ctypes.data, g.ctypes.data, n, int(min_rung),
                                int(bool(do_out)), float(dt_max), float(eta), float(soft_len), float(G), vo.ctypes.data,
                                ro.ctypes.data, mr.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_kick: %d" % rc)
    return vo, ro, int(mr[0])


def drift(x, v, mrung):
    """The reference's part_vect_drift (src/part_vect.cpp:493-540) by
    rung_to_dt(mrung) (t_max = 1): the new int32 positions."""
    x = np.ascontiguousarray(x, np.int32)
    v = np.ascontiguousarray(v, np.float32)
    xo = np.zeros_like(x)
    rc = _lib(("drift", len(x))).reftree_drift(x.ctypes.data, v.ctypes.data, len(x), int(mrung), xo.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_drift: %d" % rc)
    return xo


def fof(x, link_len, leaf_max=64):
    """The reference's friends-of-friends partition (tree::find_groups and
    part_vect_find_groups driven as solve_gravity drives them): per caller
    particle its group id (the reference's smallest storage index in the
    group), -1 without friends."""
    x = np.ascontiguousarray(x, np.int32)
    n = len(x)
    label = np.zeros(n, np.int64)
    rc = _lib(("fof", n, float(link_len), int(leaf_max))).reftree_fof(x.ctypes.data, n, float(link_len),
                                                                      int(leaf_max), label.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_fof: %d" % rc)
    return label


def fof_catalog(x, v, link_len, leaf_max=64, cap=1 << 16):
    """The partition of fof() and the reference's catalogue of it (groups.cpp
    fed by the output kick, a = 1): (label, dict of arrays id (the
    reference's group id), N, x, v, dv, rmax, rc)."""
    x = np.ascontiguousarray(x, np.int32)
    v = np.ascontiguousarray(v, np.float32)
    n = len(x)
    label = np.zeros(n, np.int64)
    cat = np.zeros((cap, 13))
    ng = np.zeros(1, np.int64)
    rc = _lib(("fofcat", n, float(link_len), int(leaf_max))).reftree_fof_catalog(
        x.ctypes.data, v.ctypes.data, n, float(link_len), int(leaf_max), label.ctypes.data, cap, cat.ctypes.data,
        ng.ctypes.data)
    if rc != 0 or ng[0] > cap:
        raise RuntimeError("reftree_fof_catalog: %d (%d groups)" % (rc, ng[0]))
    c = cat[:ng[0]]
    return label, dict(id=c[:, 0].astype(np.int64), N=c[:, 1].astype(np.int64), x=c[:, 2:5], v=c[:, 5:8],
                       dv=c[:, 8:11], rmax=c[:, 11], rc=c[:, 12])


def load_gadget1(path, cap=1 << 22):
    """The reference's load_particles (src/load.cpp:34-96): int32 positions
    and float velocities of a Gadget-1 file."""
    x = np.zeros((cap, 3), np.int32)
    v = np.zeros((cap, 3), np.float32)
    n = np.zeros(1, np.int64)
    rc = _lib(("load",)).reftree_load_gadget1(str(path).encode(), cap, x.ctypes.data, v.ctypes.data, n.ctypes.data)
    if rc != 0:
        raise RuntimeError("reftree_load_gadget1: %d" % rc)
    return x[:n[0]].copy(), v[:n[0]].copy()
