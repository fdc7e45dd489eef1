"""Host-side mirror of TigerGrav's gravity-path interface over the C ABI.

``GravitySolver`` plays the role of the reference's tree_client plus the
particle store for the gravity path:

  reference                                         here
  ------------------------------------------------  ---------------------------
  options (theta, soft_len, m_tot/N, G, ewald,       GravitySolver(theta=..., ...)
  parts_per_node)  tigergrav/options.hpp:5-82
  part_vect_init   src/part_vect.cpp:654-673         set_particles(x, v)
  tree::refine     src/tree.cpp:122-201              build()
  tree::compute_multipoles  src/tree.cpp:203-296     multipoles()
  tree::kick_fmm (lists)    src/tree.cpp:378-635     walk()
  tree::kick_fmm (kernels)                           forces()
  solve_gravity    src/main.cpp:31-73                solve_gravity()
  part_vect_kick / part_vect_drift                   kick(dt) / drift(dt)
  interaction_stats  tigergrav/tree.hpp:84-114       stats()

Arrays may be numpy (host) or torch CUDA tensors (device); results come back
in the caller's particle order.  Every call goes to the CUDA library; errors
raise ``TGError`` (the reference aborts instead).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import lib, check, tg_params, tg_stats, tg_cosmo_params, tg_rung_params, tg_rung_state, tg_cosmo_rung_state, TG_HOST, TG_DEVICE, TG_PREC_F32, TG_PREC_F64, \
    LIST_KINDS


def _is_torch_cuda(a) -> bool:
    return hasattr(a, "is_cuda") and bool(getattr(a, "is_cuda"))


def _ptr(a):
    if a is None:
        return None, TG_HOST
    if _is_torch_cuda(a):
        assert a.is_contiguous()
        return C.c_void_p(a.data_ptr()), TG_DEVICE
    if hasattr(a, "data_ptr"):  # torch CPU tensor (pinned ones are copied without staging)
        assert a.is_contiguous()
        return C.c_void_p(a.data_ptr()), TG_HOST
    assert isinstance(a, np.ndarray) and a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data), TG_HOST


def _stream(stream):
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return C.c_void_p(stream.cuda_stream)
    return C.c_void_p(int(stream))


def make_params(theta=0.7, soft_len=None, m=None, G=1.0, ewald=True, leaf_max=64, precision="f32", device=0,
                n=None) -> tg_params:
    if soft_len is None:
        soft_len = 0.02 * float(n) ** (-1.0 / 3.0)
    if m is None:
        m = 1.0 / float(n)
    prec = {"f32": TG_PREC_F32, "f64": TG_PREC_F64}[precision] if isinstance(precision, str) else int(precision)
    return tg_params(theta, soft_len, m, G, int(bool(ewald)), int(leaf_max), prec, int(device))


class GravitySolver:
    """One periodic box on one GPU.  Parameters default to the reference's
    (soft_len = 0.02 N^-1/3, src/options.cpp:86-88; m = 1/N; leaf 64)."""

    def __init__(self, n: int, theta=0.7, soft_len=None, m=None, G=1.0, ewald=True, leaf_max=64,
                 precision="f32", device=0):
        self.n = int(n)
        self.params = make_params(theta, soft_len, m, G, ewald, leaf_max, precision, device, n=n)
        h = C.c_void_p()
        check("tg_create", lib.tg_create(C.byref(self.params), C.byref(h)))
        self.h = h
        self.stream = None

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.tg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- particles ----
    def set_particles(self, x, v=None, stream=None):
        assert len(x) == self.n
        px, wx = _ptr(x)
        pv, wv = _ptr(v)
        if v is not None:
            assert wv == wx, "x and v must both be host or both device arrays"
        check("tg_set_particles", lib.tg_set_particles(self.h, px, pv, self.n, wx, _stream(stream)))
        return self

    def get_particles(self):
        x = np.zeros((self.n, 3), np.int32)
        v = np.zeros((self.n, 3), np.float32)
        check("tg_get_particles", lib.tg_get_particles(self.h, x.ctypes.data, v.ctypes.data, TG_HOST, None))
        return x, v

    # ---- the gravity path ----
    def build(self, stream=None):
        check("tg_build", lib.tg_build(self.h, _stream(stream)))
        return self

    def multipoles(self, stream=None):
        check("tg_multipoles", lib.tg_multipoles(self.h, _stream(stream)))
        return self

    def walk(self, stream=None):
        check("tg_walk", lib.tg_walk(self.h, _stream(stream)))
        return self

    def set_walk_capacity(self, entries: int):
        """First capacity of every list pool for the following walks (0: sized
        from the tree); a small value exercises the regrowth path."""
        check("tg_set_walk_capacity", lib.tg_set_walk_capacity(self.h, int(entries)))
        return self

    def forces(self, stream=None):
        check("tg_forces", lib.tg_forces(self.h, _stream(stream)))
        return self

    def solve_gravity(self, stream=None):
        check("tg_solve_gravity", lib.tg_solve_gravity(self.h, _stream(stream)))
        return self

    def get_forces(self, dtype=np.float64, out_phi=None, out_g=None, stream=None):
        """(phi[n], g[n,3]) in caller order; numpy by default, or fill torch CUDA tensors."""
        if out_phi is not None or out_g is not None:
            pp, w = _ptr(out_phi)
            pg, w2 = _ptr(out_g)
            w = w if out_phi is not None else w2
            t = out_phi if out_phi is not None else out_g
            is64 = str(t.dtype).endswith("float64")
            fn = lib.tg_get_forces_f64 if is64 else lib.tg_get_forces
            check("tg_get_forces", fn(self.h, pp, pg, w, _stream(stream)))
            return out_phi, out_g
        phi = np.zeros(self.n, dtype)
        g = np.zeros((self.n, 3), dtype)
        fn = lib.tg_get_forces_f64 if dtype == np.float64 else lib.tg_get_forces
        check("tg_get_forces", fn(self.h, phi.ctypes.data, g.ctypes.data, TG_HOST, _stream(stream)))
        return phi, g

    def kick(self, dt, stream=None):
        check("tg_kick", lib.tg_kick(self.h, float(dt), _stream(stream)))

    def drift(self, dt, stream=None):
        check("tg_drift", lib.tg_drift(self.h, float(dt), _stream(stream)))

    def kick_drift(self, dt_close, dt_open, dt_drift, stream=None):
        """The closing kick of one step, the opening kick of the next and the
        drift, in one pass (dt_close = 0 skips the first kick)."""
        check("tg_kick_drift", lib.tg_kick_drift(self.h, float(dt_close), float(dt_open), float(dt_drift),
                                                 _stream(stream)))
        return self

    def leapfrog(self, dt, n_steps, stream=None):
        check("tg_leapfrog", lib.tg_leapfrog(self.h, float(dt), int(n_steps), _stream(stream)))

    # ---- differentiation ----
    def forward(self, dt, n_steps, stream=None):
        """n_steps leapfrog steps with checkpoints for backward()."""
        check("tg_forward", lib.tg_forward(self.h, float(dt), int(n_steps), _stream(stream)))
        return self

    def backward(self, gx, gv=None, stream=None):
        """(dL/dx0, dL/dv0) from dL/dx, dL/dv after the last forward() step (n x 3, caller order)."""
        gx = np.ascontiguousarray(gx, np.float64)
        gv = None if gv is None else np.ascontiguousarray(gv, np.float64)
        gx0 = np.zeros((self.n, 3))
        gv0 = np.zeros((self.n, 3))
        check("tg_backward", lib.tg_backward(self.h, gx.ctypes.data, None if gv is None else gv.ctypes.data,
                                             gx0.ctypes.data, gv0.ctypes.data, TG_HOST, _stream(stream)))
        return gx0, gv0

    def tidal(self, u, stream=None):
        """J u (J = dg/dx per unit G) at the current particles and lists (n x 3, caller order)."""
        u = np.ascontiguousarray(u, np.float64)
        out = np.zeros((self.n, 3))
        check("tg_tidal", lib.tg_tidal(self.h, u.ctypes.data, out.ctypes.data, TG_HOST, _stream(stream)))
        return out

    def find_groups(self, link_len=0.2, stream=None):
        """Friends-of-friends groups (tree::find_groups, src/tree.cpp:637-759;
        the friend test of src/part_vect.cpp:85-124): per caller index the
        group id (the smallest caller index in the group) or -1 for a particle
        without friends.  link_len is in mean interparticle spacings."""
        g = np.zeros(self.n, np.int64)
        ng = C.c_int64(0)
        check("tg_find_groups", lib.tg_find_groups(self.h, float(link_len), g.ctypes.data, C.byref(ng), TG_HOST,
                                                   _stream(stream)))
        return g

    def group_catalog(self, a=1.0, stream=None) -> dict:
        """Statistics of the groups of the last find_groups (src/groups.cpp:124-226),
        ids ascending: id, N, x (n,3), v (n,3), dv (n,3), rmax, rc."""
        ng = C.c_int64(0)
        check("tg_group_catalog", lib.tg_group_catalog(self.h, float(a), None, 0, C.byref(ng), _stream(stream)))
        out = np.zeros((max(ng.value, 1), 14))
        check("tg_group_catalog", lib.tg_group_catalog(self.h, float(a), out.ctypes.data, ng.value, C.byref(ng),
                                                       _stream(stream)))
        out = out[:ng.value]
        return dict(id=out[:, 0].astype(np.int64), N=out[:, 1].astype(np.int64), x=out[:, 2:5], v=out[:, 5:8],
                    dv=out[:, 8:11], rmax=out[:, 11], rc=out[:, 12])

    def groups_output(self, path, a=1.0, min_size=10, stream=None):
        """The group file of groups_output (src/groups.cpp:78-100): one line
        per group of at least min_size members: id, N, rmax, rc, |v|, |dv|."""
        c = self.group_catalog(a, stream)
        with open(path, "wt") as fp:
            keep = np.nonzero(c["N"] >= min_size)[0]
            for k in keep:
                fp.write("%16li %5i %12e %12e %12e %12e\n" % (c["id"][k], c["N"][k], c["rmax"][k], c["rc"][k],
                                                             np.linalg.norm(c["v"][k]), np.linalg.norm(c["dv"][k])))
            if len(keep) == 0:
                fp.write("No groups\n")
        return len(keep)

    def rung_step(self, state=None, t_max=1.0, dt_max=None, eta=0.2, all_forces=False, stream=None):
        """One step of hierarchical (rung) time stepping (src/main.cpp:266-313,
        src/part_vect.cpp:340-381); state None starts at itime 0.  Returns the
        new state dict: itime, max_rung, min_rung, num_active, t."""
        st = tg_rung_state(0, -1, 0, 0, 0, 0.0)
        if state is not None:
            st.itime, st.max_rung, st.min_rung = state["itime"], state["max_rung"], state["min_rung"]
            st.num_active, st.t = state["num_active"], state["t"]
        p = tg_rung_params(float(t_max), float(t_max if dt_max is None else dt_max), float(eta))
        check("tg_rung_step", lib.tg_rung_step(self.h, C.byref(p), C.byref(st), int(bool(all_forces)),
                                               _stream(stream)))
        return dict(itime=st.itime, max_rung=st.max_rung, min_rung=st.min_rung, num_active=st.num_active, t=st.t)

    def rung_step_cosmo(self, state, cstate, H0, omega_m=0.3, omega_lambda=0.7, t_max=1.0, dt_max=None, eta=0.2,
                        all_forces=False, stream=None):
        """rung_step with the reference's cosmological kick and drift factors.
        cstate: a tg_cosmo_rung_state (from cosmo_rung_state()), updated in place."""
        st = tg_rung_state(0, -1, 0, 0, 0, 0.0)
        if state is not None:
            st.itime, st.max_rung, st.min_rung = state["itime"], state["max_rung"], state["min_rung"]
            st.num_active, st.t = state["num_active"], state["t"]
        p = tg_rung_params(float(t_max), float(t_max if dt_max is None else dt_max), float(eta))
        cp = tg_cosmo_params(float(H0), float(omega_m), float(omega_lambda))
        check("tg_rung_step_cosmo", lib.tg_rung_step_cosmo(self.h, C.byref(p), C.byref(st), C.byref(cp),
                                                           C.byref(cstate), int(bool(all_forces)), _stream(stream)))
        return dict(itime=st.itime, max_rung=st.max_rung, min_rung=st.min_rung, num_active=st.num_active, t=st.t)

    def rungs(self, stream=None) -> np.ndarray:
        """Per-particle rungs in caller order (int8)."""
        r = np.zeros(self.n, np.int8)
        check("tg_get_rungs", lib.tg_get_rungs(self.h, r.ctypes.data, TG_HOST, _stream(stream)))
        return r

    def leapfrog_cosmo(self, dt, n_steps, state, H0, omega_m=0.3, omega_lambda=0.7, stream=None):
        """n_steps comoving KDK steps with the cosmological factors; state = [a, da/dt, tau] (updated)."""
        st = np.ascontiguousarray(state, np.float64)
        p = tg_cosmo_params(H0, omega_m, omega_lambda)
        check("tg_leapfrog_cosmo", lib.tg_leapfrog_cosmo(self.h, C.byref(p), st.ctypes.data, float(dt), int(n_steps),
                                                         _stream(stream)))
        return st

    def energy(self, stream=None) -> dict:
        out = np.zeros(5)
        check("tg_energy", lib.tg_energy(self.h, out.ctypes.data, _stream(stream)))
        return dict(ekin=out[0], epot=out[1], momentum=out[2:5].copy())

    def stats(self) -> dict:
        s = tg_stats()
        check("tg_get_stats", lib.tg_get_stats(self.h, C.byref(s)))
        kinds = ("PP_D", "PP_E", "PC_D", "PC_E", "CC_D", "CC_E", "CP_D", "CP_E")
        refk = ("PP_direct", "PP_ewald", "CC_direct", "CC_ewald", "CP_direct", "CP_ewald")
        return dict(n=s.n, nodes=s.nodes, leaves=s.leaves, depth=s.depth, walk_retries=s.walk_retries,
                    ref_stats=dict(zip(refk, map(int, s.ref_stats))), counts=dict(zip(kinds, map(int, s.counts))),
                    flops=s.flops, launches=s.launches, device_bytes=s.device_bytes, ms=dict(build=s.ms_build, multipoles=s.ms_multipoles, walk=s.ms_walk,
                                           nodes=s.ms_nodes, leaves=s.ms_leaves, pp=s.ms_pp,
                                           kick_drift=s.ms_kick_drift))

    def memory(self) -> dict:
        """Device bytes per buffer of this handle (and "total")."""
        buf = C.create_string_buffer(1 << 16)
        check("tg_memory_report", lib.tg_memory_report(self.h, buf, len(buf)))
        return {k: int(v) for k, v in (ln.split() for ln in buf.value.decode().splitlines())}

    # ---- introspection ----
    @property
    def num_nodes(self) -> int:
        return int(lib.tg_num_nodes(self.h))

    def nodes(self) -> dict:
        nn = self.num_nodes
        d = dict(boxid=np.zeros(nn, np.uint64), level=np.zeros(nn, np.int32), pbegin=np.zeros(nn, np.int64),
                 pend=np.zeros(nn, np.int64), child0=np.zeros(nn, np.int32), parent=np.zeros(nn, np.int32),
                 x=np.zeros((nn, 3), np.int32), r=np.zeros(nn, np.float32), rmax=np.zeros(nn, np.float32),
                 m=np.zeros((nn, 17), np.float32))
        check("tg_get_nodes", lib.tg_get_nodes(self.h, *[d[k].ctypes.data for k in
                                                           ("boxid", "level", "pbegin", "pend", "child0", "parent",
                                                            "x", "r", "rmax", "m")]))
        return d

    def perm(self) -> np.ndarray:
        p = np.zeros(self.n, np.int64)
        check("tg_get_perm", lib.tg_get_perm(self.h, p.ctypes.data))
        return p

    def list(self, kind: str):
        k = LIST_KINDS[kind]
        tot = lib.tg_list_size(self.h, k)
        if tot < 0:
            raise _lib.TGError("tg_list_size", _lib.TG_ERR_STATE, "no lists")
        off = np.zeros(self.num_nodes + 1, np.int64)
        ids = np.zeros(max(tot, 1), np.int32)
        check("tg_get_list", lib.tg_get_list(self.h, k, off.ctypes.data, ids.ctypes.data))
        return off, ids[:tot]

    def truth(self, samples, alpha=8.0):
        """FP64 direct Ewald sum at the sample particles (caller indices)."""
        s = np.ascontiguousarray(samples, np.int64)
        phi = np.zeros(len(s))
        g = np.zeros((len(s), 3))
        check("tg_truth", lib.tg_truth(self.h, s.ctypes.data, len(s), float(alpha), phi.ctypes.data, g.ctypes.data,
                                       None))
        return phi, g


class GravityBatch:
    """Many independent periodic unit boxes (counts[b] particles each, m = 1/N_b,
    soft_len = 0.02 N_b^-1/3) evaluated together on nstreams streams."""

    def __init__(self, counts, theta=0.7, G=1.0, ewald=True, leaf_max=64, precision="f32", device=0, nstreams=16):
        self.counts = np.ascontiguousarray(counts, np.int64)
        self.n = int(self.counts.sum())
        self.params = make_params(theta, 1.0, 1.0, G, ewald, leaf_max, precision, device)
        h = C.c_void_p()
        check("tg_batch_create", lib.tg_batch_create(C.byref(self.params), len(self.counts), self.counts.ctypes.data,
                                                     int(nstreams), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib.tg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_particles(self, x, v=None):
        x = np.ascontiguousarray(x, np.int32)
        assert x.shape == (self.n, 3)
        v = None if v is None else np.ascontiguousarray(v, np.float32)
        check("tg_batch_set_particles", lib.tg_batch_set_particles(self.h, x.ctypes.data,
                                                                   None if v is None else v.ctypes.data, TG_HOST))
        return self

    def autotune(self, leaf_sizes=(16, 32, 64, 128)):
        ls = np.ascontiguousarray(leaf_sizes, np.int32)
        chosen = np.zeros(len(self.counts), np.int32)
        check("tg_batch_autotune", lib.tg_batch_autotune(self.h, ls.ctypes.data, len(ls), chosen.ctypes.data))
        return chosen

    def solve(self):
        check("tg_batch_solve", lib.tg_batch_solve(self.h))
        return self

    def leapfrog(self, dt, n_steps):
        check("tg_batch_leapfrog", lib.tg_batch_leapfrog(self.h, float(dt), int(n_steps)))
        return self

    def get_forces(self):
        phi = np.zeros(self.n, np.float32)
        g = np.zeros((self.n, 3), np.float32)
        check("tg_batch_get_forces", lib.tg_batch_get_forces(self.h, phi.ctypes.data, g.ctypes.data, TG_HOST))
        return phi, g


def cosmo_rung_state(a=1.0, adot=None, H0=None):
    """A fresh cosmological rung-step state at scale factor a (adot defaults to H0)."""
    cs = tg_cosmo_rung_state()
    check("tg_cosmo_rung_init", lib.tg_cosmo_rung_init(C.byref(cs), float(a), float(H0 if adot is None else adot)))
    return cs


def cosmo_kdk(state, dt, H0, omega_m=0.3, omega_lambda=0.7):
    """One KDK step's cosmological factors (src/cosmo.cpp:50-106,187-218):
    returns (new state [a, da/dt, tau], [kick1, drift, kick2])."""
    st = np.array(state, np.float64)
    f = np.zeros(3)
    p = tg_cosmo_params(H0, omega_m, omega_lambda)
    check("tg_cosmo_kdk", lib.tg_cosmo_kdk(C.byref(p), st.ctypes.data, float(dt), f.ctypes.data))
    return st, f


def load_gadget1(path):
    """N-GenIC / Gadget-1 initial conditions as the reference loads them
    (src/load.cpp:34-96): (header dict, x int32 (n,3) fixed point, v float32 (n,3))."""
    hdr = np.zeros(8)
    n = C.c_int64(0)
    check("tg_load_gadget1", lib.tg_load_gadget1(str(path).encode(), hdr.ctypes.data, None, None, 0, C.byref(n)))
    x = np.zeros((n.value, 3), np.int32)
    v = np.zeros((n.value, 3), np.float32)
    check("tg_load_gadget1", lib.tg_load_gadget1(str(path).encode(), hdr.ctypes.data, x.ctypes.data, v.ctypes.data,
                                                 n.value, C.byref(n)))
    keys = ("npart", "redshift", "mass", "omega_m", "omega_lambda", "hubble_param", "box_size", "time")
    h = dict(zip(keys, hdr.tolist()))
    h["npart"] = int(h["npart"])
    return h, x, v


def device_fp32_peak(device=0) -> float:
    """Measured FP32 FMA throughput of the device in TFLOP/s."""
    t = C.c_double(0)
    check("tg_device_fp32_peak", lib.tg_device_fp32_peak(int(device), C.byref(t), None))
    return t.value


# ---- kernel-level seams (torch CUDA tensors) ----
def _dp(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def gravity_PP(kind, params, sink_off, sink_x, src_off, src_x, f, do_phi=True, stream=None):
    fl = C.c_uint64(0)
    ng = len(sink_off) - 1
    if kind == "direct":
        check("tg_gravity_PP_direct", lib.tg_gravity_PP_direct(C.byref(params), ng, _dp(sink_off), _dp(sink_x),
                                                               _dp(src_off), _dp(src_x), _dp(f), int(do_phi),
                                                               C.byref(fl), _stream(stream)))
    else:
        check("tg_gravity_PP_ewald", lib.tg_gravity_PP_ewald(C.byref(params), ng, _dp(sink_off), _dp(sink_x),
                                                             _dp(src_off), _dp(src_x), _dp(f), C.byref(fl),
                                                             _stream(stream)))
    return fl.value


def gravity_PC(kind, params, sink_off, sink_x, src_off, src_m, src_x, f, stream=None):
    fl = C.c_uint64(0)
    ng = len(sink_off) - 1
    fn = lib.tg_gravity_PC_direct if kind == "direct" else lib.tg_gravity_PC_ewald
    check("tg_gravity_PC_" + kind, fn(C.byref(params), ng, _dp(sink_off), _dp(sink_x), _dp(src_off), _dp(src_m),
                                      _dp(src_x), _dp(f), C.byref(fl), _stream(stream)))
    return fl.value


def gravity_CC(kind, params, sink_x, src_off, src_m, src_x, L, stream=None):
    fl = C.c_uint64(0)
    ng = len(src_off) - 1
    fn = lib.tg_gravity_CC_direct if kind == "direct" else lib.tg_gravity_CC_ewald
    check("tg_gravity_CC_" + kind, fn(C.byref(params), ng, _dp(sink_x), _dp(src_off), _dp(src_m), _dp(src_x),
                                      _dp(L), C.byref(fl), _stream(stream)))
    return fl.value


def gravity_CP(kind, params, sink_x, src_off, src_x, L, stream=None):
    fl = C.c_uint64(0)
    ng = len(src_off) - 1
    fn = lib.tg_gravity_CP_direct if kind == "direct" else lib.tg_gravity_CP_ewald
    check("tg_gravity_CP_" + kind, fn(C.byref(params), ng, _dp(sink_x), _dp(src_off), _dp(src_x), _dp(L),
                                      C.byref(fl), _stream(stream)))
    return fl.value
