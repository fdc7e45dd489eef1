"""tg_energy_noalloc: the energy / momentum reduction for callers that cannot
allocate device memory (a host code that owns a fixed memory arena, an
allocation-free time loop).  It must give what tg_energy gives for the same
particles, call after call, while keeping its partial sums in the library's
fixed scratch array instead of a cudaMalloc'd buffer.  Both are also checked
against a plain FP64 sum on the host, so the pair cannot agree on a shared
mistake.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # FP64 reductions of the same FP32 values, in different orders


def _check(ref, got, what):
    for k, (a, b) in enumerate(zip(ref, got)):
        scale = max(abs(a), 1e-300)
        assert abs(a - b) <= REL_TOL * scale + 1e-300, (what, k, a, b)


def _host_sums(v, phi, m, G):
    """E_kin, E_pot, mean velocity in FP64 on the host (the definition)."""
    v64 = v.astype(np.float64)
    ekin = float(np.sum(0.5 * m * np.sum(v64 * v64, axis=1)))
    epot = 0.0 if phi is None else float(np.sum(0.5 * m * phi.astype(np.float64) * G))
    mom = (np.sum(v64, axis=0) / len(v)).tolist()
    return [ekin, epot, *mom]


def _noalloc(v_d, phi_d, n, m, G, out):
    import torch
    from tigergrav_b200 import _lib
    out.fill_(float("nan"))
    rc = _lib.lib.tg_energy_noalloc(C.c_void_p(v_d.data_ptr()),
                                    None if phi_d is None else C.c_void_p(phi_d.data_ptr()), n, m, G,
                                    C.c_void_p(out.data_ptr()), 0, None)
    assert rc == _lib.TG_OK, _lib.lib.tg_error_string(rc)
    torch.cuda.synchronize()
    assert torch.cuda.current_device() == 0
    return out.cpu().numpy().tolist()


def test_noalloc_energy_matches_tg_energy_twice():
    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics

    x = ics.clustered(16, 3)
    n = len(x)
    rng = np.random.Generator(np.random.PCG64(12))
    v = rng.normal(scale=0.01, size=(n, 3)).astype(np.float32)
    with tg.GravitySolver(n, theta=0.7) as s:
        s.set_particles(x, v)
        s.solve_gravity()
        e = s.energy()
        ref = [e["ekin"], e["epot"], *e["momentum"]]
        phi, _ = s.get_forces(dtype=np.float32)
    _check(_host_sums(v, phi, 1.0 / n, 1.0), ref, "tg_energy vs host FP64")
    v_d = torch.tensor(v, device="cuda")
    phi_d = torch.tensor(phi, device="cuda")
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    for _ in range(2):
        _check(ref, _noalloc(v_d, phi_d, n, 1.0 / n, 1.0, out), "noalloc vs tg_energy")


def test_noalloc_larger_then_smaller_call_and_no_potential():
    """A call over fewer particles after one over more must not pick up the
    earlier call's partial sums left in the shared array; phi = NULL gives
    E_pot = 0."""
    import torch
    rng = np.random.Generator(np.random.PCG64(13))
    n_big = 3 * 1024 * 7 + 517
    v = rng.normal(scale=0.02, size=(n_big, 3)).astype(np.float32)
    phi = rng.normal(loc=-1.0, scale=0.3, size=n_big).astype(np.float32)
    v_d = torch.tensor(v, device="cuda")
    phi_d = torch.tensor(phi, device="cuda")
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    m, G = 1.0 / n_big, 1.3
    for n in (n_big, n_big // 3 + 7, 1, n_big):
        _check(_host_sums(v[:n], phi[:n], m, G), _noalloc(v_d, phi_d, n, m, G, out), "n=%d" % n)
    got = _noalloc(v_d, None, n_big // 3 + 7, m, G, out)
    assert got[1] == 0.0
    _check(_host_sums(v[:n_big // 3 + 7], None, m, G), got, "phi=NULL")


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from tigergrav_b200 import _lib
    rc = _lib.lib.tg_energy_noalloc(C.c_void_p(16), None, _lib.TG_NOALLOC_MAX_N + 1, 1.0, 1.0, C.c_void_p(16), 0,
                                    None)
    assert rc == _lib.TG_ERR_SIZE
    assert b"TG_NOALLOC_MAX_N" in _lib.lib.tg_error_string(rc)
