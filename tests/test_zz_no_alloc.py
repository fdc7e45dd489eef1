"""tg_energy_noalloc: the energy / momentum reduction for callers that cannot
allocate device memory (a host code that owns a fixed memory arena, an
allocation-free time loop).  It must give what tg_energy gives for the same
particles, call after call, while keeping its partial sums in the library's
fixed scratch array instead of a cudaMalloc'd buffer.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10  # both are FP64 reductions of the same FP32 values, in different orders


def _check(ref, got):
    for k, (a, b) in enumerate(zip(ref, got)):
        scale = max(abs(a), 1e-300)
        assert abs(a - b) <= REL_TOL * scale + 1e-300, (k, a, b)


def test_noalloc_energy_matches_tg_energy_twice():
    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import _lib, ics

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
    v_d = torch.tensor(v, device="cuda")
    phi_d = torch.tensor(phi, device="cuda")
    out = torch.empty(5, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        rc = _lib.lib.tg_energy_noalloc(C.c_void_p(v_d.data_ptr()), C.c_void_p(phi_d.data_ptr()), n,
                                        1.0 / n, 1.0, C.c_void_p(out.data_ptr()), 0, None)
        assert rc == _lib.TG_OK, _lib.lib.tg_error_string(rc)
        torch.cuda.synchronize()
        _check(ref, out.cpu().numpy().tolist())


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from tigergrav_b200 import _lib
    rc = _lib.lib.tg_energy_noalloc(C.c_void_p(16), None, _lib.TG_NOALLOC_MAX_N + 1, 1.0, 1.0, C.c_void_p(16), 0,
                                    None)
    assert rc == _lib.TG_ERR_SIZE
    assert b"TG_NOALLOC_MAX_N" in _lib.lib.tg_error_string(rc)
