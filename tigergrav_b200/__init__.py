"""tigergrav_b200 -- B200 (sm_100a) periodic tree gravity with TigerGrav's method.

The compute lives in ``libtigergrav_b200.so`` (C ABI: include/tigergrav_b200.h);
this package is its host-side binding.  ``ics`` (seeded workloads) needs no GPU;
``GravitySolver`` and the kernel-level seams load the CUDA library on first use
and raise if it is missing.
"""
__all__ = ["GravitySolver", "GravityBatch", "make_params", "gravity_PP", "gravity_PC", "gravity_CC", "gravity_CP"]


def __getattr__(name):
    if name in ("GravitySolver", "GravityBatch", "make_params", "gravity_PP", "gravity_PC", "gravity_CC",
                "gravity_CP"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
