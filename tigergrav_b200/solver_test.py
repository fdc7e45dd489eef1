"""The reference's solver test (src/main.cpp:137-165, compute_error in
src/output.cpp:17-51) on the GPU path: the forces at theta = 1e-10 (every
interaction a particle pair) are the "direct" solution, then theta runs from
1.0 down to 0.2 in steps of 0.1, printing time, GFLOP/s in the reference's
flop convention, the mean and 99th-percentile per-particle relative force
error against the direct solution, and the mean acceleration.

    python -m tigergrav_b200.solver_test --n 4096 [--clustered] [--precision f64]
"""
import argparse

import numpy as np


def run(x, precision="f32", thetas=None, ewald=True):
    import torch
    from .solver import GravitySolver
    n = len(x)
    thetas = thetas if thetas is not None else [round(1.0 - 0.1 * k, 1) for k in range(9)]
    with GravitySolver(n, theta=1e-10, ewald=ewald, precision=precision) as s:
        s.set_particles(x).solve_gravity()
        _, gd = s.get_forces()
    rows = []
    for th in thetas:
        with GravitySolver(n, theta=th, ewald=ewald, precision=precision) as s:
            s.set_particles(x).solve_gravity()  # warm-up: buffers and tables
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            s.solve_gravity()
            b.record()
            torch.cuda.synchronize()
            sec = a.elapsed_time(b) * 1e-3
            st = s.stats()
            _, g = s.get_forces()
        # src/output.cpp:33-35: |dg| / |g_test|, mean and the top-1% threshold
        e = np.linalg.norm(g - gd, axis=1) / np.linalg.norm(g, axis=1)
        gm = g.mean(axis=0) / n
        rows.append(dict(theta=th, time=sec, gflops=st["flops"] / sec / 1024 ** 3, error=float(e.mean()),
                         error99=float(np.sort(e)[-max(1, n // 100)]), g=gm.tolist()))
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--clustered", action="store_true")
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()
    from . import ics
    x = ics.clustered(round(args.n ** (1 / 3)), args.seed) if args.clustered else ics.uniform(args.n, args.seed)
    print("%11s %11s %11s %11s %11s %11s %11s %11s" % ("theta", "time", "GFLOPS", "error", "error99", "gx", "gy",
                                                       "gz"))
    for r in run(x, args.precision):
        print("%11.4e %11.4e %11.4e %11.4e %11.4e %11.4e %11.4e %11.4e" % (
            r["theta"], r["time"], r["gflops"], r["error"], r["error99"], *r["g"]))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
