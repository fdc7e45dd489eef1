"""A fixed, small force-evaluation run for profilers (ncu -k/-s/-c captures).

    python -m tigergrav_b200.profile --nside 128 --theta 0.3 --reps 2

Builds the seeded clustered box (seed 2), evaluates the forces `reps` times
and prints the per-phase device times of the last evaluation.  Each
evaluation launches every kernel of the path once per phase, so `ncu -s k -c m
-k regex:<kernel>` selects evaluation k+1 onwards.
"""
import argparse


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nside", type=int, default=128)
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--seed", type=int, default=2)
    args = ap.parse_args()
    import torch
    from . import ics
    from .solver import GravitySolver
    x = ics.clustered(args.nside, args.seed)
    with GravitySolver(len(x), theta=args.theta, precision=args.precision) as s:
        s.set_particles(x)
        for _ in range(args.reps):
            s.solve_gravity()
        torch.cuda.synchronize()
        st = s.stats()
    print({k: round(float(v), 3) for k, v in st["ms"].items()}, {k: int(v) for k, v in st["counts"].items()})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
