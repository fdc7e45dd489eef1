"""Benchmark: periodic tree gravity on B200 (one JSON line on stdout).

Workload (default): 128^3 = 2,097,152 particles on a lattice displaced by a
seeded Gaussian random field with P(k) ~ k^-2 (rms displacement 0.5 spacing),
periodic unit box, theta = 0.7, Ewald on, leaf 64, FP32 path.
A step is one kick-drift-kick leapfrog step at dt = 1e-3: half kick, drift,
a full force evaluation (tree build, multipoles, walk, all interaction
kernels), half kick.  value = particles / step time = Mparticles/s per force
evaluation.  Inputs stay resident in HBM; L2 is flushed (256 MB write, untimed)
between timed steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  torchrun --nproc-per-node N bench.py --gpus N ...   (independent replicas)

--impl reference times the reference's own CPU kernels (src/gravity.cpp,
compiled from the reference sources into oracle/_ref) driven by the oracle's
restatement of its tree and walk, on the host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "clustered128": dict(kind="clustered", nside=128, seed=2),
    "clustered64": dict(kind="clustered", nside=64, seed=5),
    "clustered256": dict(kind="clustered", nside=256, seed=8),
    "uniform32": dict(kind="uniform", n=32768, seed=1),
}

# FP32 operations per PP pair in k_pp_f32's inner loop, counted from the
# source with an FMA as 2: separation 9 (per axis two differences of split
# coordinates and their sum), r^2 5 (1 mul + 2 fma), min 1, clamp 1,
# rsqrt 1, 1/r^3 2, phi sum 1, three force FMAs 6 -> 26 (the Kahan fold,
# ~1.3 per pair, is not counted).  Roofline numerator.
EXEC_FLOPS = {"PP_D": 26}
# DRAM bytes per PP pair of k_pp_f32 (ncu capture, filled in from profiles/)
TRAFFIC_PP_BYTES_PER_PAIR = 0.0


def make_particles(w):
    from tigergrav_b200 import ics
    if w["kind"] == "clustered":
        return ics.clustered(w["nside"], w["seed"])
    return ics.uniform(w["n"], w["seed"])


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 4 + k and r[4 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_reference(x, theta, nthreads, leaf_max=64):
    """One force evaluation with the reference's kernels on the host cores.
    Returns (seconds_total, seconds_tree_walk, stats)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if O.ref_lib() is None:
        kind = "port"
    else:
        kind = "reference"
    o = O.Oracle(theta=theta, ewald=True, leaf_max=leaf_max).set_particles(x)
    t0 = time.perf_counter()
    o.build().multipoles().walk()
    t1 = time.perf_counter()
    o.evaluate(use_ref=(kind == "reference"), nthreads=nthreads)
    t2 = time.perf_counter()
    return t2 - t0, t1 - t0, kind, o


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clustered128", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 Ewald error measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    w = WORKLOADS[args.workload]
    cfg = {"workload": "%s: %s, theta %.2g, Ewald, leaf 64, KDK dt %g" % (
        args.workload, "128^3 clustered P(k)~k^-2" if args.workload == "clustered128" else args.workload,
        args.theta, args.dt), "particles_per_gpu": None, "theta": args.theta, "leaf_max": 64,
        "precision": args.precision, "l2": "256 MB flush between timed steps (untimed)",
        "parallelism": "replicas x%d" % world}

    if args.impl == "reference":
        if rank != 0:
            return 0
        x = make_particles(w)
        n = len(x)
        nth = os.cpu_count() or 1
        times = []
        for it in range(args.warmup + args.steps):
            t, ttree, kind, o = cpu_reference(x, args.theta, nth)
            if it >= args.warmup:
                times.append(t)
            del o
        sec = float(np.mean(times))
        v = n / sec / 1e6
        cfg["particles_per_gpu"] = n
        line = {"impl": "reference", "metric": "Mparticles/s per force eval (128^3 clustered, theta 0.7, Ewald)",
                "value": v, "unit": "Mparticles/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32 (FP64 sums)", "data": "synthetic (seeded)", "config": cfg,
                "cpu_baseline": {"value": v, "unit": "Mparticles/s", "cores": nth, "kind": kind,
                                 "sample": "full force evaluation (tree + walk single-threaded, kernels on %d threads)"
                                           % nth},
                "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200.solver import device_fp32_peak

    dist = world > 1
    if dist:
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    dev = local_rank if dist else 0
    torch.cuda.set_device(dev)
    x = make_particles(w)
    n = len(x)
    cfg["particles_per_gpu"] = n
    stream = torch.cuda.current_stream()

    s = tg.GravitySolver(n, theta=args.theta, ewald=True, leaf_max=64, precision=args.precision, device=dev)
    s.set_particles(x)
    s.solve_gravity(stream=stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    dt = args.dt

    def kdk():
        s.kick(0.5 * dt, stream=stream)
        s.drift(dt, stream=stream)
        s.solve_gravity(stream=stream)
        s.kick(0.5 * dt, stream=stream)

    for _ in range(args.warmup):
        kdk()
    torch.cuda.synchronize()
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    pp_ms, launches0 = [], s.stats()["launches"]
    with ClockSampler(dev) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            kdk()
            ev[k][1].record(stream)
            torch.cuda.synchronize()
            st = s.stats()
            pp_ms.append(st["ms"]["pp"])
    torch.cuda.synchronize()
    launches = s.stats()["launches"] - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(np.sum(step_ms))
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        total_ms = float(t.item())
        tdist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * n / (ms_per_step * 1e-3) / 1e6
    st = s.stats()

    # ---- end to end through the public API with host buffers ----
    # page-locked host buffers, as a production caller would hold them
    xh = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    vh = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    phi_h = torch.zeros(n, dtype=torch.float32).pin_memory()
    g_h = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    e2e_ms = []
    s2 = tg.GravitySolver(n, theta=args.theta, ewald=True, leaf_max=64, precision=args.precision, device=dev)
    for k in range(args.warmup + args.steps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s2.set_particles(xh, vh, stream=stream)
        s2.solve_gravity(stream=stream)
        s2.get_forces(out_phi=phi_h, out_g=g_h, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e_ms.append(a.elapsed_time(b))
    s2.close()
    e2e_step = float(np.mean(e2e_ms))
    e2e_val = world * n / (e2e_step * 1e-3) / 1e6
    if dist:
        t = torch.tensor([e2e_val], device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MIN)
        e2e_val = float(t.item())

    # ---- roofline of the dominant kernel (PP direct, k_pp_f32) ----
    peak = device_fp32_peak(dev)
    cnt = st["counts"]
    pp_s = float(np.mean(pp_ms)) * 1e-3
    exec_flops = cnt["PP_D"] * EXEC_FLOPS["PP_D"]
    achieved = exec_flops / pp_s / 1e12 if pp_s > 0 else None
    roof = {"kernel": "k_pp_f32 (PP direct, FP32)", "bound": "fp32", "achieved": achieved,
            "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if achieved else None,
            "traffic": TRAFFIC_PP_BYTES_PER_PAIR * cnt["PP_D"],
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of k_pp_f32 on clustered64, "
                              "scaled by PP pairs",
            "peak_source": "measured FP32 FMA kernel on this GPU (tg_device_fp32_peak)",
            "flops_per_launch": exec_flops, "flop_convention": "FP32 lane operations per PP pair (%d)" % EXEC_FLOPS["PP_D"],
            "ms_per_launch": pp_s * 1e3, "phase_ms": st["ms"], "interactions": cnt,
            "ref_convention_gflop_per_eval": st["flops"] / 1e9}

    line = {"metric": "Mparticles/s per force eval (128^3 clustered, theta 0.7, Ewald)", "value": value,
            "unit": "Mparticles/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "f32" else "f64", "data": "synthetic (seeded)", "config": cfg,
            "e2e": {"value": e2e_val, "unit": "Mparticles/s", "h2d_bytes_per_step": int(n * 24),
                    "d2h_bytes_per_step": int(n * 16), "ms_per_step": e2e_step},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary(),
            "interactions_per_s": float(sum(cnt.values())) / (ms_per_step * 1e-3)}

    if rank == 0 and not args.no_error:
        # FP64 direct Ewald sum at 4096 seeded samples (outside the timed region)
        from tigergrav_b200 import ics
        smp = ics.samples(n, 4096, 3)
        s.set_particles(x)
        s.solve_gravity(stream=stream)
        phi, g = s.get_forces()
        tphi, tgr = s.truth(smp)
        e = np.linalg.norm(g[smp] - tgr, axis=1) / np.linalg.norm(tgr, axis=1)
        line["force_error_vs_fp64_ewald"] = {"rms": float(np.sqrt(np.mean(e ** 2))), "max": float(e.max()),
                                             "median": float(np.median(e)), "samples": int(len(smp))}
    if rank == 0 and world == 1 and not args.no_cpu:
        nth = os.cpu_count() or 1
        tcpu, ttree, kind, o = cpu_reference(x, args.theta, nth)
        del o
        line["cpu_baseline"] = {"value": n / tcpu / 1e6, "unit": "Mparticles/s", "cores": nth, "kind": kind,
                                "sample": "one full force evaluation of this workload: oracle tree+walk "
                                          "(1 thread, %.2f s) + reference kernels (%d threads)" % (ttree, nth)}
    s.close()
    if dist:
        import torch.distributed as tdist
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
