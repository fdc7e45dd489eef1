"""Benchmark: periodic tree gravity on B200 (one JSON line on stdout).

Metric: Mparticles/s per force evaluation at RMS relative force error <= 1e-4
against the FP64 direct Ewald sum; adjoint / forward cost.

Headline workload (default, ``clustered256``): 256^3 = 16,777,216 particles on a
lattice displaced by a seeded Gaussian random field with P(k) ~ k^-2 (rms
displacement 0.5 spacing, seed 8), periodic unit box, Ewald on, the FP32
compensated path, leaf size 48.  RMS <= 1e-4 needs theta = 0.19 on this
workload (theta 0.2 gives 1.24e-4 at leaf 64, 1.26e-4 at 48); among the leaf
sizes 24..64 at theta 0.19, 48 is the fastest that meets it (32: 1.07e-4),
so the headline runs there and every run re-measures the error at 4096
seeded samples.

A step is one kick-drift-kick leapfrog step at dt = 1e-3: the previous step's
closing half kick, this step's opening half kick and the drift in one fused
pass, then a full force evaluation (tree build, multipoles, walk, every
interaction kernel).  value = particles / step time.  Inputs stay resident in
HBM; L2 is flushed (256 MB write, untimed) between timed steps.

The same JSON line carries:
  e2e              the evaluation through the public API from page-locked host
                   buffers (positions + velocities in, phi + g out, copies
                   inside the timed region);
  fp64_path        the plain FP64 path (TG_PREC_F64) on the same particles and
                   GPU, one force evaluation timed after a warm-up one, with its
                   error; fp32_over_fp64 = its time / the FP32 evaluation time;
  adjoint          the differentiation workload: 64^3 clustered (seed 5),
                   L = sum w.x(T) (w ~ N(0,1), seed 6) after 8 steps at
                   dt = 1e-3: tg_forward and tg_backward times, their ratio, and
                   central finite differences (h = 1e-4, FP64 path) on 32
                   coordinates (seed 7);
  secondary        the 128^3 clustered box (seed 2) at theta 0.2 and at the
                   literal theta 0.7;
  roofline         the dominant interaction kernel against the measured FP32
                   FMA peak of the GPU;
  cpu_baseline     the reference's own kernels (src/gravity.cpp compiled from
                   the reference sources into oracle/_ref) on all host cores.

CPU baseline and --impl reference: a force evaluation of the reference's CPU
path at 256^3 and theta 0.19 takes hours, so its time is assembled from
measured parts: the tree build and multipoles (the oracle's serial
restatement of src/tree.cpp, timed), the walk (restated kick_fmm on all host
threads, timed in full), and per interaction kind the evaluation's count
times that kind's host throughput, sampled by running the reference kernel
over random sinks of this workload with their real lists.  The reference arm
also times full evaluations with the reference kernels on all host cores
where one fits in seconds: the 32^3 uniform box and the 128^3 clustered box,
both at theta 0.7 (``measured_full``), and the 32^3 box once more with the
reference's own tree, walk and kernels (src/tree.cpp, part_vect.cpp,
gravity.cpp compiled into oracle/_ref) run serially on one core, its
interaction counts checked against the restated walk's.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
  torchrun --nproc-per-node N bench.py --gpus N ...   (independent replicas)
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
    "clustered256": dict(kind="clustered", nside=256, seed=8, theta_rms=0.19, leaf=48,
                         label="256^3 clustered P(k)~k^-2, rms displacement 0.5 spacing, seed 8"),
    "clustered128": dict(kind="clustered", nside=128, seed=2, theta_rms=0.2,
                         label="128^3 clustered P(k)~k^-2, rms displacement 0.5 spacing, seed 2"),
    "clustered64": dict(kind="clustered", nside=64, seed=5, theta_rms=0.2, label="64^3 clustered, seed 5"),
    # a profiling case: the headline's theta and leaf size (so its near / far
    # mix of PP source leaves) on a box whose ncu capture stays a few GB
    "clustered72": dict(kind="clustered", nside=72, seed=2, theta_rms=0.19, leaf=48,
                        label="72^3 clustered, seed 2 (profiling case)"),
    "uniform32": dict(kind="uniform", n=32768, seed=1, theta_rms=0.3, label="32^3 uniform, seed 1"),
    "batch64": dict(kind="batch", nboxes=64, seed=4, theta_rms=0.7,
                    label="64 boxes, N = 2^U[12,18], half uniform, half clustered"),
}
METRIC = "Mparticles/s per force eval at RMS err<=1e-4 vs FP64 Ewald; adjoint/fwd cost"
KINDS = ("PP_D", "PP_E", "PC_D", "PC_E", "CC_D", "CC_E", "CP_D", "CP_E")

# FP32 operations per PP pair in k_pp_leaf's inner loop for far source
# leaves (nearly all pairs at the headline workload), counted from the source
# with an FMA as 2: separation 3, r^2 5 (1 mul + 2 fma), rsqrt 1, 1/r^3 2,
# phi sum 1, three force FMAs 6 -> 18 (near leaves: 6 more for the split
# separation and 2 for the softening clamp; the Kahan fold, ~1.3 per pair,
# is not counted).
PP_FLOPS = 18
# FP32 operations per interaction of the Ewald and multipole kernels, counted
# from the source the same way.  One real-space image: separation and r^2 8,
# rsqrt and powers of 1/r 8, erfc/exp 18, d0..d4 31, the moment sums 120 ->
# 185; 38.8 images on average inside the FP32 cut r < 2.1 (4/3 pi 2.1^3);
# finish 105 -> 7.3k per green_ewald without its reciprocal terms.  The 61
# reciprocal terms of PC_E / PP_E are not evaluated per interaction: each
# chunk sums its sources' m_k (cos, sin) per vector h in the leaf kernels
# (tg_ewald_sep.cuh): per PC_E source node 56 ops x 61 shared by the sink
# leaf's particles (~32: +110 per interaction); per PP_E source leaf 4 x 61
# shared by its pairs (negligible).  The per-particle evaluation of the sums
# (61 terms) is not counted.  The node kernels keep the per-interaction
# reciprocal sum: one term of the half sum h.X 5, reduction and sin/cos 5,
# 35 FMAs 70 -> 80, x 61 = 4.9k.  Contractions: M2L 858, M2P 414, P2L 70
# (direct kernels: the reference's constants).
# PP_E pair (cut r < 2, origin separate): 32.5 images x 44 + 30 = 1.46k.
NODE_FLOPS = {"CC_D": 1025, "CP_D": 455, "CC_E": 13100, "CP_E": 12300}
LEAF_FLOPS = {"PC_D": 581, "PC_E": 7800, "PP_E": 1460}
# DRAM bytes per interaction of each kernel group, from ncu captures
# (dram__bytes_read.sum + dram__bytes_write.sum over the capture's
# interactions): k_pp_leaf and k_node_ewald on the 72^3 clustered box at
# theta 0.19, leaf 48 (the clustered72 workload); k_ewald_chunk on the 128^3
# clustered box at theta 0.3.  Scaled by this run's counts on the assumption
# that traffic grows with the interactions.
TRAFFIC = {"pp": {"PP_D": 4.6e-3}, "nodes": {"CC_E": 2.65, "CP_E": 2.65}, "leaf": {"PP_E": 1.61, "PC_E": 1.61}}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum per interaction of a small capture, "
                  "scaled by this run's interaction counts")


T_START = time.perf_counter()


def log(msg):
    """progress on stderr (the JSON line is the only stdout)"""
    print("[bench %7.1f s] %s" % (time.perf_counter() - T_START, msg), file=sys.stderr, flush=True)


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


def reduce_over_ranks(v, op, device):
    """max (slowest replica's time) or min of a value over the ranks of the
    default process group (NCCL on the GPUs, gloo in the CPU tests)."""
    import torch
    import torch.distributed as tdist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX if op == "max" else tdist.ReduceOp.MIN)
    return float(t.item())


# ---------------------------------------------------------------- CPU side --

def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_walk(x, theta, nthreads, leaf=64):
    """The reference's tree build, multipoles (serial restatement, timed) and
    walk (restated kick_fmm on nthreads threads, timed).  Returns the oracle
    and the seconds of each part."""
    O = _oracle()
    o = O.Oracle(theta=theta, ewald=True, leaf_max=leaf).set_particles(x)
    t0 = time.perf_counter()
    o.build().multipoles()
    t1 = time.perf_counter()
    o.walk(nthreads=nthreads)
    t2 = time.perf_counter()
    return o, {"build_multipoles_s": t1 - t0, "walk_s": t2 - t1}


def cpu_estimate(o, parts, nthreads, budget_s, seed):
    """Seconds of one evaluation on the host: the timed tree and walk plus,
    per kind, this evaluation's interaction count x the reference kernel's
    sampled host throughput (all nthreads threads)."""
    O = _oracle()
    kind = "reference" if O.ref_lib() is not None else "port"
    _, counts, _ = o.stats()
    costs = o.kind_costs(use_ref=(kind == "reference"), nthreads=nthreads, budget_s=budget_s, seed=seed)
    t_kern = sum(counts[k] * costs[k][0] * 1e-9 for k in KINDS)
    return {"seconds": parts["build_multipoles_s"] + parts["walk_s"] + t_kern, "kernels_s": t_kern, "kind": kind,
            "ns_per_interaction": {k: costs[k][0] for k in KINDS},
            "sampled_interactions": {k: int(costs[k][1]) for k in KINDS}, **parts}


def cpu_line(r, n, nth, budget_s):
    v = n / r["seconds"] / 1e6
    return {"value": v, "unit": "Mparticles/s", "cores": nth, "kind": r["kind"],
            "sample": "tree build + multipoles (serial, %.1f s) and walk (%d threads, %.1f s) timed in full; each of "
                      "the 8 reference kernels run over random sinks of this workload with their lists for <=%g s "
                      "(%d interactions sampled), scaled by this evaluation's interaction counts (%.0f s)" % (
                          r["build_multipoles_s"], nth, r["walk_s"], budget_s,
                          sum(r["sampled_interactions"].values()), r["kernels_s"]),
            "seconds_per_eval": r["seconds"], "ns_per_interaction": r["ns_per_interaction"]}


def cpu_full_eval(x, theta, nthreads):
    """One full evaluation with the reference's kernels on the host: tree,
    multipoles, walk and every interaction (the reference's own kernels on
    nthreads threads), timed end to end."""
    O = _oracle()
    use_ref = O.ref_lib() is not None
    t0 = time.perf_counter()
    o = O.Oracle(theta=theta, ewald=True, leaf_max=64).set_particles(x)
    o.build().multipoles().walk(nthreads=nthreads)
    o.evaluate(use_ref=use_ref, nthreads=nthreads)
    sec = time.perf_counter() - t0
    return {"seconds": sec, "mparticles_per_s": len(x) / sec / 1e6, "theta": theta, "n": int(len(x)),
            "kind": "reference" if use_ref else "port", "cores": nthreads}


def reference_code_eval(x, theta):
    """One full evaluation by the reference's own code -- src/tree.cpp's
    refine, compute_multipoles and kick_fmm, src/part_vect.cpp and its
    kernels -- compiled where it lies into oracle/_ref/libtg_reftree.so and
    run serially on one core through a single-locality HPX stand-in (the
    reference runs it on HPX threads).  None when that library was not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_tree
    if not ref_tree.available():
        return None
    t0 = time.perf_counter()
    r = ref_tree.solve(x, theta, True, 64)
    sec = time.perf_counter() - t0
    O = _oracle()
    o = O.Oracle(theta=theta, ewald=True, leaf_max=64).set_particles(x)
    o.build().multipoles().walk(nthreads=os.cpu_count() or 1)
    same = o.stats()[0] == r["stats"]
    return {"seconds": sec, "mparticles_per_s": len(x) / sec / 1e6, "theta": theta, "n": int(len(x)), "cores": 1,
            "kind": "reference code (serial)", "interaction_stats": r["stats"],
            "stats_equal_restated_walk": bool(same)}


def reference_arm(args, w, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from tigergrav_b200 import ics
    x = make_particles(w)
    n = len(x)
    nth = os.cpu_count() or 1
    o, parts = cpu_walk(x, args.theta, nth, args.leaf)  # the walk is deterministic: timed once, in full
    times, last = [], None
    for it in range(args.warmup + args.steps):
        r = cpu_estimate(o, parts, nth, budget_s=0.5, seed=1 + it)
        if it >= args.warmup:
            times.append(r["seconds"])
        last = r
    del o
    sec = float(np.mean(times))
    v = n / sec / 1e6
    cb = cpu_line(last, n, nth, 0.5)
    cb["value"] = v
    full = {"uniform32_theta0.7": cpu_full_eval(ics.uniform(32768, 1), 0.7, nth),
            "clustered128_theta0.7": cpu_full_eval(ics.clustered(128, 2), 0.7, nth)}
    own = reference_code_eval(ics.uniform(32768, 1), 0.7)
    if own is not None:
        full["uniform32_theta0.7_reference_code"] = own
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mparticles/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 sums)", "data": "synthetic (seeded)",
            "config": cfg, "cpu_baseline": cb, "measured_full": full,
            "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- GPU side --

def timed_steps(s, stream, flush, steps, warmup, dt, clock_dev=None):
    """KDK steps with events around each; returns (per-step ms, launches, clocks, stats per step)."""
    import torch

    first = [True]

    def kdk():
        # the previous step's closing half kick, this step's opening half kick
        # and the drift in one pass (tg_kick_drift), then the force evaluation
        s.kick_drift(0.0 if first[0] else 0.5 * dt, 0.5 * dt, dt, stream=stream)
        first[0] = False
        s.solve_gravity(stream=stream)

    for _ in range(warmup):
        kdk()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    stats = []
    launches0 = s.stats()["launches"]
    clk = ClockSampler(clock_dev) if clock_dev is not None else None
    if clk:
        clk.__enter__()
    try:
        for k in range(steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            kdk()
            ev[k][1].record(stream)
            torch.cuda.synchronize()
            stats.append(s.stats())
    finally:
        if clk:
            clk.__exit__()
    launches = s.stats()["launches"] - launches0
    return [a.elapsed_time(b) for a, b in ev], launches, (clk.summary() if clk else None), stats


def eval_ms(s, x, stream, flush, reps):
    """Device time of force evaluations (solve_gravity alone) at positions x."""
    import torch
    out = []
    s.set_particles(x)
    for k in range(reps):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.solve_gravity(stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b))
    return out


def truth_at(s, x, smp):
    s.set_particles(x)
    return s.truth(smp)


def error_vs(g, smp, tgr):
    e = np.linalg.norm(g[smp] - tgr, axis=1) / np.linalg.norm(tgr, axis=1)
    nw = np.sqrt(np.mean(np.sum((g[smp] - tgr) ** 2, 1)) / np.mean(np.sum(tgr ** 2, 1)))
    return {"rms": float(np.sqrt(np.mean(e ** 2))), "max": float(e.max()), "median": float(np.median(e)),
            "normwise": float(nw), "samples": int(len(smp)),
            "definition": "per-particle |g - g_true| / |g_true| at 4096 seeded samples, FP64 direct Ewald truth"}


def forces_at(s, x, stream):
    s.set_particles(x)
    s.solve_gravity(stream=stream)
    return s.get_forces()


def e2e_run(s, x, stream, flush, steps):
    """The evaluation through the public API from page-locked host buffers."""
    import torch
    n = len(x)
    xh = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    vh = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    phi_h = torch.zeros(n, dtype=torch.float32).pin_memory()
    g_h = torch.zeros((n, 3), dtype=torch.float32).pin_memory()
    ms = []
    for k in range(steps + 1):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        s.set_particles(xh, vh, stream=stream)
        s.solve_gravity(stream=stream)
        s.get_forces(out_phi=phi_h, out_g=g_h, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        if k >= 1:  # the first call is a warm-up
            ms.append(a.elapsed_time(b))
    return ms


def adjoint_run(dev, theta=0.7, fd_samples=32):
    """The differentiation workload (64^3 clustered, seed 5; 8 steps at
    dt = 1e-3; L = sum w.x(T), w ~ N(0,1) seed 6): tg_forward / tg_backward
    times on the FP32 path (host clock around the synchronous calls), and
    central finite differences of the FP64 path (h = 1e-4) against the FP64
    backward on 32 coordinates (seed 7).  A coordinate whose +h and -h runs
    have different interaction lists is skipped (a tree force is piecewise
    smooth) and counted."""
    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x0 = ics.clustered(64, 5)
    n = len(x0)
    w = np.random.default_rng(6).standard_normal((n, 3))
    dt, steps, h = 1e-3, 8, 1e-4
    res = {"workload": "64^3 clustered (seed 5), 8 KDK steps at dt 1e-3, theta %g, L = sum w.x(T)" % theta}
    with tg.GravitySolver(n, theta=theta, precision="f32", device=dev) as s:
        s.set_particles(x0).forward(dt, steps)
        s.backward(w)
        fw, bw = [], []
        for _ in range(3):
            s.set_particles(x0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.forward(dt, steps)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            s.backward(w)
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            fw.append(t1 - t0)
            bw.append(t2 - t1)
    res.update({"forward_ms": 1e3 * float(np.median(fw)), "backward_ms": 1e3 * float(np.median(bw)),
                "precision": "f32", "timing": "host clock around the synchronous calls, median of 3"})
    res["ratio"] = res["backward_ms"] / res["forward_ms"]

    p2d = ics.pos_to_double
    xd0 = p2d(x0)
    with tg.GravitySolver(n, theta=theta, precision="f64", device=dev) as s64:
        s64.set_particles(x0).forward(dt, steps)
        gx0, _ = s64.backward(w)

        def loss(xpos):
            s64.set_particles(xpos).solve_gravity()
            sig = []
            for _ in range(steps):
                s64.kick(0.5 * dt)
                s64.drift(dt)
                s64.solve_gravity()
                s64.kick(0.5 * dt)
                sig.append(tuple(s64.stats()["counts"].values()))
            xt, _ = s64.get_particles()
            disp = (p2d(xt) - xd0 + 0.5) % 1.0 - 0.5
            return float(np.sum(w * (xd0 + disp))), tuple(sig)

        rng = np.random.default_rng(7)
        idx = rng.choice(n, fd_samples, replace=False)
        dims = rng.integers(0, 3, fd_samples)
        errs, nonid, skipped = [], [], 0
        for i, d in zip(idx, dims):
            xp, xm = x0.copy(), x0.copy()
            xp[i, d] = ics.double_to_pos(np.array([xd0[i, d] + h]))[0]
            xm[i, d] = ics.double_to_pos(np.array([xd0[i, d] - h]))[0]
            hh = ((p2d(xp[i, d]) - p2d(xm[i, d]) + 0.5) % 1.0) - 0.5
            (lp, sp), (lm, sm) = loss(xp), loss(xm)
            if sp != sm:
                skipped += 1
                continue
            fd = (lp - lm) / hh
            errs.append(abs(gx0[i, d] - fd) / abs(fd))
            nonid.append(abs((gx0[i, d] - w[i, d]) - (fd - w[i, d])) / max(abs(fd - w[i, d]), 1e-300))
    errs = np.array(errs)
    res["fd"] = {"h": h, "samples": fd_samples, "skipped": skipped, "path": "f64",
                 "median_rel_err": float(np.median(errs)), "p90_rel_err": float(np.percentile(errs, 90)),
                 "max_rel_err": float(errs.max()), "non_identity_median_rel_err": float(np.median(nonid))}
    return res


def secondary_run(args, dev, stream, flush):
    """The 128^3 clustered box (seed 2) at theta 0.2 and at the literal 0.7."""
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    x = ics.clustered(128, 2)
    n = len(x)
    smp = ics.samples(n, 4096, 3)
    out = {}
    tphi = tgr = None
    for theta in (0.2, 0.7):
        with tg.GravitySolver(n, theta=theta, precision=args.precision, device=dev) as s:
            if tgr is None:
                tphi, tgr = truth_at(s, x, smp)
            _, g = forces_at(s, x, stream)
            s.solve_gravity(stream=stream)
            ms, _, _, st = timed_steps(s, stream, flush, 5, 3, args.dt)
            out["clustered128_theta%g" % theta] = {
                "theta": theta, "value": n / (float(np.mean(ms)) * 1e-3) / 1e6, "unit": "Mparticles/s",
                "ms_per_step": float(np.mean(ms)),
                "phase_ms": {k: float(np.mean([q["ms"][k] for q in st])) for k in st[-1]["ms"]},
                "force_error_vs_fp64_ewald": error_vs(g, smp, tgr)}
    return out


def roofline(phase_ms, cnt, peak):
    """FP32 roofline of the kernel with the largest share of the evaluation.
    achieved = executed FP32 operations (per-interaction counts from the
    kernel source, FMA = 2) / that kernel's CUDA-event phase time."""
    leaf_far = max(phase_ms["leaves"] - phase_ms.get("pp", 0.0), 1e-9)
    kern = {"k_pp_leaf (PP direct)": (phase_ms.get("pp", 0.0), {"PP_D": PP_FLOPS}, "pp"),
            "k_node + k_node_ewald<float> (CC/CP direct + Ewald)": (phase_ms["nodes"], NODE_FLOPS, "nodes"),
            "k_ewald_chunk<float> + k_ewald_reduce + k_leaf (PC/PP Ewald, L2P, PC direct)":
                (leaf_far, LEAF_FLOPS, "leaf")}
    name = max(kern, key=lambda k: kern[k][0])
    ms, fl, tk = kern[name]
    flops = sum(cnt[k] * v for k, v in fl.items())
    achieved = flops / (ms * 1e-3) / 1e12
    traffic = sum(cnt[k] * v for k, v in TRAFFIC[tk].items())
    return {"kernel": name, "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "traffic_source": TRAFFIC_SOURCE,
            "peak_source": "measured FP32 FMA kernel on this GPU (tg_device_fp32_peak); MEASURED_PEAKS.json has no "
                           "FP32 figure",
            "flops_per_launch": flops, "flops_per_interaction": fl, "ms_per_launch": ms}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clustered256", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="f32", choices=["f32", "f64"])
    ap.add_argument("--theta", type=float, default=None,
                    help="opening angle (default: the workload's theta for RMS error <= 1e-4)")
    ap.add_argument("--leaf", type=int, default=None,
                    help="leaf size (parts_per_node; default: the workload's, 48 at 256^3, else 64)")
    ap.add_argument("--dt", type=float, default=1e-3)
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--no-error", action="store_true", help="skip the FP64 Ewald error measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-path comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the differentiation workload")
    ap.add_argument("--no-secondary", action="store_true", help="skip the 128^3 runs")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.theta is None:
        args.theta = w["theta_rms"]
    if args.leaf is None:
        args.leaf = w.get("leaf", 64)
    if args.impl == "ours":
        args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cfg = {"workload": "%s (%s), theta %.3g (%s), Ewald, leaf %d, KDK dt %g" % (
        args.workload, w["label"], args.theta,
        ("the batching config's theta" if w["kind"] == "batch" else "RMS force error <= 1e-4 on this workload")
        if args.theta == w["theta_rms"] else "set by --theta", args.leaf, args.dt),
        "particles_per_gpu": (w["nside"] ** 3 if w["kind"] == "clustered" else w.get("n")),
        "theta": args.theta, "leaf_max": args.leaf, "precision": args.precision,
        "l2": "256 MB flush between timed steps (untimed)", "parallelism": "replicas x%d" % world}
    if args.impl == "reference":
        if w["kind"] == "batch":
            print(json.dumps({"impl": "reference", "unavailable": "the batch workload is measured for this "
                              "implementation only; the reference arm runs the single-box workloads"}))
            return 0
        return reference_arm(args, w, cfg)
    if w["kind"] == "batch":
        return bench_batch(args, w, cfg)

    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    from tigergrav_b200.solver import device_fp32_peak

    dist = world > 1
    if dist:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = local_rank if dist else 0
    torch.cuda.set_device(dev)
    x = make_particles(w)
    n = len(x)
    log("particles ready: %d" % n)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    s = tg.GravitySolver(n, theta=args.theta, ewald=True, leaf_max=args.leaf, precision=args.precision, device=dev)
    s.set_particles(x)
    s.solve_gravity(stream=stream)
    if dist:
        tdist.barrier()
    torch.cuda.synchronize()
    step_ms, launches, clocks, stats = timed_steps(s, stream, flush, args.steps, args.warmup, args.dt, dev)
    total_ms = float(np.sum(step_ms))
    if dist:
        total_ms = reduce_over_ranks(total_ms, "max", "cuda")
        tdist.barrier()
    ms_per_step = total_ms / args.steps
    value = world * n / (ms_per_step * 1e-3) / 1e6
    log("timed steps done: %.1f ms per step" % ms_per_step)
    st = stats[-1]
    phase_ms = {k: float(np.mean([q["ms"][k] for q in stats])) for k in st["ms"]}

    # ---- one force evaluation alone (the unit of the FP32 / FP64 comparison) ----
    ev32 = eval_ms(s, x, stream, flush, 2)

    # ---- end to end through the public API with page-locked host buffers ----
    e2e_ms = e2e_run(s, x, stream, flush, args.e2e_steps)
    e2e_step = float(np.mean(e2e_ms))
    log("eval %.1f ms, e2e %.1f ms" % (np.mean(ev32), e2e_step))
    e2e_val = world * n / (e2e_step * 1e-3) / 1e6
    if dist:
        e2e_val = reduce_over_ranks(e2e_val, "min", "cuda")

    # ---- roofline of the dominant kernel ----
    peak = device_fp32_peak(dev)
    cnt = st["counts"]
    roof = roofline(phase_ms, cnt, peak)
    roof["phase_ms"] = phase_ms
    roof["interactions"] = cnt
    roof["ref_convention_gflop_per_eval"] = st["flops"] / 1e9

    line = {"metric": METRIC, "value": value, "unit": "Mparticles/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "f32" else "f64",
            "data": "synthetic (seeded)", "config": cfg,
            "e2e": {"value": e2e_val, "unit": "Mparticles/s", "h2d_bytes_per_step": int(n * 24),
                    "d2h_bytes_per_step": int(n * 16), "ms_per_step": e2e_step, "steps": len(e2e_ms),
                    "step": "set_particles (host) + solve_gravity + get_forces (host)"},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clocks,
            "interactions_per_s": float(sum(cnt.values())) / (ms_per_step * 1e-3),
            "eval_ms": float(np.mean(ev32))}

    smp = ics.samples(n, 4096, 3)
    tgr = None
    if rank == 0 and not args.no_error:
        _, tgr = truth_at(s, x, smp)
        _, g = forces_at(s, x, stream)
        line["force_error_vs_fp64_ewald"] = error_vs(g, smp, tgr)
        line["accuracy_met"] = line["force_error_vs_fp64_ewald"]["rms"] <= 1e-4
        del g
        log("force error: %s" % line["force_error_vs_fp64_ewald"]["rms"])
    s.close()

    if not args.no_fp64 and args.precision == "f32":
        # the plain FP64 port-equivalent path on the same particles and GPU
        with tg.GravitySolver(n, theta=args.theta, ewald=True, leaf_max=args.leaf, precision="f64",
                              device=dev) as s64:
            s64.set_particles(x).solve_gravity(stream=stream)  # warm-up (allocations)
            ev64 = eval_ms(s64, x, stream, flush, 1)
            fp = {"eval_ms": float(np.mean(ev64)), "value": n / (float(np.mean(ev64)) * 1e-3) / 1e6,
                  "unit": "Mparticles/s per force evaluation", "theta": args.theta}
            if tgr is not None:
                _, g64 = s64.get_forces()
                fp["force_error_vs_fp64_ewald"] = error_vs(g64, smp, tgr)
                del g64
        line["fp64_path"] = fp
        line["fp32_over_fp64"] = fp["eval_ms"] / line["eval_ms"]
        log("fp64 path: %.1f ms" % fp["eval_ms"])

    if not args.no_adjoint and rank == 0:
        line["adjoint"] = adjoint_run(dev)
        log("adjoint: %s" % line["adjoint"])

    if not args.no_secondary and args.workload != "clustered128" and rank == 0:
        line["secondary"] = secondary_run(args, dev, stream, flush)
        log("secondary done")

    if rank == 0 and world == 1 and not args.no_cpu:
        nth = os.cpu_count() or 1
        o, parts = cpu_walk(x, args.theta, nth, args.leaf)
        r = cpu_estimate(o, parts, nth, budget_s=1.5, seed=1)
        del o
        line["cpu_baseline"] = cpu_line(r, n, nth, 1.5)
        log("cpu baseline: %s" % line["cpu_baseline"]["sample"])
    if dist:
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def bench_batch(args, w, cfg):
    """The batching workload: all boxes per step through tg_batch_solve (boxes
    on 16 streams, leaf size autotuned per box over 16..128).  The batch runs on
    its own streams from host threads, so a step is timed by the host clock
    around the call (which returns after every stream has finished)."""
    import torch
    import tigergrav_b200 as tg
    from tigergrav_b200 import ics
    counts, x = ics.batch(w["nboxes"], w["seed"])
    n = int(counts.sum())
    b = tg.GravityBatch(counts, theta=args.theta, precision=args.precision, nstreams=16)
    b.set_particles(x)
    t0 = time.perf_counter()
    chosen = b.autotune((16, 32, 64, 128))
    t_tune = time.perf_counter() - t0
    for _ in range(args.warmup):
        b.solve()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ms = []
    with ClockSampler(0) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))
            torch.cuda.synchronize()
            t = time.perf_counter()
            b.solve()
            ms.append((time.perf_counter() - t) * 1e3)
    # the same boxes one after another on one stream, for comparison
    ser = []
    for k in range(len(counts)):
        off = int(counts[:k].sum())
        s = tg.GravitySolver(int(counts[k]), theta=args.theta, leaf_max=int(chosen[k]), precision=args.precision)
        s.set_particles(x[off:off + int(counts[k])])
        s.solve_gravity()
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.solve_gravity()
        torch.cuda.synchronize()
        ser.append((time.perf_counter() - t) * 1e3)
        s.close()
    b.close()
    mps = float(np.mean(ms))
    cfg.update({"particles_total": n, "boxes": int(len(counts)), "leaf_sizes_chosen": chosen.tolist(),
                "autotune_s": t_tune, "streams": 16, "timing": "host clock around each batched call"})
    line = {"metric": "Mparticles/s per batched force eval (64 boxes)", "value": n / (mps * 1e-3) / 1e6,
            "unit": "Mparticles/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": mps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.precision,
            "data": "synthetic (seeded)", "config": cfg, "clocks": clk.summary(),
            "serial_ms": float(np.sum(ser)), "speedup_vs_serial": float(np.sum(ser)) / mps}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
