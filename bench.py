"""Benchmark: Brownian dynamics with hydrodynamic interactions, N=1024.

Workload (the reference's headline configuration): 1024 beads, radii uniform
in [10, 40] A, non-overlapping random positions (rejection sampling, seed 0)
in a periodic cubic box of 1500 A; RPY tensor under Smith's Ewald summation
(alpha = sqrt(pi), ewald_real = 2, ewald_imag = 4); Cholesky noise;
Ermak-McCammon update, dt = 0.5 ps, T = 293.15 K, eta = 0.01005 P; overlap
check on.  A step is one Box.propagate: Ewald build of D (3072 x 3072),
Cholesky factor B, D F and B xi products, overlap test, update and wrap.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm times the mixed-precision path (FP32 Ewald tensor and Cholesky
trailing updates, FP64 diagonal tiles and positions) and, for the metric's
"vs FP64" part, the plain FP64 GPU path on the same inputs.  The reference
arm times the reference's own CPU implementation (its C library compiled
from source into oracle/_ref with OpenMP, NumPy LAPACK for the Cholesky)
on the host cores.  With --gpus N > 1 every rank advances an independent
replica (weak scaling, no collective on the data path).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BD steps/s, N=1024 RPY-Ewald: mixed vs FP64 (rel err ≤1e-5); serve p50/p99 ms"
WORKLOAD = {"workload": "BD-HI N=1024 polydisperse a~U[10,40] L=1500 Smith-Ewald m=2 n=4 Ermak dt=0.5",
            "n_beads": 1024, "box_length": 1500.0, "ewald_real": 2, "ewald_imag": 4, "dt": 0.5,
            "seed": 0}


def bench_config(world):
    """The `config` of the JSON line, identical in both arms (the reference
    arm times the same workload on the host cores)."""
    return dict(WORKLOAD, parallelism=f"replicas x{world}" if world > 1 else "single system",
                l2="GPU arm: L2 flushed between timed steps (256 MiB write)")


def bead_config(seed, N, L, a_lo, a_hi, gap=0.0):
    """Sequential rejection sampling: radius, then a uniform position in
    [-L/2, L/2)^3, rejected if the minimum-image distance to any placed bead
    is <= a_i + a_j + gap."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((N, 3))
    radii = np.zeros(N)
    k = 0
    while k < N:
        a = rng.uniform(a_lo, a_hi)
        p = rng.uniform(-L / 2, L / 2, size=3)
        if k:
            d = pos[:k] - p
            d -= L * np.round(d / L)
            if np.any(np.sqrt((d * d).sum(1)) <= radii[:k] + a + gap):
                continue
        pos[k], radii[k] = p, a
        k += 1
    return pos, radii


def lub_workload():
    """Stokesian dynamics with Jeffrey-Onishi lubrication: 512 beads of radius
    20 A at volume fraction 0.30 (box edge from the volume fraction), minimum
    gap 0.05 a at placement, lubrication for surface gaps < 1 a
    (lubrication_cutoff 0.5 in units of a_i + a_j), Cichocki correction,
    midpoint scheme (m = 100), dt = 0.1 ps, seed 0."""
    N, a, phi = 512, 20.0, 0.30
    L = (N * 4.0 * math.pi * a ** 3 / 3.0 / phi) ** (1.0 / 3.0)
    return {"workload": "SD N=512 a=20 phi=0.30 rpy_smith_lub JO cutoff 0.5 Cichocki midpoint m=100 dt=0.1",
            "n_beads": N, "radius": a, "volume_fraction": phi, "box_length": L, "min_gap": 0.05 * a,
            "lubrication_cutoff": 0.5, "m_midpoint": 100.0, "dt": 0.1, "seed": 0}


def lub_input(precision):
    w = lub_workload()
    inp = box_input(precision)
    inp.update({"box_length": w["box_length"], "hydrodynamics": "rpy_smith_lub",
                "lubrication_cutoff": w["lubrication_cutoff"], "cichocki_correction": True,
                "propagation_scheme": "midpoint", "m_midpoint": w["m_midpoint"]})
    return inp


def box_input(precision):
    return {"box_length": WORKLOAD["box_length"], "T": 293.15, "viscosity": 0.01005, "seed": 0,
            "hydrodynamics": "rpy_smith", "ewald_alpha": math.sqrt(math.pi),
            "ewald_real": WORKLOAD["ewald_real"], "ewald_imag": WORKLOAD["ewald_imag"],
            "propagation_scheme": "ermak", "immobile_labels": [], "check_overlaps": True,
            "overlap_treshold": 0.0, "max_move_attempts": 1000000, "external_force": [0.0, 0.0, 0.0],
            "energy_unit": "joule", "verbose": False, "debug": False, "precision": precision,
            "lennard_jones_6": False, "lennard_jones_12": False, "custom_interactions": False}


# ----------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        mx = float(parts[2])
                    except ValueError:
                        continue
                    for nm, v in zip(names, parts[5:9]):
                        if v.lower() == "active":
                            reasons.add(nm)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.remove(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- our arm

class DeviceRun:
    """Device-resident stepping through the C ABI: state, D, B and the noise
    pool live in HBM; one pbg_run call per step (from the second step one
    CUDA graph launch, the move attempts under a device-side WHILE node)."""

    def __init__(self, pos, radii, precision, n_noise_steps, seed, torch, inp=None):
        from pybrown_b200 import _lib
        from pybrown_b200.bead import Bead
        from pybrown_b200.box import Box
        self._lib, self.torch = _lib, torch
        self.box = Box([Bead(p, a) for p, a in zip(pos, radii)], inp or box_input(precision))
        self.n = 3 * len(radii)
        rs = np.random.RandomState(seed)
        self.pool = torch.tensor(rs.normal(0.0, 1.0, size=(n_noise_steps + 64) * self.n), dtype=torch.float64,
                                 device="cuda")
        self.cursor = 0  # draws consumed
        self.j = 0
        self.report = _lib.PbgStepReport()

    def step(self, dt):
        _lib, h = self._lib, self.box._h
        base = self.pool.data_ptr() + 8 * self.cursor
        _lib.call("pbg_run", h, self.j, 1, float(dt), 1, 1, 1, base, self.pool.numel() - self.cursor, None)
        _lib.lib.pbg_run_report(h, _lib.ctypes.byref(self.report), None)
        self.cursor += self.report.draws_consumed
        self.j += 1

    def positions(self):
        out = np.empty(self.n)
        self._lib.call("pbg_get_positions", self.box._h, out.ctypes.data, None)
        self.torch.cuda.synchronize()
        return out.reshape(-1, 3)


def l2_flush(torch, buf):
    buf.add_(1.0)  # 256 MiB read + write: evicts the 126 MB L2


def timed_steps(torch, fn, steps, flush_buf):
    """Per-step CUDA-event timing with an L2 flush between steps (outside
    the timed interval).  Returns total milliseconds of the K steps."""
    total = 0.0
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    for _ in range(steps):
        l2_flush(torch, flush_buf)
        torch.cuda.synchronize()
        start.record()
        fn()
        end.record()
        torch.cuda.synchronize()
        total += start.elapsed_time(end)
    return total


def cholesky_kernel_timing(torch, box, reps):
    """Average device time of the Cholesky factorisation of this step's D
    (the dominant kernel), on the launching stream."""
    from pybrown_b200 import _lib
    n = 3 * len(box.beads)
    ld = (n + 63) // 64 * 64
    dtype = torch.float32 if box.precision == "mixed" else torch.float64
    D = torch.tensor(box.D, dtype=dtype, device="cuda")
    A0 = torch.zeros((ld, ld), dtype=dtype, device="cuda")
    A0[:n, :n] = D
    A = A0.clone()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    prec = 1 if box.precision == "mixed" else 0
    times = []
    for r in range(reps + 1):
        A.copy_(A0)
        torch.cuda.synchronize()
        start.record()
        _lib.call("pbg_dev_cholesky", A.data_ptr(), n, ld, prec, info.data_ptr(), None)
        end.record()
        torch.cuda.synchronize()
        if r:
            times.append(start.elapsed_time(end))
    return sum(times) / len(times), int(info.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_reference_steps(N, steps, warmup, threads=None):
    """The reference's CPU path: its C library (compiled from source with
    OpenMP into oracle/_ref) for the pair vectors, Smith-Ewald tensor and
    overlap test, NumPy LAPACK for the Cholesky, driven step by step like
    Box.propagate.  Returns (steps/s, cores, kind, sample)."""
    from oracle.oracle import REF_LIB, REF_OMP_LIB, ORACLE_LIB, CLib, OracleBox
    cores = threads or len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    lib, kind = None, "reference"
    for path in (REF_OMP_LIB, REF_LIB):
        if os.path.exists(path):
            lib = CLib(path)
            break
    if lib is None:
        lib, kind = CLib(ORACLE_LIB), "port"
    pos, radii = bead_config(WORKLOAD["seed"], N, WORKLOAD["box_length"], 10.0, 40.0)
    inp = box_input("fp64")
    box = OracleBox(pos, radii, inp, clib=lib)
    for _ in range(warmup):
        box.propagate(WORKLOAD["dt"])
    t0 = time.perf_counter()
    for _ in range(steps):
        box.propagate(WORKLOAD["dt"])
    dt = time.perf_counter() - t0
    sample = (f"{steps} Box.propagate steps of the N={N} workload after {warmup} warm-up step(s); "
              f"{os.path.basename(lib.path)} + NumPy cholesky, OMP threads={cores}")
    return steps / dt, cores, kind, sample


def mixed_vs_oracle(pos, radii, seed, steps=5):
    """Accuracy of the mixed path against the FP64 oracle (the checker, run
    outside every timed region): D, B and B xi at the start positions (the
    first step's matrices and noise) and the displacement after `steps`
    steps, both fed the same RandomState noise.  Errors are
    max |a - b| / max |b|."""
    from oracle.oracle import ORACLE_OMP_LIB, ORACLE_LIB, CLib, OracleBox
    from pybrown_b200.bead import Bead
    from pybrown_b200.box import Box
    lib = CLib(ORACLE_OMP_LIB if os.path.exists(ORACLE_OMP_LIB) else ORACLE_LIB)
    inp = box_input("mixed")
    inp["seed"] = seed
    box = Box([Bead(p.copy(), a) for p, a in zip(pos, radii)], inp)
    ref_inp = dict(inp)
    ref_inp.pop("precision")
    ref = OracleBox(pos, radii, ref_inp, clib=lib)
    dt, L = WORKLOAD["dt"], WORKLOAD["box_length"]

    def rel(a, b):
        return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))

    box.propagate(dt)
    ref.propagate(dt)
    xi = np.random.RandomState(seed).normal(0.0, 1.0, 3 * len(radii))
    B = np.tril(box.B)
    out = {"D": rel(box.D, ref.D), "B": rel(B, ref.B), "Bxi": rel(B @ xi, ref.B @ xi)}
    for _ in range(steps - 1):
        box.propagate(dt)
        ref.propagate(dt)
    got = np.array([b.r for b in box.beads])
    dg, dr = got - pos, ref.pos - pos
    dg -= L * np.round((dg - dr) / L)
    out["disp"] = rel(dg, dr)
    out["steps"] = steps
    out["same_draws"] = bool(box.draw_count == ref.draw_count)
    out["oracle"] = os.path.basename(lib.path)
    return out


# DRAM bytes (read + write) of one mixed factorisation of the N=1024 matrix,
# from one ncu capture of the same kernel on the same order
# (profiles/chol_df_mixed_order3072_full.md):
#   ncu --set full --clock-control none -k regex:chol_df -s 1 -c 1 \
#       python -m pybrown_b200.profile_cases cholesky --order 3072 --precision mixed --reps 1
# (19,468,544 + 1,830,912 B); re-measure when the factorisation changes.
CHOL_MIXED_TRAFFIC_BYTES = 19468544 + 1830912


def replica_seed(rank):
    """Each rank advances an independent replica of the workload."""
    return WORKLOAD["seed"] + rank


def max_over_ranks(torch, dist, value, device="cuda"):
    """The slowest rank's time (every rank takes part; identity without a
    process group)."""
    if dist is None:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, torch, dist, rank, world):
    from pybrown_b200 import _lib
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    N = WORKLOAD["n_beads"]
    seed = replica_seed(rank)
    pos, radii = bead_config(seed, N, WORKLOAD["box_length"], 10.0, 40.0)
    dt = WORKLOAD["dt"]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    results = {}
    for prec in ("mixed", "fp64"):
        run = DeviceRun(pos, radii, prec, args.warmup + args.steps + 8, seed, torch)
        for _ in range(args.warmup):
            run.step(dt)
        barrier()
        launches0 = _lib.lib.pbg_launch_count()
        sampler = ClockSampler(local) if prec == "mixed" else None
        if sampler:
            sampler.__enter__()
        ms = timed_steps(torch, lambda: run.step(dt), args.steps, flush)
        if sampler:
            sampler.__exit__(None, None, None)
        launches = _lib.lib.pbg_launch_count() - launches0
        barrier()
        ms = max_over_ranks(torch, dist, ms)
        results[prec] = {"ms": ms, "launches": launches, "run": run,
                         "clocks": sampler.summary() if sampler else None}

    # mixed vs FP64 displacement error after the same warm-up + timed steps
    p_mixed = results["mixed"]["run"].positions()
    p_fp64 = results["fp64"]["run"].positions()
    disp_m = p_mixed - pos
    disp_d = p_fp64 - pos
    L = WORKLOAD["box_length"]
    disp_m -= L * np.round((disp_m - disp_d) / L)
    rel_err = float(np.max(np.abs(disp_m - disp_d)) / np.max(np.abs(disp_d)))

    # e2e through the public API: Box.propagate with host RandomState noise,
    # H2D of positions and noise, D2H of positions, every step.
    from pybrown_b200.bead import Bead
    from pybrown_b200.box import Box
    box = Box([Bead(p, a) for p, a in zip(pos, radii)], box_input("mixed"))
    for _ in range(args.warmup):
        box.propagate(dt)
    barrier()
    e2e_ms = timed_steps(torch, lambda: box.propagate(dt), args.steps, flush)
    e2e_ms = max_over_ranks(torch, dist, e2e_ms)

    # the same with an .xyz frame every step through the drivers' writer thread
    e2e_xyz_ms = None
    if world == 1:
        from pybrown_b200.io import AsyncXYZWriter
        labels = [b.label for b in box.beads]
        with tempfile.TemporaryDirectory() as d, open(os.path.join(d, "t.xyz"), "w", buffering=1) as f, \
                AsyncXYZWriter(f, "t.xyz", labels) as writer:
            j = [0]

            def step_with_frame():
                writer.write(j[0], dt, box.positions())
                box.propagate(dt)
                j[0] += 1

            e2e_xyz_ms = timed_steps(torch, step_with_frame, args.steps, flush)
            writer.flush()

    # dominant kernel: the Cholesky factorisation of D (3072 x 3072)
    chol_ms, info = cholesky_kernel_timing(torch, results["mixed"]["run"].box, 3)
    n = 3 * N
    flops = n ** 3 / 3.0
    peaks, peak_kind = measured_peaks()
    achieved_tflops = flops / (chol_ms * 1e-3) / 1e12

    if rank != 0:
        return None
    ms_step = results["mixed"]["ms"] / args.steps
    value = world * args.steps / (results["mixed"]["ms"] * 1e-3)
    fp64_value = world * args.steps / (results["fp64"]["ms"] * 1e-3)
    cpu = None
    accuracy = None
    if world == 1 and not args.no_oracle_check:
        accuracy = mixed_vs_oracle(pos, radii, seed)
    if world == 1 and not args.no_cpu_baseline:
        sps, cores, kind, sample = cpu_reference_steps(N, steps=2, warmup=1)
        cpu = {"value": sps, "unit": "steps/s", "cores": cores, "kind": kind, "sample": sample}
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64 (mixed: FP32 tensor/trailing updates, FP64 diagonal tiles "
                                       "and positions)", "data": "synthetic (seeded bead configurations)",
        "config": bench_config(world),
        "fp64_value": fp64_value, "mixed_over_fp64": value / fp64_value,
        "mixed_vs_fp64_displacement_rel_err": rel_err,
        "mixed_vs_oracle": accuracy,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "steps/s",
                "h2d_bytes_per_step": 8 * 3 * N * 2 + 8 * N, "d2h_bytes_per_step": 8 * 3 * N},
        "e2e_with_xyz_every_step": (None if e2e_xyz_ms is None else
                                    {"value": args.steps / (e2e_xyz_ms * 1e-3), "unit": "steps/s",
                                     "writer": "drivers' .xyz writer thread, one frame per step"}),
        "gpu_launches": results["mixed"]["launches"],
        "roofline": {"kernel": "cholesky (mixed)", "bound": "tensor", "achieved": achieved_tflops,
                     "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                     "frac": achieved_tflops / peaks["bf16_tflops"], "traffic": CHOL_MIXED_TRAFFIC_BYTES,
                     "note": f"(3N)^3/3 = {flops:.3e} flop per factorisation in {chol_ms:.3f} ms; "
                             f"peak is the {peak_kind} dense bf16 figure; the factorisation is bound "
                             f"by its 48-panel dependency chain, not by a throughput unit; traffic "
                             f"(bytes per launch) from one ncu capture of the same order"},
        "cpu_baseline": cpu,
        "clocks": results["mixed"]["clocks"],
    }
    # A failure in a secondary section is reported in its own key (the
    # exception type and message) instead of costing the whole line.
    sections = (("lubrication", args.no_lub, run_lub_section), ("batch", args.no_batch, run_batch_section),
                ("serve", args.no_serve, run_serve_section),
                ("serve_full_stream", args.no_serve or args.no_serve_full, run_serve_full_section),
                ("serve_full_stream_smallest_work", args.no_serve or args.no_serve_full or args.no_serve_sjf,
                 lambda a, t: run_serve_full_section(a, t, policy="smallest_work")))
    for key, skip, fn in sections:
        if world != 1 or skip:
            continue
        try:
            line[key] = fn(args, torch)
        except Exception as e:  # noqa: BLE001 -- recorded in the line, not hidden
            line[key] = {"error": f"{type(e).__name__}: {e}"}
    return line


def cpu_reference_lub_steps(steps=1):
    """The reference's CPU path on the lubricated workload: its C library
    (OpenMP build in oracle/_ref) for the tensors, NumPy LAPACK for the
    inverses and the Cholesky, driven like Box.propagate (midpoint).  Returns
    (steps/s, cores, kind, sample)."""
    from oracle.oracle import REF_OMP_LIB, REF_LIB, ORACLE_LIB, CLib, OracleBox
    cores = len(os.sched_getaffinity(0))
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    lib, kind = None, "reference"
    for path in (REF_OMP_LIB, REF_LIB):
        if os.path.exists(path):
            lib = CLib(path)
            break
    if lib is None:
        lib, kind = CLib(ORACLE_LIB), "port"
    w = lub_workload()
    pos, radii = bead_config(w["seed"], w["n_beads"], w["box_length"], w["radius"], w["radius"], gap=w["min_gap"])
    inp = lub_input("fp64")
    inp.pop("precision", None)
    box = OracleBox(pos, radii, inp, clib=lib)
    t0 = time.perf_counter()
    for _ in range(steps):
        box.propagate(w["dt"])
    dt = time.perf_counter() - t0
    sample = (f"{steps} midpoint Box.propagate step(s) of the lubricated N=512 workload; "
              f"{os.path.basename(lib.path)} + NumPy inv/cholesky, OMP threads={cores}")
    return steps / dt, cores, kind, sample


def run_lub_section(args, torch, precisions=("fp64", "mixed")):
    """The lubricated workload (lub_workload) stepped on the device: per-step
    CUDA events with an L2 flush between steps, like the main workload."""
    w = lub_workload()
    pos, radii = bead_config(w["seed"], w["n_beads"], w["box_length"], w["radius"], w["radius"], gap=w["min_gap"])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    out = {"workload": w["workload"], "box_length": w["box_length"], "steps": args.steps}
    runs = {}
    for prec in precisions:
        run = DeviceRun(pos, radii, prec, 4 * (args.warmup + args.steps) + 64, w["seed"], torch, inp=lub_input(prec))
        for _ in range(args.warmup):
            run.step(w["dt"])
        torch.cuda.synchronize()
        ms = timed_steps(torch, lambda: run.step(w["dt"]), args.steps, flush)
        runs[prec] = run
        out[prec] = {"ms_per_step": ms / args.steps, "steps_per_s": args.steps / (ms * 1e-3),
                     "move_attempts": run.cursor // run.n}
    if "fp64" in runs and "mixed" in runs:
        d_ref = runs["fp64"].positions() - pos
        d_mix = runs["mixed"].positions() - pos
        d_mix -= w["box_length"] * np.round((d_mix - d_ref) / w["box_length"])
        out["mixed_vs_fp64_displacement_rel_err"] = float(np.max(np.abs(d_mix - d_ref)) / np.max(np.abs(d_ref)))
        out["mixed_over_fp64"] = out["mixed"]["steps_per_s"] / out["fp64"]["steps_per_s"]
    if not args.no_cpu_baseline:
        sps, cores, kind, sample = cpu_reference_lub_steps(steps=1)
        out["cpu_baseline"] = {"value": sps, "unit": "steps/s", "cores": cores, "kind": kind, "sample": sample}
    return out


def run_batch_section(args, torch):
    """256 independent replicas, N uniform in [32, 512] (seed 1), radii uniform
    in [10, 30], volume fraction 0.05 each, Smith-Ewald m=2 n=4, mixed
    precision, device noise streams, dt 0.5 ps: one batched step advances all."""
    from pybrown_b200 import _lib
    from pybrown_b200.batch import ReplicaBatch
    from pybrown_b200.serve import place_beads
    rng = np.random.default_rng(1)
    Ns = rng.integers(32, 513, size=256)
    batch = ReplicaBatch(precision="mixed")
    for k, N in enumerate(Ns):
        radii = rng.uniform(10.0, 30.0, size=int(N))
        L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
        batch.add(place_beads(rng, radii, L), radii, L, seed=k, noise="device")
    for _ in range(args.warmup):
        batch.propagate(0.5)
    tune = batch.autotune(reps=2)  # schedule of the batched factorisation (results unchanged)
    torch.cuda.synchronize()
    launches0 = _lib.lib.pbg_launch_count()
    calls0 = _lib.lib.pbg_host_launch_count()
    attempts = 0
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        batch.propagate(0.5)
        attempts += max(batch.last_move_attempts(s) for s in batch.slots())
    end.record()
    torch.cuda.synchronize()
    ms = start.elapsed_time(end)
    launches = (_lib.lib.pbg_launch_count() - launches0) / args.steps
    calls = (_lib.lib.pbg_host_launch_count() - calls0) / args.steps
    graph = batch.graph_state()
    beads = int(Ns.sum())
    batch.close()
    return {"workload": "256 replicas, N~U[32,512] (seed 1), a~U[10,30], phi=0.05, Smith-Ewald m=2 n=4, "
                        "mixed, dt=0.5, device Philox noise", "replicas": 256, "beads": beads,
            "steps": args.steps, "ms_per_step": ms / args.steps,
            "bead_steps_per_s": beads * args.steps / (ms * 1e-3),
            "replica_steps_per_s": 256 * args.steps / (ms * 1e-3), "gpu_launches_per_step": launches,
            "host_launch_calls_per_step": calls, "attempt_rounds_per_step": attempts / args.steps,
            "step_graph": {1: "one CUDA graph launch per step (attempt rounds under a device-side WHILE node)",
                           0: "direct launches", -1: "capture refused"}[graph],
            "schedule": {"merge_order": tune["merge_order"], "ctas_per_sm": tune["ctas_per_sm"],
                         "factorisation_ms": {f"{o}/{c}": round(v, 4) for (o, c), v in tune["ms"].items()}}}


def run_serve_section(args, torch):
    """Continuous batching of a Poisson request stream (50 requests/s, N
    log-uniform in [16, 2048], radii uniform in [10, 40], phi 0.05, dt 1 ps),
    scaled to finish in a bench run: a shorter arrival window and fewer steps
    per request than the full stream (stated in the workload string)."""
    from pybrown_b200.batch import ReplicaBatch
    from pybrown_b200.serve import Server, make_stream
    lo, hi = args.serve_steps
    stream = make_stream(4, rate=50.0, duration=args.serve_seconds, steps_min=lo, steps_max=hi, dt=1.0)
    server = Server(ReplicaBatch(precision="mixed"), keep_positions=False)
    recs, summary = server.run(stream, clock="wall")
    server.batch.close()
    summary["workload"] = (f"Poisson 50 req/s for {args.serve_seconds:g} s, N log-U[16,2048], a~U[10,40], "
                           f"phi=0.05, steps U[{lo},{hi}] (full stream: 60 s, steps U[100,5000], about 150x "
                           f"the work per request), dt=1, mixed, device noise")
    summary["offered_bead_steps_per_s"] = sum(r.n_beads * r.steps for r in stream) / args.serve_seconds
    summary["memory_budget_gb"] = summary.pop("memory_budget") / 1e9
    summary["peak_gb"] = summary.pop("peak_bytes") / 1e9
    return summary


def run_serve_full_section(args, torch, policy="fifo"):
    """The full serving stream: Poisson 50 requests/s for 60 s, N log-uniform
    in [16, 2048], radii uniform in [10, 40], phi 0.05, steps uniform in
    [100, 5000], dt 1 ps, mixed precision, device noise; wall clock.  One B200
    cannot keep up with it (about 5e7 bead-steps/s offered), so the run is
    cut: admissions end when the stream ends and the loop stops a drain time
    later; the requests still waiting or running are reported as backlog,
    latencies are those of the completed requests.  policy: the admission
    order among arrived requests (FIFO, or least remaining work first)."""
    from pybrown_b200.batch import ReplicaBatch
    from pybrown_b200.serve import Server, make_stream
    duration = 60.0
    stream = make_stream(4, rate=50.0, duration=duration, steps_min=100, steps_max=5000, dt=1.0, lazy=True)
    server = Server(ReplicaBatch(precision="mixed"), keep_positions=False, max_active=args.serve_max_active,
                    policy=policy)
    recs, summary = server.run(stream, clock="wall", stop_admission_at=duration, drain_limit=args.serve_drain)
    server.batch.close()
    summary["workload"] = ("Poisson 50 req/s for 60 s, N log-U[16,2048], a~U[10,40], phi=0.05, steps U[100,5000], "
                           "dt=1, mixed, device noise; admissions end at 60 s, the loop "
                           f"{args.serve_drain:g} s later; at most {args.serve_max_active} requests run together; "
                           f"admission {policy}")
    summary["offered_bead_steps_per_s"] = sum(r.n_beads * r.steps for r in stream) / duration
    summary["completed_bead_steps"] = sum(r.n_beads * r.steps for r in recs if math.isfinite(r.completed))
    summary["memory_budget_gb"] = summary.pop("memory_budget") / 1e9
    summary["peak_gb"] = summary.pop("peak_bytes") / 1e9
    used = summary.pop("peak_device_used_bytes")
    summary["peak_device_used_gb"] = None if used is None else used / 1e9
    return summary


def run_reference(args, rank):
    if rank != 0:
        return None
    N = WORKLOAD["n_beads"]
    from oracle.oracle import REF_OMP_LIB
    if not os.path.exists(REF_OMP_LIB):
        return {"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent at build)"}
    sps, cores, kind, sample = cpu_reference_steps(N, steps=args.steps, warmup=min(args.warmup, 1))
    return {"impl": "reference", "metric": METRIC, "value": sps, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / sps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bead configurations)",
            "config": bench_config(args.gpus),
            "cpu_baseline": {"value": sps, "unit": "steps/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": sps, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-check", action="store_true",
                    help="skip the mixed-vs-FP64-oracle accuracy check (D, B, B xi, displacement)")
    ap.add_argument("--no-lub", action="store_true", help="skip the lubricated (Stokesian dynamics) section")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-replicas section")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving section")
    ap.add_argument("--serve-seconds", type=float, default=6.0, help="arrival window of the serving stream")
    ap.add_argument("--serve-steps", type=int, nargs=2, default=(5, 30), help="steps per request: min max")
    ap.add_argument("--no-serve-full", action="store_true", help="skip the full 60 s serving stream")
    ap.add_argument("--no-serve-sjf", action="store_true",
                    help="skip the full stream under the least-remaining-work admission policy")
    ap.add_argument("--serve-drain", type=float, default=60.0,
                    help="full serving stream: seconds the loop runs on after admissions end")
    ap.add_argument("--serve-max-active", type=int, default=256,
                    help="full serving stream: requests running together at most")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line))
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        line = run_ours(args, torch, dist, rank, world)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
