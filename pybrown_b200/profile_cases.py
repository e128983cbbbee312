"""Run one hot-path kernel on a seeded synthetic case (for profilers).

    python -m pybrown_b200.profile_cases cholesky --order 768 --precision mixed
    python -m pybrown_b200.profile_cases smith --beads 512 --precision fp64
    python -m pybrown_b200.profile_cases batch --replicas 64 --precision mixed
    python -m pybrown_b200.profile_cases lub --beads 512 --precision fp64
    python -m pybrown_b200.profile_cases forces --beads 1024 --precision mixed

`cholesky` factors the Smith-Ewald diffusion matrix of a random bead
configuration (order 3 x beads, padded to a multiple of 64); `smith` builds it;
`batch` advances a batch of replicas (N uniform in [32, 512], seed 1) by one
step; `lub` takes one midpoint step of a lubricated box (rpy_smith_lub,
radius 20, volume fraction 0.30, cutoff 0.5, Cichocki, m = 100, dt 0.1);
`forces` steps a box of bonded chains (16 beads each, bond angles at their
150-degree equilibrium, harmonic bonds and angles, Lennard-Jones 6-12,
rpy_smith, Ermak, dt 0.05), so that the force kernels run every step.
Each case runs `--reps` times after one warm-up and prints the mean CUDA-event
time of one launch; `--reps 0` runs the warm-up call only (a batch's first
step is made of direct kernel launches, the later ones replay a CUDA graph).
"""
import argparse
import math

import numpy as np


def _config(seed, n, L, a_lo=10.0, a_hi=40.0, gap=0.0):
    rng = np.random.default_rng(seed)
    pos = np.zeros((n, 3))
    radii = np.zeros(n)
    k = 0
    while k < n:
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


def _time(torch, fn, reps):
    """Mean CUDA-event time (ms) of `reps` calls of fn after one warm-up call;
    None for reps = 0 (the warm-up call only)."""
    fn()
    torch.cuda.synchronize()
    if reps <= 0:
        return None
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total = 0.0
    for _ in range(reps):
        start.record()
        fn()
        end.record()
        torch.cuda.synchronize()
        total += start.elapsed_time(end)
    return total / reps


def _ms(t):
    return "warm-up only" if t is None else f"{t:.3f} ms"


def main(argv=None):
    import torch

    from . import _lib
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("kernel", choices=("cholesky", "smith", "batch", "lub", "forces"))
    ap.add_argument("--replicas", type=int, default=64)
    ap.add_argument("--beads", type=int, default=256)
    ap.add_argument("--order", type=int, default=0, help="cholesky: matrix order (default 3 x beads)")
    ap.add_argument("--precision", choices=("fp64", "mixed", "mixed_fp64_diag"), default="mixed",
                    help="mixed_fp64_diag: cholesky only, the FP32 factorisation with FP64 diagonal tiles")
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--merge-order", default="larger_first", help="batch: task merge order")
    ap.add_argument("--ctas", type=int, default=0, help="batch: factorisation CTAs per SM (0 = as many as fit)")
    a = ap.parse_args(argv)
    if a.kernel == "batch":
        return _batch(a, torch)
    if a.kernel == "lub":
        return _lub(a, torch)
    if a.kernel == "forces":
        return _forces(a, torch)
    chol_prec = {"fp64": 0, "mixed": 1, "mixed_fp64_diag": 2}[a.precision]
    prec = min(chol_prec, 1)  # the Ewald build: FP64 or FP32
    dtype = torch.float64 if prec == 0 else torch.float32
    beads = a.order // 3 if a.order else a.beads
    L = 1500.0 * (beads / 1024.0) ** (1.0 / 3.0)  # volume fraction of the N=1024 workload
    pos, radii = _config(0, beads, L)
    n = 3 * beads
    ld = (n + 63) // 64 * 64
    dpos = torch.tensor(pos.reshape(-1), dtype=torch.float64, device="cuda")
    drad = torch.tensor(radii, dtype=torch.float64, device="cuda")
    M = torch.zeros((ld, ld), dtype=dtype, device="cuda")
    scale = 1.380649e-23 * 293.15 * 1e19 / 0.01005

    def smith():
        _lib.call("pbg_dev_smith_matrix", dpos.data_ptr(), drad.data_ptr(), beads, L, math.sqrt(math.pi), 2, 4,
                  scale, prec, M.data_ptr(), ld, None)

    smith()
    torch.cuda.synchronize()
    A0 = M.clone()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")

    def cholesky():
        M.copy_(A0)
        _lib.call("pbg_dev_cholesky", M.data_ptr(), n, ld, chol_prec, info.data_ptr(), None)

    t = _time(torch, smith if a.kernel == "smith" else cholesky, a.reps)
    extra = f" info={int(info.item())}" if a.kernel == "cholesky" else ""
    print(f"{a.kernel} n={n} ({a.precision}): {_ms(t)} per launch{extra}")


def _batch(a, torch):
    from .batch import ReplicaBatch
    from .serve import place_beads
    rng = np.random.default_rng(1)
    Ns = rng.integers(32, 513, size=a.replicas)
    batch = ReplicaBatch(precision=a.precision)
    for k, N in enumerate(Ns):
        radii = rng.uniform(10.0, 30.0, size=int(N))
        L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
        batch.add(place_beads(rng, radii, L), radii, L, seed=k, noise="device")
    batch.set_schedule(a.merge_order, a.ctas)
    t = _time(torch, lambda: batch.propagate(0.5), a.reps)
    print(f"batch {a.replicas} replicas ({int(Ns.sum())} beads, {a.precision}, {a.merge_order}, "
          f"{a.ctas or 'max'} CTAs/SM): {_ms(t)} per step")
    batch.close()


def _lub(a, torch):
    from .bead import Bead
    from .box import Box
    N, radius, phi = a.beads, 20.0, 0.30
    L = (N * 4.0 * math.pi * radius ** 3 / 3.0 / phi) ** (1.0 / 3.0)
    pos, radii = _config(0, N, L, radius, radius, gap=0.05 * radius)
    inp = {"box_length": L, "T": 293.15, "viscosity": 0.01005, "seed": 0, "hydrodynamics": "rpy_smith_lub",
           "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 4, "lubrication_cutoff": 0.5,
           "cichocki_correction": True, "propagation_scheme": "midpoint", "m_midpoint": 100.0,
           "immobile_labels": [], "check_overlaps": True, "overlap_treshold": 0.0, "max_move_attempts": 1000000,
           "external_force": [0.0, 0.0, 0.0], "energy_unit": "joule", "verbose": False, "debug": False,
           "precision": a.precision, "lennard_jones_6": False, "lennard_jones_12": False,
           "custom_interactions": False}
    box = Box([Bead(p, r) for p, r in zip(pos, radii)], inp)
    t = _time(torch, lambda: box.propagate(0.1), a.reps)
    print(f"lub N={N} L={L:.1f} ({a.precision}): {_ms(t)} per step")


def _chains(n_beads, length=16, seed=0):
    """Chains of beads (radius 2, bond length 4.2 A, every bond angle at its
    150-degree equilibrium, random dihedrals) in a box at about 2 % volume
    fraction, bonded along each chain (rest length 4.2, k 5) with angle terms
    (150 degrees, k 2).  No three consecutive beads are collinear: the
    harmonic angle force divides by sin(angle), which vanishes at 180 degrees."""
    from .bead import Bead
    rng = np.random.default_rng(seed)
    n_chains = max(1, n_beads // length)
    L = (n_chains * length * 4.0 / 3.0 * math.pi * 8.0 / 0.02) ** (1.0 / 3.0)
    turn = math.radians(180.0 - 150.0)
    beads, pts_all = [], []

    def walk():
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        pts = [rng.uniform(-L / 2, L / 2, 3)]
        for _ in range(length - 1):
            w = rng.normal(size=3)
            w -= (w @ u) * u
            w /= np.linalg.norm(w)
            if len(pts) > 1:
                u = math.cos(turn) * u + math.sin(turn) * w
            pts.append(pts[-1] + 4.2 * u)
        return pts

    def clear(p, others):
        for q in others:
            d = p - q
            d -= L * np.round(d / L)
            if d @ d <= 4.5 ** 2:
                return False
        return True

    for c in range(n_chains):
        while True:
            pts = walk()
            ok = all(clear(p, pts[:max(0, i - 1)]) for i, p in enumerate(pts))
            ok = ok and all(clear(p, pts_all) for p in pts)
            if ok:
                break
        base = len(beads) + 1
        for i, p in enumerate(pts):
            p = p - L * np.round(p / L)
            beads.append(Bead(p, 2.0, label="P", hard_core_radius=1.9, epsilon_LJ=0.2, bead_id=base + i))
        pts_all.extend(pts)
        for i in range(length - 1):
            beads[base - 1 + i].bonded_with.append(base + i + 1)
            beads[base - 1 + i].bonded_how[base + i + 1] = [4.2, 5.0]
        for i in range(length - 2):
            beads[base - 1 + i].angled_with.append([base + i + 1, base + i + 2])
            beads[base - 1 + i].angled_how[(base + i + 1, base + i + 2)] = [150.0, 2.0]
    return beads, L


def _forces(a, torch):
    from .box import Box
    beads, L = _chains(a.beads)
    inp = {"box_length": L, "T": 293.15, "viscosity": 0.01005, "seed": 0, "hydrodynamics": "rpy_smith",
           "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 4, "propagation_scheme": "ermak",
           "immobile_labels": [], "check_overlaps": True, "overlap_treshold": 0.0, "max_move_attempts": 1000000,
           "external_force": [0.0, 0.0, 0.0], "energy_unit": "kcal/mol", "verbose": False, "debug": False,
           "precision": a.precision, "lennard_jones_6": True, "lennard_jones_12": True, "lennard_jones_alpha": 4.0,
           "custom_interactions": False}
    box = Box(beads, inp)
    t = _time(torch, lambda: box.propagate(0.05), a.reps)
    print(f"forces N={len(beads)} L={L:.1f} ({a.precision}): {_ms(t)} per step, E={box.E:.4g}")


if __name__ == "__main__":
    main()
