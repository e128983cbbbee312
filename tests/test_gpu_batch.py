"""Batched replicas (pybrown_b200.batch.ReplicaBatch) on the GPU.

Each replica in a batch must follow its own reference trajectory exactly as
a single system does (FP64 bar: displacement relative error <= 1e-10 and the
same accept/reject decisions), whatever else shares the batch:
  * reference trajectories (tests/golden/trajectories.npz) run inside a mix
    of other replicas, one of them with an external force, one with overlap
    rejections;
  * replicas of uneven N against the CPU oracle run alone;
  * D and B of a replica against the oracle's;
  * the mixed-precision batch against the FP64 oracle (displacement <= 1e-5);
  * a replica alone and in a mix whose membership changes between steps:
    bit-identical positions and noise-stream positions.
"""
import json
import math

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _config(seed, N, phi, a_lo, a_hi):
    rng = np.random.default_rng(seed)
    radii = rng.uniform(a_lo, a_hi, size=N)
    L = (np.sum(4.0 / 3.0 * np.pi * radii ** 3) / phi) ** (1.0 / 3.0)
    pos = []
    for a in radii:
        while True:
            p = rng.uniform(-L / 2, L / 2, size=3)
            ok = True
            for q, b in zip(pos, radii):
                d = p - q
                d -= L * np.round(d / L)
                if np.linalg.norm(d) <= a + b:
                    ok = False
                    break
            if ok:
                pos.append(p)
                break
    return np.array(pos), radii, float(L)


def _inp(L, seed, hydro, **kw):
    d = {"box_length": L, "T": 293.15, "viscosity": 0.01005, "seed": seed, "hydrodynamics": hydro,
         "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 4, "propagation_scheme": "ermak",
         "check_overlaps": True, "overlap_treshold": 0.0, "max_move_attempts": 1000000,
         "external_force": [0.0, 0.0, 0.0]}
    d.update(kw)
    return d


def _add(batch, init, radii, inp, noise="numpy"):
    N = len(radii)
    force = None
    Fex = np.asarray(inp.get("external_force", [0.0, 0.0, 0.0]), dtype=float)
    if np.any(Fex != 0):
        force = np.tile(Fex, N)
    return batch.add(init, radii, inp["box_length"], T=inp["T"], viscosity=inp["viscosity"], seed=inp["seed"],
                     noise=noise, check_overlaps=inp["check_overlaps"], overlap_treshold=inp["overlap_treshold"],
                     max_move_attempts=inp["max_move_attempts"], force=force)


def _golden(trajectories, name):
    inp = json.loads(str(trajectories[f"{name}/config"]))
    init = trajectories[f"{name}/init"]
    radii = np.full(len(init), float(trajectories[f"{name}/radius"]))
    return inp, init, radii, float(trajectories[f"{name}/dt"])


# one batch per reference trajectory: a batch shares one set of Ewald parameters
@pytest.mark.parametrize("hydro,names", [("rpy", ("ermak_rpy_reject",)), ("rpy", ("ermak_rpy",)),
                                         ("rpy_smith", ("ermak_smith",)),
                                         ("rpy_smith", ("ermak_smith_force",))])
def test_reference_trajectories_inside_a_mix(trajectories, oracle_lib, hydro, names):
    from oracle.oracle import OracleBox
    from pybrown_b200.batch import ReplicaBatch
    golden = [_golden(trajectories, n) for n in names]
    dt = golden[0][3]
    assert all(g[3] == dt for g in golden)
    ew = {k: golden[0][0][k] for k in ("ewald_alpha", "ewald_real", "ewald_imag")}
    batch = ReplicaBatch(precision="fp64", hydrodynamics=hydro, **ew)
    slots, refs = [], []
    # other replicas first, so the reference ones do not sit at slot 0
    for k, N in enumerate((9, 20)):
        pos, radii, L = _config(40 + k, N, 0.05, 1.0, 2.0)
        inp = _inp(L, 7 + k, hydro, T=298.0, viscosity=0.01, **ew)
        refs.append((_add(batch, pos, radii, inp), OracleBox(pos, radii, inp, clib=oracle_lib), pos))
    for (inp, init, radii, _), n in zip(golden, names):
        slots.append((_add(batch, init, radii, inp), n, init))
    steps = min(len(trajectories[f"{n}/traj"]) for n in names)
    draws = {s: 0 for s, _, _ in slots}
    for k in range(steps):
        batch.propagate(dt)
        for s, n, init in slots:
            draws[s] += 3 * len(init) * batch.last_move_attempts(s)
            ref = trajectories[f"{n}/traj"][k]
            assert draws[s] == trajectories[f"{n}/draws"][k], (n, k)
            assert rel_err(batch.positions(s) - init, ref - init) <= 1e-10, (n, k)
        for s, box, init in refs:
            box.propagate(dt)
            assert rel_err(batch.positions(s) - init, box.pos - init) <= 1e-10, (s, k)
    batch.close()


def test_uneven_replicas_match_oracle_alone(oracle_lib):
    """Four rpy_smith replicas of N = 12 .. 64 in one FP64 batch, each against
    the oracle run alone; then D and B of the largest."""
    from oracle.oracle import OracleBox
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision="fp64")
    reps = []
    for k, N in enumerate((12, 30, 47, 64)):
        pos, radii, L = _config(k, N, 0.05, 10.0, 30.0)
        inp = _inp(L, 100 + k, "rpy_smith")
        reps.append((_add(batch, pos, radii, inp), OracleBox(pos, radii, inp, clib=oracle_lib), pos))
    draws = {s: 0 for s, _, _ in reps}
    for step in range(5):
        batch.propagate(1.0)
        for s, box, init in reps:
            box.propagate(1.0)
            draws[s] += 3 * len(init) * batch.last_move_attempts(s)
            assert draws[s] == box.draw_count, (s, step)
            assert rel_err(batch.positions(s) - init, box.pos - init) <= 1e-10, (s, step)
    s, box, _ = reps[-1]
    assert rel_err(batch.matrix(s, "D"), box.D) <= 1e-10
    assert rel_err(np.tril(batch.matrix(s, "B")), np.tril(box.B)) <= 1e-10
    batch.close()


def test_mixed_batch_against_fp64_oracle(oracle_lib):
    from oracle.oracle import OracleBox
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision="mixed")
    reps = []
    for k, N in enumerate((24, 64, 96)):
        pos, radii, L = _config(10 + k, N, 0.05, 10.0, 30.0)
        inp = _inp(L, 200 + k, "rpy_smith")
        reps.append((_add(batch, pos, radii, inp), OracleBox(pos, radii, inp, clib=oracle_lib), pos))
    for _ in range(5):
        batch.propagate(0.5)
        for s, box, init in reps:
            box.propagate(0.5)
    for s, box, init in reps:
        assert rel_err(batch.positions(s) - init, box.pos - init) <= 1e-5, s
    batch.close()


def test_alone_equals_mix_with_changing_membership():
    """Device noise, mixed precision: one replica alone, and the same replica in
    a batch that gains and loses other replicas between steps, give identical
    positions and noise-stream positions."""
    from pybrown_b200.batch import ReplicaBatch
    pos, radii, L = _config(77, 50, 0.05, 10.0, 30.0)

    def run(mix):
        batch = ReplicaBatch(precision="mixed")
        others = []
        if mix:
            for k, N in enumerate((17, 120)):
                p, r, l = _config(300 + k, N, 0.05, 10.0, 30.0)
                others.append(batch.add(p, r, l, seed=900 + k, noise="device"))
        s = batch.add(pos, radii, L, seed=12345, noise="device")
        out = []
        for step in range(6):
            if mix and step == 2:
                p, r, l = _config(400, 33, 0.05, 10.0, 30.0)
                others.append(batch.add(p, r, l, seed=901, noise="device"))
            if mix and step == 4:
                batch.remove(others.pop(0))
            batch.propagate(1.0)
            out.append(batch.positions(s).copy())
        d = batch.draws(s)
        batch.close()
        return np.array(out), d

    alone, d_alone = run(False)
    mixed, d_mixed = run(True)
    assert d_alone == d_mixed and d_alone >= 6 * 150
    assert np.array_equal(alone, mixed)
    assert np.all(np.isfinite(alone)) and not np.array_equal(alone[0], alone[-1])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_autotuned_schedule_changes_no_result(precision):
    """The schedule autotuner (merge order of the replicas' task segments,
    L2-sized chunks of replicas included, x CTAs per SM) times every
    candidate on the current matrices and keeps the fastest; trajectories with the tuned schedule, and with each fixed
    schedule, are bit-identical to the default one."""
    from pybrown_b200.batch import ReplicaBatch
    configs = [_config(500 + k, N, 0.05, 10.0, 30.0) for k, N in enumerate((40, 130, 75, 200, 33))]

    def run(schedule):
        batch = ReplicaBatch(precision=precision)
        slots = [batch.add(p, r, l, seed=70 + k, noise="device") for k, (p, r, l) in enumerate(configs)]
        tuned = None
        out = []
        for step in range(5):
            if step == 1 and schedule == "auto":
                tuned = batch.autotune(reps=1)
            elif step == 1 and schedule is not None:
                batch.set_schedule(*schedule)
            batch.propagate(1.0)
            out.append(np.concatenate([batch.positions(s).ravel() for s in slots]))
        batch.close()
        return np.array(out), tuned

    ref, _ = run(None)
    got, tuned = run("auto")
    assert np.array_equal(ref, got)
    # every merge order at each CTAs-per-SM count the factorisation kernel
    # can keep resident (one for both kernels of this build)
    ctas = {c for _, c in tuned["ms"]}
    assert ctas and ctas <= {1, 2}
    assert set(tuned["ms"]) == {(o, c) for o in ReplicaBatch.MERGE_ORDERS for c in ctas}
    assert all(v > 0 for v in tuned["ms"].values())
    assert tuned["ms"][(tuned["merge_order"], tuned["ctas_per_sm"])] == min(tuned["ms"].values())
    for sched in (("replica_major", 1), ("smaller_first", 0), ("added", 1), ("chunk_32M", 0)):
        assert np.array_equal(ref, run(sched)[0]), sched


def test_graph_replay_matches_direct_launches():
    """From the second step with an unchanged membership the start of a step
    replays one CUDA graph; the trajectories equal, bit for bit, those of a
    batch whose schedule is switched every step (a rebuild, so its kernels are
    launched one by one)."""
    from pybrown_b200.batch import ReplicaBatch
    configs = [_config(600 + k, N, 0.05, 10.0, 30.0) for k, N in enumerate((64, 150, 90))]

    def run(toggle):
        batch = ReplicaBatch(precision="mixed")
        slots = [batch.add(p, r, l, seed=30 + k, noise="device") for k, (p, r, l) in enumerate(configs)]
        out, states = [], []
        for step in range(5):
            if toggle:
                batch.set_schedule("added" if step % 2 else "larger_first")
            batch.propagate(1.0)
            states.append(batch.graph_state())
            out.append(np.concatenate([batch.positions(s).ravel() for s in slots]))
        batch.close()
        return np.array(out), states

    graph, g_states = run(False)
    direct, d_states = run(True)
    assert g_states == [0, 1, 1, 1, 1]
    assert d_states == [0, 0, 0, 0, 0]
    assert np.array_equal(graph, direct)


def test_device_noise_is_standard_normal():
    """The counter-based stream has mean 0, variance 1 and no correlation
    between neighbouring draws, seen through the moves of a very dilute rpy
    replica (D almost diagonal, so a move is sqrt(2 dt D_ii) xi_i)."""
    from pybrown_b200.batch import ReplicaBatch
    N = 1000
    L = 1.0e5  # very dilute: D is almost diagonal, D_ii = kBT 1e19 / (6 pi eta a)
    rng = np.random.default_rng(5)
    pos = rng.uniform(-L / 2, L / 2, size=(N, 3))
    radii = np.full(N, 10.0)
    batch = ReplicaBatch(precision="fp64", hydrodynamics="rpy")
    s = batch.add(pos, radii, L, seed=2024, noise="device", check_overlaps=False)
    moves = []
    for _ in range(4):
        before = batch.positions(s).copy()
        batch.propagate(1.0)
        d = batch.positions(s) - before
        d -= L * np.round(d / L)
        moves.append(d.reshape(-1))
    m = np.concatenate(moves)
    kBT = 1.380649e-23 * 293.15
    sigma = math.sqrt(2 * 1.0 * kBT * 1e19 / (6 * math.pi * 0.01005 * 10.0))
    z = m / sigma
    assert abs(z.mean()) < 0.05
    assert abs(z.var() - 1.0) < 0.05
    assert abs(np.corrcoef(z[:-1], z[1:])[0, 1]) < 0.05
    assert batch.draws(s) == 4 * 3 * N
    batch.close()


def test_device_step_loop_matches_host_driven_attempts():
    """pbg_batch_step (every attempt round on the device, one CUDA graph per
    repeated step) gives, bit for bit, the positions, attempt counts and noise
    stream positions of the attempt-by-attempt path driven from the host,
    including replicas with rejected moves (dense boxes) and a membership
    change between steps."""
    from pybrown_b200.batch import ReplicaBatch
    configs = [_config(700 + k, N, phi, 10.0, 30.0) for k, (N, phi) in
               enumerate(((64, 0.05), (150, 0.30), (90, 0.25), (40, 0.05)))]

    def run(device_loop):
        batch = ReplicaBatch(precision="mixed")
        slots = [batch.add(p, r, l, seed=70 + k, noise="device") for k, (p, r, l) in enumerate(configs[:3])]
        out, att, states = [], [], []
        for step in range(6):
            if step == 3:
                slots.append(batch.add(*configs[3], seed=73, noise="device"))
            batch.propagate(10.0, device_loop=device_loop)  # long steps: rejections in the dense boxes
            states.append(batch.graph_state())
            out.append(np.concatenate([batch.positions(s).ravel() for s in slots]))
            att.append([batch.last_move_attempts(s) for s in slots])
        draws = [batch.draws(s) for s in slots]
        batch.close()
        return out, att, draws, states

    dev = run(True)
    host = run(False)
    for a, b in zip(dev[0], host[0]):
        assert np.array_equal(a, b)
    assert dev[1] == host[1]
    assert dev[2] == host[2]
    assert max(max(a) for a in dev[1]) > 1  # some moves were rejected and redrawn
    assert dev[3] == [0, 1, 1, 0, 1, 1]  # captured on a repeat, dropped by the membership change


def test_device_step_loop_attempt_limit():
    """A replica that can never be accepted (two beads overlapping at the
    start) stops after max_move_attempts with every move undone and the
    step raises, as box.py:248 asserts."""
    from pybrown_b200.batch import ReplicaBatch
    pos = np.array([[0.0, 0.0, 0.0], [5.0, 0.0, 0.0], [40.0, 40.0, 40.0]])
    radii = np.array([10.0, 10.0, 10.0])
    batch = ReplicaBatch(precision="fp64")
    s = batch.add(pos, radii, 200.0, seed=3, noise="device", max_move_attempts=5)
    other = batch.add(*_config(5, 30, 0.05, 10.0, 20.0), seed=4, noise="device")
    with pytest.raises(AssertionError):
        batch.propagate(0.01)
    assert batch.last_move_attempts(s) == 5
    assert batch.last_move_attempts(other) >= 1
    assert np.allclose(batch.positions(s), pos, rtol=0, atol=1e-12)
    batch.close()


def test_long_graph_replay_with_autotuner_matches_direct_launches():
    """The batched configuration's shape -- 256 replicas, N uniform in
    [32, 512] (seed 1), radii U[10, 30], volume fraction 0.05, mixed
    precision, device noise -- stepped 200 times as graph replays (whole steps
    on the device), then autotuned, then 200 more, against the same batch
    stepped with every kernel launched directly (a schedule switch before
    every step forces a rebuild, and the attempts are driven from the host):
    identical positions bit for bit, and no step reports a failed
    factorisation."""
    from pybrown_b200.batch import ReplicaBatch
    from pybrown_b200.serve import place_beads
    rng = np.random.default_rng(1)
    Ns = rng.integers(32, 513, size=256)
    configs = []
    for N in Ns:
        radii = rng.uniform(10.0, 30.0, size=int(N))
        L = float((np.sum(4.0 / 3.0 * np.pi * radii ** 3) / 0.05) ** (1.0 / 3.0))
        configs.append((place_beads(rng, radii, L), radii, L))

    def run(direct):
        batch = ReplicaBatch(precision="mixed")
        slots = [batch.add(p, r, l, seed=k, noise="device") for k, (p, r, l) in enumerate(configs)]
        snaps = []
        for phase in range(2):
            for step in range(200):
                if direct:
                    batch.set_schedule(("larger_first", "added")[step % 2])
                batch.propagate(0.5, device_loop=not direct)
                if not direct and step >= 1:
                    assert batch.graph_state() == 1
                if step % 50 == 49:
                    snaps.append(np.concatenate([batch.positions(s).ravel() for s in slots[::17]]))
            if phase == 0:
                batch.autotune(reps=1)
        final = np.concatenate([batch.positions(s).ravel() for s in slots])
        batch.close()
        return snaps, final

    g_snaps, g_final = run(False)
    d_snaps, d_final = run(True)
    for a, b in zip(g_snaps, d_snaps):
        assert np.array_equal(a, b)
    assert np.array_equal(g_final, d_final)


def test_check_factor_of_healthy_replicas():
    """pbg_batch_check_factor factors a copy of a replica's D with the
    single-matrix kernel: 0 for every replica of a healthy batch, and the
    batch's own B is left unchanged."""
    import ctypes
    from pybrown_b200 import _lib
    from pybrown_b200.batch import ReplicaBatch
    batch = ReplicaBatch(precision="mixed")
    slots = [batch.add(*_config(800 + k, N, 0.05, 10.0, 30.0), seed=k, noise="device")
             for k, N in enumerate((40, 130))]
    batch.propagate(0.5)
    for s in slots:
        B = batch.matrix(s, "B")
        info = ctypes.c_int(-5)
        _lib.call("pbg_batch_check_factor", batch._h, s, ctypes.byref(info), None)
        assert info.value == 0
        assert np.array_equal(batch.matrix(s, "B"), B)
    batch.close()
