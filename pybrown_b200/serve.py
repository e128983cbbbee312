"""Serving loop: continuous batching of BD-with-HI simulation requests.

Requests (bead configuration, step count, seed) arrive over time.  The loop
admits a request as soon as it has arrived and its device footprint -- the
(3N)^2 tensor and factor plus tables and state, ``pbg_batch_footprint`` --
fits in the memory budget next to the requests already running; admitted
requests join one ``ReplicaBatch`` and advance together, one batched step at
a time, so their work overlaps on the device; a request leaves the batch when
its last step is done, freeing its memory for the next ones.  State stays on
the device from admission to completion.

Each request draws its noise from its own counter-based device stream keyed
by its seed, so its result does not depend on what else was running: it is
the same alone and in the mix.

Completion latency = completion time - arrival time.  ``run`` returns the
per-request records and a summary with p50/p99 latency of the completed
requests, the bead-steps/s the batched steps delivered, and -- when the run
is cut off (admissions end at ``stop_admission_at``, the loop ``drain_limit``
seconds later) -- the backlog of requests still waiting or running.

Two clocks: ``"wall"`` (real time; arrivals are released when the wall clock
reaches them) and ``"virtual"`` (time advances by ``tick`` per batched step
and jumps to the next arrival when idle; deterministic, for tests).
"""
import collections
import heapq
import math
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float          # s since the start of the stream
    positions: np.ndarray   # N x 3, Angstrom (None: placed on first use, see placement_seed)
    radii: np.ndarray       # N, Angstrom
    box_length: float       # Angstrom
    steps: int
    seed: int
    dt: float = 1.0         # ps
    T: float = 293.15
    viscosity: float = 0.01005
    placement_seed: int = None  # positions = place_beads_fast(default_rng(placement_seed), radii, box)

    def __post_init__(self):
        if self.positions is None and self.placement_seed is None:
            raise ValueError("a request needs positions or a placement seed")

    def materialize(self):
        """Places the beads now if they were left for first use."""
        if self.positions is None:
            self.positions = place_beads_fast(np.random.default_rng(self.placement_seed), self.radii,
                                              self.box_length)
        return self.positions

    @property
    def n_beads(self):
        return len(self.radii)


@dataclass
class Record:
    rid: int
    n_beads: int
    steps: int
    arrival: float
    admitted: float = math.nan
    completed: float = math.nan
    positions: np.ndarray = field(default=None, repr=False)
    failed: dict = None   # set when the request's factorisation failed: {"status", "recheck"}

    @property
    def latency(self):
        return self.completed - self.arrival


def make_stream(seed, rate, duration, n_min=16, n_max=2048, a_lo=10.0, a_hi=40.0, phi=0.05,
                steps_min=100, steps_max=5000, dt=1.0, lazy=False):
    """Poisson arrivals at `rate` per second for `duration` seconds; N
    log-uniform in [n_min, n_max], radii uniform in [a_lo, a_hi], random
    non-overlapping positions in a periodic cubic box at volume fraction phi,
    step count uniform in [steps_min, steps_max].  With lazy=True each
    request's beads are placed when it is first used (admission), from its
    own seeded generator, so that a long stream costs nothing up front."""
    rng = np.random.default_rng(seed)
    t, out, rid = 0.0, [], 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        N = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        radii = rng.uniform(a_lo, a_hi, size=N)
        L = (np.sum(4.0 / 3.0 * np.pi * radii ** 3) / phi) ** (1.0 / 3.0)
        if lazy:
            pos, pseed = None, int(rng.integers(0, 2 ** 63))
        else:
            pos, pseed = place_beads(rng, radii, L), None
        steps = int(rng.integers(steps_min, steps_max + 1))
        out.append(Request(rid, t, pos, radii, float(L), steps, int(rng.integers(0, 2 ** 63)), dt,
                           placement_seed=pseed))
        rid += 1
    return out


def place_beads_fast(rng, radii, L, max_rounds=1000):
    """Random non-overlapping placement (minimum image) for dilute boxes:
    every bead drawn uniformly in the box at once, then, round by round, the
    higher-indexed bead of each overlapping pair (found with a periodic k-d
    tree) drawn again, until no pair overlaps."""
    from scipy.spatial import cKDTree
    N = len(radii)
    pos = rng.uniform(-L / 2, L / 2, size=(N, 3))
    reach = 2.0 * float(np.max(radii))
    for _ in range(max_rounds):
        tree = cKDTree(np.mod(pos + L / 2, L), boxsize=L)
        pairs = tree.query_pairs(reach, output_type="ndarray")
        if len(pairs):
            d = pos[pairs[:, 0]] - pos[pairs[:, 1]]
            d -= L * np.round(d / L)
            hit = np.einsum("ij,ij->i", d, d) <= (radii[pairs[:, 0]] + radii[pairs[:, 1]]) ** 2
            pairs = pairs[hit]
        if not len(pairs):
            return pos
        redo = np.unique(np.max(pairs, axis=1))
        pos[redo] = rng.uniform(-L / 2, L / 2, size=(len(redo), 3))
    raise RuntimeError("bead placement did not converge (box too dense)")


def place_beads(rng, radii, L):
    """Sequential random placement without overlaps (minimum image), on a cell
    grid so that large N stays fast."""
    N = len(radii)
    amax = float(np.max(radii))
    ncell = max(1, int(L // (2 * amax)))
    cell = L / ncell
    grid = collections.defaultdict(list)
    pos = np.empty((N, 3))
    for i, a in enumerate(radii):
        while True:
            p = rng.uniform(-L / 2, L / 2, size=3)
            c = np.floor((p + L / 2) / cell).astype(int) % ncell
            ok = True
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((c[0] + dx) % ncell, (c[1] + dy) % ncell, (c[2] + dz) % ncell)
                        for j in grid.get(key, ()):
                            d = p - pos[j]
                            d -= L * np.round(d / L)
                            if np.dot(d, d) <= (a + radii[j]) ** 2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                pos[i] = p
                grid[tuple(c)].append(i)
                break
    return pos


class Server:
    """Continuous-batching request loop over one ReplicaBatch.

    batch: a ReplicaBatch (or an object with add/remove/propagate/positions/
    footprint); memory_budget: device bytes the admitted requests may take
    (default: 80 % of the free device memory at start); max_active: optional
    cap on concurrent requests; policy: the admission order among the
    requests that have arrived -- "fifo" (arrival order; a request that does
    not fit holds back the ones behind it) or "smallest_work" (least
    remaining work first, work = steps x (3N)^3, the factorisation's cost per
    step, ties in arrival order)."""

    POLICIES = ("fifo", "smallest_work")

    def __init__(self, batch=None, memory_budget=None, max_active=None, precision="mixed", keep_positions=True,
                 policy="fifo"):
        if policy not in self.POLICIES:
            raise ValueError(f"unknown admission policy {policy!r}")
        self.policy = policy
        if batch is None:
            from .batch import ReplicaBatch
            batch = ReplicaBatch(precision=precision)
        self.batch = batch
        if memory_budget is None:
            import torch
            free, _ = torch.cuda.mem_get_info()
            memory_budget = int(0.8 * free)
        self.memory_budget = int(memory_budget)
        self.max_active = max_active
        self.keep_positions = keep_positions
        # device memory in use (total - free), sampled during the run
        self.device_memory = None
        try:
            import torch
            if torch.cuda.is_available():
                def used():
                    free, total = torch.cuda.mem_get_info()
                    return int(total - free)
                self.device_memory = used
        except ImportError:
            pass

    def _propagate(self, dt):
        """One batched step; returns the replicas whose factorisation failed
        as (slot, status, status of a single-matrix recheck)."""
        try:
            self.batch.propagate(dt)
        except Exception as e:  # noqa: BLE001 -- only a failed factorisation is handled here
            slots = getattr(e, "slots", None)
            if not slots:
                raise
            return [(s, info, getattr(e, "recheck", {}).get(s)) for s, info in slots.items()]
        return []

    def run(self, requests, clock="wall", tick=1e-3, stop_admission_at=None, drain_limit=None):
        """Serves `requests` until all are done, or -- with stop_admission_at
        (s) -- admits nothing after that time and stops drain_limit s later
        (then the ones still waiting or running are the backlog)."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            if self.batch.footprint(r.n_beads) > self.memory_budget:
                raise ValueError(f"request {r.rid} (N={r.n_beads}) does not fit in the memory budget")
        pending = collections.deque(reqs)
        arrived = []  # smallest_work: heap of the arrived requests
        records = {r.rid: Record(r.rid, r.n_beads, r.steps, r.arrival) for r in reqs}
        active = {}  # slot -> [request, steps left, bytes]
        used = 0
        peak_used, peak_active, batched_steps = 0, 0, 0
        t_step = t_admin = 0.0
        bead_steps_done = 0
        peak_device_used = 0
        start = time.perf_counter()
        vnow = 0.0
        end_at = None if stop_admission_at is None else stop_admission_at + (drain_limit or 0.0)

        def now():
            return vnow if clock == "virtual" else time.perf_counter() - start

        def next_candidate():
            if self.policy == "fifo":
                return pending[0] if pending and pending[0].arrival <= t else None
            while pending and pending[0].arrival <= t:
                r = pending.popleft()
                heapq.heappush(arrived, (r.steps * (3 * r.n_beads) ** 3, r.arrival, r.rid, r))
            return arrived[0][3] if arrived else None

        def take(r):
            if self.policy == "fifo":
                pending.popleft()
            else:
                heapq.heappop(arrived)

        while pending or arrived or active:
            t = now()
            if end_at is not None and t >= end_at:
                break
            admitting = stop_admission_at is None or t < stop_admission_at
            if not admitting and not active:
                break
            # admission: arrived requests in policy order, while they fit
            while admitting:
                r = next_candidate()
                if r is None:
                    break
                fp = self.batch.footprint(r.n_beads)
                if used + fp > self.memory_budget or (self.max_active and len(active) >= self.max_active):
                    break
                take(r)
                t0 = time.perf_counter()
                slot = self.batch.add(r.materialize(), r.radii, r.box_length, T=r.T, viscosity=r.viscosity,
                                      seed=r.seed, noise="device")
                t_admin += time.perf_counter() - t0
                active[slot] = [r, r.steps, fp]
                used += fp
                records[r.rid].admitted = now()
            peak_used = max(peak_used, used)
            peak_active = max(peak_active, len(active))
            if not active:
                if not pending:
                    break  # admission closed with requests still waiting
                # idle until the next arrival
                nxt = pending[0].arrival
                if stop_admission_at is not None and nxt >= stop_admission_at:
                    break
                if clock == "virtual":
                    vnow = max(vnow, nxt)
                else:
                    time.sleep(max(0.0, nxt - now()))
                continue
            dts = {a[0].dt for a in active.values()}
            if len(dts) != 1:
                raise ValueError("requests running together must share dt")
            t0 = time.perf_counter()
            failed = self._propagate(dts.pop())
            t_step += time.perf_counter() - t0
            for slot, info, recheck in failed:
                # a request whose factorisation failed leaves with an error; the others go on
                r, _, fp = active.pop(slot)
                rec = records[r.rid]
                rec.failed = {"status": info, "recheck": recheck}
                self.batch.remove(slot)
                used -= fp
            batched_steps += 1
            bead_steps_done += sum(a[0].n_beads for a in active.values())
            if self.device_memory and batched_steps % 16 == 1:
                peak_device_used = max(peak_device_used, self.device_memory())
            if clock == "virtual":
                vnow += tick
            done = []
            for slot, a in active.items():
                a[1] -= 1
                if a[1] == 0:
                    done.append(slot)
            if done:
                t_done = now()
                t0 = time.perf_counter()
                for slot in done:
                    r, _, fp = active.pop(slot)
                    rec = records[r.rid]
                    rec.completed = t_done
                    if self.keep_positions:
                        rec.positions = self.batch.positions(slot).copy()
                    self.batch.remove(slot)
                    used -= fp
                t_admin += time.perf_counter() - t0
        elapsed = now() if clock == "virtual" else time.perf_counter() - start
        for slot in list(active):  # stopped by the drain limit: leave the batch empty
            self.batch.remove(slot)
        recs = [records[r.rid] for r in reqs]
        completed = [x for x in recs if np.isfinite(x.completed)]
        lat = np.array([x.latency for x in completed]) if completed else np.array([math.nan])
        failures = [{"rid": x.rid, "n_beads": x.n_beads, **x.failed} for x in recs if x.failed]
        summary = {
            "requests": len(recs),
            "completed": len(completed),
            "failed": len(failures),
            "failures": failures[:16],
            "backlog_waiting": sum(1 for x in recs if not np.isfinite(x.admitted)),
            "backlog_running": len(active),
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3),
            "bead_steps_per_s": bead_steps_done / elapsed if elapsed > 0 else math.inf,
            "elapsed_s": elapsed,
            "batched_steps": batched_steps,
            "peak_active": peak_active,
            "step_s": t_step,      # wall time inside batched steps (membership rebuilds included)
            "admin_s": t_admin,    # wall time adding and removing replicas (bead placement included)
            "peak_bytes": peak_used,
            "peak_device_used_bytes": peak_device_used or None,
            "memory_budget": self.memory_budget,
        }
        return recs, summary
