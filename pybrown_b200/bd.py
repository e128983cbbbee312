"""The BD.py and BD-restart.py drivers (src/bdsim/BD.py, src/bdsim/BD-restart.py).

    python -m pybrown_b200.bd input.json [--batch]
    python -m pybrown_b200.bd --restart job.rst [-j patch.json]

Same JSON keywords, defaults, job loop over ``filename_range``, ``.xyz``,
``.enr`` and ``.rst`` output as the reference drivers, with ``Box`` from
``pybrown_b200.box`` (device-resident state).  The reference's
``measure_concentration`` / ``measure_flux`` outputs belong to subsystems
outside the accelerated path and raise ``NotImplementedError`` (as ``Box``
does for their keywords).

``--batch`` runs all jobs of a ``filename_range`` together as replicas of one
``ReplicaBatch`` (rpy / rpy_smith hydrodynamics, Ermak scheme, no bonds or
immobile beads, no restart output): every job keeps its own
``RandomState(seed)`` noise in the reference's order, so each job's
trajectory is the one it has when run alone.  Runs that batching does not
cover go through the sequential loop.
"""
import argparse
import pickle
import sys
import time
from contextlib import ExitStack

import numpy as np

from .io import (AsyncXYZWriter, InputData, read_str_file, timestamp, truncate_output_file_during_restart,
                 write_to_enr_file, write_to_restart_file)

REQUIRED_KEYWORDS = ["output_xyz_filename", "input_str_filename", "box_length", "T", "viscosity", "dt",
                     "number_of_steps"]

# BD.py:40-56
DEFAULTS = {"debug": False, "verbose": False, "hydrodynamics": "nohi",
            "ewald_alpha": float(np.sqrt(np.pi)), "ewald_real": 0, "ewald_imag": 0,
            "diff_freq": 1, "lub_freq": 1, "chol_freq": 1, "xyz_write_freq": 1,
            "lubrication_cutoff": 1, "progress_bar": False, "seed": None, "immobile_labels": [],
            "propagation_scheme": "ermak", "m_midpoint": 100, "divergence_term": False,
            "check_overlaps": True, "external_force": [0.0, 0.0, 0.0],
            "lennard_jones_6": False, "lennard_jones_12": False, "lennard_jones_alpha": 4.0,
            "energy_unit": "joule", "custom_interactions": False, "cichocki_correction": True,
            "overlap_treshold": 0.0, "max_move_attempts": 1000000}

ALL_KEYWORDS = REQUIRED_KEYWORDS + list(DEFAULTS) + [
    "output_rst_filename", "rst_write_freq", "output_enr_filename", "enr_write_freq", "filename_range",
    "custom_interactions_filename", "auxiliary_custom_interactions_keywords", "external_force_region",
    "measure_flux", "measure_concentration", "walls",
    # this implementation: arithmetic of the hot path ("fp64" or "mixed")
    "precision"]


def _names(template, inp):
    if "filename_range" in inp:
        return [template.format(j) for j in range(*inp["filename_range"])]
    return [template]


def _unsupported_outputs(inp):
    for key in ("measure_concentration", "measure_flux"):
        if key in inp:
            raise NotImplementedError("keyword {!r} is outside the accelerated hot path".format(key))


def batch_eligible(inp, beads_per_job):
    """True when the jobs can run as replicas of one ReplicaBatch."""
    if inp["hydrodynamics"] not in ("rpy", "rpy_smith") or inp["propagation_scheme"] != "ermak":
        return False
    if "rst_write_freq" in inp or inp.get("immobile_labels") or inp.get("divergence_term"):
        return False
    if inp.get("lennard_jones_6") or inp.get("lennard_jones_12") or inp.get("custom_interactions"):
        return False
    for beads in beads_per_job:
        if any(b.bonded_with or b.angled_with for b in beads):
            return False
    return True


def _forces(inp, N):
    from .box import eV_to_joule, kcal_per_mole_to_joule
    F = np.array(list(np.asarray(inp["external_force"], dtype=float)) * N)
    if inp["energy_unit"] == "kcal/mol":
        F = kcal_per_mole_to_joule(F)
    elif inp["energy_unit"] == "eV":
        F = eV_to_joule(F)
    return F


def run_sequential(inp, jobs):
    """BD.py:132-200: one Box per job, in order."""
    from .box import Box
    dt, n_steps = inp["dt"], inp["number_of_steps"]
    n_write, n_diff, n_lub, n_chol = inp["xyz_write_freq"], inp["diff_freq"], inp["lub_freq"], inp["chol_freq"]
    restart = "rst_write_freq" in inp
    energy = "enr_write_freq" in inp
    for index, job in enumerate(jobs):
        timestamp("{} job", job["str"])
        start = time.time()
        box = Box(read_str_file(job["str"]), inp)
        timestamp("Random seed: {}", box.seed)
        with ExitStack() as stack:
            xyz = stack.enter_context(open(job["xyz"], "w", buffering=1))
            enr = stack.enter_context(open(job["enr"], "w", buffering=1)) if energy else None
            _loop(box, inp, index, job, xyz, enr, 0, n_steps, dt, n_write, n_diff, n_lub, n_chol, restart, energy)
        print("{} seconds elapsed".format(time.time() - start))


def _loop(box, inp, index, job, xyz, enr, j0, n_steps, dt, n_write, n_diff, n_lub, n_chol, restart, energy):
    """BD.py:160-186.  The .xyz frames go through a writer thread (the loop
    hands over a copy of the positions); a restart file waits for the frames
    written so far, since it records the .xyz file's length."""
    extra = [job["enr"]] if energy else []
    with AsyncXYZWriter(xyz, job["xyz"], [b.label for b in box.beads]) as writer:
        for j in range(j0, n_steps):
            if inp["debug"]:
                print("STEP {}\n".format(j))
            if j % n_write == 0:
                writer.write(j, dt, box.positions())
            box.propagate(dt, j % n_diff == 0, j % n_lub == 0, j % n_chol == 0)
            if energy and j % inp["enr_write_freq"] == 0:
                write_to_enr_file(enr, j, dt, box.E, inp["energy_unit"])
            if restart and j != 0 and j % inp["rst_write_freq"] == 0:
                writer.flush()
                write_to_restart_file(job["rst"], index, j, box, job["xyz"], extra)


class _FrameBuffers:
    """Rings of pinned host buffers for the batched .xyz frames: a frame's
    positions are copied device-to-host asynchronously (on the batch's
    stream, so before the next step moves them) and the writer threads wait
    for an event recorded after the copies.  Each ring has depth + 2 buffers,
    so a buffer is reused only after its writer has formatted it (a writer
    holds at most depth pending frames and one being written)."""

    depth = 4

    def __init__(self, sizes):
        import torch
        self.torch = torch
        self.rings = [torch.empty((self.depth + 2, n, 3), dtype=torch.float64, pin_memory=True) for n in sizes]
        self.k = 0

    def capture(self, batch, slots):
        from . import _lib
        k = self.k % (self.depth + 2)
        self.k += 1
        bufs = []
        for ring, s in zip(self.rings, slots):
            buf = ring[k]
            _lib.call("pbg_batch_get_positions_async", batch._h, int(s), buf.data_ptr(), batch._stream)
            bufs.append(buf.numpy())
        ev = self.torch.cuda.Event()
        ev.record(self.torch.cuda.current_stream() if batch._stream is None else
                  self.torch.cuda.ExternalStream(batch._stream))
        return bufs, ev.synchronize


def run_batched(inp, jobs, beads_per_job):
    """All jobs as replicas of one ReplicaBatch; per-job RandomState(seed)."""
    from .batch import ReplicaBatch
    from .bead import build_connection_matrix, check_overlaps
    dt, n_steps = inp["dt"], inp["number_of_steps"]
    n_write, n_diff, n_chol = inp["xyz_write_freq"], inp["diff_freq"], inp["chol_freq"]
    energy = "enr_write_freq" in inp
    batch = ReplicaBatch(precision=inp.get("precision", "fp64"), hydrodynamics=inp["hydrodynamics"],
                         ewald_alpha=inp["ewald_alpha"], ewald_real=inp["ewald_real"],
                         ewald_imag=inp["ewald_imag"])
    slots = []
    for job, beads in zip(jobs, beads_per_job):
        if inp["check_overlaps"]:
            conn = build_connection_matrix(beads)
            assert not check_overlaps(beads, inp["box_length"], inp["overlap_treshold"], conn), \
                "starting configuration contains overlaps"
        seed = inp["seed"] if inp["seed"] is not None else np.random.randint(2 ** 32 - 1)
        timestamp("{} job, random seed: {}", job["str"], seed)
        F = _forces(inp, len(beads))
        s = batch.add(np.array([b.r for b in beads]), np.array([b.a for b in beads]), inp["box_length"],
                      T=inp["T"], viscosity=inp["viscosity"], seed=seed, noise="numpy",
                      check_overlaps=inp["check_overlaps"], overlap_treshold=inp["overlap_treshold"],
                      max_move_attempts=inp["max_move_attempts"], force=F if np.any(F != 0) else None)
        slots.append(s)
    start = time.time()
    frames = _FrameBuffers([len(beads) for beads in beads_per_job])
    with ExitStack() as stack:
        xyz = [stack.enter_context(open(job["xyz"], "w", buffering=1)) for job in jobs]
        enr = [stack.enter_context(open(job["enr"], "w", buffering=1)) for job in jobs] if energy else None
        writers = [stack.enter_context(AsyncXYZWriter(f, job["xyz"], [b.label for b in beads], frames.depth))
                   for f, job, beads in zip(xyz, jobs, beads_per_job)]
        for j in range(n_steps):
            if j % n_write == 0:
                # device-to-host copies into pinned buffers, ordered before the next step
                bufs, ready = frames.capture(batch, slots)
                for w, buf in zip(writers, bufs):
                    w.write(j, dt, buf, ready)
            batch.propagate(dt, build_D=j % n_diff == 0, cholesky=j % n_chol == 0)
            if energy and j % inp["enr_write_freq"] == 0:
                for f in enr:
                    write_to_enr_file(f, j, dt, 0.0, inp["energy_unit"])
    batch.close()
    print("{} seconds elapsed".format(time.time() - start))


def run(input_filename, batch=False):
    """BD.py main()."""
    timestamp("Reading input from {} file", input_filename)
    i = InputData(input_filename, REQUIRED_KEYWORDS, DEFAULTS, ALL_KEYWORDS)
    timestamp("Input data:\n{}", i)
    inp = i.input_data
    _unsupported_outputs(inp)
    jobs = [{"str": s, "xyz": x} for s, x in zip(_names(inp["input_str_filename"], inp),
                                                  _names(inp["output_xyz_filename"], inp))]
    if "rst_write_freq" in inp:
        for job, r in zip(jobs, _names(inp["output_rst_filename"], inp)):
            job["rst"] = r
    if "enr_write_freq" in inp:
        for job, e in zip(jobs, _names(inp["output_enr_filename"], inp)):
            job["enr"] = e
    if batch:
        beads_per_job = [read_str_file(job["str"]) for job in jobs]
        if batch_eligible(inp, beads_per_job):
            return run_batched(inp, jobs, beads_per_job)
        timestamp("--batch: this configuration runs job by job")
    return run_sequential(inp, jobs)


def restart(restart_filename, json_filename=None):
    """BD-restart.py main(): continue from a .rst file, optionally patching the input."""
    from .box import Box
    timestamp("Reading restart from {} file", restart_filename)
    patch = InputData(json_filename).input_data if json_filename is not None else {}
    with open(restart_filename, "rb") as f:
        index_rst = pickle.load(f)
        j_rst = pickle.load(f)
        box_rst = pickle.load(f)
        xyz_len = pickle.load(f)
        enr_len = pickle.load(f) if box_rst.is_energy else None
    inp = box_rst.inp
    for key, value in patch.items():
        if key in inp:
            timestamp("Keyword {} updated: from {} to {}", key, inp[key], value)
        else:
            timestamp("Keyword {} introduced: {}", key, value)
        inp[key] = value
    _unsupported_outputs(inp)
    jobs = [{"str": s, "xyz": x, "rst": r} for s, x, r in zip(_names(inp["input_str_filename"], inp),
                                                              _names(inp["output_xyz_filename"], inp),
                                                              _names(inp["output_rst_filename"], inp))]
    energy = box_rst.is_energy
    if energy:
        for job, e in zip(jobs, _names(inp["output_enr_filename"], inp)):
            job["enr"] = e
        truncate_output_file_during_restart(jobs[index_rst]["enr"], enr_len)
    truncate_output_file_during_restart(jobs[index_rst]["xyz"], xyz_len)
    dt, n_steps = inp["dt"], inp["number_of_steps"]
    n_write, n_diff, n_lub, n_chol = inp["xyz_write_freq"], inp["diff_freq"], inp["lub_freq"], inp["chol_freq"]
    for index in range(index_rst, len(jobs)):
        job = jobs[index]
        start = time.time()
        if index == index_rst:
            box, j0, mode = box_rst, j_rst + 1, "a"
        else:
            box, j0, mode = Box(read_str_file(job["str"]), inp), 0, "w"
        timestamp("Random seed: {}", box.seed)
        with ExitStack() as stack:
            xyz = stack.enter_context(open(job["xyz"], mode, buffering=1))
            enr = stack.enter_context(open(job["enr"], mode, buffering=1)) if energy else None
            _loop(box, inp, index, job, xyz, enr, j0, n_steps, dt, n_write, n_diff, n_lub, n_chol, True, energy)
        print("{} seconds elapsed".format(time.time() - start))


def main(argv=None):
    ap = argparse.ArgumentParser(description="Brownian dynamics on the GPU (pyBrown BD.py / BD-restart.py)")
    ap.add_argument("input_filename", nargs="?", help="JSON input (BD.py)")
    ap.add_argument("--batch", action="store_true", help="run the jobs of filename_range as one batch of replicas")
    ap.add_argument("--restart", metavar="RST", help="continue from a restart file (BD-restart.py)")
    ap.add_argument("-j", "--json-filename", help="input patch for --restart")
    a = ap.parse_args(argv)
    if a.restart:
        restart(a.restart, a.json_filename)
    elif a.input_filename:
        run(a.input_filename, batch=a.batch)
    else:
        ap.error("give an input file or --restart")


if __name__ == "__main__":
    sys.exit(main())
