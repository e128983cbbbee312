"""The BD.py / BD-restart.py drivers (pybrown_b200.bd) on the GPU: a
filename_range job loop against the oracle, the batched job loop against the
sequential one, and a restart that resumes the .xyz trajectory bit for bit."""
import json
import math
import os
import shutil

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def _beads(seed, N, L):
    from pybrown_b200.bead import Bead
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < N:
        a = rng.uniform(1.0, 2.0)
        p = rng.uniform(-L / 2, L / 2, size=3)
        if all(np.linalg.norm((p - b.r) - L * np.round((p - b.r) / L)) > a + b.a for b in out):
            out.append(Bead(p, a, label="B", hard_core_radius=a, bead_id=len(out) + 1))
    return out


def _setup(tmp_path, jobs=3, **extra):
    from pybrown_b200.io import write_str_file
    L = 30.0
    for j in range(jobs):
        write_str_file(str(tmp_path / f"in{j}.str"), _beads(10 + j, 8 + 3 * j, L))
    inp = {"input_str_filename": str(tmp_path / "in{}.str"), "output_xyz_filename": str(tmp_path / "out{}.xyz"),
           "filename_range": [0, jobs], "box_length": L, "T": 298.0, "viscosity": 0.01, "dt": 0.002,
           "number_of_steps": 6, "xyz_write_freq": 2, "hydrodynamics": "rpy_smith",
           "ewald_alpha": math.sqrt(math.pi), "ewald_real": 2, "ewald_imag": 2, "seed": 3}
    inp.update(extra)
    path = tmp_path / "input.json"
    path.write_text(json.dumps(inp))
    return str(path), inp


def _frames(path):
    lines = open(path).read().splitlines()
    frames, k = [], 0
    while k < len(lines):
        n = int(lines[k])
        frames.append(np.array([[float(v) for v in ln.split()[1:4]] for ln in lines[k + 2:k + 2 + n]]))
        k += 2 + n
    return frames


def test_job_loop_matches_the_oracle(tmp_path, oracle_lib):
    from oracle.oracle import OracleBox
    from pybrown_b200 import bd
    from pybrown_b200.io import read_str_file
    path, inp = _setup(tmp_path)
    bd.run(path)
    full = dict(bd.DEFAULTS)
    full.update(inp)
    for j in range(3):
        beads = read_str_file(str(tmp_path / f"in{j}.str"))
        init = np.array([b.r for b in beads])
        box = OracleBox(init, [b.a for b in beads], full, clib=oracle_lib)
        frames = _frames(str(tmp_path / f"out{j}.xyz"))
        assert len(frames) == 3
        for step in range(6):
            if step % 2 == 0:
                assert rel_err(frames[step // 2] - init, box.pos - init) <= 1e-10 or step == 0
            box.propagate(inp["dt"])


def test_batched_job_loop_equals_the_sequential_one(tmp_path):
    from pybrown_b200 import bd
    path, _ = _setup(tmp_path)
    bd.run(path)
    seq = [_frames(str(tmp_path / f"out{j}.xyz")) for j in range(3)]
    for j in range(3):
        os.remove(str(tmp_path / f"out{j}.xyz"))
    bd.run(path, batch=True)
    for j in range(3):
        got = _frames(str(tmp_path / f"out{j}.xyz"))
        assert len(got) == len(seq[j])
        for a, b in zip(got, seq[j]):
            assert np.array_equal(a, b), j


def test_restart_resumes_bit_for_bit(tmp_path):
    from pybrown_b200 import bd
    path, _ = _setup(tmp_path, jobs=1, filename_range=[0, 1], number_of_steps=11, xyz_write_freq=1,
                     rst_write_freq=4, output_rst_filename=str(tmp_path / "out{}.rst"))
    bd.run(path)
    xyz = str(tmp_path / "out0.xyz")
    full = open(xyz).read()
    shutil.copy(xyz, xyz + ".full")
    # the last restart point is step 8; resuming rewrites the frames of steps 9 and 10
    bd.restart(str(tmp_path / "out0.rst"))
    assert open(xyz).read() == full
