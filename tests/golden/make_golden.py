"""Generate the golden fixtures of the parity tests from the reference itself.

Run in a container that has the reference tree and the reference's C library
compiled by oracle/Makefile (oracle/_ref/libpyBrown.so):

    make -C oracle ref && python tests/golden/make_golden.py

It imports the reference's Python package (src/bdsim/pyBrown) with its
ctypes library redirected to oracle/_ref/libpyBrown.so, evaluates the
hot-path functions on seeded inputs and writes:

  tensors.npz        -- pair vectors, free-space RPY, Smith-Ewald RPY,
                        Jeffrey-Onishi two-body R, lubrication corrections,
                        overlap flags (inputs and outputs)
  trajectories.npz   -- Box.propagate trajectories (positions after each
                        step, RNG draw counts) for Ermak (nohi, rpy,
                        rpy_smith, with overlap rejections) and midpoint
                        (rpy_smith_lub) runs
  known_answers.json -- the HYDROLIB / BD_BOX golden numbers held in the
                        reference's test files, read as text

The GPU box has none of the reference: the tests only read these files.
"""
import ast
import ctypes.util
import json
import math
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# root of the reference checkout; PYBROWN_REFERENCE overrides the default
REFERENCE_BDSIM = os.path.join(os.environ.get("PYBROWN_REFERENCE", "/root/reference"), "src", "bdsim")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libpyBrown.so")


def _import_reference():
    if not os.path.exists(REF_LIB):
        raise SystemExit(f"{REF_LIB} missing: run `make -C oracle ref` first")
    real = ctypes.util.find_library
    ctypes.util.find_library = lambda name: REF_LIB if name == "pyBrown" else real(name)
    sys.path.insert(0, REFERENCE_BDSIM)
    from pyBrown import bead, box, diffusion  # noqa: E402
    return bead, box, diffusion


def mock_input(**kw):
    """Keyword set of the reference's Box tests (src/bdsim/tests/test_box.py:39-46)."""
    d = {"hydrodynamics": "nohi", "box_length": 35.0, "T": 298.0, "viscosity": 0.01,
         "external_force": [0, 0, 0], "immobile_labels": [], "propagation_scheme": "ermak",
         "check_overlaps": True, "lennard_jones_6": False, "lennard_jones_12": False,
         "energy_unit": "joule", "custom_interactions": False, "debug": False, "verbose": False,
         "overlap_treshold": 0.0, "max_move_attempts": 1000000, "cichocki_correction": True,
         "divergence_term": False, "seed": 0, "ewald_alpha": math.sqrt(math.pi),
         "ewald_real": 0, "ewald_imag": 0, "lubrication_cutoff": 1, "m_midpoint": 100}
    d.update(kw)
    return d


def tensor_cases(bead, diffusion):
    Bead = bead.Bead
    out = {}
    rng = np.random.default_rng(20240611)

    def beads_of(pos, radii):
        return [Bead(np.array(p, float), float(a)) for p, a in zip(pos, radii)]

    cases = []
    grid = [[x, y, z] for x in (-3.0, 0.0, 3.0) for y in (-3.0, 0.0, 3.0) for z in (-3.0, 0.0, 3.0)]
    cases.append(("grid27", np.array(grid), np.ones(27), 20.0))
    pos = rng.uniform(-15, 15, size=(20, 3))
    pos[1] = pos[0] + np.array([1.2, 0.3, -0.2])   # overlapping pair (intermediate regime)
    pos[3] = pos[2] + np.array([0.05, 0.0, 0.02])  # a small bead inside a big one
    radii = rng.uniform(0.5, 1.5, size=20)
    radii[2], radii[3] = 1.5, 0.4
    cases.append(("poly20", pos, radii, 30.0))
    pos = rng.uniform(-25, 25, size=(33, 3))
    cases.append(("rand33", pos, rng.uniform(0.8, 1.2, size=33), 50.0))
    for name, pos, radii, L in cases:
        b = beads_of(pos, radii)
        rij = bead.compute_pointer_pbc_matrix(b, L)
        out[f"{name}/pos"] = pos
        out[f"{name}/radii"] = radii
        out[f"{name}/L"] = np.array(L)
        out[f"{name}/rij"] = rij
        out[f"{name}/rpy"] = diffusion.RPY_M_matrix(b, rij)
        for (m, n) in ((0, 0), (1, 1), (2, 4), (3, 3)):
            out[f"{name}/smith_m{m}_n{n}"] = diffusion.RPY_Smith_M_matrix(b, rij, L, math.sqrt(math.pi), m, n)
        out[f"{name}/smith_alpha2_m2_n2"] = diffusion.RPY_Smith_M_matrix(b, rij, L, 2.0, 2, 2)
        for cutoff in (1.0, 10.0):
            for cich in (True, False):
                out[f"{name}/lub_c{cutoff:g}_{int(cich)}"] = diffusion.JO_R_lubrication_correction_matrix(
                    b, rij, cutoff, cich)
    # two-body JO resistance
    jo_in, jo_out = [], []
    for s in (2.001, 2.01, 2.1, 2.5, 3.0, 4.0, 6.0):
        for ai, aj in ((1.0, 1.0), (1.0, 0.5), (0.5, 1.0), (2.0, 0.7)):
            d = s * (ai + aj) / 2
            direction = rng.normal(size=3)
            direction /= np.linalg.norm(direction)
            bi, bj = Bead(np.zeros(3), ai), Bead(d * direction, aj)
            jo_in.append([ai, aj, *(d * direction)])
            jo_out.append(diffusion.JO_2B_R_matrix(bi, bj))
    out["jo2b/in"] = np.array(jo_in)
    out["jo2b/out"] = np.array(jo_out)
    # minimum image at and near the +-L/2 ties
    L = 10.0
    pos = np.array([[0.0, 0.0, 0.0], [5.0, -5.0, 4.999999], [-5.0, 5.0, -4.9999999],
                    [4.5, 0.5, -0.5], [-4.99, 2.5, 7.5]])
    b = beads_of(pos, np.ones(len(pos)))
    out["pbc/pos"] = pos
    out["pbc/L"] = np.array(L)
    out["pbc/rij"] = bead.compute_pointer_pbc_matrix(b, L)
    # overlap flags, including the axis pre-filter with a positive threshold
    ov_pos, ov_rad, ov_thr, ov_flag = [], [], [], []
    for k in range(40):
        n = 12
        p = rng.uniform(-6, 6, size=(n, 3))
        r = rng.uniform(0.4, 1.0, size=n)
        thr = [0.0, 0.3][k % 2]
        bb = beads_of(p, r)
        conn = np.zeros((n, n), dtype=np.int32)
        ov_pos.append(p)
        ov_rad.append(r)
        ov_thr.append(thr)
        ov_flag.append(bead.check_overlaps(bb, 12.0, thr, conn))
    out["overlap/pos"] = np.array(ov_pos)
    out["overlap/radii"] = np.array(ov_rad)
    out["overlap/thr"] = np.array(ov_thr)
    out["overlap/flag"] = np.array(ov_flag, dtype=np.int32)
    out["overlap/L"] = np.array(12.0)
    return out


def trajectory_cases(bead, box):
    Bead = bead.Bead
    out = {}
    grid3 = [[x, y, z] for x in (-3.0, 0.0, 3.0) for y in (-3.0, 0.0, 3.0) for z in (-3.0, 0.0, 3.0)]
    grid22 = [[x, y, z] for x in (-2.2, 0.0, 2.2) for y in (-2.2, 0.0, 2.2) for z in (-2.2, 0.0, 2.2)]
    runs = [
        ("ermak_nohi", grid3, 1.0, mock_input(hydrodynamics="nohi"), 1e-3, 20),
        ("ermak_rpy", grid3, 1.0, mock_input(hydrodynamics="rpy"), 1e-3, 20),
        ("ermak_smith", grid3, 1.0, mock_input(hydrodynamics="rpy_smith", ewald_real=2, ewald_imag=2), 1e-3, 20),
        ("ermak_smith_force", grid3, 1.0,
         mock_input(hydrodynamics="rpy_smith", ewald_real=1, ewald_imag=2, external_force=[2e-21, 0.0, -4e-21]),
         1e-3, 10),
        # close packing and a long step: many overlap rejections
        ("ermak_rpy_reject", [[0.0, 0.0, 0.0], [2.05, 0.0, 0.0], [0.0, 2.05, 0.0], [-2.05, 0.0, 0.0]], 1.0,
         mock_input(hydrodynamics="rpy", box_length=12.0, max_move_attempts=10000), 2e-3, 12),
        ("midpoint_smith_lub", grid22, 1.0,
         mock_input(hydrodynamics="rpy_smith_lub", propagation_scheme="midpoint", lubrication_cutoff=10,
                    ewald_real=1, ewald_imag=1, m_midpoint=10.0), 1e-3, 10),
        ("midpoint_lub_reject", [[0.0, 0.0, 0.0], [2.03, 0.0, 0.0], [0.0, 2.03, 0.0], [-2.03, 0.0, 0.0]], 1.0,
         mock_input(hydrodynamics="rpy_lub", propagation_scheme="midpoint", lubrication_cutoff=1.0,
                    box_length=12.0, m_midpoint=2.0, max_move_attempts=10000), 0.2, 8),
    ]
    for name, coords, a, inp, dt, steps in runs:
        beads = [Bead(np.array(c, float), a) for c in coords]
        b = box.Box(beads, dict(inp))
        traj, draws = [], []
        for _ in range(steps):
            b.propagate(dt)
            traj.append(np.array([bb.r for bb in b.beads]))
            draws.append(b.draw_count)
        out[f"{name}/init"] = np.array(coords, float)
        out[f"{name}/radius"] = np.array(a)
        out[f"{name}/dt"] = np.array(dt)
        out[f"{name}/traj"] = np.array(traj)
        out[f"{name}/draws"] = np.array(draws)
        out[f"{name}/config"] = np.array(json.dumps(inp))
    return out


def _assigned_arrays(src, var):
    """Value of `var = np.array(...)` / float literal assignments in a test file."""
    vals = []
    tree = ast.parse(src)
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef):
            for st in node.body:
                if isinstance(st, ast.Assign) and len(st.targets) == 1 and isinstance(st.targets[0], ast.Name):
                    if re.fullmatch(var, st.targets[0].id):
                        try:
                            if isinstance(st.value, ast.Call) and getattr(st.value.func, "attr", "") == "array":
                                vals.append((node.name, st.targets[0].id, ast.literal_eval(st.value.args[0])))
                            else:
                                vals.append((node.name, st.targets[0].id, ast.literal_eval(st.value)))
                        except ValueError:
                            pass
    return vals


def known_answers():
    """Golden numbers of the HYDROLIB / BD_BOX comparisons, read as text."""
    tests = os.path.join(REFERENCE_BDSIM, "tests")
    ka = {"hydrolib_2body": {}, "bdbox": []}
    with open(os.path.join(tests, "test_diffusion_vs_hydrolib.py")) as f:
        src = f.read()
    m = re.search(r"self\.R_hydrolib_infty\s*=\s*([0-9.eE+-]+)", src)
    ka["hydrolib_R_infty"] = float(m.group(1))
    for fn, var, val in _assigned_arrays(src, r"R_hydrolib_\d[_\d]*"):
        sep = var.replace("R_hydrolib_", "").replace("_", ".")
        ka["hydrolib_2body"][sep] = {"test": fn, "R": val}
    with open(os.path.join(tests, "test_diffusion_vs_bdbox.py")) as f:
        src = f.read()
    tree = ast.parse(src)
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name.startswith("test_"):
            vals = {}
            for st in node.body:
                if isinstance(st, ast.Assign) and isinstance(st.targets[0], ast.Name):
                    try:
                        vals[st.targets[0].id] = ast.literal_eval(st.value)
                    except ValueError:
                        pass
            beads = re.findall(r"Bead\(\[([^\]]*)\],\s*([0-9.]+)\)", ast.get_source_segment(src, node))
            vals["beads"] = [[[float(x) for x in c.split(",")], float(a)] for c, a in beads]
            vals["test"] = node.name
            ka["bdbox"].append(vals)
    return ka


def main():
    bead, box, diffusion = _import_reference()
    t = tensor_cases(bead, diffusion)
    np.savez_compressed(os.path.join(HERE, "tensors.npz"), **t)
    tr = trajectory_cases(bead, box)
    np.savez_compressed(os.path.join(HERE, "trajectories.npz"), **tr)
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(known_answers(), f, indent=1)
    for name in ("tensors.npz", "trajectories.npz", "known_answers.json"):
        print(name, os.path.getsize(os.path.join(HERE, name)), "bytes")


if __name__ == "__main__":
    main()
