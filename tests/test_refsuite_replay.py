"""The reference's own unit-test suites, replayed call by call.

tests/golden/make_golden_refsuite.py ran the reference's hot-path suites
(src/bdsim/tests/test_diffusion_vs_python.py, test_diffusion_vs_bdbox.py,
test_diffusion_vs_hydrolib.py, test_diffusion.py, test_box.py, test_bead.py)
unchanged against the reference's own C build and recorded the calls they
make into its seven exports (the first calls of each export in each test),
with the reference library's results.  The reference binds these exports with
``ctypes.cdll.LoadLibrary(find_library("pyBrown"))``
(src/bdsim/pyBrown/diffusion.py:24-26, bead.py:24-26); substituting
libpybrown_b200.so there means these exact calls reach it.  Here every recorded
call is made again, in order, on

  * the oracle (CPU; pins the restatement against the suites' calls), and
  * libpybrown_b200.so's exports of the same names (GPU),

and each result is compared with the reference library's: the pair-vector
matrices bit for bit, check_overlaps' flag exactly, the mobility matrices to
a relative 1e-10 (FP64), the lubrication corrections to 1e-10 of the larger of
their own size and the two-body resistance scale 6 pi a (the correction is a
difference of two such matrices).
"""
import ctypes
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_err

TOL = 1e-10
FIXTURE = os.path.join(GOLDEN, "refsuite_calls.npz")


@pytest.fixture(scope="module")
def recorded():
    z = np.load(FIXTURE)
    return json.loads(str(z["index"])), z


def _replay(fn, call, z):
    """Make one recorded call on `fn`; returns (result, output array)."""
    args, keep = [], []
    n = len(call["args"])
    for j, kind in enumerate(call["args"]):
        tag, value = kind
        if tag == "int":
            args.append(ctypes.c_int(value))
        elif tag == "double":
            args.append(ctypes.c_double(value))
        elif tag == "f64[]":
            is_out = call["fn"] != "check_overlaps" and j == n - 1
            a = np.zeros(value) if is_out else np.array(z[f"c{call['id']}_a{j}"], dtype=np.float64)
            keep.append(a)
            args.append(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        elif tag == "int32[]":
            a = np.ascontiguousarray(z[f"c{call['id']}_a{j}"], dtype=np.int32)
            keep.append(a)
            args.append(a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        else:
            raise AssertionError(f"unknown argument kind {kind}")
    result = fn(*args)
    return result, keep[-1]


def _check(lib, index, z):
    bad = []
    for i, call in enumerate(index["calls"]):
        call = dict(call, id=i)
        result, out = _replay(getattr(lib, call["fn"]), call, z)
        where = f"call {i} {call['fn']} from {call['test']}"
        if call["fn"] == "check_overlaps":
            if int(result) != call["result"]:
                bad.append(f"{where}: flag {int(result)} != {call['result']}")
        elif "out_sha256" in call:
            if hashlib.sha256(out.tobytes()).hexdigest() != call["out_sha256"]:
                bad.append(f"{where}: pair vectors differ from the reference's bits")
        elif call["fn"] == "JO_R_lubrication_correction_matrix":
            # R_JO - R_RPY of two-body resistance matrices whose entries are of
            # order 6 pi a: for far pairs (test_JO_R_3inline_3000: r = 3000 a)
            # the correction is ~1e-12 of that, rounding residue of the
            # subtraction, so its error is measured against the operands' scale
            ref = z[call["out"]]
            a_max = float(np.max(z[f"c{i}_a0"]))
            scale = max(float(np.max(np.abs(ref))), 6.0 * np.pi * a_max)
            err = float(np.max(np.abs(out - ref))) / scale if np.all(np.isfinite(ref)) else rel_err(out, ref)
            if not err <= TOL:
                bad.append(f"{where}: error {err:.3g} of the two-body scale")
        else:
            err = rel_err(out, z[call["out"]])
            if not err <= TOL:
                bad.append(f"{where}: relative error {err:.3g}")
    assert not bad, "\n".join(bad[:20])


def test_fixture_covers_the_suites(recorded):
    index, _ = recorded
    assert index["tests_run"] == 75 and index["failures"] == 0 and index["errors"] == 0
    fns = {c["fn"] for c in index["calls"]}
    assert fns == {"RPY_M_matrix", "RPY_Smith_M_matrix", "JO_2B_R_matrix",
                   "JO_R_lubrication_correction_matrix", "pointer_pbc_matrix",
                   "pointer_immobile_pbc_matrix", "check_overlaps"}
    suites = {t.split(".")[0] for t in index["tests_with_calls"]}
    assert suites == set(index["suites"])
    # both outcomes of the overlap test are exercised
    assert {c["result"] for c in index["calls"] if c["fn"] == "check_overlaps"} == {0, 1}


def test_oracle_replays_reference_suites(recorded):
    from oracle import oracle
    if not os.path.exists(oracle.ORACLE_LIB):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
    lib = ctypes.CDLL(oracle.ORACLE_LIB)
    lib.check_overlaps.restype = ctypes.c_int
    index, z = recorded
    _check(lib, index, z)


@pytest.mark.gpu
def test_gpu_library_replays_reference_suites(recorded):
    from pybrown_b200 import _lib
    index, z = recorded
    _check(_lib.lib, index, z)
