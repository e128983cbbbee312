"""Record the reference's own unit-test suites' calls into its C library.

Run in a container that has the reference tree and the reference's C library
compiled by oracle/Makefile (oracle/_ref/libpyBrown.so):

    make -C oracle ref && python tests/golden/make_golden_refsuite.py

The reference's hot-path suites (src/bdsim/tests/test_diffusion_vs_python.py,
test_diffusion_vs_bdbox.py, test_diffusion_vs_hydrolib.py, test_diffusion.py,
test_box.py, test_bead.py) reach the native code only through the seven
exports that src/bdsim/pyBrown/diffusion.py:24-175 and bead.py:24-443 bind
with ctypes.  This script runs those suites unchanged with the library
redirected to the reference's own C build and wraps every export so that each
call's arguments and result are recorded:

  refsuite_calls.npz -- for each recorded call: the export's name, the test
                        that made it, its scalar arguments, its input arrays
                        and the reference library's output (the matrix it
                        filled, the SHA-256 of the pair-vector matrices, whose
                        bar is bit-exact, or check_overlaps' return value);
                        plus the suites' own outcome with the reference
                        library.

The GPU box has no reference tree, so the suites cannot run there; the replay
test (tests/test_refsuite_replay.py) feeds the same calls, in the same order
and with the same arguments, to libpybrown_b200.so's exports of the same
names and compares each result with the reference library's.

The suites' long simulations (test_box) make thousands of calls with the same
shapes; the first CAP_MATRIX calls of each export in each test are kept (all
distinct configurations appear there), and the first CAP_OVERLAP calls of
check_overlaps in test_bead, whose random configurations are small.
"""
import ctypes
import ctypes.util
import hashlib
import json
import os
import sys
import tempfile
import unittest

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# root of the reference checkout; PYBROWN_REFERENCE overrides the default
REFERENCE_BDSIM = os.path.join(os.environ.get("PYBROWN_REFERENCE", "/root/reference"), "src", "bdsim")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libpyBrown.so")
OUT = os.path.join(HERE, "refsuite_calls.npz")

SUITES = [
    "test_diffusion_vs_python",
    "test_diffusion_vs_bdbox",
    "test_diffusion_vs_hydrolib",
    "test_diffusion",
    "test_box",
    "test_bead",
]
EXPORTS = ("RPY_M_matrix", "RPY_Smith_M_matrix", "JO_2B_R_matrix",
           "JO_R_lubrication_correction_matrix", "pointer_pbc_matrix",
           "pointer_immobile_pbc_matrix", "check_overlaps")
BIT_EXACT = ("pointer_pbc_matrix", "pointer_immobile_pbc_matrix")
CAP_MATRIX = 3
CAP_OVERLAP = 150


class Recorder:
    def __init__(self):
        self.test = None
        self.calls = []          # index entries (json)
        self.arrays = {}         # npz payload
        self.seen = {}

    def keep(self, fn):
        key = (self.test, fn)
        self.seen[key] = self.seen.get(key, 0) + 1
        random_overlaps = fn == "check_overlaps" and self.test.startswith("test_bead.")
        cap = CAP_OVERLAP if random_overlaps else CAP_MATRIX
        return self.seen[key] <= cap

    def record(self, fn, args, result):
        i = len(self.calls)
        kinds = []
        for j, a in enumerate(args):
            if isinstance(a, ctypes.Array):
                self.arrays[f"c{i}_a{j}"] = np.frombuffer(a, dtype=np.float64).copy()
                kinds.append(["f64[]", len(a)])
            elif isinstance(a, np.ndarray):
                self.arrays[f"c{i}_a{j}"] = np.ascontiguousarray(a).copy()
                kinds.append([f"{a.dtype.name}[]", a.size])
            elif isinstance(a, ctypes.c_int):
                kinds.append(["int", a.value])
            elif isinstance(a, ctypes.c_double):
                kinds.append(["double", a.value])
            else:
                raise TypeError(f"{fn}: unexpected argument {type(a)}")
        entry = {"fn": fn, "test": self.test, "args": kinds}
        out = f"c{i}_a{len(args) - 1}"
        if fn == "check_overlaps":
            entry["result"] = int(result)
        elif fn in BIT_EXACT:
            # the pair vectors are compared bit for bit: their digest stands for them
            entry["out_sha256"] = hashlib.sha256(self.arrays.pop(out).tobytes()).hexdigest()
        else:
            # every other export fills its last argument
            entry["out"] = out
        self.calls.append(entry)


REC = Recorder()


class _Export:
    def __init__(self, name, fn):
        object.__setattr__(self, "_name", name)
        object.__setattr__(self, "_fn", fn)

    def __setattr__(self, key, value):       # argtypes / restype set by bead.py:422
        setattr(self._fn, key, value)

    def __call__(self, *args):
        if not REC.keep(self._name):
            return self._fn(*args)
        before = [np.frombuffer(a, dtype=np.float64).copy() if isinstance(a, ctypes.Array) else None
                  for a in args]
        result = self._fn(*args)
        n_in = len(args) if self._name == "check_overlaps" else len(args) - 1
        for j in range(n_in):
            if before[j] is not None:      # the inputs are recorded after the call: unchanged by it
                assert np.array_equal(before[j], np.frombuffer(args[j], dtype=np.float64))
        REC.record(self._name, args, result)
        return result


class _Library:
    def __init__(self, lib):
        self._lib = lib

    def __getattr__(self, name):
        fn = getattr(self._lib, name)
        wrapped = _Export(name, fn) if name in EXPORTS else fn
        setattr(self, name, wrapped)
        return wrapped


class _Result(unittest.TextTestResult):
    def startTest(self, test):
        REC.test = test.id()
        super().startTest(test)


def main():
    if not os.path.exists(REF_LIB):
        raise SystemExit(f"{REF_LIB} missing: run `make -C oracle ref` first")
    real_find = ctypes.util.find_library
    ctypes.util.find_library = lambda name: REF_LIB if name == "pyBrown" else real_find(name)
    real_load = ctypes.cdll.LoadLibrary
    ctypes.cdll.LoadLibrary = lambda path: _Library(real_load(path)) if path == REF_LIB else real_load(path)
    sys.path.insert(0, os.path.join(REFERENCE_BDSIM, "tests"))
    sys.path.insert(0, REFERENCE_BDSIM)

    loader = unittest.TestLoader()
    suite = unittest.TestSuite(loader.loadTestsFromName(s) for s in SUITES)
    cwd = os.getcwd()
    os.chdir(tempfile.mkdtemp(prefix="pybrown_refsuite_"))  # test_box writes scratch files
    try:
        np.random.seed(0)
        result = unittest.TextTestRunner(verbosity=1, resultclass=_Result).run(suite)
    finally:
        os.chdir(cwd)
    tests = sorted({c["test"] for c in REC.calls})
    index = {
        "suites": SUITES,
        "tests_run": result.testsRun,
        "failures": len(result.failures),
        "errors": len(result.errors),
        "cap_matrix": CAP_MATRIX,
        "cap_overlap": CAP_OVERLAP,
        "calls_seen": {f"{t}::{fn}": n for (t, fn), n in REC.seen.items()},
        "tests_with_calls": tests,
        "calls": REC.calls,
    }
    np.savez_compressed(OUT, index=np.array(json.dumps(index)), **REC.arrays)
    print(f"{len(REC.calls)} calls from {len(tests)} tests; suites: ran {result.testsRun}, "
          f"failures {len(result.failures)}, errors {len(result.errors)}; "
          f"{os.path.getsize(OUT) / 1e6:.2f} MB -> {OUT}")
    return 0 if result.wasSuccessful() else 1


if __name__ == "__main__":
    sys.exit(main())
