"""Run the reference's own unittest suites against a chosen shared library.

Test infrastructure only.  This is how the in-house oracle
(oracle/pybrown_oracle.c) is pinned: the reference's hot-path suites
(src/bdsim/tests/test_diffusion_vs_python.py, test_diffusion_vs_bdbox.py,
test_diffusion_vs_hydrolib.py, test_diffusion.py, test_box.py, test_bead.py)
load their native library with ``ctypes.cdll.LoadLibrary(find_library("pyBrown"))``
(src/bdsim/pyBrown/diffusion.py:24-26, bead.py:24-26).  Here
``ctypes.util.find_library`` is redirected to the library under test, so every
known-answer value those suites hold (HYDROLIB and BD_BOX golden numbers, the
pure-Python restatement, the seeded trajectories) is checked against it.

It reads the reference tree in place and only runs in a container that has it.

    python oracle/run_reference_suite.py --lib oracle/_build/libpybrown_oracle.so
    python oracle/run_reference_suite.py --lib oracle/_ref/libpyBrown.so
"""
import argparse
import ctypes.util
import os
import sys
import tempfile
import unittest

# root of the reference checkout; PYBROWN_REFERENCE overrides the default
REFERENCE_BDSIM = os.path.join(os.environ.get("PYBROWN_REFERENCE", "/root/reference"), "src", "bdsim")

HOT_PATH_SUITES = [
    "test_diffusion_vs_python",
    "test_diffusion_vs_bdbox",
    "test_diffusion_vs_hydrolib",
    "test_diffusion",
    "test_box",
    "test_bead",
]


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--lib", required=True, help="shared library exporting the pyBrown C ABI")
    ap.add_argument("--suite", action="append", help="run only these suites (module names)")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)

    lib = os.path.abspath(args.lib)
    if not os.path.exists(lib):
        raise SystemExit(f"library not found: {lib}")
    if not os.path.isdir(REFERENCE_BDSIM):
        raise SystemExit(f"reference tree not present at {REFERENCE_BDSIM}")

    real_find = ctypes.util.find_library
    ctypes.util.find_library = lambda name: lib if name == "pyBrown" else real_find(name)

    sys.path.insert(0, os.path.join(REFERENCE_BDSIM, "tests"))
    sys.path.insert(0, REFERENCE_BDSIM)

    suites = args.suite or HOT_PATH_SUITES
    loader = unittest.TestLoader()
    tests = unittest.TestSuite(loader.loadTestsFromName(s) for s in suites)
    workdir = tempfile.mkdtemp(prefix="pybrown_refsuite_")
    cwd = os.getcwd()
    os.chdir(workdir)  # test_box writes scratch files into the working directory
    try:
        result = unittest.TextTestRunner(verbosity=2 if args.verbose else 1).run(tests)
    finally:
        os.chdir(cwd)
    print(f"library under test: {lib}")
    print(f"ran {result.testsRun}, failures {len(result.failures)}, errors {len(result.errors)}")
    return 0 if result.wasSuccessful() else 1


if __name__ == "__main__":
    sys.exit(main())
