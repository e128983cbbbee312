"""The FP32 Ewald path's erfc (csrc/ewald.cu, erfc_as): Abramowitz & Stegun,
Handbook of Mathematical Functions, 7.1.26, |error| < 1.5e-7 for x >= 0.

Host-only: the constants are read from the kernel source and the formula is
evaluated in FP64 against math.erfc, so a mistyped constant shows here; the
device path itself is bounded by test_gpu_tensors.py (the FP32 Smith-Ewald
tensor within 2e-6 of the FP64 oracle)."""
import math
import os
import re

import numpy as np

from conftest import ROOT


def _constants():
    src = open(os.path.join(ROOT, "pybrown_b200", "csrc", "ewald.cu")).read()
    body = src[src.index("__device__ __forceinline__ float erfc_as("):]
    body = body[:body.index("\n}\n")]
    nums = [float(v) for v in re.findall(r"(-?\d+\.\d+)f", body)]
    # 1 / (p x + 1), then a5, a4, a3, a2, a1 in Horner order (signs included)
    assert len(nums) == 8 and nums[0] == 1.0 and nums[2] == 1.0
    return nums[1], nums[3], nums[4:]


def test_abramowitz_stegun_erfc_bound():
    p, a5, rest = _constants()
    a4, a3, a2, a1 = rest
    xs = np.linspace(0.0, 6.0, 20001)
    t = 1.0 / (1.0 + p * xs)
    poly = ((((a5 * t + a4) * t + a3) * t + a2) * t + a1) * t
    approx = poly * np.exp(-xs * xs)
    exact = np.array([math.erfc(x) for x in xs])
    assert np.max(np.abs(approx - exact)) < 1.5e-7
