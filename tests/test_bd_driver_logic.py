"""Host logic of the BD.py driver (pybrown_b200.bd): keyword defaults and
validation, filename_range expansion, which runs can be batched.  No GPU."""
import json

import numpy as np
import pytest

from pybrown_b200 import bd
from pybrown_b200.bead import Bead
from pybrown_b200.io import InputData


def _inp(tmp_path, **kw):
    d = {"input_str_filename": "in{}.str", "output_xyz_filename": "out{}.xyz", "box_length": 10.0, "T": 298.0,
         "viscosity": 0.01, "dt": 0.1, "number_of_steps": 3}
    d.update(kw)
    p = tmp_path / "i.json"
    p.write_text(json.dumps(d))
    return InputData(str(p), bd.REQUIRED_KEYWORDS, bd.DEFAULTS, bd.ALL_KEYWORDS).input_data


def test_defaults_and_filename_range(tmp_path):
    inp = _inp(tmp_path, filename_range=[2, 5])
    assert inp["hydrodynamics"] == "nohi" and inp["diff_freq"] == 1 and inp["seed"] is None
    assert bd._names(inp["input_str_filename"], inp) == ["in2.str", "in3.str", "in4.str"]


def test_unknown_and_missing_keywords(tmp_path):
    with pytest.raises(AssertionError):
        _inp(tmp_path, not_a_keyword=1)
    p = tmp_path / "j.json"
    p.write_text(json.dumps({"box_length": 1.0}))
    with pytest.raises(AssertionError):
        InputData(str(p), bd.REQUIRED_KEYWORDS, bd.DEFAULTS, bd.ALL_KEYWORDS)


def test_batch_eligibility(tmp_path):
    beads = [[Bead(np.zeros(3), 1.0), Bead(np.ones(3), 1.0)]]
    assert bd.batch_eligible(_inp(tmp_path, hydrodynamics="rpy_smith"), beads)
    assert not bd.batch_eligible(_inp(tmp_path, hydrodynamics="rpy_smith_lub"), beads)
    assert not bd.batch_eligible(_inp(tmp_path, hydrodynamics="rpy", propagation_scheme="midpoint"), beads)
    assert not bd.batch_eligible(_inp(tmp_path, hydrodynamics="rpy", rst_write_freq=2,
                                      output_rst_filename="r"), beads)
    bonded = [[Bead(np.zeros(3), 1.0, bead_id=1), Bead(np.ones(3), 1.0, bead_id=2)]]
    bonded[0][0].bonded_with.append(2)
    assert not bd.batch_eligible(_inp(tmp_path, hydrodynamics="rpy"), bonded)


def test_out_of_scope_outputs_raise(tmp_path):
    with pytest.raises(NotImplementedError):
        bd._unsupported_outputs(_inp(tmp_path, measure_flux={"output_flux_filename": "f"}))
