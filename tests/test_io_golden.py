"""File formats against the reference's own input/output code (CPU).

tests/golden/io.json holds what the reference's `read_str_file`,
`write_to_xyz_file`, `write_to_enr_file`, `truncate_output_file_during_restart`
and `InputData` produced (tests/golden/make_golden_io.py); the same inputs go
through pybrown_b200.io here and must give the same fields and the same bytes.
"""
import json
import os

import pytest

from pybrown_b200 import io

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "io.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _beads(golden, tmp_path):
    p = tmp_path / "s.str"
    p.write_text(golden["str_text"])
    return io.read_str_file(str(p))


def test_read_str_file_fields(golden, tmp_path):
    beads = _beads(golden, tmp_path)
    assert len(beads) == len(golden["beads"])
    for b, g in zip(beads, golden["beads"]):
        assert b.label == g["label"] and b.bead_id == g["bead_id"]
        assert [float(x) for x in b.r] == g["r"] and b.a == g["a"]
        assert b.hard_core_radius == g["hard_core_radius"] and b.epsilon_LJ == g["epsilon_LJ"]
        assert list(b.bonded_with) == g["bonded_with"]
        assert {str(k): v for k, v in b.bonded_how.items()} == g["bonded_how"]
        assert [list(x) for x in b.angled_with] == g["angled_with"]
        assert {"{},{}".format(*k): v for k, v in b.angled_how.items()} == g["angled_how"]


def test_xyz_enr_and_truncation_bytes(golden, tmp_path):
    beads = _beads(golden, tmp_path)
    xyz = tmp_path / "t.xyz"
    with open(xyz, "w") as f:
        io.write_to_xyz_file(f, "t.xyz", 0, 0.5, beads)
        beads[0].r[0] += 0.125
        io.write_to_xyz_file(f, "t.xyz", 1, 0.5, beads)
    assert xyz.read_text() == golden["xyz_text"]
    enr = tmp_path / "e.enr"
    with open(enr, "w") as f:
        io.write_to_enr_file(f, 0, 0.5, 1.5e-20, "joule")
        io.write_to_enr_file(f, 1, 0.5, -2.25e-21, "joule")
    assert enr.read_text() == golden["enr_text"]
    io.truncate_output_file_during_restart(str(xyz), 3)
    assert xyz.read_text() == golden["truncated_xyz_text"]


def test_input_data_defaults(golden, tmp_path):
    cfg = tmp_path / "c.json"
    cfg.write_text(json.dumps(golden["config"]))
    inp = io.InputData(str(cfg), golden["required"], golden["defaults"], golden["all_keywords"])
    assert inp.input_data == golden["input_data"]


def test_async_xyz_writer_bytes(golden, tmp_path):
    """The writer thread gives the reference's bytes: frames handed over as
    position copies (the caller goes on changing its array) and frames whose
    buffer is filled later, behind a ready() wait."""
    import threading

    import numpy as np
    beads = _beads(golden, tmp_path)
    labels = [b.label for b in beads]
    pos = np.array([b.r for b in beads])
    xyz = tmp_path / "a.xyz"
    with open(xyz, "w") as f, io.AsyncXYZWriter(f, "t.xyz", labels, depth=1) as w:
        w.write(0, 0.5, pos)
        pos[0, 0] += 0.125  # after the hand-over: frame 0 keeps the old value
        w.write(1, 0.5, pos)
    assert xyz.read_text() == golden["xyz_text"]
    # a frame filled after its hand-over (an asynchronous copy in the drivers)
    buf = np.zeros_like(pos)
    gate = threading.Event()
    xyz2 = tmp_path / "b.xyz"
    with open(xyz2, "w") as f, io.AsyncXYZWriter(f, "t.xyz", labels) as w:
        w.write(0, 0.5, np.array([b.r for b in beads]))
        w.write(1, 0.5, buf, gate.wait)
        buf[...] = pos
        gate.set()
        w.flush()
        assert xyz2.read_text() == golden["xyz_text"]


def test_async_xyz_writer_reraises():
    class Broken:
        def write(self, text):
            raise OSError("disk full")

        def flush(self):
            pass

    import numpy as np
    w = io.AsyncXYZWriter(Broken(), "x.xyz", ["A"])
    w.write(0, 1.0, np.zeros((1, 3)))
    with pytest.raises(OSError):
        w.flush()
    w.close()
