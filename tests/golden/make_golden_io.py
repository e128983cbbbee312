"""Generate tests/golden/io.json from the reference's own input/output code.

Run in a container that has the reference tree and oracle/_ref built:

    make -C oracle ref && python tests/golden/make_golden_io.py

It feeds a structure file written here (beads with labels and ids, bonds,
angles) to the reference's `read_str_file` (src/bdsim/pyBrown/input.py:113-172)
and records every parsed field; writes two `.xyz` frames and two `.enr`
lines with the reference's writers (output.py:63-69, 108-118); truncates a
file with `truncate_output_file_during_restart` (output.py:44-60); and
completes a JSON configuration with `InputData` (input.py:24-109).  The GPU
box has none of the reference: tests/test_io_golden.py only reads io.json.
"""
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _import_reference  # noqa: E402

STR_TEXT = """sub A 1 0.5 -1.25 3.0 2.0 0.0 4.0 0.3 1.0
sub B 2 1.5 -0.25 3.5 2.5 0.0 5.0 0.2 1.0
sub A 3 2.5 0.75 4.0 2.0 0.0 4.0 0.3 1.0
sub C 7 -3.0 2.0 -1.0 1.0 0.0 2.0 0.1 1.0
bond 1 2 4.5 0 10.0
bond 2 3 4.25 0 12.5
angle 0 1 2 3 2.0 7.5
angle 0 2 3 7 1.5 3.0
"""

DEFAULTS = {"T": 298.15, "seed": None, "dt": 1.0}
REQUIRED = ["box_length"]
ALL = ["box_length", "T", "seed", "dt", "hydrodynamics"]
CONFIG = {"box_length": 75.0, "hydrodynamics": "rpy"}


def main():
    _import_reference()
    from pyBrown import input as ref_input  # noqa: E402
    from pyBrown import output as ref_output  # noqa: E402
    out = {"str_text": STR_TEXT, "defaults": DEFAULTS, "required": REQUIRED, "all_keywords": ALL,
           "config": CONFIG}
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "s.str")
        with open(p, "w") as f:
            f.write(STR_TEXT)
        beads = ref_input.read_str_file(p)
        out["beads"] = [{"label": b.label, "bead_id": b.bead_id, "r": [float(x) for x in b.r], "a": b.a,
                         "hard_core_radius": b.hard_core_radius, "epsilon_LJ": b.epsilon_LJ,
                         "bonded_with": list(b.bonded_with),
                         "bonded_how": {str(k): v for k, v in b.bonded_how.items()},
                         "angled_with": [list(x) for x in b.angled_with],
                         "angled_how": {"{},{}".format(*k): v for k, v in b.angled_how.items()}}
                        for b in beads]
        xyz = os.path.join(d, "t.xyz")
        with open(xyz, "w") as f:
            ref_output.write_to_xyz_file(f, "t.xyz", 0, 0.5, beads)
            beads[0].r[0] += 0.125
            ref_output.write_to_xyz_file(f, "t.xyz", 1, 0.5, beads)
        out["xyz_text"] = open(xyz).read()
        enr = os.path.join(d, "e.enr")
        with open(enr, "w") as f:
            ref_output.write_to_enr_file(f, 0, 0.5, 1.5e-20, "joule")
            ref_output.write_to_enr_file(f, 1, 0.5, -2.25e-21, "joule")
        out["enr_text"] = open(enr).read()
        ref_output.truncate_output_file_during_restart(xyz, 3)
        out["truncated_xyz_text"] = open(xyz).read()
        cfg = os.path.join(d, "c.json")
        with open(cfg, "w") as f:
            json.dump(CONFIG, f)
        inp = ref_input.InputData(cfg, REQUIRED, DEFAULTS, ALL)
        out["input_data"] = inp.input_data
    with open(os.path.join(HERE, "io.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "io.json"))


if __name__ == "__main__":
    main()
