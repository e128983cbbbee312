"""Input and output formats (drop-in for pyBrown.input / pyBrown.output).

JSON configuration with defaults and keyword validation
(src/bdsim/pyBrown/input.py:24-109), `.str` structure files
(input.py:113-172), `.xyz` trajectories (output.py:63-69) and pickled `.rst`
restart files with a `.rst2` backup (output.py:72-84).  Byte formats are the
reference's.
"""
import json
import os
import pickle
import shutil
import time

import numpy as np

from .bead import Bead


class InputData:
    """input.py:24-109: JSON keywords completed with defaults; missing
    required keywords and unknown keywords raise AssertionError."""

    def __init__(self, input_filename, obligatory_keywords=(), defaults=None, all_keywords=None):
        with open(input_filename, "r") as f:
            self.input_data = json.load(f)
        for k, v in (defaults or {}).items():
            if k not in self.input_data:
                self.input_data[k] = v
        for k in obligatory_keywords:
            assert k in self.input_data, "Missing {} keyword in input JSON file.".format(k)
        if all_keywords is not None:
            for k in self.input_data:
                assert k in all_keywords, "Unrecognized {} keyword in input JSON file.".format(k)

    def __str__(self):
        return "".join("{}: {}\n".format(k, v) for k, v in self.input_data.items())

    __repr__ = __str__


def read_str_file(input_str_filename):
    """input.py:113-172: `sub`, `bond` and `angle` lines -> list of Bead."""
    beads = []
    with open(input_str_filename) as f:
        for line in f:
            seg = line.split()
            if not seg:
                continue
            if seg[0] == "sub":
                beads.append(Bead(coords=np.array([float(seg[i]) for i in range(3, 6)]),
                                  hydrodynamic_radius=float(seg[6]), label=seg[1],
                                  hard_core_radius=float(seg[8]) / 2, epsilon_LJ=float(seg[9]),
                                  bead_id=int(seg[2])))
            elif seg[0] == "bond":
                id1, id2 = int(seg[1]), int(seg[2])
                b1 = next(b for b in beads if b.bead_id == id1)
                b1.bonded_with.append(id2)
                b1.bonded_how[id2] = [float(seg[3]), float(seg[5])]
            elif seg[0] == "angle":
                id1, id2, id3 = int(seg[2]), int(seg[3]), int(seg[4])
                b1 = next(b for b in beads if b.bead_id == id1)
                b1.angled_with.append([id2, id3])
                b1.angled_how[(id2, id3)] = [float(seg[5]), float(seg[6])]
    return beads


def write_str_file(filename, beads):
    """Writes beads as `sub` lines (label id x y z a charge 2*lj_radius lj_energy mass)."""
    with open(filename, "w") as f:
        for i, b in enumerate(beads):
            bid = b.bead_id if b.bead_id is not None else i + 1
            f.write("sub {} {} {!r} {!r} {!r} {!r} 0 {!r} {!r} 1\n".format(
                b.label, bid, float(b.r[0]), float(b.r[1]), float(b.r[2]), float(b.a),
                2 * float(b.hard_core_radius), float(b.epsilon_LJ)))


def timestamp(message, *variables):
    date = time.asctime(time.localtime(time.time()))
    print("{}: ".format(date) + message.format(*variables) + "\n")


def write_to_xyz_file(xyz_file, xyz_filename, j, dt, beads):
    """output.py:63-69."""
    xyz_file.write("{}\n".format(len(beads)))
    xyz_file.write("{} time [ps] {}\n".format(xyz_filename, j * dt))
    for bead in beads:
        xyz_file.write("{} {} {} {}\n".format(bead.label, *bead.r))


def _xyz_frame(xyz_filename, j, dt, labels, positions):
    """The text of one frame in the format of write_to_xyz_file (the
    shortest round-trip repr of each coordinate, as str.format gives for a
    float), built from Python floats in one pass."""
    x, y, z = np.asarray(positions, dtype=np.float64).reshape(-1, 3).T.tolist()
    head = "{}\n{} time [ps] {}\n".format(len(labels), xyz_filename, j * dt)
    return head + "".join(map("{} {!r} {!r} {!r}\n".format, labels, x, y, z))


class AsyncXYZWriter:
    """.xyz frames (output.py:63-69) written by a background thread, so that a
    step loop hands over a frame and goes on.  Each frame is a snapshot of the
    positions (an array copied at hand-over, or a buffer that an asynchronous
    device-to-host copy is filling, with `ready` a callable that blocks until
    the copy is done).  The thread waits for the copy, formats the frame
    exactly as write_to_xyz_file does and writes frames in order.  At most
    `depth` frames are pending; flush() waits for all of them (before the
    file's length is read, e.g. for a restart file) and re-raises an error of
    the thread; close() waits for them and stops the thread."""

    def __init__(self, xyz_file, xyz_filename, labels, depth=4):
        import queue
        import threading
        self._file = xyz_file
        self._name = xyz_filename
        self._labels = list(labels)
        self._queue = queue.Queue(maxsize=max(1, int(depth)))
        self._error = None
        self._thread = threading.Thread(target=self._run, name="xyz-writer", daemon=True)
        self._thread.start()

    def _run(self):
        while True:
            item = self._queue.get()
            try:
                if item is None:
                    return
                j, dt, positions, ready = item
                if self._error is None:
                    if ready is not None:
                        ready()
                    self._file.write(_xyz_frame(self._name, j, dt, self._labels, positions))
            except BaseException as e:  # noqa: BLE001 -- re-raised in the caller's thread
                self._error = e
            finally:
                self._queue.task_done()

    def _check(self):
        if self._error is not None:
            err, self._error = self._error, None
            raise err

    def write(self, j, dt, positions, ready=None):
        """Queues frame j (time j * dt).  Without `ready` the positions are
        copied now; with it they are read once ready() has returned."""
        self._check()
        pos = np.array(positions, dtype=np.float64, copy=True) if ready is None else positions
        self._queue.put((j, dt, pos, ready))

    def flush(self):
        """Waits until every frame handed over is written and flushed to the
        file (a restart file records the .xyz file's length)."""
        self._queue.join()
        self._check()
        self._file.flush()

    def close(self):
        if self._thread.is_alive():
            self._queue.put(None)
            self._thread.join()
        self._check()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _file_length(filename):
    i = -1
    with open(filename, "r") as f:
        for i, _ in enumerate(f):
            pass
    return i + 1


def write_to_restart_file(restart_filename, index, j, box, xyz_filename, extra_output_filenames=(),
                          extra_data=None):
    """output.py:72-84: pickle (index, j, box, output lengths) and copy to .rst2."""
    with open(restart_filename, "wb", buffering=0) as f:
        pickle.dump(index, f)
        pickle.dump(j, f)
        pickle.dump(box, f)
        pickle.dump(_file_length(xyz_filename), f)
        for name in extra_output_filenames:
            pickle.dump(_file_length(name), f)
        if extra_data is not None:
            pickle.dump(extra_data, f)
    shutil.copy(restart_filename, restart_filename + "2")


def truncate_output_file_during_restart(filename, line):
    """output.py:44-60."""
    tmp = filename + ".tmp"
    with open(filename, "r") as src, open(tmp, "w") as dst:
        for _ in range(line):
            dst.write(src.readline())
    with open(tmp, "r") as src, open(filename, "w") as dst:
        for ln in src:
            dst.write(ln)
    if os.path.exists(tmp):
        os.remove(tmp)


def write_to_enr_file(enr_file, j, dt, E, energy_unit_string):
    """output.py:108-118."""
    if j == 0:
        enr_file.write("time/ps energy/{}\n".format(energy_unit_string))
    enr_file.write("{} {}\n".format(j * dt, E))
