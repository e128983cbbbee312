"""pbg_run: the multi-step loop fed by a noise pool (include/pybrown_b200.h)
against the reference's own trajectory with overlap rejections
(tests/golden/trajectories.npz, ermak_rpy_reject): same positions, noise
consumption equal to the reference's RNG draw count, and the rollback when
the pool or the move attempts run out."""
import ctypes
import json

import numpy as np
import pytest

from conftest import rel_err
from test_gpu_box import _box

pytestmark = pytest.mark.gpu

NAME = "ermak_rpy_reject"


def _setup(trajectories, **override):
    from pybrown_b200.bd import DEFAULTS
    inp = dict(DEFAULTS)
    inp.update(json.loads(str(trajectories[f"{NAME}/config"])))
    inp.update(override)
    init = trajectories[f"{NAME}/init"]
    radii = np.full(len(init), float(trajectories[f"{NAME}/radius"]))
    return _box(init, radii, inp), inp, init


def _run(box, n_steps, dt, pool):
    from pybrown_b200 import _lib
    rc = _lib.lib.pbg_run(box._h, 0, n_steps, float(dt), 1, 1, 1, pool.ctypes.data, pool.size, None)
    rep = _lib.PbgStepReport()
    assert _lib.lib.pbg_run_report(box._h, ctypes.byref(rep), None) == 0
    pos = np.empty((len(box.mobile_beads), 3))
    _lib.call("pbg_get_positions", box._h, pos.ctypes.data, None)
    return rc, rep, pos


def test_run_matches_reference(trajectories):
    box, inp, init = _setup(trajectories)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]))
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool)
    assert rc == 0 and rep.status == 0
    assert rep.steps_done == len(traj) and rep.draws_consumed == draws[-1]
    assert rep.max_attempts == max(np.diff(np.concatenate([[0], draws])) // (3 * len(init)))
    assert rel_err(pos - init, traj[-1] - init) <= 1e-10


def test_run_rolls_back_when_the_pool_runs_out(trajectories):
    from pybrown_b200 import _lib
    box, inp, init = _setup(trajectories)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]) - 1)
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool)
    assert rc == _lib.PBG_ERR_NOISE and rep.status == rc
    assert rep.steps_done == len(traj) - 1 and rep.draws_consumed == draws[-2]
    assert rel_err(pos - init, traj[-2] - init) <= 1e-10


def test_run_stops_at_max_move_attempts(trajectories):
    from pybrown_b200 import _lib
    box, inp, init = _setup(trajectories, max_move_attempts=1)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    per_step = np.diff(np.concatenate([[0], draws])) // (3 * len(init))
    first = int(np.argmax(per_step > 1))
    assert first > 0 and per_step[first] > 1
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]))
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool)
    assert rc == _lib.PBG_ERR_ATTEMPTS
    assert rep.steps_done == first
    assert rel_err(pos - init, traj[first - 1] - init) <= 1e-10
