"""pbg_run: the multi-step loop fed by a noise pool (include/pybrown_b200.h)
against the reference's own trajectory with overlap rejections
(tests/golden/trajectories.npz, ermak_rpy_reject): same positions, noise
consumption equal to the reference's RNG draw count, and the rollback when
the pool or the move attempts run out.  With the pool in host memory the
steps are driven from the host; with the pool in device memory they run on
the device (one CUDA graph per step from the second step with the same flags,
the attempts under a conditional WHILE node): both are checked, and against
each other bit for bit."""
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


def _run(box, n_steps, dt, pool, where="host", j0=0):
    from pybrown_b200 import _lib
    if where == "device":
        import torch
        dpool = torch.tensor(pool, dtype=torch.float64, device="cuda")
        ptr = dpool.data_ptr()
    else:
        ptr = pool.ctypes.data
    rc = _lib.lib.pbg_run(box._h, j0, n_steps, float(dt), 1, 1, 1, ptr, pool.size, None)
    rep = _lib.PbgStepReport()
    assert _lib.lib.pbg_run_report(box._h, ctypes.byref(rep), None) == 0
    pos = np.empty((len(box.mobile_beads), 3))
    _lib.call("pbg_get_positions", box._h, pos.ctypes.data, None)
    return rc, rep, pos


@pytest.mark.parametrize("where", ["host", "device"])
def test_run_matches_reference(trajectories, where):
    box, inp, init = _setup(trajectories)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]))
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool, where)
    assert rc == 0 and rep.status == 0
    assert rep.steps_done == len(traj) and rep.draws_consumed == draws[-1]
    assert rep.max_attempts == max(np.diff(np.concatenate([[0], draws])) // (3 * len(init)))
    assert rel_err(pos - init, traj[-1] - init) <= 1e-10


@pytest.mark.parametrize("where", ["host", "device"])
def test_run_rolls_back_when_the_pool_runs_out(trajectories, where):
    from pybrown_b200 import _lib
    box, inp, init = _setup(trajectories)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]) - 1)
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool, where)
    assert rc == _lib.PBG_ERR_NOISE and rep.status == rc
    assert rep.steps_done == len(traj) - 1 and rep.draws_consumed == draws[-2]
    assert rel_err(pos - init, traj[-2] - init) <= 1e-10


@pytest.mark.parametrize("where", ["host", "device"])
def test_run_stops_at_max_move_attempts(trajectories, where):
    from pybrown_b200 import _lib
    box, inp, init = _setup(trajectories, max_move_attempts=1)
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    per_step = np.diff(np.concatenate([[0], draws])) // (3 * len(init))
    first = int(np.argmax(per_step > 1))
    assert first > 0 and per_step[first] > 1
    pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]))
    rc, rep, pos = _run(box, len(traj), trajectories[f"{NAME}/dt"], pool, where)
    assert rc == _lib.PBG_ERR_ATTEMPTS
    assert rep.steps_done == first
    assert rel_err(pos - init, traj[first - 1] - init) <= 1e-10


def test_device_steps_equal_host_steps_call_by_call(trajectories):
    """One step per pbg_run call, as a step loop makes them: with the pool on
    the device every call from the second replays the captured step graph;
    positions and draws equal the host-driven steps' bit for bit, call by
    call."""
    import torch
    from pybrown_b200 import _lib
    traj, draws = trajectories[f"{NAME}/traj"], trajectories[f"{NAME}/draws"]
    dt = trajectories[f"{NAME}/dt"]
    out = {}
    for where in ("host", "device"):
        box, inp, init = _setup(trajectories)
        pool = np.random.RandomState(inp["seed"]).normal(0.0, 1.0, int(draws[-1]))
        dpool = torch.tensor(pool, dtype=torch.float64, device="cuda")
        n = 3 * len(init)
        cursor, steps = 0, []
        for j in range(len(traj)):
            base = dpool.data_ptr() + 8 * cursor if where == "device" else pool.ctypes.data + 8 * cursor
            rc = _lib.lib.pbg_run(box._h, j, 1, float(dt), 1, 1, 1, base, pool.size - cursor, None)
            assert rc == 0
            rep = _lib.PbgStepReport()
            assert _lib.lib.pbg_run_report(box._h, ctypes.byref(rep), None) == 0
            cursor += rep.draws_consumed
            pos = np.empty((len(box.mobile_beads), 3))
            _lib.call("pbg_get_positions", box._h, pos.ctypes.data, None)
            steps.append((pos.copy(), cursor))
        assert cursor == draws[-1]
        out[where] = steps
    for (p_h, c_h), (p_d, c_d) in zip(out["host"], out["device"]):
        assert c_h == c_d
        assert np.array_equal(p_h, p_d)
