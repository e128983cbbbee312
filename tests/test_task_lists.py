"""The batched factorisation's task lists (host only, no GPU).

The persistent batched kernels take tasks in list order from an atomic
counter and spin (bounded) on the flags of the tasks they depend on, so the
factorisation cannot stall only if every task depends on earlier tasks of its
replica's list alone (a merge of several replicas' lists keeps each one's own
order).  These tests replay each list sequentially against the kernels' flag
semantics (csrc/cholesky_df.cu: batch_worker_loop, ll_task) and check that
every wait is already satisfied when its task is reached, and that every
lower tile of L is finished exactly once.
"""
import ctypes

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401  (puts the repository on sys.path)

PREC_FP64, PREC_MIXED = 0, 1
LL_DIAG, LL_UPDATE, LL_SOLVE = 0, 1, 2
TASK_F, TASK_S, TASK_U, TASK_U2 = 0, 1, 2, 4


def _lib():
    from pybrown_b200 import _lib as L
    return L.lib


def task_list(nt, precision):
    lib = _lib()
    cap, seg_cap = nt * nt * nt + 16, 4 * nt + 8
    tasks = (ctypes.c_int * (4 * cap))()
    seg = (ctypes.c_int * seg_cap)()
    n_tasks, n_segs = ctypes.c_int(), ctypes.c_int()
    rc = lib.pbg_cholesky_task_list(nt, precision, tasks, cap, seg, seg_cap, ctypes.byref(n_tasks),
                                    ctypes.byref(n_segs))
    assert rc == 0
    t = np.frombuffer(tasks, dtype=np.int32)[: 4 * n_tasks.value].reshape(-1, 4)
    return t, list(seg[: n_segs.value])


def replay_left_looking(nt, tasks):
    """fin[r]: finished tiles of row r; upd[r]: columns of row r whose U is
    stored.  Returns the set of finished tiles, in finishing order."""
    fin = np.zeros(nt, dtype=int)
    upd = np.zeros(nt, dtype=int)
    done = []
    for kind, i, j, _ in tasks:
        rows = [i] + ([i + 1] if i + 1 < nt else [])
        if kind in (LL_DIAG, LL_UPDATE):
            # the products read L_rk, L_jk for k < j: rows i, i+1, j finished through column j-1
            for r in rows + [j]:
                assert fin[r] >= j, (kind, i, j, r, fin[r])
        if kind == LL_DIAG:
            assert i == j
            for r in rows:
                assert fin[r] == j  # a row's tiles finish in column order
                fin[r] = j + 1
                done.append((r, j))
        elif kind == LL_UPDATE:
            assert i >= j + 2
            for r in rows:
                assert upd[r] == j
                upd[r] = j + 1
        elif kind == LL_SOLVE:
            assert i >= j + 2
            assert fin[j] >= j + 1  # F(j): inv(L_jj) published
            for r in rows:
                assert upd[r] >= j + 1  # U_rj stored
                assert fin[r] == j
                fin[r] = j + 1
                done.append((r, j))
        else:
            raise AssertionError(f"unknown kind {kind}")
    return done


def replay_right_looking(nt, tasks):
    """upd[i][j]: panels applied to tile (i, j); fin[i][j]: tile final."""
    upd = np.zeros((nt, nt), dtype=int)
    fin = np.zeros((nt, nt), dtype=bool)
    done = []
    for kind, i, j, k in tasks:
        if kind in (TASK_U, TASK_U2):
            for r in ([i, i + 1] if kind == TASK_U2 else [i]):
                assert fin[r, k] and fin[j, k] and upd[r, j] == k, (kind, r, j, k)
                upd[r, j] = k + 1
        elif kind in (TASK_F, TASK_S):
            col = j
            if col > 0:
                # the task applies panel col - 1 itself
                assert fin[i, col - 1] and fin[col, col - 1] and upd[i, col] == col - 1, (kind, i, col)
                upd[i, col] = col
            if kind == TASK_S:
                assert fin[col, col], (i, col)
            assert not fin[i, col]
            fin[i, col] = True
            done.append((i, col))
        else:
            raise AssertionError(f"unknown kind {kind}")
    return done


@pytest.mark.parametrize("nt", [1, 2, 3, 5, 8, 24, 96])
def test_left_looking_list_is_ordered_and_complete(nt):
    tasks, seg = task_list(nt, PREC_MIXED)
    assert seg[0] == 0 and seg[-1] == len(tasks) and len(seg) == 2 * nt + 1
    assert all(a <= b for a, b in zip(seg, seg[1:]))
    done = replay_left_looking(nt, tasks)
    tiles = [(r, c) for c in range(nt) for r in range(c, nt)]
    assert sorted(done) == sorted(tiles) and len(done) == len(set(done))
    # segment 2c: the diagonal pair and the updates of column c; 2c + 1: the solves
    for c in range(nt):
        a = tasks[seg[2 * c]:seg[2 * c + 1]]
        b = tasks[seg[2 * c + 1]:seg[2 * c + 2]]
        assert a[0][0] == LL_DIAG and a[0][2] == c and all(t[0] == LL_UPDATE and t[2] == c for t in a[1:])
        assert all(t[0] == LL_SOLVE and t[2] == c for t in b)
        assert [t[1] for t in a[1:]] == [t[1] for t in b]


@pytest.mark.parametrize("nt", [1, 2, 3, 5, 8, 24])
def test_right_looking_list_is_ordered_and_complete(nt):
    tasks, seg = task_list(nt, PREC_FP64)
    assert seg[0] == 0 and seg[-1] == len(tasks)
    done = replay_right_looking(nt, tasks)
    tiles = [(r, c) for c in range(nt) for r in range(c, nt)]
    assert sorted(done) == sorted(tiles) and len(done) == len(set(done))


def test_merged_lists_keep_each_replicas_order():
    """The batch merges the replicas' lists segment by segment (any order of
    replicas within a segment number): each replica's subsequence is its own
    list, so the replay above holds for each one in the merged list."""
    rng = np.random.default_rng(3)
    nts = [int(x) for x in rng.integers(1, 12, size=6)]
    lists = [task_list(nt, PREC_MIXED) for nt in nts]
    merged = []
    for s in range(max(len(seg) - 1 for _, seg in lists)):
        for q in rng.permutation(len(lists)):
            tasks, seg = lists[q]
            if s + 1 < len(seg):
                merged += [(q, tuple(t)) for t in tasks[seg[s]:seg[s + 1]]]
    for q, (tasks, _) in enumerate(lists):
        mine = np.array([t for r, t in merged if r == q]).reshape(-1, 4)
        assert np.array_equal(mine, tasks)
        replay_left_looking(nts[q], mine)


def test_bad_arguments_are_refused():
    lib = _lib()
    tasks = (ctypes.c_int * 64)()
    seg = (ctypes.c_int * 8)()
    n, m = ctypes.c_int(), ctypes.c_int()
    assert lib.pbg_cholesky_task_list(0, PREC_MIXED, tasks, 16, seg, 8, ctypes.byref(n), ctypes.byref(m)) == -2
    # too small for nt = 8: refused, with the sizes it would need
    assert lib.pbg_cholesky_task_list(8, PREC_MIXED, tasks, 16, seg, 8, ctypes.byref(n), ctypes.byref(m)) == -2
    assert n.value > 16 and m.value == 17
