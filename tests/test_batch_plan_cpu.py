"""The device scheduler's task list (host-only planner, batch.cu
xg_batch_plan): every task of every field's tile Cholesky appears exactly
once, and replaying the list in order with the scheduler's own dependency
rules never meets a task whose dependencies are not already in the list --
the condition under which persistent CTAs that take tasks in list order
cannot deadlock.  Runs without a GPU."""
import ctypes

import numpy as np
import pytest

POTRF, TRSM, GEMM = 0, 1, 2


def _plan(xg, nts, workers):
    L = xg.lib()
    f = L.exageostat_b200_batch_plan
    f.restype = ctypes.c_longlong
    f.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_void_p]
    arr = (ctypes.c_int * len(nts))(*nts)
    n = f(len(nts), arr, workers, None)
    out = np.zeros(4 * n, dtype=np.int32)
    assert f(len(nts), arr, workers, out.ctypes.data) == n
    return out.reshape(n, 4)


def _expected(nt):
    return {(POTRF, k, k, k) for k in range(nt)} | \
        {(TRSM, i, k, k) for k in range(nt) for i in range(k + 1, nt)} | \
        {(GEMM, i, j, k) for k in range(nt) for j in range(k + 1, nt) for i in range(j, nt)}


@pytest.mark.parametrize("nts,workers", [([1], 4), ([5], 1), ([7, 3, 1, 7], 3), ([12, 9, 4, 2, 11, 6], 148)])
def test_plan_is_a_complete_topological_order(xg, nts, workers):
    tl = _plan(xg, nts, workers)
    seen = [set() for _ in nts]
    ucnt = [dict() for _ in nts]
    tdone = [set() for _ in nts]
    pdone = [set() for _ in nts]
    for code, i, j, k in tl:
        typ, f = int(code) & 3, int(code) >> 2
        key = (typ, int(i), int(j), int(k))
        assert key not in seen[f], "task listed twice"
        seen[f].add(key)
        u = ucnt[f]
        # the device scheduler's waits, all satisfied by tasks earlier in the list
        if typ == POTRF:
            assert u.get((k, k), 0) == k
            pdone[f].add(k)
        elif typ == TRSM:
            assert k in pdone[f] and u.get((i, k), 0) == k
            tdone[f].add((i, k))
        else:
            assert (i, k) in tdone[f] and (j, k) in tdone[f] and u.get((i, j), 0) == k
            u[(i, j)] = k + 1
    for f, nt in enumerate(nts):
        assert seen[f] == _expected(nt)


def test_plan_starts_the_next_panel_before_the_step_ends(xg):
    """Critical path first: with fewer CTAs than a step's updates, a field's
    POTRF(k + 1) is listed before the last trailing update of its step k (the
    lookahead a step-by-step order lacks)."""
    tl = _plan(xg, [10], 4)
    pos = {tuple(int(v) for v in r): q for q, r in enumerate(tl)}
    for k in range(8):
        last_update = max(q for (code, i, j, kk), q in pos.items() if (code & 3) == GEMM and kk == k)
        assert pos[(POTRF, k + 1, k + 1, k + 1)] < last_update
