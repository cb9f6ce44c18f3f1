"""The runtime-plugin boundary, on the host (no GPU).

The reference's own CHAMELEON_dposv_Tile (compute/zposv.c:222-245: one
chameleon_pdpotrf and two chameleon_pdtrsm, compute/pzpotrf.c:84-194,
compute/pztrsm.c:58-200, d precision) is linked with the B200 runtime plugin
(chameleon_b200/runtime/runtime_b200.c) in place of StarPU/OpenMP, by
oracle/build_plugin.sh.  In record-only mode its INSERT_TASK_* calls are kept,
not run.  The recorded task set must equal the DAG the executor builds itself
for the same shape (C1: N=2048, NB=320, nrhs=1; C2: N=16384, NB=512, nrhs=64;
both triangles), and the executor must accept the records in their submission
order (its device wait predicates replayed on the scheduled list).
"""
import ctypes
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PLUGIN = os.path.join(ROOT, "oracle", "_ref", "libchamb200rt.so")
FACT, SOLVE = 1, 2

pytestmark = pytest.mark.skipif(not os.path.exists(PLUGIN), reason="plugin test library not built (needs the "
                                                                   "reference sources: oracle/build_plugin.sh)")


def recorded(uplo, N, NB, nrhs):
    L = ctypes.CDLL(PLUGIN)
    cap = 6 * (N // NB + 2) ** 3
    dag = (ctypes.c_int * (5 * cap))()
    n = ctypes.c_int()
    rc = L.harness_posv(uplo, N, NB, nrhs, None, N, None, N, 1, dag, cap, ctypes.byref(n))
    assert rc == 0 and 0 < n.value <= cap
    return np.frombuffer(dag, dtype=np.int32)[:5 * n.value].reshape(-1, 5).copy()


@pytest.mark.parametrize("uplo", [121, 122])
@pytest.mark.parametrize("N,NB,nrhs", [(2048, 320, 1), (16384, 512, 64), (1000, 256, 40)])
def test_reference_algorithms_record_the_executor_dag(cb_host, uplo, N, NB, nrhs):
    rec = recorded(uplo, N, NB, nrhs)
    got = {tuple(int(v) for v in r) if r[0] > 3 else (int(r[0]), int(r[1]), int(r[2]), int(r[3]), 0) for r in rec}
    assert len(got) == len(rec)                      # every tile task submitted once
    sched = cb_host.schedule(FACT | SOLVE, N, NB, nrhs, NB, 148, 0, 1)
    want = {(int(t[0]), int(t[2]), int(t[3]), int(t[4]), int(t[5]) if t[0] > 3 else 0) for t in sched}
    assert got == want
    # the executor schedules the records in their submission order
    L = cb_host.lib()
    dag = ctypes.c_void_p()
    assert L.CHAM_B200_Dag_Create(ctypes.byref(dag)) == 0
    try:
        for r in rec:
            assert L.CHAM_B200_Dag_Record(dag, *(int(v) for v in r)) == 0
        n = L.CHAM_B200_Dag_Schedule(dag, N, NB, nrhs, NB, 148, None, 0)
        assert n == len(sched)
    finally:
        L.CHAM_B200_Dag_Destroy(dag)


def test_records_out_of_order_are_refused(cb_host):
    """An update of a tile recorded before an earlier panel's update of the
    same tile cannot run on the executor's in-order counters: refused, not
    deadlocked."""
    L = cb_host.lib()
    dag = ctypes.c_void_p()
    assert L.CHAM_B200_Dag_Create(ctypes.byref(dag)) == 0
    try:
        for r in [(1, 0, 0, 0, 0), (2, 1, 0, 0, 0), (2, 2, 0, 0, 0), (3, 1, 1, 0, 0), (3, 2, 1, 0, 0),
                  (3, 2, 2, 0, 0), (1, 1, 1, 1, 0), (2, 2, 1, 1, 0), (1, 2, 2, 2, 0),   # POTRF(2) before UPD(2,2,1)
                  (3, 2, 2, 1, 0)]:
            assert L.CHAM_B200_Dag_Record(dag, *r) == 0
        assert L.CHAM_B200_Dag_Schedule(dag, 300, 100, 0, 100, 4, None, 0) == -103   # NOT_SUPPORTED
    finally:
        L.CHAM_B200_Dag_Destroy(dag)


@pytest.fixture(scope="module")
def cb_host():
    import chameleon_b200 as cb
    return cb
