"""GPU tests of the serving loop (CHAM_B200_Serve_*; no reference counterpart).

Each request's result is checked against the oracle's tiled dposv with the
reference's solve check (threshold 60), and the result a request gets inside a
mix of concurrent requests (batched small systems, mixed-precision large
systems on several streams, kept factors) is bitwise the result it gets alone.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
THRESH = 60.0


def make_case(orc, N, nrhs, seed, uplo=122):
    A = orc.dplgsy(float(N), N, 51 + seed)
    B = orc.dplrnt(N, nrhs, 5673 + seed)
    if uplo == 121:
        Ain = np.asfortranarray(np.triu(A))
    else:
        Ain = np.asfortranarray(np.tril(A))
    return A, Ain, B


def solve_alone(cb, Ain, B, uplo, slots=1, small_n=512, key=-1):
    X = np.zeros_like(B, order="F")
    with cb.Server(slots=slots, small_n=small_n) as sv:
        r = sv.submit(Ain, B, X, uplo=uplo, factor_key=key)
        sv.drain()
        assert r.status == 0, r.status
    return X


CASES = [  # (N, nrhs, uplo): small ones take the batched path, large the mixed path
    (17, 1, 122), (64, 3, 122), (200, 8, 121), (512, 2, 122),
    (513, 4, 122), (1000, 5, 121), (2048, 16, 122), (4500, 3, 122),
]


def test_mix_equals_alone(cb, orc):
    cases = [make_case(orc, N, k, i, u) + (u,) for i, (N, k, u) in enumerate(CASES)]
    alone = [solve_alone(cb, Ain, B, u) for (_, Ain, B, u) in cases]
    for (A, _, B, _), X in zip(cases, alone):
        assert orc.check_solve(A, X, B) < THRESH
    with cb.Server(slots=3) as sv:
        outs, reqs = [], []
        for rep in range(2):   # every case twice, interleaved
            for (A, Ain, B, u) in cases:
                X = np.zeros_like(B, order="F")
                reqs.append(sv.submit(Ain, B, X, uplo=u))
                outs.append(X)
        sv.drain()
        st = sv.stats()
    assert all(r.status == 0 for r in reqs), [r.status for r in reqs]
    for i, X in enumerate(outs):
        assert np.array_equal(X, alone[i % len(cases)]), CASES[i % len(cases)]
    assert st["completed"] == 2 * len(cases)
    assert st["batched_requests"] == 2 * sum(1 for (N, _, _) in CASES if N <= 512)


def test_kept_factor_reuse(cb, orc):
    N = 3000
    A, Ain, B = make_case(orc, N, 4, 11)
    B2 = orc.dplrnt(N, 7, 999)
    X = np.zeros_like(B, order="F")
    X2 = np.zeros_like(B2, order="F")
    X3 = np.zeros_like(B2, order="F")
    with cb.Server(slots=2) as sv:
        r1 = sv.submit(Ain, B, X, factor_key=42)
        sv.drain()
        r2 = sv.submit(None, B2, X2, N=N, factor_key=42)
        r3 = sv.submit(None, B2, X3, N=N, factor_key=43)   # nothing kept under 43
        sv.drain()
        st = sv.stats()
    assert r1.status == 0 and r2.status == 0
    assert r3.status == cb.CHAMELEON_ERR_NOT_FOUND
    assert orc.check_solve(A, X, B) < THRESH
    assert orc.check_solve(A, X2, B2) < THRESH
    assert st["reused_factors"] == 1 and st["kept_factors"] == 1
    # the same right-hand sides solved from scratch give the same bits
    X4 = solve_alone(cb, Ain, B2, 122)
    assert np.abs(X4 - X2).max() <= 1e-12 * np.abs(X4).max()


def test_admission_under_small_budget(cb, orc):
    """A budget below one request still serves every request (one at a time)."""
    cases = [make_case(orc, N, 2, 20 + i) for i, N in enumerate([1500, 2500, 700, 300, 100])]
    with cb.Server(slots=2, hbm_budget_bytes=8e6) as sv:
        outs, reqs = [], []
        for (A, Ain, B) in cases:
            X = np.zeros_like(B, order="F")
            reqs.append(sv.submit(Ain, B, X))
            outs.append(X)
        sv.drain()
        st = sv.stats()
    assert all(r.status == 0 for r in reqs)
    for (A, _, B), X in zip(cases, outs):
        assert orc.check_solve(A, X, B) < THRESH
    assert st["bytes_in_use"] == 0


def test_not_spd_request_is_isolated(cb, orc):
    good = [make_case(orc, N, 2, 30 + i) for i, N in enumerate([40, 90, 300])]
    Abad = np.asfortranarray(np.eye(64))
    Abad[10, 10] = -1.0
    Bbad = np.ones((64, 1), order="F")
    with cb.Server(slots=1) as sv:
        outs, reqs = [], []
        for (A, Ain, B) in good:
            X = np.zeros_like(B, order="F")
            reqs.append(sv.submit(Ain, B, X))
            outs.append(X)
        rb = sv.submit(Abad, Bbad, np.zeros_like(Bbad, order="F"))
        sv.drain()
    assert rb.status == 11
    assert all(r.status == 0 for r in reqs)
    for (A, _, B), X in zip(good, outs):
        assert orc.check_solve(A, X, B) < THRESH


def test_submit_rejects_bad_arguments(cb):
    B = np.ones((8, 1), order="F")
    X = np.zeros_like(B)
    with cb.Server(slots=1) as sv:
        with pytest.raises(cb.ChameleonError):
            sv.submit(None, B, X, N=8)            # no matrix and no key
        with pytest.raises(cb.ChameleonError):
            sv.submit(np.eye(8, order="F"), B, X, N=8, lda=4)
