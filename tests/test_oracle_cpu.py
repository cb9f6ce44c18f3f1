"""The CPU oracle pinned against the reference's own outputs (golden fixtures).

The fixtures under tests/golden were produced by the reference library built
from its sources (tests/golden/make_golden.py); here the C restatement
(oracle/cham_oracle.c) must reproduce them: generators bit-exact, factor and
solution within the reference's testing tolerance.
"""
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_generators_bitexact_vs_reference(orc):
    g = np.load(os.path.join(GOLDEN, "gen_37.npz"))
    assert np.array_equal(orc.dplgsy(37.0, 37, 51), g["A"])
    assert np.array_equal(orc.dplrnt(37, 3, 5673), g["B"])


def test_known_answers(orc):
    kat = json.load(open(os.path.join(GOLDEN, "kat.json")))
    for n, s, v in kat["lcg_skip"]:
        assert orc.lcg_skip(n, s) == v
    assert orc.dplgsy(2048.0, 4, 51, bigM=2048)[0, 0] == kat["dplgsy_2048_seed51_A00"] == 2048.5
    assert orc.dplrnt(1, 1, 5673, bigM=2048)[0, 0] == kat["dplrnt_2048_seed5673_B0"]


def test_generator_symmetric_and_bump(orc):
    A = orc.dplgsy(50.0, 50, 7)
    assert np.array_equal(A, A.T)
    off = A - np.diag(np.diag(A))
    assert np.all(np.abs(off) <= 0.5) and np.all(np.diag(A) > 49.4)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "posv_*.npz"))))
def test_oracle_posv_matches_reference(orc, path):
    g = np.load(path)
    uplo, N, NB, nrhs = (int(x) for x in os.path.basename(path)[5:-4].split("_"))
    A, B = g["A"], g["B"]
    assert np.array_equal(A, orc.dplgsy(float(N), N, 51))
    F, info = orc.dpotrf_tiled(uplo, A, NB)
    assert info == 0 == int(g["info"])
    X = orc.dpotrs_tiled(uplo, F, B, NB)
    tri = np.triu if uplo == 121 else np.tril
    # element-wise agreement with the reference's factor / solution
    assert np.abs(tri(F) - g["F"]).max() <= 64 * N * 1.11e-16 * np.abs(A).max()
    assert np.abs(X - g["X"]).max() <= 64 * N * 1.11e-16 * max(1.0, np.abs(g["X"]).max())
    # the reference's own checks (testing/testing_zcheck_facto.c), threshold 60
    assert orc.check_factorization(uplo, A, F) < 60.0
    assert orc.check_solve(A, X, B) < 60.0


def test_checks_detect_a_planted_error(orc):
    """A wrong factor planted in the oracle's output must fail the check."""
    N, NB = 35, 16
    A = orc.dplgsy(float(N), N, 51)
    F, _ = orc.dpotrf_tiled(122, A, NB)
    F[20, 3] += 1e-6
    assert orc.check_factorization(122, A, F) > 60.0


def test_oracle_non_spd_info(orc):
    N, NB = 40, 16
    A = orc.dplgsy(float(N), N, 3)
    A[25, 25] = -100.0
    _, info = orc.dpotrf_tiled(122, A, NB)
    assert info == 26


def test_live_reference_agrees_when_built(orc):
    if not orc.reference_available():
        pytest.skip("reference library not built on this host")
    N, NB = 77, 17
    A = orc.dplgsy(float(N), N, 51)
    B = orc.dplrnt(N, 4, 5673)
    for uplo in (121, 122):
        F, X, info, _ = orc.ref_dposv(uplo, A, B, NB)
        assert info == 0
        assert orc.check_solve(A, X, B) < 60.0
        Xp = orc.dpotrs_tiled(uplo, orc.dpotrf_tiled(uplo, A, NB)[0], B, NB)
        assert np.abs(Xp - X).max() < 1e-13
