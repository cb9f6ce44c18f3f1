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


def test_gered_restatement_rule():
    """The oracle's gered (compute/pzgered.c:160-260 with the CUDA rule of
    codelet_zgered.c): a hand-checked 2 x 2 tile case."""
    from oracle import oracle as o
    mb = 4
    A = np.zeros((8, 8))
    A[:4, :4] = 10 * np.eye(4)            # diagonal tiles: ||.||_F = 20 each
    A[4:, 4:] = 10 * np.eye(4)
    A[4:, :4] = 1e-3                      # off-diagonal tile: ||.||_F = 4e-3
    A[:4, 4:] = 1e-3
    # lower: gnorm = sqrt(20^2 + 20^2 + 4e-3^2) ~ 28.28; prec 1e-6 -> threshold
    # 1e-6 * 28.28 / 2 = 1.41e-5: 4e-3 < 1.41e-5 / 1e-4 = 0.141 -> FP16
    R, tags = o.gered(122, 1e-6, A, mb)
    assert tags.tolist() == [[0, 0], [2, 0]]
    assert np.array_equal(R[4:, :4], np.float64(np.float16(1e-3)) * np.ones((4, 4)))
    assert np.array_equal(R[:4, 4:], A[:4, 4:])            # outside the triangle: untouched
    # prec 1e-9: threshold 1.41e-8; FP16 needs < 1.41e-4, FP32 < 1.41e-8 / 2^-24 = 0.237 -> FP32
    R, tags = o.gered(122, 1e-9, A, mb)
    assert tags.tolist() == [[0, 0], [1, 0]]
    # the diagonal tiles use the FP32 unit roundoff once prec exceeds it
    R, tags = o.gered(122, 1e-2, A, mb)
    assert tags[0, 0] == 0 and tags[1, 1] == 0
