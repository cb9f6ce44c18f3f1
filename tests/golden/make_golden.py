"""Generate the golden fixtures of tests/golden from the reference's own library.

Run in a checkout that has the reference sources (it builds
oracle/_ref/libchamref.so with oracle/build_ref.sh, then calls the reference's
CHAMELEON_dplgsy / dplrnt / dposv through oracle/ref_driver.c):

    python tests/golden/make_golden.py

Fixtures (all small):
  * kat.json      -- known-answer values: first elements of the reference's
                     dplgsy/dplrnt at N=2048 (seeds 51 / 5673), and LCG
                     skip-ahead states of the restatement (regression values;
                     the states themselves are pinned through gen_37.npz,
                     which the reference generated)
  * gen_37.npz    -- the reference's dplgsy (N=37, seed 51) and dplrnt
                     (37 x 3, seed 5673)
  * batch_<uplo>.npz -- the reference's CHAMELEON_dpotrf_batch_Tile and
                     CHAMELEON_dtrsm_batch_Tile on 6 matrices of order 40
  * posv_<uplo>_<N>_<NB>_<nrhs>.npz -- the reference's dposv on the
                     testing/input/posv.in-style odd sizes: A (full symmetric
                     input), B, factor F (uplo triangle) and solution X.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402

# testing/input/posv.in style: nb 16/17, n 15/21/35, nrhs 1/13/22/33, both uplo
CASES = [
    (121, 15, 16, 1), (122, 15, 16, 13), (121, 21, 17, 22), (122, 21, 16, 33),
    (121, 35, 17, 13), (122, 35, 16, 1), (121, 37, 17, 22), (122, 64, 16, 5),
    (121, 100, 32, 3), (122, 130, 48, 7),
]
SEED_A, SEED_B = 51, 5673


def main():
    O.build_ref()
    kat = {
        "lcg_skip": [[n, s, int(O.lcg_skip(n, s))] for n, s in
                     [(0, 51), (1, 51), (2, 51), (12345, 51), (2**40 + 3, 5673), (2**63 - 1, 1804289383)]],
        "dplgsy_2048_seed51_A00": float(O.ref_dplgsy(2048.0, 123, 2048, SEED_A, 320)[0, 0]),
        "dplrnt_2048_seed5673_B0": float(O.ref_dplrnt(2048, 1, SEED_B, 320)[0, 0]),
    }
    A37 = O.ref_dplgsy(37.0, 123, 37, SEED_A, 17)
    B37 = O.ref_dplrnt(37, 3, SEED_B, 17)
    np.savez_compressed(os.path.join(HERE, "gen_37.npz"), A=A37, B=B37)
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(kat, f, indent=1)
    for uplo, N, NB, nrhs in CASES:
        A = O.ref_dplgsy(float(N), 123, N, SEED_A, NB)
        B = O.ref_dplrnt(N, nrhs, SEED_B, NB)
        F, X, info, _ = O.ref_dposv(uplo, A, B, NB)
        tri = np.triu(F) if uplo == 121 else np.tril(F)
        np.savez_compressed(os.path.join(HERE, "posv_%d_%d_%d_%d.npz" % (uplo, N, NB, nrhs)),
                            A=A, B=B, F=tri, X=X, info=info)
    import ctypes
    L = O.reference()
    n, count, nrhs = 40, 6, 3
    for uplo in (121, 122):
        # stacked column-major (count*n) x n array; tile i (mb = nb = n) is matrix i
        A = np.asfortranarray(np.concatenate([O.ref_dplgsy(float(n), 123, n, 100 + i, n) for i in range(count)]))
        Ain = A.copy()
        t = ctypes.c_double()
        assert L.chamref_dpotrf_batch(uplo, n, count, O._ptr(A), ctypes.byref(t)) == 0
        B = np.asfortranarray(np.concatenate([O.ref_dplrnt(n, nrhs, 7 + i, n) for i in range(count)]))
        Bin = B.copy()
        # forward solve with the factors: op(T) lower-effective (L, or U^T)
        trans = 112 if uplo == 121 else 111
        assert L.chamref_dtrsm_batch(141, uplo, trans, 131, 1.0, n, nrhs, count, O._ptr(A), O._ptr(B)) == 0
        np.savez_compressed(os.path.join(HERE, "batch_%d.npz" % uplo), A=Ain, F=A, B=Bin, Y=B, n=n, count=count,
                            nrhs=nrhs, trans=trans)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
