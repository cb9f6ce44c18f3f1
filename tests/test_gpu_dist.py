"""The multi-GPU dispatcher's product path on one GPU: a world of one rank
(gloo group in this process), whose worker is the library's serving loop on
cuda:0.  Mixed orders take both of the server's paths (batched FP64 and the
mixed solver); results are checked against an FP64 solve."""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_dispatcher_world_of_one_on_the_gpu(cb, orc):
    import torch.distributed as dist
    from chameleon_b200 import dist as cd
    port = _free_port()
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=timedelta(seconds=30))
    dist.init_process_group("gloo", store=store, rank=0, world_size=1, timeout=timedelta(seconds=30))
    try:
        d = cd.Dispatcher(cd.make_group(), store_addr=("127.0.0.1", port))
        rng = np.random.default_rng(3)
        sizes = [16, 100, 300, 700, 1500, 40, 2600]
        mats = [orc.dplgsy(float(n), n, 11 + i) for i, n in enumerate(sizes)]
        reqs = [cd.Request(A, rng.standard_normal((A.shape[0], 1 + i % 4)), factor_key=i)
                for i, A in enumerate(mats)]
        d.dposv_batch(reqs)
        for r, A in zip(reqs, mats):
            assert r.status == 0 and r.rank == 0
            assert np.abs(A @ r.X - r.B).max() <= 1e-10 * np.abs(r.B).max() * A.shape[0]
        # serving: reuse the kept factors
        again = [d.submit(cd.Request(None, rng.standard_normal((A.shape[0], 2)), factor_key=i))
                 for i, A in enumerate(mats)]
        d.drain()
        for r, A in zip(again, mats):
            assert r.status == 0
            assert np.abs(A @ r.X - r.B).max() <= 1e-10 * np.abs(r.B).max() * A.shape[0]
        d.close()
    finally:
        dist.destroy_process_group()
