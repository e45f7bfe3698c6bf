"""The device-resident split regular force (RankSplit.regf_device) through
the real library on the GPU: one NCCL rank (each GPU call here has one GPU,
and two ranks may not share a device), so the all-gather is the trivial
one, but every other step is the multi-rank one -- nb6_regf_device_ on
device-resident i data in calls of at most 1024, each call's output rows
copied on the library's stream into the send buffer, NCCL on that stream.
The rows must equal gpunb_regf_'s on the same inputs, bit for bit."""
import datetime
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_device_split_one_nccl_rank_equals_gpunb_regf(nb6):
    import torch
    import torch.distributed as dist
    from nb6b200 import ics
    from nb6b200.rank_split import RankSplit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    cl = ics.plummer(20000, seed=3, imf=True)
    nb6.gpunb_open(cl.n + 10, 0)
    try:
        nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
        isel = np.sort(np.random.default_rng(4).choice(cl.n, 2500, replace=False))
        h2, dtr, x, v = cl.h2(0)[isel], cl.dtr[isel], cl.pos[isel], cl.vel[isel]
        split = RankSplit(nb6)
        dev = split.device
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
        rec, lst = split.regf_device(t(h2), t(dtr), t(x), t(v), 512, 400, 0)
        rec, lst = rec.cpu().numpy(), lst.cpu().numpy()
        W = lst.shape[1]
        assert rec.shape == (2500, 7) and W == 401
        for a in range(0, 2500, 1024):
            b = min(2500, a + 1024)
            acc, jrk, pot, l = nb6.gpunb_regf(h2[a:b], dtr[a:b], x[a:b], v[a:b], 512, 400, 0)
            np.testing.assert_array_equal(rec[a:b, 0:3], acc)
            np.testing.assert_array_equal(rec[a:b, 3:6], jrk)
            np.testing.assert_array_equal(rec[a:b, 6], pot)
            for r in range(b - a):
                n = l[r, 0]
                assert lst[a + r, 0] == n
                if n > 0:
                    np.testing.assert_array_equal(lst[a + r, 1:1 + n], l[r, 1:1 + n])
    finally:
        nb6.gpunb_close()
        dist.destroy_process_group()
