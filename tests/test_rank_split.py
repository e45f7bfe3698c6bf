"""The regular force and the potential split over ranks (nb6b200.rank_split)
on CPU: gloo ranks, one process each as torchrun launches them, with the FP64
oracle standing in for each rank's GPU library.  Every rank must end with the
results of a single-rank call over the whole active list, bit for bit:
ragged pieces, pieces that are empty, pieces that cross the per-call limit,
and overflowing neighbour lists (-nnb rows) included; and likewise for the
potential of every body, split above a size threshold, and for the
irregular force of an active list."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _OracleForceLib:
    """gpunb_send / gpunb_regf of the FP64 oracle (the checker), with the
    ForceLib call signatures."""

    def __init__(self, orc):
        self.orc = orc
        self.j = None

    def gpunb_send(self, m, x, v):
        self.j = (np.array(m), np.array(x), np.array(v))

    def gpunb_regf(self, h2, dtr, xi, vi, lmax, nnbmax, m_flag=0):
        return self.orc.regf(*self.j, h2, dtr, xi, vi, lmax, nnbmax, m_flag)

    def gpupot(self, m, x, istart=1, ni=None, irank=0):
        return self.orc.pot(m, x, istart, ni)

    def irr_state(self, *state):
        self.irr = state

    def irr_firr_vec(self, ti, addr):
        return self.orc.firr(ti, addr, *self.irr)


# (active count, chunk, nnbmax): ragged pieces, an empty list, fewer active
# particles than ranks, pieces crossing the call limit, overflowing lists.
CASES = [(256, 1024, 40), (5, 1024, 40), (1, 1024, 40), (0, 1024, 40), (200, 7, 40), (97, 16, 3)]
# (bodies, split threshold): split with ragged pieces, a piece that is empty,
# and a set small enough to be evaluated whole on every rank.
POT_CASES = [(256, 100), (5, 0), (2, 0), (256, 50000)]
# active counts of an irregular block: ragged, fewer than ranks, empty.
IRR_CASES = [256, 77, 2, 0]


def _irr_state(cl, k=12):
    """Irregular state of the cluster: records at t0 = 0 and lists of the k
    nearest bodies (rows [nnb, 1-based ids])."""
    rng = np.random.default_rng(3)
    n = cl.n
    d2 = ((cl.pos[:, None, :] - cl.pos[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    near = np.argsort(d2, axis=1)[:, :k]
    lists = np.zeros((n, k + 4), dtype=np.int32)
    lists[:, 0] = k
    lists[:, 1:k + 1] = np.sort(near, axis=1) + 1
    acc2 = rng.normal(scale=0.5, size=(n, 3))
    jrk6 = rng.normal(scale=0.1, size=(n, 3))
    return (cl.pos, cl.vel, acc2, jrk6, cl.mass, np.zeros(n), lists)


def _cases():
    import oracle
    from nb6b200 import ics
    cl = ics.plummer(256, seed=43532, nnbopt=20)
    h2 = cl.h2(0)
    rng = np.random.default_rng(7)
    out = []
    for nl, chunk, nnbmax in CASES:
        act = np.sort(rng.choice(cl.n, size=nl, replace=False))
        out.append((cl, h2[act], cl.dtr[act], cl.pos[act], cl.vel[act], chunk, nnbmax))
    return oracle, out


def _rank(rank, world, port, out):
    import datetime
    import sys
    for p in (os.path.join(ROOT, "nbody6ppgpu-beijing_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch.distributed as dist
    from nb6b200.rank_split import RankSplit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc, cases = _cases()
        res = []
        for cl, h2, dtr, xi, vi, chunk, nnbmax in cases:
            lmax = 64
            split = RankSplit(_OracleForceLib(orc), chunk=chunk)
            split.send(cl.mass, cl.pos, cl.vel)
            got = split.regf(h2, dtr, xi, vi, lmax, nnbmax, 0)
            want = orc.regf(cl.mass, cl.pos, cl.vel, h2, dtr, xi, vi, lmax, nnbmax, 0)
            same = all(np.array_equal(g, w) for g, w in zip(got, want))
            shapes = tuple(g.shape for g in got)
            nover = int((got[3][:, 0] < 0).sum()) if len(got[3]) else 0
            res.append((same, shapes, split.piece(len(h2)), nover))
        pots = []
        for n, split_min in POT_CASES:
            cl = cases[0][0]
            m, x = cl.mass[:n], cl.pos[:n]
            got = split.gpupot(m, x, split_min)
            pots.append((got.shape, bool(np.array_equal(got, orc.pot(m, x)))))
        irrs = []
        cl = cases[0][0]
        lib = _OracleForceLib(orc)
        lib.irr_state(*_irr_state(cl))
        split = RankSplit(lib)
        rng = np.random.default_rng(11)
        for nl in IRR_CASES:
            addr = (np.sort(rng.choice(cl.n, size=nl, replace=False)) + 1).astype(np.int32)
            got = split.firr(0.01, addr)
            want = orc.firr(0.01, addr, *lib.irr)
            irrs.append((tuple(g.shape for g in got), all(np.array_equal(g, w) for g, w in zip(got, want))))
        out[rank] = (res, pots, irrs)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_end_with_the_single_rank_results(world):
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    from nb6b200.rank_split import active_split
    for rank in range(world):
        regs, pots, irrs = res[rank]
        assert len(regs) == len(CASES)
        for nl, (shapes, same) in zip(IRR_CASES, irrs):
            assert shapes == ((nl, 3), (nl, 3), (nl,)) and same, (rank, nl)
        for (n, _), (shape, same) in zip(POT_CASES, pots):
            assert shape == (n,) and same, (rank, n)
        for (nl, chunk, nnbmax), (same, shapes, piece, nover) in zip(CASES, regs):
            assert same, (rank, nl, chunk, nnbmax)
            assert shapes == ((nl, 3), (nl, 3), (nl,), (nl, 64))
            start, count = active_split(nl, world)
            assert piece == (start[rank], count[rank])
            if nnbmax == 3 and nl > 0:
                assert nover > 0  # the overflow rows travelled too


def _fortran_split(nl, isize):
    """intgrt.F:955-968 as written, 1-based ista, inum zeroed past the list."""
    inl = nl // isize
    idiff = nl - isize * inl
    irun, ista, inum = 0, [], []
    for ix in range(1, isize + 1):
        n = inl + (1 if ix <= idiff else 0)
        s = irun + 1
        if s > nl:
            n = 0
        ista.append(s)
        inum.append(n)
        irun += n
    return ista, inum


def test_active_split_matches_the_reference_cut():
    from nb6b200.rank_split import active_split
    for size in range(1, 9):
        for nl in list(range(0, 40)) + [1023, 1024, 1025, 65536, 996147]:
            ista, inum = _fortran_split(nl, size)
            start, count = active_split(nl, size)
            assert count == inum
            assert sum(count) == nl
            for s, i, c in zip(start, ista, count):
                if c:
                    assert s == i - 1


def test_one_rank_without_a_process_group_evaluates_everything():
    import oracle
    from nb6b200 import ics
    from nb6b200.rank_split import RankSplit
    cl = ics.plummer(128, seed=5, nnbopt=20)
    h2 = cl.h2(0)
    split = RankSplit(_OracleForceLib(oracle), chunk=50)
    assert (split.rank, split.size) == (0, 1)
    split.send(cl.mass, cl.pos, cl.vel)
    got = split.regf(h2, cl.dtr, cl.pos, cl.vel, 64, 40, 0)
    want = oracle.regf(cl.mass, cl.pos, cl.vel, h2, cl.dtr, cl.pos, cl.vel, 64, 40, 0)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert np.array_equal(split.gpupot(cl.mass, cl.pos, 0), oracle.pot(cl.mass, cl.pos))


def test_chunk_outside_the_call_limit_is_rejected():
    from nb6b200.rank_split import RankSplit
    with pytest.raises(ValueError):
        RankSplit(None, chunk=0)
    with pytest.raises(ValueError):
        RankSplit(None, chunk=1025)


def _rank_device(rank, world, port, out):
    """The device-resident split with gloo ranks on CPU: each rank's piece
    comes from the FP64 oracle as CPU tensors in place of the library's
    device output rows, then the padded all-gather of regf_device."""
    import datetime
    import sys
    for p in (os.path.join(ROOT, "nbody6ppgpu-beijing_b200"), os.path.join(ROOT, "oracle")):
        sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    from nb6b200.rank_split import NREC, RankSplit
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        orc, cases = _cases()
        res = []
        for cl, h2, dtr, xi, vi, chunk, nnbmax in cases:
            lmax = 64
            W = min(nnbmax, lmax - 1) + 1
            split = RankSplit(None, chunk=chunk)

            def own(d_h2, d_dtr, d_xi, d_vi, lmax_, nnbmax_, m_flag, s, n, pad):
                rec = torch.zeros((pad, NREC), dtype=torch.float64)
                lst = torch.zeros((pad, W), dtype=torch.int32)
                if n:
                    a, j, p, l = orc.regf(cl.mass, cl.pos, cl.vel, d_h2[s:s + n].numpy(), d_dtr[s:s + n].numpy(),
                                          d_xi[s:s + n].numpy(), d_vi[s:s + n].numpy(), lmax_, nnbmax_, m_flag)
                    rec[:n, 0:3] = torch.from_numpy(a)
                    rec[:n, 3:6] = torch.from_numpy(j)
                    rec[:n, 6] = torch.from_numpy(p)
                    lst[:n] = torch.from_numpy(l[:, :W])
                return rec, lst, None

            split._own_device = own
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64))
            rec, lst = split.regf_device(t(h2), t(dtr), t(xi), t(vi), lmax, nnbmax, 0)
            want = orc.regf(cl.mass, cl.pos, cl.vel, h2, dtr, xi, vi, lmax, nnbmax, 0)
            same = (np.array_equal(rec[:, 0:3].numpy(), want[0]) and np.array_equal(rec[:, 3:6].numpy(), want[1])
                    and np.array_equal(rec[:, 6].numpy(), want[2])
                    and np.array_equal(lst.numpy(), want[3][:, :W]))
            res.append((same, tuple(rec.shape), tuple(lst.shape)))
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_device_split_gathers_the_single_rank_rows(world):
    import torch.multiprocessing as mp
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_device, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        assert len(res[rank]) == len(CASES)
        for (nl, chunk, nnbmax), (same, rshape, lshape) in zip(CASES, res[rank]):
            assert same, (rank, nl, chunk, nnbmax)
            assert rshape == (nl, 7) and lshape == (nl, min(nnbmax, 63) + 1)
