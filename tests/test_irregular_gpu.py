"""irr_simd_* (irregular force over resident lists): CUDA library vs the
FP64 oracle (nbint.F with jpred_int.f prediction) and the reference's own
irr.avx.cpp outputs.  Tolerances: acc <= 1e-6 and jerk <= 1e-5 relative vs
FP64 per particle; nnbid identical except exact FP64 ties."""
import os

import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load_state(lib, g):
    n = g["x0"].shape[0]
    lib.irr_open(n, g["lists"].shape[1], 0)
    lib.irr_set_jp_all(g["x0"], g["v0"], g["acc2"], g["jrk6"], g["mass"], g["t0"])
    for i in range(n):
        lib.irr_set_list(i + 1, g["lists"][i])


def test_irregular_golden(nb6, orc):
    g = dict(np.load(os.path.join(GOLD, "irr_plummer1k.npz")))
    load_state(nb6, g)
    try:
        acc, jrk, nnbid = nb6.irr_firr_vec(float(g["ti"]), g["addr"])
    finally:
        nb6.irr_close(0)
    oa, oj, oid = orc.firr(float(g["ti"]), g["addr"], g["x0"], g["v0"], g["acc2"], g["jrk6"],
                           g["mass"], g["t0"], g["lists"])
    ok = g["lists"][g["addr"] - 1, 0] > 0
    assert rel_err_vec(acc[ok], oa[ok]).max() <= 1e-6
    assert rel_err_vec(jrk[ok], oj[ok]).max() <= 1e-5
    np.testing.assert_array_equal(nnbid, oid)
    assert np.all(nnbid[~ok] == -1) and np.all(acc[~ok] == 0)
    # vs the reference library (FP32 predictor): ~1e-5
    assert np.median(rel_err_vec(acc[ok], g["acc"][ok])) < 1e-5
    assert (nnbid[ok] != g["nnbid"][ok]).sum() <= 2


def _random_state(n, lmax, seed):
    from nb6b200 import ics
    rng = np.random.default_rng(seed)
    cl = ics.plummer(n, seed=seed, imf=True)
    f2 = rng.normal(size=(n, 3)) * 0.5
    fd6 = rng.normal(size=(n, 3)) * 0.2
    t0 = -rng.integers(0, 16, n) / 2048.0
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        k = int(rng.integers(0, lmax))
        ids = np.sort(rng.choice(np.delete(np.arange(1, n + 1), i), size=min(k, n - 1),
                                 replace=False))
        lists[i, 0] = len(ids)
        lists[i, 1:1 + len(ids)] = ids
    return {"x0": cl.pos, "v0": cl.vel, "acc2": f2, "jrk6": fd6, "mass": cl.mass, "t0": t0,
            "lists": lists}


@pytest.mark.parametrize("n,lmax,ni", [(40, 9, 40), (3000, 601, 1), (3000, 601, 777),
                                       (20000, 130, 5000)])
def test_irregular_random(nb6, orc, n, lmax, ni):
    g = _random_state(n, lmax, seed=n + lmax)
    addr = np.sort(np.random.default_rng(1).choice(n, ni, replace=False) + 1).astype(np.int32)
    load_state(nb6, g)
    try:
        for ti in (0.0, 1.0 / 1024):
            acc, jrk, nnbid = nb6.irr_firr_vec(ti, addr)
            oa, oj, oid = orc.firr(ti, addr, g["x0"], g["v0"], g["acc2"], g["jrk6"],
                                   g["mass"], g["t0"], g["lists"])
            ok = g["lists"][addr - 1, 0] > 0
            assert rel_err_vec(acc[ok], oa[ok]).max() <= 1e-6
            assert rel_err_vec(jrk[ok], oj[ok]).max() <= 1e-5
            np.testing.assert_array_equal(nnbid, oid)
    finally:
        nb6.irr_close(0)


def test_irregular_large_call_in_chunks(nb6, orc):
    """A large call runs in chunks whose results are downloaded and copied
    into the caller's arrays while later chunks compute: 50,000 bodies (four
    ragged chunks) against the oracle, and bit for bit against the same
    bodies split over two calls, with preallocated output arrays reused."""
    from nb6b200 import ics
    n, lmax, ni = 60000, 80, 50000
    rng = np.random.default_rng(21)
    cl = ics.plummer(n, seed=21)
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        ids = np.unique((i + rng.integers(1, n, int(rng.integers(0, lmax)))) % n) + 1
        lists[i, 0] = len(ids)
        lists[i, 1:1 + len(ids)] = ids
    g = {"x0": cl.pos, "v0": cl.vel, "acc2": rng.normal(size=(n, 3)) * 0.5,
         "jrk6": rng.normal(size=(n, 3)) * 0.2, "mass": cl.mass,
         "t0": -rng.integers(0, 16, n) / 2048.0, "lists": lists}
    addr = np.sort(rng.choice(n, ni, replace=False) + 1).astype(np.int32)
    load_state(nb6, g)
    try:
        ti = 1.0 / 1024
        out = (np.full((ni, 3), np.nan), np.full((ni, 3), np.nan), np.full(ni, -7, np.int32))
        acc, jrk, nnbid = nb6.irr_firr_vec(ti, addr, out)
        oa, oj, oid = orc.firr(ti, addr, g["x0"], g["v0"], g["acc2"], g["jrk6"], g["mass"], g["t0"], lists)
        ok = lists[addr - 1, 0] > 0
        assert ok.sum() > 0.9 * ni
        assert rel_err_vec(acc[ok], oa[ok]).max() <= 1e-6
        assert rel_err_vec(jrk[ok], oj[ok]).max() <= 1e-5
        np.testing.assert_array_equal(nnbid, oid)
        first = [a.copy() for a in (acc, jrk, nnbid)]
        h = 23457
        for part in (slice(0, h), slice(h, ni)):
            pa, pj, pn = nb6.irr_firr_vec(ti, addr[part])
            np.testing.assert_array_equal(pa, first[0][part])
            np.testing.assert_array_equal(pj, first[1][part])
            np.testing.assert_array_equal(pn, first[2][part])
        acc, jrk, nnbid = nb6.irr_firr_vec(ti, addr, out)        # the same arrays again
        for a, b in zip((acc, jrk, nnbid), first):
            np.testing.assert_array_equal(a, b)
    finally:
        nb6.irr_close(0)


def test_predicted_set_walk_equals_record_walk_bit_for_bit(nb6, orc):
    """The walk over the predicted set (every record predicted to the call's
    time once, nb6_irr_pv_ 2) and the walk that predicts each neighbour from
    its record (nb6_irr_pv_ 0) give the same bits, for a small and a large
    call; the default (1) picks one of them by size."""
    import ctypes as C
    from nb6b200 import ics
    n, lmax = 20000, 72
    rng = np.random.default_rng(33)
    cl = ics.plummer(n, seed=33)
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        ids = np.unique((i + rng.integers(1, n, int(rng.integers(0, lmax)))) % n) + 1
        lists[i, 0] = len(ids)
        lists[i, 1:1 + len(ids)] = ids
    g = {"x0": cl.pos, "v0": cl.vel, "acc2": rng.normal(size=(n, 3)) * 0.5,
         "jrk6": rng.normal(size=(n, 3)) * 0.2, "mass": cl.mass,
         "t0": -rng.integers(0, 16, n) / 2048.0, "lists": lists}
    load_state(nb6, g)
    ti = 3.0 / 4096
    mode = lambda k: nb6.lib.nb6_irr_pv_(C.byref(C.c_int(k)))    # noqa: E731
    try:
        for ni in (97, 15000):
            addr = np.sort(rng.choice(n, ni, replace=False) + 1).astype(np.int32)
            res = {}
            for k in (0, 2, 1):
                mode(k)
                res[k] = [a.copy() for a in nb6.irr_firr_vec(ti, addr)]
            for k in (2, 1):
                for a, b in zip(res[k], res[0]):
                    np.testing.assert_array_equal(a, b)
            oa, oj, oid = orc.firr(ti, addr, g["x0"], g["v0"], g["acc2"], g["jrk6"], g["mass"], g["t0"], lists)
            ok = lists[addr - 1, 0] > 0
            assert rel_err_vec(res[2][0][ok], oa[ok]).max() <= 1e-6
            assert rel_err_vec(res[2][1][ok], oj[ok]).max() <= 1e-5
            np.testing.assert_array_equal(res[2][2], oid)
    finally:
        mode(1)
        nb6.irr_close(0)


def test_irregular_updates_between_calls(nb6, orc):
    """set_jp / set_list after a firr call take effect on the next call; a
    second set of the same particle before a flush wins."""
    g = _random_state(2000, 64, seed=4)
    addr = np.arange(1, 2001, dtype=np.int32)
    load_state(nb6, g)
    try:
        nb6.irr_firr_vec(0.0, addr)
        rng = np.random.default_rng(9)
        for i in rng.choice(2000, 300, replace=False):
            g["x0"][i] += rng.normal(size=3) * 1e-3
            g["t0"][i] = 1.0 / 4096
            nb6.irr_set_jp(i + 1, g["x0"][i] + 5.0, g["v0"][i], g["acc2"][i], g["jrk6"][i],
                           g["mass"][i], g["t0"][i])     # superseded below
            nb6.irr_set_jp(i + 1, g["x0"][i], g["v0"][i], g["acc2"][i], g["jrk6"][i],
                           g["mass"][i], g["t0"][i])
            row = g["lists"][i].copy()
            row[0] = max(0, row[0] - 3)
            row[1 + row[0]:] = 0
            g["lists"][i] = row
            nb6.irr_set_list(i + 1, row)
        acc, jrk, nnbid = nb6.irr_firr_vec(1.0 / 2048, addr)
        oa, oj, oid = orc.firr(1.0 / 2048, addr, g["x0"], g["v0"], g["acc2"], g["jrk6"],
                               g["mass"], g["t0"], g["lists"])
        ok = g["lists"][:, 0] > 0
        assert rel_err_vec(acc[ok], oa[ok]).max() <= 1e-6
        np.testing.assert_array_equal(nnbid, oid)
    finally:
        nb6.irr_close(0)


def test_gpuirr_aliases(nb6):
    lib = nb6.lib
    for s in ("gpuirr_open_", "gpuirr_close_", "gpuirr_set_jp_", "gpuirr_set_list_"):
        assert hasattr(lib, s)
