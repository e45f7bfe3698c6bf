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
