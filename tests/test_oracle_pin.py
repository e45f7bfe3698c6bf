"""Pin the FP64 oracle against the reference's own outputs (CPU only).

The reference ships no golden vectors; tests/golden/*.npz were produced by its
CPU libraries (reg.avx.cpp, pot.avx.cpp, irr.avx.cpp) -- see make_golden.py.
The reference regular kernel works on FP32 absolute coordinates with one
Newton step (reg.avx.cpp:250-291), so it agrees with FP64 to ~1e-5 relative;
pot.avx.cpp uses hi/lo differences and 2-sum accumulation (~1e-7);
irr.avx.cpp predicts in FP32 on hi/lo positions (~1e-6).
"""
import os

import numpy as np
import pytest

from parity import align_to_lists, compare_lists, rel_err_vec

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


REG_CASES = ["reg_plummer1k", "reg_plummer1k_overflow", "reg_kroupa2k_mflag"]


@pytest.mark.parametrize("case", REG_CASES)
def test_oracle_regular_vs_reference_golden(orc, case):
    g = _load(case)
    m_flag = int(g["m_flag"])
    acc, jrk, pot, lst = orc.regf(g["mj"], g["xj"], g["vj"], g["h2"], g["dtr"], g["xi"],
                                  g["vi"], int(g["lmax"]), int(g["nnbmax"]), m_flag)
    # move boundary pairs the two sides classify differently before comparing
    acc, jrk, pot = align_to_lists(acc, jrk, pot, lst, g["list"], g)
    ok = (lst[:, 0] >= 0) & (g["list"][:, 0] >= 0)
    ea = rel_err_vec(acc[ok], g["acc"][ok])
    ej = rel_err_vec(jrk[ok], g["jrk"][ok])
    ep = rel_err_vec(pot[ok], g["pot"][ok])
    # reference = FP32 absolute coordinates: ~1e-5 relative to FP64
    assert np.median(ea) < 2e-5 and ea.max() < 5e-4, (np.median(ea), ea.max())
    assert np.median(ej) < 5e-5 and ej.max() < 5e-3, (np.median(ej), ej.max())
    assert np.median(ep) < 2e-5 and ep.max() < 5e-4, (np.median(ep), ep.max())
    # lists: identical except pairs inside the FP32 boundary band
    res = compare_lists(lst, g["list"], g, band=1e-4, m_flag=m_flag)
    assert res["pairs_out_of_band"] == 0, res
    assert res["overflow_mismatch"] == 0, res
    assert res["unsorted_rows"] == 0, res
    # overflow rows carry -nnb, same count on both sides up to band pairs
    both = (lst[:, 0] < 0) & (g["list"][:, 0] < 0)
    assert np.all(np.abs(lst[both, 0] - g["list"][both, 0]) <= 2)


def test_oracle_overflow_case_has_both_kinds():
    g = _load("reg_plummer1k_overflow")
    n = g["list"][:, 0]
    assert (n < 0).any() and (n >= 0).any()


@pytest.mark.parametrize("case", ["pot_plummer1k", "pot_kroupa2k_partial"])
def test_oracle_potential_vs_reference_golden(orc, case):
    g = _load(case)
    pot = orc.pot(g["m"], g["x"], int(g["istart"]), int(g["ni"]))
    e = rel_err_vec(pot, g["pot"])
    assert e.max() < 2e-6, e.max()


def test_oracle_irregular_vs_reference_golden(orc):
    g = _load("irr_plummer1k")
    acc, jrk, nnbid = orc.firr(float(g["ti"]), g["addr"], g["x0"], g["v0"], g["acc2"],
                               g["jrk6"], g["mass"], g["t0"], g["lists"])
    nnb = g["lists"][g["addr"] - 1, 0]
    ok = nnb > 0
    ea = rel_err_vec(acc[ok], g["acc"][ok])
    ej = rel_err_vec(jrk[ok], g["jrk"][ok])
    assert np.median(ea) < 1e-5 and ea.max() < 1e-3, (np.median(ea), ea.max())
    assert np.median(ej) < 1e-4 and ej.max() < 1e-2, (np.median(ej), ej.max())
    # nearest neighbour agrees except FP32 near-ties
    mism = np.nonzero(nnbid[ok] != g["nnbid"][ok])[0]
    assert len(mism) <= 2, mism
    # empty lists: the oracle returns -1 (nbint.F:27), forces are zero
    assert np.all(nnbid[~ok] == -1)
    assert np.all(acc[~ok] == 0.0)


def test_live_reference_reproduces_golden(orc):
    """When the reference libraries are built here, they reproduce the
    committed fixtures bit for bit (the fixtures are not stale)."""
    if not orc.ref_available("reg"):
        pytest.skip("reference CPU libraries not built")
    import nb6b200.abi as abi
    g = _load("reg_plummer1k")
    lib = abi.ForceLib(orc.ref_lib("reg"), "ref")
    lib.gpunb_open(len(g["mj"]) + 10, 0)
    lib.gpunb_send(g["mj"], g["xj"], g["vj"])
    acc, jrk, pot, lst = lib.gpunb_regf(g["h2"], g["dtr"], g["xi"], g["vi"], int(g["lmax"]),
                                        int(g["nnbmax"]), int(g["m_flag"]))
    lib.gpunb_close()
    np.testing.assert_array_equal(acc, g["acc"])
    np.testing.assert_array_equal(pot, g["pot"])
    np.testing.assert_array_equal(lst, g["list"])
