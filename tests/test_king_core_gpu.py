"""Regular force on a King W0=6 cluster of 262,144 stars (5% binaries as c.m.
bodies), every i of two 1024-i calls against the FP64 oracle.

The j set is above the spatial order's minimum size, so the packed kernel
runs with its far-tile loop (tile-relative differences, 1/r from the
approximation) on most (warp, tile) pairs.  One call is a slice of the
full-evaluation call sequence (bodies in random radial order, a sample of
the whole cluster); the other is the 1024 bodies nearest the centre, the
King core, where each body's regular force is a sum of many near terms that
cancel most.  Both run on the autotuned plan and on the packed kernel
forced.  Tolerances: acceleration and potential <= 1e-6 relative per
particle, jerk <= 1e-5; neighbour lists identical row for row.
"""
import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu

N_STARS = 262144


@pytest.fixture(scope="module")
def king():
    from nb6b200 import ics
    return ics.king(N_STARS, w0=6.0, seed=777, imf=True, binary_fraction=0.05, nnbopt=50)


def _calls(cl, chunk=1024):
    n = cl.n
    centre = (cl.mass[:, None] * cl.pos).sum(0) / cl.mass.sum()
    byr = np.argsort(((cl.pos - centre) ** 2).sum(1), kind="stable")
    k = (n // chunk) // 2
    return {"sequence": np.arange(k * chunk, (k + 1) * chunk),
            "core": np.sort(byr[:chunk])}


@pytest.mark.parametrize("variant", [0, 11])
def test_king_core_and_sequence_calls_vs_fp64(nb6, orc, king, variant):
    import ctypes as C
    cl = king
    h2 = cl.rs ** 2
    raw = nb6.lib
    raw.nb6_regf_tune_(C.byref(C.c_int(variant)), C.byref(C.c_int(0)))
    nb6.gpunb_open(cl.n + 10, 0)
    try:
        nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
        for name, idx in _calls(cl).items():
            acc, jrk, pot, lst = nb6.gpunb_regf(h2[idx], cl.dtr[idx], cl.pos[idx], cl.vel[idx],
                                                512, 400, 0)
            oa, oj, op, ol = orc.regf(cl.mass, cl.pos, cl.vel, h2[idx], cl.dtr[idx], cl.pos[idx],
                                      cl.vel[idx], 512, 400, 0)
            np.testing.assert_array_equal(lst, ol, err_msg=name)
            ok = ol[:, 0] >= 0
            assert ok.sum() > 900, (name, ok.sum())
            ea = rel_err_vec(acc[ok], oa[ok])
            ej = rel_err_vec(jrk[ok], oj[ok])
            ep = rel_err_vec(pot[ok], op[ok])
            print(f"{name} variant {variant}: acc max {ea.max():.2e} p99.9 "
                  f"{np.quantile(ea, 0.999):.2e}, jerk max {ej.max():.2e}, pot max {ep.max():.2e}")
            assert ea.max() <= 1e-6, (name, ea.max())
            assert ep.max() <= 1e-6, (name, ep.max())
            assert ej.max() <= 1e-5, (name, ej.max())
    finally:
        nb6.gpunb_close()
        raw.nb6_regf_tune_(C.byref(C.c_int(0)), C.byref(C.c_int(0)))
