"""Plummer N = 65,536 with a Kroupa IMF: the active set of each
power-of-two timestep level (a block at a time that is a multiple of 2^-l
activates every body whose regular step is at most 2^-l).  Levels are drawn
so that each holds about half the bodies of the one above, so N_active runs
from all N bodies down to one.  Force, jerk and potential errors against
the FP64 oracle, reported per level, each within the stated tolerances
(acc and pot <= 1e-6, jerk <= 1e-5); neighbour lists identical."""
import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu


def test_force_error_per_timestep_level(nb6, orc):
    from nb6b200 import ics
    cl = ics.plummer(65536, seed=2026, imf=True)
    # levels drawn so that each deeper level holds about half the bodies of
    # the one above: N_active runs from N down to a single body
    u = np.random.default_rng(7).random(cl.n)
    lev = np.minimum(3 + np.floor(-np.log2(u)).astype(int), 22)
    cl.dtr = 2.0 ** -lev.astype(float)
    h2 = cl.h2(0)
    nb6.gpunb_open(cl.n + 10, 0)
    rows = []
    try:
        nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
        for l in range(lev.min(), lev.max() + 1):
            act = np.nonzero(lev >= l)[0]
            if len(act) == 0:
                continue
            acc, jrk, pot, lst = nb6.gpunb_regf(h2[act], cl.dtr[act], cl.pos[act], cl.vel[act],
                                                512, 400, 0)
            sel = np.sort(np.random.default_rng(l).choice(len(act), min(len(act), 384), replace=False))
            a = act[sel]
            oa, oj, op, ol = orc.regf(cl.mass, cl.pos, cl.vel, h2[a], cl.dtr[a], cl.pos[a],
                                      cl.vel[a], 512, 400, 0)
            np.testing.assert_array_equal(lst[sel, 0], ol[:, 0])
            for r, s in enumerate(sel):
                n = lst[s, 0]
                if n > 0:
                    np.testing.assert_array_equal(lst[s, 1:1 + n], ol[r, 1:1 + n])
            ok = ol[:, 0] >= 0
            ea = rel_err_vec(acc[sel][ok], oa[ok])
            ej = rel_err_vec(jrk[sel][ok], oj[ok])
            ep = rel_err_vec(pot[sel][ok], op[ok])
            rows.append((l, len(act), ea.max(), np.median(ea), ej.max(), ep.max()))
            assert ea.max() <= 1e-6 and ep.max() <= 1e-6 and ej.max() <= 1e-5, rows[-1]
    finally:
        nb6.gpunb_close()
    print("\nlevel  dt        N_active  acc max   acc med   jrk max   pot max")
    for l, na, am, amed, jm, pm in rows:
        print(f"{l:5d}  2^-{l:<5d}  {na:8d}  {am:.2e}  {amed:.2e}  {jm:.2e}  {pm:.2e}")
    assert rows[0][1] == cl.n and rows[-1][1] <= 4
