"""Randomised parity of the regular force against the FP64 oracle, aimed at
the spatially ordered j set and its far-tile path: clusters above the order's
minimum size with escapers far out, close pairs, ragged radii and regular
steps, both m_flag values, N_active from a few to all bodies.  Lists must be
identical and forces within the parity tolerances."""
import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", range(8))
def test_regular_random_configurations(nb6, orc, seed):
    from nb6b200 import ics
    rng = np.random.default_rng(seed)
    n = int(rng.choice([33000, 40000, 50000]))
    cl = ics.plummer(n, seed=seed, imf=bool(seed % 2))
    x, v = cl.pos.copy(), cl.vel.copy()
    k = rng.choice(n, n // 100, replace=False)
    x[k] *= 30.0                                          # escapers
    v[k] *= 3.0
    k = rng.choice(n, n // 20, replace=False)
    x[k[1:]] = x[k[:-1]] + rng.normal(size=(len(k) - 1, 3)) * 1e-4   # close pairs
    rs = cl.rs * rng.uniform(0.3, 3.0, n)
    dtr = 2.0 ** -rng.integers(3, 12, n).astype(float)
    mf = int(seed % 4 == 1)
    h2 = rs ** 2 if not mf else rs ** 2 / cl.mass.mean()
    ni = int(rng.choice([7, 300, 1024, 4096]))
    isel = np.sort(rng.choice(n, ni, replace=False))
    nb6.gpunb_open(n + 10, 0)
    try:
        nb6.gpunb_send(cl.mass, x, v)
        acc, jrk, pot, lst = nb6.gpunb_regf(h2[isel], dtr[isel], x[isel], v[isel], 512, 400, mf)
    finally:
        nb6.gpunb_close()
    oa, oj, op, ol = orc.regf(cl.mass, x, v, h2[isel], dtr[isel], x[isel], v[isel], 512, 400, mf)
    np.testing.assert_array_equal(lst[:, 0], ol[:, 0])
    for r in range(ni):
        c = lst[r, 0]
        if c > 0:
            np.testing.assert_array_equal(lst[r, 1:1 + c], ol[r, 1:1 + c])
    ok = ol[:, 0] >= 0
    if ok.any():
        assert rel_err_vec(acc[ok], oa[ok]).max() <= 1e-6
        assert rel_err_vec(pot[ok], op[ok]).max() <= 1e-6
        assert rel_err_vec(jrk[ok], oj[ok]).max() <= 1e-5
