"""gpupot_ (N^2 potential): CUDA library vs the FP64 oracle and the
reference's own CPU library (golden fixtures).  Tolerance: relative error
<= 1e-6 per particle vs FP64 (FP32 pair math on hi/lo differences,
double-single sums)."""
import os

import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-6


@pytest.mark.parametrize("case", ["pot_plummer1k", "pot_kroupa2k_partial"])
def test_potential_golden(nb6, orc, case):
    g = dict(np.load(os.path.join(GOLD, case + ".npz")))
    p = nb6.gpupot(g["m"], g["x"], istart=int(g["istart"]), ni=int(g["ni"]))
    po = orc.pot(g["m"], g["x"], int(g["istart"]), int(g["ni"]))
    assert rel_err_vec(p, po).max() <= TOL
    assert rel_err_vec(p, g["pot"]).max() <= 2e-6     # reference: hi/lo + 2-sum


@pytest.mark.parametrize("n,istart,ni", [(1, 1, 1), (2, 2, 1), (129, 1, 129), (1000, 17, 500),
                                         (5000, 4001, 1000), (70000, 1, 70000)])
def test_potential_sizes(nb6, orc, n, istart, ni):
    from nb6b200 import ics
    cl = ics.plummer(max(n, 2), seed=n, imf=True)
    m, x = cl.mass[:n], cl.pos[:n]
    p = nb6.gpupot(m, x, istart=istart, ni=ni)
    if n * ni > 2e9:
        sel = np.random.default_rng(0).choice(ni, 512, replace=False)
        po = np.array([orc.pot(m, x, istart + k, 1)[0] for k in sel])
        assert rel_err_vec(p[sel], po).max() <= TOL
    else:
        po = orc.pot(m, x, istart, ni)
        assert rel_err_vec(p, po).max() <= TOL if n > 1 else np.all(p == 0)


def test_potential_coincident_and_repeat(nb6, orc):
    """Coincident bodies (r2 = 0) are skipped (gpupot.gpu.cu:52); repeated
    calls with different n reuse the buffers."""
    from nb6b200 import ics
    cl = ics.plummer(3000, seed=1)
    x = cl.pos.copy()
    x[10] = x[11]
    for n in (3000, 1500, 3000):
        p = nb6.gpupot(cl.mass[:n], x[:n])
        po = orc.pot(cl.mass[:n], x[:n])
        assert rel_err_vec(p, po).max() <= TOL


def test_potential_energy_plummer(nb6):
    """Henon units: W = -1/2 sum m phi ~ -0.5 for a Plummer sphere."""
    from nb6b200 import ics
    cl = ics.plummer(20000, seed=3)
    p = nb6.gpupot(cl.mass, cl.pos)
    w = -0.5 * float((cl.mass * p).sum())
    assert abs(w + 0.5) < 0.03


def test_potential_ordered_path_stress(nb6, orc):
    """A whole-set call above 32,768 bodies takes the Morton-ordered path
    (packed far loop on tile-relative coordinates): every body's potential
    within the tolerance of the FP64 oracle, with escapers far out, close
    and coincident pairs, results in the caller's order."""
    from nb6b200 import ics
    cl = ics.king(40000, w0=6.0, seed=11, imf=True, binary_fraction=0.05)
    x = cl.pos.copy()
    rng = np.random.default_rng(2)
    k = rng.choice(len(x), len(x) // 100, replace=False)
    x[k] *= 50.0                                            # escapers
    k = rng.choice(len(x), len(x) // 20, replace=False)
    x[k[1:]] = x[k[:-1]] + rng.normal(size=(len(k) - 1, 3)) * 1e-5   # close pairs
    x[7] = x[8]                                             # a coincident pair
    p = nb6.gpupot(cl.mass, x)
    po = orc.pot(cl.mass, x)
    assert rel_err_vec(p, po).max() <= TOL
