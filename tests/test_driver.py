"""The C++ block-step driver (Hermite + Ahmad-Cohen, singles) on the
reference's own CPU force libraries: a CPU-only check that the driver itself
conserves energy and keeps neighbour counts near NNBOPT, so that the GPU
comparison (test_driver_gpu.py) isolates the force path."""
import numpy as np
import pytest


def _ref_backend(orc):
    for lib in ("reg", "irr", "pot"):
        if not orc.ref_available(lib):
            pytest.skip("reference CPU libraries not built")
    return {"reg": orc.ref_path("reg"), "irr": orc.ref_path("irr"), "pot": orc.ref_path("pot")}


def test_driver_reference_backend_plummer1k_t1(orc):
    from nb6b200 import drive, ics
    cl = ics.plummer(1024, seed=43532)
    r = drive.run(_ref_backend(orc), cl.mass, cl.pos, cl.vel, tcrit=1.0, dt_out=0.125)
    assert r.stats["t_end"] == 1.0
    assert r.de_max < 1e-5, r.de_max
    nb = r.stats["nb_sum"] / r.stats["reg_steps"]
    assert 25 < nb < 100, nb
    assert abs(r.etot[0] + 0.25) < 0.03          # Henon units
    assert np.all(np.isfinite(r.x)) and np.all(np.isfinite(r.v))


def test_driver_is_deterministic(orc):
    from nb6b200 import drive, ics
    cl = ics.plummer(512, seed=3)
    b = _ref_backend(orc)
    r1 = drive.run(b, cl.mass, cl.pos, cl.vel, tcrit=0.25)
    r2 = drive.run(b, cl.mass, cl.pos, cl.vel, tcrit=0.25)
    np.testing.assert_array_equal(r1.x, r2.x)
    assert r1.stats["blocks"] == r2.stats["blocks"]
