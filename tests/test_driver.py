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


def test_ensemble_per_cluster_calls_reproduce_each_cluster_alone(orc):
    """The ensemble driver (all clusters on one block clock, one irregular
    call per block for all of them) with per-cluster regular calls follows
    each cluster's own trajectory exactly: on the reference's deterministic
    CPU libraries the final state and energies equal those of the
    single-cluster driver run on each cluster alone, bit for bit."""
    from nb6b200 import drive, ics
    b = _ref_backend(orc)
    cls = [ics.plummer(300, seed=11), ics.plummer(520, seed=12, imf=True), ics.plummer(200, seed=13)]
    ens = drive.run_ensemble(b, cls, batched=False, tcrit=0.25, dt_out=0.125)
    assert ens.stats["t_end"] == 0.25
    for c, cl in enumerate(cls):
        alone = drive.run(b, cl.mass, cl.pos, cl.vel, tcrit=0.25, dt_out=0.125)
        np.testing.assert_array_equal(ens.x[c], alone.x)
        np.testing.assert_array_equal(ens.v[c], alone.v)
        np.testing.assert_array_equal(ens.energy[:, c, 2], alone.etot)
    # blocks: the union of the clusters' block times
    assert ens.stats["irr_steps"] > 0 and ens.stats["reg_steps"] > 0


def test_driver_logs_learning_samples(orc):
    """mlp_mode 1 keeps the Ahmad-Cohen trajectory unchanged and logs one
    (features, target) sample per regular step that has a predecessor."""
    from nb6b200 import drive, ics
    b = _ref_backend(orc)
    cl = ics.plummer(400, seed=21)
    plain = drive.run(b, cl.mass, cl.pos, cl.vel, tcrit=0.25)
    logged = drive.run(b, cl.mass, cl.pos, cl.vel, tcrit=0.25, mlp_mode=1, sample_cap=100000)
    np.testing.assert_array_equal(plain.x, logged.x)
    s = logged.samples
    assert s.shape[1] == 6 and len(s) == logged.stats["nsamples"]
    assert len(s) >= logged.stats["reg_steps"] - 2 * cl.n
    assert np.all(np.isfinite(s))
    # feature 0 is log(1 + nnb) with self counted: nnb in a sane range
    nnb = np.exp(s[:, 0]) - 1
    assert 5 < np.median(nnb) < 200
