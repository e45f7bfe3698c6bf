"""Ensemble of independent clusters on libnb6b200 (the 256-cluster method at small
size): every force kind issued once per block for all clusters
(nb6_irr_predict_send_ + nb6_regf_seg_ + one irr_simd_firr_vec_), against
each cluster integrated alone with the plain method on the same GPU."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clusters(k, seed):
    from nb6b200 import ics
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(512), np.log(2048), k)).astype(int)
    return [ics.plummer(int(n), seed=seed + 10 * c, imf=True) for c, n in enumerate(sizes)]


def test_ensemble_unbatched_equals_alone_bit_for_bit(nb6):
    """With per-cluster regular calls and the autotuner off (fixed kernel
    choice), the GPU ensemble reproduces each cluster alone exactly."""
    from nb6b200 import drive
    ours = drive.backend_paths("nb6b200")
    cls = _clusters(3, 40)
    raw = nb6.lib
    raw.nb6_regf_autotune_(C.byref(C.c_int(0)))
    try:
        ens = drive.run_ensemble(ours, cls, batched=False, tcrit=0.25)
        for c, cl in enumerate(cls):
            alone = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=0.25)
            np.testing.assert_array_equal(ens.x[c], alone.x)
            np.testing.assert_array_equal(ens.energy[:, c, 2], alone.etot)
    finally:
        raw.nb6_regf_autotune_(C.byref(C.c_int(1)))


def test_ensemble_batched_energy_matches_alone(nb6):
    """Batched ensemble to T = 1: every cluster conserves energy as well as
    when integrated alone (the forces differ only by rounding), with far
    fewer regular-force calls."""
    from nb6b200 import drive
    ours = drive.backend_paths("nb6b200")
    cls = _clusters(8, 60)
    ens = drive.run_ensemble(ours, cls, batched=True, tcrit=1.0, dt_out=0.125)
    assert ens.stats["t_end"] == 1.0
    de_alone, calls_alone, wall_alone = [], 0, 0.0
    for cl in cls:
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=1.0, dt_out=0.125)
        de_alone.append(r.de_max)
        calls_alone += r.stats["reg_calls"]
        wall_alone += r.stats["wall_total"]
    de_alone = np.array(de_alone)
    de_ens = ens.de_max
    print(f"\nper-cluster dE ensemble {np.array2string(de_ens, precision=2)}\n"
          f"per-cluster dE alone    {np.array2string(de_alone, precision=2)}\n"
          f"regular calls {ens.stats['reg_calls']} vs {calls_alone}; wall {ens.stats['wall_total']:.2f}s "
          f"vs {wall_alone:.2f}s")
    # energy error per cluster within 10% of the same cluster alone (the
    # contract's bound on drift vs the plain method)
    assert np.all(de_ens <= 1.10 * de_alone + 1e-7), (de_ens, de_alone)
    assert ens.stats["reg_calls"] < calls_alone
    # the same initial energies (same bodies, FP64-accurate potentials)
    e0 = np.array([drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=0.0).etot[0] for cl in cls])
    np.testing.assert_allclose(ens.energy[0, :, 2], e0, rtol=1e-12)


def test_device_corrector_equals_host_corrector_bit_for_bit(nb6):
    """The batched ensemble with the irregular corrector on the device
    (nb6_irr_correct_) follows exactly the trajectory of the same run with
    the corrector on the host: same final state and energies, bit for bit."""
    from nb6b200 import drive
    ours = drive.backend_paths("nb6b200")
    cls = _clusters(4, 80)
    dev = drive.run_ensemble(ours, cls, batched=True, dev_corrector=True, tcrit=0.5, dt_out=0.125)
    host = drive.run_ensemble(ours, cls, batched=True, dev_corrector=False, tcrit=0.5, dt_out=0.125)
    assert dev.stats["irr_steps"] == host.stats["irr_steps"] > 0
    assert dev.stats["reg_steps"] == host.stats["reg_steps"]
    for c in range(len(cls)):
        np.testing.assert_array_equal(dev.x[c], host.x[c])
        np.testing.assert_array_equal(dev.v[c], host.v[c])
    np.testing.assert_array_equal(dev.energy, host.energy)


@pytest.mark.parametrize("small_lists,m_flag", [(False, 0), (True, 0), (False, 1)])
def test_device_regular_corrector_equals_host_corrector_bit_for_bit(nb6, small_lists, m_flag):
    """Both correctors on the device (nb6_irr_correct_ + nb6_regf_correct_),
    and both plus the block clock (nb6_blocks_run_), against both on the
    host (the same segmented regular-force call for every block): same
    blocks, steps, neighbour counts, final state and
    energies, bit for bit.  With small_lists the neighbour lists overflow
    (NNBMAX 24) so the shrink-and-retry path runs too."""
    from nb6b200 import drive
    ours = drive.backend_paths("nb6b200")
    cls = _clusters(4, 90)
    kw = dict(batched=True, tcrit=0.5, dt_out=0.125, m_flag=m_flag)
    if small_lists:
        kw.update(nnbopt=12, nnbmax=24, lmax=32, tcrit=0.25)
    dev = drive.run_ensemble(ours, cls, dev_corrector=2, **kw)
    host = drive.run_ensemble(ours, cls, dev_corrector=0, seg_single=True, **kw)
    # and with the block clock on the device as well (nb6_blocks_run_)
    clk = drive.run_ensemble(ours, cls, dev_corrector=3, **kw)
    for run in (dev, clk):
        for key in ("blocks", "irr_steps", "reg_steps", "reg_calls", "overflow_retries", "nb_sum"):
            assert run.stats[key] == host.stats[key], key
        assert run.stats["reg_steps"] > 0
        if small_lists:
            assert host.stats["overflow_retries"] > 0
        for c in range(len(cls)):
            np.testing.assert_array_equal(run.x[c], host.x[c])
            np.testing.assert_array_equal(run.v[c], host.v[c])
        np.testing.assert_array_equal(run.energy, host.energy)
        np.testing.assert_array_equal(run.times, host.times)



def test_device_clock_output_times_off_the_block_grid(nb6):
    """An output interval that no block time falls on (0.1): the device
    clock records after the first block past each output time, as the host
    clock does, with the same energies and state."""
    from nb6b200 import drive
    ours = drive.backend_paths("nb6b200")
    cls = _clusters(3, 95)
    kw = dict(batched=True, tcrit=0.3, dt_out=0.1)
    clk = drive.run_ensemble(ours, cls, dev_corrector=3, **kw)
    host = drive.run_ensemble(ours, cls, dev_corrector=2, **kw)
    assert clk.stats["blocks"] == host.stats["blocks"]
    np.testing.assert_array_equal(clk.times, host.times)
    np.testing.assert_array_equal(clk.energy, host.energy)
    for c in range(len(cls)):
        np.testing.assert_array_equal(clk.x[c], host.x[c])
