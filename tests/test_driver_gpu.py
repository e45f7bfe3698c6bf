"""The same block-step driver on libnb6b200 (GPU) and on the reference's own
CPU libraries.  Plummer N = 1024, equal masses, Henon units,
integrated to T = 1; energy drift over 10 N-body times compared with the
reference's under the identical driver (contract: within 10%; a smaller drift
passes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _backends(orc):
    from nb6b200 import drive
    for lib in ("reg", "irr", "pot"):
        if not orc.ref_available(lib):
            pytest.skip("reference CPU libraries not built")
    ref = {"reg": orc.ref_path("reg"), "irr": orc.ref_path("irr"), "pot": orc.ref_path("pot")}
    return drive.backend_paths("nb6b200"), ref


def test_config1_plummer1k_to_t1(orc):
    from nb6b200 import drive, ics
    ours, ref = _backends(orc)
    cl = ics.plummer(1024, seed=43532)
    r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=1.0, dt_out=0.125)
    rr = drive.run(ref, cl.mass, cl.pos, cl.vel, tcrit=1.0, dt_out=0.125)
    print(f"\nT=1  dE ours {r.de_max:.3e}  reference {rr.de_max:.3e}; "
          f"blocks {r.stats['blocks']} vs {rr.stats['blocks']}; "
          f"wall {r.stats['wall_total']:.2f}s vs {rr.stats['wall_total']:.2f}s")
    assert r.stats["t_end"] == 1.0
    assert r.de_max < 1e-5
    # same initial energy (identical inputs, both FP64-accurate potentials)
    assert abs(r.etot[0] / rr.etot[0] - 1) < 1e-6


SEEDS = (43532, 1, 2, 3, 4, 5, 6, 7)


def test_energy_drift_t10_within_10pct_of_reference(orc):
    """T = 10 energy drift, same driver on both backends, over 8 seeds.

    Single realisations are chaotic and the drivers integrate single stars
    without KS regularisation, so one seed's drift is set by its closest
    encounters: across these seeds max |dE/E| spans three decades on either
    backend.  The contract's 10% is therefore stated over the sample: the
    median of max |dE/E| over the seeds may exceed the reference's median by
    at most 10% (measured: 3.4e-6 and 7.3e-6 in two runs against 1.4e-5;
    the library's own median moves with the autotuner's kernel choices,
    which change the last bits and so the orbits).  Both medians are
    printed."""
    from nb6b200 import drive, ics
    ours, ref = _backends(orc)
    mo, mr = [], []
    for seed in SEEDS:
        cl = ics.plummer(1024, seed=seed)
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=10.0, dt_out=0.5)
        rr = drive.run(ref, cl.mass, cl.pos, cl.vel, tcrit=10.0, dt_out=0.5)
        assert r.stats["t_end"] == 10.0 and rr.stats["t_end"] == 10.0
        mo.append(r.de_max)
        mr.append(rr.de_max)
    med_o, med_r = float(np.median(mo)), float(np.median(mr))
    print(f"\nT=10 max |dE/E| median over {len(SEEDS)} seeds: ours {med_o:.3e}  reference {med_r:.3e}")
    assert med_o <= 1.10 * med_r
