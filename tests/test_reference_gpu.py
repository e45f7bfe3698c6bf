"""This library against the reference's own CUDA regular-force library
(gpunb.velocity.cu built for sm_100a into oracle/_ref by oracle/Makefile),
same inputs, same GPU: neighbour lists identical except pairs inside the
reference's FP32 boundary band, forces within the reference's FP32
accuracy of ours.  Skipped where the reference library was not built."""
import numpy as np
import pytest

from parity import align_to_lists, compare_lists, rel_err_vec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m_flag", [0, 1])
def test_lists_and_forces_match_the_reference_cuda_library(nb6, orc, m_flag):
    from nb6b200 import ics
    from nb6b200.abi import ForceLib
    if not orc.ref_available("gpunb_velocity"):
        pytest.skip("the reference CUDA library was not built (oracle/Makefile ref_gpu)")
    ref = ForceLib(orc.ref_lib("gpunb_velocity"), "ref-gpunb-velocity")
    cl = ics.plummer(8192, seed=77 + m_flag, imf=True)
    isel = np.arange(0, cl.n, 8)                       # 1,024 i spread over the set
    inp = {"mj": cl.mass, "xj": cl.pos, "vj": cl.vel, "h2": cl.h2(m_flag)[isel], "dtr": cl.dtr[isel],
           "xi": cl.pos[isel], "vi": cl.vel[isel], "lmax": 512, "nnbmax": 400}
    outs = []
    for lib in (nb6, ref):
        lib.gpunb_open(cl.n + 10, 0)
        try:
            lib.gpunb_send(cl.mass, cl.pos, cl.vel)
            outs.append(lib.gpunb_regf(inp["h2"], inp["dtr"], inp["xi"], inp["vi"], 512, 400, m_flag))
        finally:
            lib.gpunb_close()
    (a, j, p, l), (ra, rj, rp, rl) = outs
    res = compare_lists(l, rl, inp, band=1e-4, m_flag=m_flag)
    assert res["pairs_out_of_band"] == 0 and res["overflow_mismatch"] == 0, res
    assert res["unsorted_rows"] == 0, res
    a, j, p = align_to_lists(a, j, p, l, rl, inp)
    ok = (l[:, 0] >= 0) & (rl[:, 0] >= 0)
    ea, ej, ep = rel_err_vec(a[ok], ra[ok]), rel_err_vec(j[ok], rj[ok]), rel_err_vec(p[ok], rp[ok])
    # the reference works on FP32 absolute coordinates (~1e-5 of FP64)
    assert np.median(ea) < 2e-5 and ea.max() < 5e-4, (np.median(ea), ea.max())
    assert np.median(ej) < 5e-5 and ej.max() < 5e-3, (np.median(ej), ej.max())
    assert np.median(ep) < 2e-5 and ep.max() < 5e-4, (np.median(ep), ep.max())


def test_potential_matches_the_reference_cuda_library(nb6, orc):
    """gpupot_ of this library (ordered path above 32,768 bodies) against
    the reference's gpupot.gpu.cu built for sm_100a, whole set."""
    from nb6b200 import ics
    from nb6b200.abi import ForceLib
    if not orc.ref_available("gpupot_gpu"):
        pytest.skip("the reference CUDA potential was not built (oracle/Makefile ref_gpu)")
    ref = ForceLib(orc.ref_lib("gpupot_gpu"), "ref-gpupot-gpu")
    for n in (3000, 40000):
        cl = ics.plummer(n, seed=n, imf=True)
        p = nb6.gpupot(cl.mass, cl.pos)
        pr = ref.gpupot(cl.mass, cl.pos)
        assert rel_err_vec(p, pr).max() < 2e-6          # both hi/lo differences, FP32 pair math
