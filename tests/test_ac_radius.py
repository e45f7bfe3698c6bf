"""The oracle's Ahmad-Cohen radius rule (regcor_gpu.F:19-238) and overflow
shrink (util_gpu.F:69-100) against hand-derived cases, one per branch.

Each expected value is worked out step by step from the reference's lines
for the chosen inputs, with the reference's REAL*4 literals and FLOAT()
terms in float32 (it is built without -fdefault-real-8).  The cases pin the
oracle, which the device corrector and the drivers are then checked
against.
"""
import numpy as np
import pytest

f32 = np.float32
NNBOPT, NNBMAX = 50, 400
ZNBMIN = 4.0            # MAX(0.01*FLOAT(400), 1.0)
NBAVE = 200             # MIN(50+150, MAX(400-50, 4))
ONE3 = 1.0 / 3.0


def adj(rdens=(0.0, 0.0, 0.0), rscale=1.0, rc2=0.01, rsfac=100.0, bodym=1e-5):
    return [*rdens, rscale, rc2, rsfac, bodym]


def fac(nnb):
    return float(f32(1.0) + f32(0.1) * (f32(NNBOPT) - f32(nnb)) / f32(nnb))


def one(orc, kz39, a, nnb, nnb0, dtr, x, v, rs, xnb=None, vnb=None):
    xn = None if xnb is None else np.asarray(xnb, float).reshape(1, 3, 3)
    vn = None if vnb is None else np.asarray(vnb, float).reshape(1, 3, 3)
    out, dfi, dfd = orc.ac_radius(kz39, NNBOPT, NNBMAX, a, [nnb], [nnb0], [dtr], [x], [v], [rs], xn, vn)
    return out[0], dfi[0], dfd[0]


def test_zero_neighbours_outward_and_inward(orc):
    a = adj(rscale=0.8, bodym=2e-5)
    x, v = np.array([3.0, 4.0, 0.0]), np.array([0.3, 0.4, 0.1])       # r = 5, moving out
    rs, dfi, dfd = one(orc, 0, a, 0, 7, 0.01, x, v, 0.2)
    assert rs == max(0.75 * 0.2, float(f32(0.1)) * 0.8)                 # :125-126
    r2 = 25.0
    fij = float(f32(0.01)) * 2e-5 / (r2 * np.sqrt(r2))
    rdot = 3.0 * (x @ v) / r2
    np.testing.assert_array_equal(dfi, -fij * x)                       # :118-121
    np.testing.assert_array_equal(dfd, -(v - rdot * x) * fij)
    rs, _, _ = one(orc, 0, a, 0, 7, 0.01, x, -v, 0.2)                  # moving in
    assert rs == float(f32(1.1)) * 0.2                                  # :128


def test_growth_inside_the_core(orc):
    # nnb = 20 < NNBOPT, inside RC: no outer factors; A5 = 0.25 (RSFAC*DTR = 1)
    x, v = np.array([0.01, 0.0, 0.0]), np.array([0.0, 0.5, 0.0])
    for kz39 in (0, 1):
        rs, _, _ = one(orc, kz39, adj(rc2=0.04, rsfac=100.0), 20, 20, 0.01, x, v, 0.05)
        a3 = 20.0 * fac(20)                    # 23.0000...: FAC in float
        a4 = a3 / 20.0 - 1.0                   # 0.15 < A5
        a3b = ONE3 * a4
        a1 = 1.0 + a3b - a3b * a3b
        assert rs == a1 * 0.05


def test_outer_membership_reduction_only_with_nb_flag(orc):
    # RI = 2 > RSCALE = 1: NB_FLAG = 1 scales A3 by RSCALE/RI (:152-153)
    x, v = np.array([2.0, 0.0, 0.0]), np.zeros(3)
    a = adj(rc2=0.01)
    rs1, _, _ = one(orc, 0, a, 50, 50, 1.0, x, v, 0.3)
    a3 = 50.0 * fac(50) * max(1.0 / 2.0, float(f32(0.1)))
    a4 = a3 / 50.0
    # (A3 - NNB0)(A3 - NNB) > 0: no inertial root; RIDOT = 0: factor 1
    a4 = max(a4 - 1.0, -0.25)                  # -0.5 clamped to -A5
    a3b = ONE3 * a4
    assert rs1 == (1.0 + a3b - a3b * a3b) * 0.3
    # NB_FLAG = 0 (KZ(39) = 1): A3 = MAX(A3, ZNBMIN), no change at NNBOPT
    rs0, _, _ = one(orc, 1, a, 50, 50, 1.0, x, v, 0.3)
    assert rs0 == 0.3


def test_radial_velocity_factor(orc):
    # RC2 < RI2 < 100 RH2 with NB_FLAG = 1: A4 *= 1 + RIDOT*DTR/RI2 (:165-167)
    x, v = np.array([0.5, 0.0, 0.0]), np.array([2.0, 0.0, 0.0])
    dtr = 0.05
    rs, _, _ = one(orc, 0, adj(rc2=0.01, rsfac=100.0), 50, 50, dtr, x, v, 0.1)
    ri2 = 0.25
    a4 = (50.0 * fac(50)) / 50.0 * (1.0 + (0.5 * 2.0) * dtr / ri2)   # 1.2
    a4 = min(a4 - 1.0, 0.25)
    a3b = ONE3 * a4
    assert rs == (1.0 + a3b - a3b * a3b) * 0.1
    # the same body with KZ(39) = 1 keeps its radius (no factor, A4 = 1)
    rs, _, _ = one(orc, 1, adj(rc2=0.01, rsfac=100.0), 50, 50, dtr, x, v, 0.1)
    assert rs == 0.1


def test_step_limit_and_inertial_root(orc):
    x, v = np.array([0.05, 0.0, 0.0]), np.zeros(3)
    # small RSFAC*DTR clamps the change: A5 = 0.02 (:184-192)
    rs, _, _ = one(orc, 0, adj(rc2=0.04, rsfac=2.0), 10, 10, 0.01, x, v, 0.05)
    a4 = min((10.0 * fac(10)) / 10.0 - 1.0, 2.0 * 0.01)
    a3b = ONE3 * a4
    assert rs == (1.0 + a3b - a3b * a3b) * 0.05
    # NNB0 on the other side of the prediction: A4 = SQRT(A4) (:159)
    rs, _, _ = one(orc, 0, adj(rc2=0.04, rsfac=100.0), 30, 60, 0.01, x, v, 0.05)
    a3 = 30.0 * fac(30)                     # 32: between NNB = 30 and NNB0 = 60
    a4 = np.sqrt(a3 / 30.0) - 1.0
    a3b = ONE3 * a4
    assert rs == (1.0 + a3b - a3b * a3b) * 0.05


def test_quarter_restriction_and_large_membership(orc):
    x = np.array([0.1, 0.0, 0.0])
    # RS^2 in (RI2, 2 RI2) and NNB > 5: A1 = SQRT(A1) (:206-209)
    rs, _, _ = one(orc, 0, adj(rc2=0.04, rsfac=100.0), 20, 20, 0.01, x, np.zeros(3), 0.12)
    a4 = (20.0 * fac(20)) / 20.0 - 1.0
    a3b = ONE3 * a4
    assert rs == np.sqrt(1.0 + a3b - a3b * a3b) * 0.12
    # NNB > NBAVE moving inward: RS *= 1 - DRS, DRS in float (:215-220)
    v = np.array([-1.0, 0.0, 0.0])
    nnb = 260
    rs, _, _ = one(orc, 0, adj(rc2=0.04, rsfac=100.0), nnb, nnb, 0.01, x, v, 0.05)
    a3 = min(nnb * fac(nnb), float(f32(0.9) * f32(NBAVE)))         # capped at 180
    a4 = max(a3 / nnb - 1.0, -0.25)
    a3b = ONE3 * a4
    r = (1.0 + a3b - a3b * a3b) * 0.05
    drs = float((f32(nnb) - f32(NBAVE)) / (f32(3.0) * f32(nnb)))
    assert rs == r * (1.0 - drs)


def test_small_membership_floor(orc):
    # NNB = 3 < ZNBMIN = 4 while the prediction NBP = INT(3 FAC) = 7 > ZNBMIN;
    # far outside (RI = 10 RSCALE, NB_FLAG = 1) the membership reduction
    # makes A4 < 1, so A1 < 1 and the floor sets A1 = 1.05 (:199-201).
    # KZ(39) = 2 (M_FLAG = 1) leaves out the NNB <= 3 branch.
    x, v = np.array([10.0, 0.0, 0.0]), np.zeros(3)
    nnb = 3
    assert int(nnb * fac(nnb)) == 7
    rs, _, _ = one(orc, 2, adj(rc2=0.04, rsfac=100.0), nnb, nnb, 0.01, x, v, 0.05)
    assert rs == float(f32(1.05)) * 0.05
    # without the floor's condition (NNB0 = NNB = 5 >= ZNBMIN) the radius shrinks
    rs, _, _ = one(orc, 2, adj(rc2=0.04, rsfac=100.0), 5, 5, 0.01, x, v, 0.05)
    a3 = 5 * fac(5) * max(1.0 / 10.0, float(f32(0.1)))
    a4 = max(a3 / 5 - 1.0, -0.25)
    a3b = ONE3 * a4
    assert rs == (1.0 + a3b - a3b * a3b) * 0.05


def test_few_neighbours_radial_velocity(orc):
    # NNB <= 3, M_FLAG = 0: RS = MAX(min(2 RS, RIJ + RSDOT*DTR), 1.1 RS)
    x, v = np.array([0.05, 0.0, 0.0]), np.zeros(3)
    xnb = np.zeros((3, 3))
    vnb = np.zeros((3, 3))
    xnb[0] = [0.05, 0.3, 0.0]
    vnb[0] = [0.0, 4.0, 0.0]                  # leaving: RIJ grows
    xnb[1] = [0.05, 0.0, 0.25]
    vnb[1] = [0.0, 0.0, 5.0]
    dtr = 0.01
    rs_in = 0.2
    for kz39, expect_branch in ((1, True), (3, False)):
        rs, _, _ = one(orc, kz39, adj(rc2=0.04, rsfac=0.0), 2, 2, dtr, x, v, rs_in, xnb, vnb)
        # RSFAC = 0: A5 = 0, A1 = 1, RS unchanged by the volume rule
        if expect_branch:
            a1 = 2.0 * rs_in
            for l in range(2):
                e = x - xnb[l]
                rij = np.sqrt(e[0] ** 2 + e[1] ** 2 + e[2] ** 2)
                rsdot = (e[0] * (v[0] - vnb[l][0]) + e[1] * (v[1] - vnb[l][1]) +
                         e[2] * (v[2] - vnb[l][2])) / rij
                a1 = min(a1, rij + rsdot * dtr)
            assert rs == max(a1, float(f32(1.1)) * rs_in)
        else:
            assert rs == rs_in


@pytest.mark.parametrize("kz39", [0, 1, 2, 3])
def test_overflow_shrink(orc, kz39):
    rs = orc.ac_shrink(kz39, NNBOPT, NNBMAX, [-120, -45], [0.3, 0.3])
    if kz39 in (0, 2):
        f1 = np.power(f32(-NNBOPT) / f32(-120), f32(0.333), dtype=np.float32)
        f2 = np.power(f32(NNBOPT) / f32(NNBMAX), f32(0.4), dtype=np.float32)
        np.testing.assert_allclose(rs, [float(f1) * 0.3, float(f2) * 0.3], rtol=2e-7)
    else:
        assert rs[0] == rs[1] == float(f32(0.9)) * 0.3


def _driver():
    import ctypes as C
    from nb6b200 import drive
    lib = drive._lib()
    return lib, C


def _random_cases(seed, n=20000):
    rng = np.random.default_rng(seed)
    nnb = np.where(rng.random(n) < 0.2, rng.integers(0, 4, n), rng.integers(4, 320, n)).astype(np.int32)
    nnb0 = np.where(rng.random(n) < 0.5, nnb + rng.integers(-30, 30, n), rng.integers(0, 320, n))
    nnb0 = np.clip(nnb0, 0, 400).astype(np.int32)
    dtr = 2.0 ** -rng.integers(2, 14, n).astype(float)
    r = 10 ** rng.uniform(-2, 1.3, n)
    u = rng.normal(size=(n, 3))
    xi = u / np.linalg.norm(u, axis=1)[:, None] * r[:, None]
    vi = rng.normal(size=(n, 3)) * 0.6
    rs = 10 ** rng.uniform(-2.5, 0, n)
    xnb = xi[:, None, :] + rng.normal(size=(n, 3, 3)) * rs[:, None, None]
    vnb = vi[:, None, :] + rng.normal(size=(n, 3, 3)) * 0.5
    adj = [0.02, -0.01, 0.005, 0.8, 0.04, float(rng.uniform(1, 100)), 1e-5]
    return adj, nnb, nnb0, dtr, xi, vi, rs, xnb, vnb


@pytest.mark.parametrize("kz39", [0, 1, 2, 3])
def test_driver_rule_equals_oracle_bit_for_bit(orc, kz39):
    """The drivers' host rule (driver/hermite.h ac_radius, also restated on
    the device) gives the oracle's bits on random bodies over every branch."""
    lib, C = _driver()
    d, i = C.POINTER(C.c_double), C.POINTER(C.c_int)
    for seed in range(3):
        adj, nnb, nnb0, dtr, xi, vi, rs, xnb, vnb = _random_cases(100 * kz39 + seed)
        o_rs, o_fi, o_fd = orc.ac_radius(kz39, NNBOPT, NNBMAX, adj, nnb, nnb0, dtr, xi, vi, rs, xnb, vnb)
        n = nnb.shape[0]
        h_rs = np.ascontiguousarray(rs, dtype=np.float64).copy()
        h_fi, h_fd = np.zeros((n, 3)), np.zeros((n, 3))
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (adj, dtr, xi, vi, xnb, vnb)]
        lib.nb6drive_ac_radius(n, kz39, NNBOPT, NNBMAX, arrs[0].ctypes.data_as(d), nnb.ctypes.data_as(i),
                               nnb0.ctypes.data_as(i), arrs[1].ctypes.data_as(d), arrs[2].ctypes.data_as(d),
                               arrs[3].ctypes.data_as(d), arrs[4].ctypes.data_as(d), arrs[5].ctypes.data_as(d),
                               h_rs.ctypes.data_as(d), h_fi.ctypes.data_as(d), h_fd.ctypes.data_as(d))
        np.testing.assert_array_equal(h_rs, o_rs)
        np.testing.assert_array_equal(h_fi, o_fi)
        np.testing.assert_array_equal(h_fd, o_fd)
        assert np.mean(h_rs != rs) > 0.3          # the rule moved most radii
        neg = -np.random.default_rng(seed).integers(1, 500, n).astype(np.int32)
        h2 = rs.copy()
        lib.nb6drive_ac_shrink(n, kz39, NNBOPT, NNBMAX, neg.ctypes.data_as(i), h2.ctypes.data_as(d))
        np.testing.assert_array_equal(h2, orc.ac_shrink(kz39, NNBOPT, NNBMAX, neg, rs))


def test_driver_core_finds_the_density_centre():
    """core.f restated in the driver: the density centre of a King cluster
    displaced by a known vector lands at the displacement, within the
    scatter of the densest bodies; the core radius and velocity come out
    positive and inside the half-mass radius."""
    import ctypes as C
    from scipy.spatial import cKDTree
    from nb6b200 import ics
    lib, _ = _driver()
    cl = ics.king(20000, w0=6.0, seed=3, imf=False, nnbopt=50)
    shift = np.array([0.3, -0.2, 0.1])
    x = cl.pos + shift
    n = cl.n
    tree = cKDTree(x)
    _, idx = tree.query(x, k=51)
    ls = 64
    rows = np.zeros((n, ls), dtype=np.int32)
    rows[:, 0] = 50
    rows[:, 1:51] = np.sort(idx[:, 1:], axis=1) + 1
    rs = np.sqrt(((x[idx[:, 50]] - x) ** 2).sum(1)) * 1.0001
    io = np.array([0.0, 0.0, 0.0, 0.8, 0.0, 0.0, 0.0])
    d = C.POINTER(C.c_double)
    for _ in range(3):            # the rule iterates from the last centre
        lib.nb6drive_core(n, np.ascontiguousarray(cl.mass).ctypes.data_as(d),
                          np.ascontiguousarray(x).ctypes.data_as(d),
                          np.ascontiguousarray(cl.vel).ctypes.data_as(d), rs.ctypes.data_as(d),
                          rows.ctypes.data_as(C.POINTER(C.c_int)), ls, C.c_double(1.0),
                          io.ctypes.data_as(d))
    rc = io[4]
    assert 0.0 < rc < 0.8 and abs(io[5] - rc * rc) < 1e-15 and io[6] > 0.0
    assert np.linalg.norm(io[:3] - shift) < 0.5 * rc, (io[:3], shift, rc)
