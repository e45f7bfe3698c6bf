"""nb6_regf_seg_: the regular force of an ensemble of independent clusters in
one persistent launch.  Each cluster's results must be those of the cluster
alone: neighbour lists identical to the FP64 oracle run on that cluster
alone (ids relative to the cluster's first body), force/potential within
1e-6 and jerk within 1e-5 relative to it, and within the same bounds of
gpunb_regf_ called with only that cluster sent."""
import numpy as np
import pytest

from parity import rel_err_vec

pytestmark = pytest.mark.gpu


def _ensemble(sizes, seed):
    from nb6b200 import ics
    return [ics.plummer(n, seed=seed + k, imf=(k % 2 == 1)) for k, n in enumerate(sizes)]


def _check(out, ref, tol_acc=1e-6, tol_jrk=1e-5):
    acc, jrk, pot, lst = out
    ra, rj, rp, rl = ref
    np.testing.assert_array_equal(lst[:, 0], rl[:, 0])
    for r in range(lst.shape[0]):
        n = lst[r, 0]
        if n > 0:
            np.testing.assert_array_equal(lst[r, 1:1 + n], rl[r, 1:1 + n])
    ok = lst[:, 0] >= 0
    if ok.any():
        assert rel_err_vec(acc[ok], ra[ok]).max() <= tol_acc
        assert rel_err_vec(pot[ok], rp[ok]).max() <= tol_acc
        assert rel_err_vec(jrk[ok], rj[ok]).max() <= tol_jrk


@pytest.mark.parametrize("m_flag", [0, 1])
def test_seg_matches_each_cluster_alone(nb6, orc, m_flag):
    import ctypes as C
    sizes = [700, 3000, 2, 129, 5000, 3]
    cls = _ensemble(sizes, 500 + m_flag)
    seg_j0 = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    m = np.concatenate([c.mass for c in cls])
    x = np.concatenate([c.pos for c in cls])
    v = np.concatenate([c.vel for c in cls])
    rng = np.random.default_rng(9)
    # active sets: ragged, one cluster with none active, one with all
    act = [np.sort(rng.choice(sizes[0], 37, replace=False)), np.arange(sizes[1]), np.array([0]),
           np.array([], dtype=int), np.sort(rng.choice(sizes[4], 300, replace=False)), np.array([1])]
    iseg = np.concatenate([np.full(len(a), c) for c, a in enumerate(act)]).astype(np.int32)
    h2 = np.concatenate([cls[c].h2(m_flag)[a] for c, a in enumerate(act)])
    dtr = np.concatenate([cls[c].dtr[a] for c, a in enumerate(act)])
    xi = np.concatenate([cls[c].pos[a] for c, a in enumerate(act)])
    vi = np.concatenate([cls[c].vel[a] for c, a in enumerate(act)])
    lmax, nnbmax = 512, 400
    nb6.gpunb_open(len(m) + 10, 0)
    try:
        nb6.gpunb_send(m, x, v)
        out = nb6.regf_seg(h2, dtr, xi, vi, iseg, seg_j0, lmax, nnbmax, m_flag)
        geom = (C.c_int * 3)()
        nb6.lib.nb6_regf_last_geometry_(geom)
        assert geom[0] < 0 and geom[2] >= geom[1] >= 1      # persistent: items >= CTAs
    finally:
        nb6.gpunb_close()
    k0 = 0
    for c, a in enumerate(act):
        k1 = k0 + len(a)
        if len(a):
            part = tuple(o[k0:k1] for o in out)
            cl = cls[c]
            ref = orc.regf(cl.mass, cl.pos, cl.vel, h2[k0:k1], dtr[k0:k1], xi[k0:k1], vi[k0:k1],
                           lmax, nnbmax, m_flag)
            _check(part, ref)
            nb6.gpunb_open(cl.n + 10, 0)
            try:
                nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
                alone = nb6.gpunb_regf(h2[k0:k1], dtr[k0:k1], xi[k0:k1], vi[k0:k1], lmax, nnbmax,
                                       m_flag)
            finally:
                nb6.gpunb_close()
            _check(part, alone)
        k0 = k1


def test_seg_overflow_and_repeat(nb6, orc):
    """Overflowed rows follow the gpunb_regf_ contract; repeated calls reuse
    the buffers and give identical results."""
    sizes = [2048, 1500]
    cls = _ensemble(sizes, 77)
    seg_j0 = np.array([0, 2048, 3548], dtype=np.int32)
    m = np.concatenate([c.mass for c in cls])
    x = np.concatenate([c.pos for c in cls])
    v = np.concatenate([c.vel for c in cls])
    iseg = np.repeat([0, 1], [2048, 1500]).astype(np.int32)
    h2 = np.concatenate([c.h2(0) for c in cls])
    dtr = np.concatenate([c.dtr for c in cls])
    nb6.gpunb_open(len(m) + 10, 0)
    try:
        nb6.gpunb_send(m, x, v)
        o1 = nb6.regf_seg(h2, dtr, x, v, iseg, seg_j0, 64, 40, 0)
        o2 = nb6.regf_seg(h2, dtr, x, v, iseg, seg_j0, 64, 40, 0)
    finally:
        nb6.gpunb_close()
    for a, b in zip(o1, o2):
        np.testing.assert_array_equal(a, b)
    for c in range(2):
        sl = slice(seg_j0[c], seg_j0[c + 1])
        ol = orc.regf(cls[c].mass, cls[c].pos, cls[c].vel, h2[sl], dtr[sl], x[sl], v[sl], 64, 40, 0)[3]
        np.testing.assert_array_equal(o1[3][sl, 0], ol[:, 0])
        bad = o1[3][sl, 0] < 0
        assert bad.any() and np.all(o1[3][sl][bad, 1:] == 0)


def test_seg_rejects_bad_segments(nb6):
    import nb6b200
    cls = _ensemble([100, 50], 3)
    m = np.concatenate([c.mass for c in cls])
    x = np.concatenate([c.pos for c in cls])
    v = np.concatenate([c.vel for c in cls])
    nb6b200.set_abort_on_error(False)
    nb6.gpunb_open(200, 0)
    try:
        nb6.gpunb_send(m, x, v)
        nb6b200.last_status()
        h2 = np.full(4, 0.01)
        z = np.zeros(4)
        xi = x[:4]
        # segment ids out of order
        nb6.regf_seg(h2, z, xi, xi, [1, 0, 0, 1], [0, 100, 150], 64, 50, 0)
        assert nb6b200.last_status() == 2                  # NB6_ERR_BAD_ARG
        # segment bounds past the sent set
        nb6.regf_seg(h2, z, xi, xi, [0, 0, 1, 1], [0, 100, 151], 64, 50, 0)
        assert nb6b200.last_status() == 2
    finally:
        nb6.gpunb_close()
        nb6b200.set_abort_on_error(True)


def test_predict_send_from_irregular_records_equals_host_send(nb6):
    """nb6_irr_predict_send_ predicts the resident records on the device with
    the host predictor's operation order: forces from that j set equal, bit
    for bit, the forces from a host-predicted gpunb_send_ of the same
    bodies."""
    from nb6b200 import ics
    cls = _ensemble([1200, 800, 2500], 900)
    n = sum(c.n for c in cls)
    m = np.concatenate([c.mass for c in cls])
    x0 = np.concatenate([c.pos for c in cls])
    v0 = np.concatenate([c.vel for c in cls])
    rng = np.random.default_rng(1)
    f = rng.normal(size=(n, 3)) * 0.1                  # F = a/2
    fd = rng.normal(size=(n, 3)) * 0.01                # FDOT = adot/6
    t0 = -rng.integers(0, 16, n) / 256.0
    t = 1.0 / 128.0
    s = (t - t0)[:, None]
    xp = ((fd * s + f) * s + v0) * s + x0              # xbpredall.F:50-59
    vp = (fd * (1.5 * s) + f) * (2.0 * s) + v0
    # clusters 0 and 2 only, as the ensemble driver sends them
    seg = [(1, 1200), (2001, 2500)]
    sel = np.r_[0:1200, 2000:4500]
    seg_j0 = np.array([0, 1200, 3700], dtype=np.int32)
    isel = np.r_[0:300:7, 1200 + np.arange(0, 2500, 11)]
    iseg = (isel >= 1200).astype(np.int32)
    h2 = np.full(len(isel), 0.02)
    dtr = np.full(len(isel), 1.0 / 64)
    xi, vi = xp[sel][isel], vp[sel][isel]
    nb6.gpunb_open(n + 10, 0)
    nb6.irr_open(n, 64, 0)
    try:
        nb6.irr_set_jp_all(x0, v0, f, fd, m, t0)
        nb6.irr_predict_send(t, [a for a, _ in seg], [c for _, c in seg])
        dev = nb6.regf_seg(h2, dtr, xi, vi, iseg, seg_j0, 256, 200, 0)
        nb6.gpunb_send(m[sel], xp[sel], vp[sel])
        host = nb6.regf_seg(h2, dtr, xi, vi, iseg, seg_j0, 256, 200, 0)
    finally:
        nb6.irr_close(0)
        nb6.gpunb_close()
    for a, b in zip(dev, host):
        np.testing.assert_array_equal(a, b)
    assert (host[3][:, 0] > 0).all()


def test_seg_single_large_segment_takes_the_tile_kernels(nb6, orc):
    """One segment spanning a j set of 40,000 bodies (one big cluster) runs
    on the tuned tile kernels of gpunb_regf_: the rows equal gpunb_regf_'s
    bit for bit, and the oracle's lists and forces within the usual bounds."""
    import ctypes as C
    from nb6b200 import ics
    cl = ics.plummer(40000, seed=4242, imf=True)
    rng = np.random.default_rng(3)
    a = np.sort(rng.choice(cl.n, 700, replace=False))
    h2, dtr, xi, vi = cl.h2(0)[a], cl.dtr[a], cl.pos[a], cl.vel[a]
    nb6.gpunb_open(cl.n + 10, 0)
    try:
        nb6.gpunb_send(cl.mass, cl.pos, cl.vel)
        seg = nb6.regf_seg(h2, dtr, xi, vi, np.zeros(len(a), np.int32), [0, cl.n], 512, 400, 0)
        plain = nb6.gpunb_regf(h2, dtr, xi, vi, 512, 400, 0)
    finally:
        nb6.gpunb_close()
    for s, p in zip(seg, plain):
        np.testing.assert_array_equal(s, p)
    sub = np.sort(rng.choice(len(a), 64, replace=False))
    ref = orc.regf(cl.mass, cl.pos, cl.vel, h2[sub], dtr[sub], xi[sub], vi[sub], 512, 400, 0)
    _check(tuple(o[sub] for o in seg), ref)
