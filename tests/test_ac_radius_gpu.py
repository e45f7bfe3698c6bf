"""The device regular corrector's Ahmad-Cohen radius rule against the
oracle's restatement of regcor_gpu.F:19-238, bit for bit, for every KZ(39)
form (NB_FLAG 0/1, M_FLAG 0/1).

Two Plummer clusters (two segments, each with its own radius-rule
quantities from nb6_hermite_adjust_) are put in the irregular library's
store at TIME = 0 with old neighbour lists; nb6_irr_predict_send_ +
nb6_regf_correct_ then run the regular force and corrector of a sample of
bodies whose radii are chosen to give every membership from 0 to past
NNBMAX.  For each row that fitted, the oracle gets the same inputs -- the
new count (self removed), the old count, DTR, the body at TIME, the first
three new neighbours (read back with nb6_irr_lists_get_), RS and its
cluster's quantities -- and must give the radius the device wrote.  Rows
that overflowed come back flagged and untouched.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NNBOPT, NNBMAX, LMAX = 50, 400, 512
SIZES = (1500, 2500)
ADJ = ([0.05, 0.0, -0.02, 0.6, 0.02, 40.0, 1.0 / 1500, 0.0],
       [0.0, 0.01, 0.0, 0.9, 0.05, 8.0, 1.0 / 2500, 0.0])


def _setup(nb6, kz39, seed):
    from scipy.spatial import cKDTree
    from nb6b200 import ics
    rng = np.random.default_rng(seed)
    parts = [ics.plummer(n, seed=seed + c) for c, n in enumerate(SIZES)]
    n = sum(SIZES)
    pos = np.concatenate([p.pos for p in parts])
    vel = np.concatenate([p.vel for p in parts])
    mass = np.concatenate([p.mass for p in parts])
    a0 = np.array([1, SIZES[0] + 1, n + 1], dtype=np.int32)
    # radii from the distance to a chosen neighbour rank (0 .. 460)
    kth = np.where(rng.random(n) < 0.25, rng.integers(0, 5, n), rng.integers(5, 460, n))
    rs = np.zeros(n)
    old = []
    for c in range(2):
        lo, hi = a0[c] - 1, a0[c + 1] - 1
        x = pos[lo:hi]
        tree = cKDTree(x)
        d, idx = tree.query(x, k=462)
        k = kth[lo:hi]
        rs[lo:hi] = np.where(k == 0, 0.5 * d[:, 1], 0.5 * (d[np.arange(hi - lo), k] + d[np.arange(hi - lo), k + 1]))
        for q in range(hi - lo):          # old lists: a random subset of the nearest
            m = int(rng.integers(0, 120))
            ids = np.sort(rng.choice(idx[q, 1:200], m, replace=False)) + lo + 1
            old.append(np.concatenate([[m], ids]).astype(np.int32))
    dtr = 2.0 ** -rng.integers(3, 10, n).astype(float)
    nb6.gpunb_open(n + 10, 0)                 # the regular library takes the j set
    nb6.irr_open(n, LMAX, 0)
    z = np.zeros((n, 3))
    nb6.irr_set_jp_all(pos, vel, z, z, mass, np.zeros(n))
    for i in range(n):
        nb6.irr_set_list(i + 1, old[i])
    nb6.hermite_open(0.02, 0.125, 2.0 ** -30)
    f = rng.normal(size=(n, 3)) * 0.1
    nb6.hermite_set_all(f, f * 0.3, f * 2.0, f * 0.5, dtr / 2, -dtr, dtr, rs)
    nb6.hermite_adjust(1 if kz39 in (0, 2) else 0, a0, np.array(ADJ).reshape(-1))
    return pos, vel, mass, rs, dtr, old, a0


@pytest.mark.parametrize("kz39", [0, 1, 2, 3])
def test_device_radius_rule_equals_oracle(nb6, orc, kz39):
    m_flag = 1 if kz39 in (2, 3) else 0
    pos, vel, mass, rs, dtr, old, a0 = _setup(nb6, kz39, seed=11 + kz39)
    try:
        n = pos.shape[0]
        rng = np.random.default_rng(5)
        sel = np.sort(rng.choice(n, 1200, replace=False))
        iseg = (sel >= SIZES[0]).astype(np.int32)
        nb6.irr_predict_send(0.0, a0[:2], np.array(SIZES, dtype=np.int32))
        bodym = np.where(iseg == 0, 1.0 / SIZES[0], 1.0 / SIZES[1])
        h2 = rs[sel] ** 2 / (bodym if m_flag else 1.0)
        prm = [0.02, 0.125, 2.0 ** -30, 1.0, NNBOPT, 0.0]
        out = nb6.regf_correct(0.0, sel + 1, iseg, np.array([0, SIZES[0], n], dtype=np.int32), a0[:2], h2,
                               dtr[sel], rs[sel], pos[sel], vel[sel], LMAX, NNBMAX, m_flag, prm)
        over = out[:, 28] != 0
        assert over.sum() > 20 and (~over).sum() > 600
        assert np.all(out[over, 28] < 0)
        rows = np.zeros((n, LMAX), dtype=np.int32)
        rows[sel] = nb6.lists_get(sel + 1, LMAX)
        ok = np.nonzero(~over)[0]
        nnb = out[ok, 27].astype(np.int32)
        np.testing.assert_array_equal(rows[sel[ok], 0], nnb)
        for c in range(2):
            q = ok[iseg[ok] == c]
            if q.size == 0:
                continue
            b = sel[q]
            xnb = np.zeros((q.size, 3, 3))
            vnb = np.zeros((q.size, 3, 3))
            for r, i in enumerate(b):
                ids = rows[i, 1:1 + min(3, rows[i, 0])] - 1
                xnb[r, :len(ids)] = pos[ids]
                vnb[r, :len(ids)] = vel[ids]
            nnb0 = np.array([old[i][0] for i in b], dtype=np.int32)
            o_rs, _, _ = orc.ac_radius(kz39, NNBOPT, NNBMAX, ADJ[c][:7], out[q, 27].astype(np.int32), nnb0,
                                       dtr[b], pos[b], vel[b], rs[b], xnb, vnb)
            np.testing.assert_array_equal(out[q, 26], o_rs)
        counts = out[ok, 27]
        assert (counts == 0).any() and (counts <= 3).sum() > 5 and (counts > 200).any()
        # the radius changed for most bodies (the rule acted)
        assert np.mean(out[ok, 26] != rs[sel[ok]]) > 0.3
    finally:
        nb6.irr_close(0)
        nb6.gpunb_close()
