"""KS c.m. corrections of the irregular force (cmfirr_cor.f, cmfirr_ucor.f).

CPU: the oracle's restatement against an independent numpy evaluation of
what the corrections stand for (each perturbed pair's components in place
of its point mass) and against the limit of components at the c.m.
GPU: irr_simd_firr_vec_ / nb6_irr_correct_ with a pair table set
(nb6_ks_set_) against the oracle's irregular force plus corrections."""
import numpy as np
import pytest


def _pred(s, x0, v0, f, fd):
    s = s[:, None]
    x = ((fd * s + f) * s + v0) * s + x0                     # jpred_int.f:16-25
    v = (fd * (1.5 * s) + f) * (2.0 * s) + v0
    return x, v


def _system(seed, ns=600, npair=40, nperturbed=30, sep=3e-3, lmax=96):
    """ns singles then npair c.m. bodies (addresses ns+1 ..), random lists
    with c.m. bodies in them, perturbed pairs with components around their
    predicted c.m. and perturber lists."""
    rng = np.random.default_rng(seed)
    n = ns + npair
    x0 = rng.normal(size=(n, 3)) * 0.5
    v0 = rng.normal(size=(n, 3)) * 0.5
    f = rng.normal(size=(n, 3)) * 0.05
    fd = rng.normal(size=(n, 3)) * 0.01
    m = rng.uniform(0.5, 2.0, n) / n
    ti = 0.0625
    t0 = ti - rng.integers(0, 8, n) / 512.0
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        k = int(rng.integers(0, 60))
        others = np.delete(np.arange(1, n + 1), i)
        nb = np.sort(rng.choice(others, k, replace=False))
        lists[i, 0] = k
        lists[i, 1:1 + k] = nb
    xp, vp = _pred(ti - t0, x0, v0, f, fd)
    pert = np.sort(rng.choice(npair, nperturbed, replace=False))
    cm = (ns + 1 + pert).astype(np.int32)
    q = rng.uniform(0.2, 0.8, nperturbed)
    d = rng.normal(size=(nperturbed, 3))
    d *= (sep / np.linalg.norm(d, axis=1))[:, None]
    dv = rng.normal(size=(nperturbed, 3)) * 0.3
    mc = m[cm - 1]
    m1, m2 = q * mc, (1 - q) * mc
    # components about the predicted c.m.: m1 x1 + m2 x2 = M xcm
    xk = np.stack([xp[cm - 1] + (m2 / mc)[:, None] * d, xp[cm - 1] - (m1 / mc)[:, None] * d], axis=1)
    vk = np.stack([vp[cm - 1] + (m2 / mc)[:, None] * dv, vp[cm - 1] - (m1 / mc)[:, None] * dv], axis=1)
    mk = np.stack([m1, m2], axis=1)
    pofs = [0]
    plist = []
    for p in range(nperturbed):
        k = int(rng.integers(0, 25))
        others = np.delete(np.arange(1, n + 1), cm[p] - 1)
        plist.extend(rng.choice(others, k, replace=False).tolist())
        pofs.append(len(plist))
    slot = np.full(n, -1, dtype=np.int32)
    slot[cm - 1] = np.arange(nperturbed)
    active = np.sort(np.concatenate([rng.choice(ns, 150, replace=False) + 1, cm[:20],
                                     ns + 1 + np.setdiff1d(np.arange(npair), pert)[:5]])).astype(np.int32)
    return dict(ti=ti, x0=x0, v0=v0, f=f, fd=fd, m=m, t0=t0, lists=lists, cm=cm, xk=xk, vk=vk, mk=mk,
                pofs=np.array(pofs, dtype=np.int32), plist=np.array(plist, dtype=np.int32), slot=slot,
                active=active, xp=xp, vp=vp)


def _force(xi, vi, xs, vs, ms):
    """Force and jerk on (xi, vi) from point masses (xs, vs, ms), summed."""
    dx = xs - xi
    dv = vs - vi
    r2 = np.sum(dx * dx, axis=-1)
    r3 = ms / (r2 * np.sqrt(r2))
    rv = 3.0 * np.sum(dx * dv, axis=-1) / r2
    return (dx * r3[:, None]).sum(0), ((dv - dx * rv[:, None]) * r3[:, None]).sum(0)


def _numpy_corrections(S):
    """What the corrections stand for, evaluated directly: acc, jrk of the
    active bodies over their neighbours with every perturbed pair resolved,
    plus (for a perturbed c.m.) the mass-weighted tidal terms over its
    perturbers."""
    xp, vp, m, slot = S["xp"], S["vp"], S["m"], S["slot"]
    out_a, out_j = [], []
    for a in S["active"]:
        i = a - 1
        row = S["lists"][i]
        nb = row[1:1 + row[0]] - 1
        ca, cj = np.zeros(3), np.zeros(3)
        if row[0] > 0:
            p = slot[i]
            if p >= 0:
                pl = S["plist"][S["pofs"][p]:S["pofs"][p + 1]] - 1
                for j in pl:
                    q = slot[j]
                    if q >= 0:
                        src_x, src_v, src_m = S["xk"][q], S["vk"][q], S["mk"][q]
                    else:
                        src_x, src_v, src_m = xp[j][None], vp[j][None], m[j:j + 1]
                    w = S["mk"][p] / m[i]
                    t1 = _force(S["xk"][p][0], S["vk"][p][0], src_x, src_v, src_m)
                    t2 = _force(S["xk"][p][1], S["vk"][p][1], src_x, src_v, src_m)
                    tc = _force(xp[i], vp[i], xp[j][None], vp[j][None], m[j:j + 1])
                    ca += w[0] * t1[0] + w[1] * t2[0] - tc[0]
                    cj += w[0] * t1[1] + w[1] * t2[1] - tc[1]
            else:
                for j in nb:
                    q = slot[j]
                    if q < 0:
                        continue
                    t = _force(xp[i], vp[i], S["xk"][q], S["vk"][q], S["mk"][q])
                    tc = _force(xp[i], vp[i], xp[j][None], vp[j][None], m[j:j + 1])
                    ca += t[0] - tc[0]
                    cj += t[1] - tc[1]
        out_a.append(ca)
        out_j.append(cj)
    return np.array(out_a), np.array(out_j)


def _oracle_corrections(orc, S, acc=None, jrk=None):
    ni = len(S["active"])
    acc = np.zeros((ni, 3)) if acc is None else acc
    jrk = np.zeros((ni, 3)) if jrk is None else jrk
    return orc.ks_cmcorr(S["ti"], S["active"], S["x0"], S["v0"], S["f"], S["fd"], S["m"], S["t0"],
                         S["lists"], S["slot"], S["xk"], S["vk"], S["mk"], S["pofs"], S["plist"], acc, jrk)


def test_oracle_corrections_match_direct_evaluation(orc):
    S = _system(11)
    ca, cj = _oracle_corrections(orc, S)
    na, nj = _numpy_corrections(S)
    assert np.abs(na).max() > 0 and np.abs(nj).max() > 0
    scale_a = np.abs(na).max()
    scale_j = np.abs(nj).max()
    np.testing.assert_allclose(ca, na, rtol=0, atol=1e-9 * scale_a)
    np.testing.assert_allclose(cj, nj, rtol=0, atol=1e-9 * scale_j)


def test_oracle_corrections_vanish_for_components_at_the_cm(orc):
    """Components merged at the c.m. (separation 0 in the limit): the
    resolved forces equal the point-mass ones, so every correction goes to
    zero as the separation does (second order in the separation)."""
    big = _oracle_corrections(orc, _system(12, sep=1e-3))
    small = _oracle_corrections(orc, _system(12, sep=1e-5))
    rb = np.abs(big[0]).max()
    rs = np.abs(small[0]).max()
    assert rs < 1e-3 * rb


def test_oracle_no_pairs_is_no_correction(orc):
    S = _system(13)
    S["slot"][:] = -1
    ca, cj = _oracle_corrections(orc, S)
    assert not ca.any() and not cj.any()


@pytest.mark.gpu
def test_irregular_force_with_ks_table_matches_oracle(nb6, orc):
    S = _system(21)
    n = S["x0"].shape[0]
    lmax = S["lists"].shape[1]
    nb6.irr_open(n, lmax, 0)
    try:
        nb6.irr_set_jp_all(S["x0"], S["v0"], S["f"], S["fd"], S["m"], S["t0"])
        for a in range(1, n + 1):
            nb6.irr_set_list(a, S["lists"][a - 1])
        plain = nb6.irr_firr_vec(S["ti"], S["active"])
        nb6.ks_set(S["cm"], S["xk"], S["vk"], S["mk"], S["pofs"], S["plist"])
        corr = nb6.irr_firr_vec(S["ti"], S["active"])
        nb6.ks_set([], [], [], [], [0], [])
        again = nb6.irr_firr_vec(S["ti"], S["active"])
    finally:
        nb6.irr_close(0)
    oa, oj, _ = orc.firr(S["ti"], S["active"], S["x0"], S["v0"], S["f"], S["fd"], S["m"], S["t0"],
                         S["lists"])
    ra, rj = _oracle_corrections(orc, S, oa, oj)
    # per body, relative to its own force: FP64 on both sides (the library
    # replaces a resolved neighbour's point mass where the oracle adds and
    # subtracts it, as the reference does)
    na = np.linalg.norm(ra, axis=1)
    nj = np.linalg.norm(rj, axis=1)
    ea = np.linalg.norm(corr[0] - ra, axis=1)
    ej = np.linalg.norm(corr[1] - rj, axis=1)
    has = S["lists"][S["active"] - 1, 0] > 0
    assert np.all(ea[has] <= 1e-11 * na[has]), ea[has].max()
    assert np.all(ej[has] <= 1e-10 * nj[has]), ej[has].max()
    np.testing.assert_array_equal(corr[2], plain[2])       # nearest neighbour unchanged
    for x, y in zip(plain, again):                          # cleared table: plain forces
        np.testing.assert_array_equal(x, y)
    moved = np.linalg.norm(corr[0] - plain[0], axis=1)
    assert (moved[has] > 1e-6 * na[has]).sum() >= 20       # the corrections are not trivial
