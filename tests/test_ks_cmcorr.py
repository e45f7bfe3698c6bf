"""KS c.m. corrections of the irregular force (cmfirr_cor.f, cmfirr_ucor.f).

CPU: the oracle's restatement against the two routines restated statement
by statement (bit for bit), against an independent numpy evaluation of
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
    return dict(ti=ti, x0=x0, v0=v0, f=f, fd=fd, m=m, t0=t0, lists=lists, cm=cm, xk=xk, vk=vk, mk=mk, n_single=ns,
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


def _reference_routines(S):
    """CMFIRR_COR (cmfirr_cor.f:1-136) and CMFIRR_UCOR (cmfirr_ucor.f:1-116)
    as nbint_cor.f:40-79 calls them, statement by statement in the
    routines' own order and control flow: a perturbed c.m. body gets
    CMFIRR_COR over its first component's perturber list (and no
    CMFIRR_UCOR, nbint_cor.f:66-75); any other body CMFIRR_UCOR over the
    c.m. bodies at the end of its ascending neighbour list
    (nbint_cor.f:77-79).  X, XDOT are the predicted bodies (jpred_int.f),
    the components of perturbed pairs stand for X(J1), X(J2).  Returns the
    corrections alone (FIRR, FD starting at zero)."""
    xp, vp, m, slot = S["xp"], S["vp"], S["m"], S["slot"]
    N = S["n_single"]       # bodies 0 .. N-1 are singles, the rest c.m. bodies
    out_a, out_j = [], []

    def pert(j):            # LIST(1,J1) > 0: the pair of c.m. body j (0-based) is perturbed
        return slot[j] >= 0

    for a in S["active"]:
        I = a - 1
        firr = [0.0, 0.0, 0.0]
        fd = [0.0, 0.0, 0.0]
        row = S["lists"][I]
        nnb0 = int(row[0])
        if nnb0 == 0:                       # nbint_cor.f:44-55 is the caller's own force
            out_a.append(firr)
            out_j.append(fd)
            continue
        if pert(I):
            # CMFIRR_COR(I, I1, FIRR, FD)
            p = slot[I]
            x1, x2 = S["xk"][p]
            v1, v2 = S["vk"][p]
            b1, b2 = S["mk"][p]
            for J in S["plist"][S["pofs"][p]:S["pofs"][p + 1]] - 1:
                K = J
                xk = [None, None]
                vk = [None, None]
                bk = [None, None]
                if slot[J] >= 0:            # J > N with LIST(1,J1) > 0
                    q = slot[J]
                    xk = [S["xk"][q][0], S["xk"][q][1]]
                    vk = [S["vk"][q][0], S["vk"][q][1]]
                    bk = [S["mk"][q][0], S["mk"][q][1]]
                    K = -1                  # K = J1
                if K == J:
                    xk[0], vk[0], bk[0] = xp[J], vp[J], m[J]
                A1 = xp[J][0] - xp[I][0]
                A2 = xp[J][1] - xp[I][1]
                A3 = xp[J][2] - xp[I][2]
                RIJ2 = A1 * A1 + A2 * A2 + A3 * A3
                DV = [vp[J][0] - vp[I][0], vp[J][1] - vp[I][1], vp[J][2] - vp[I][2]]
                DR2I = 1.0 / RIJ2
                DR3I = m[J] * DR2I * np.sqrt(DR2I)
                DRDV = 3.0 * (A1 * DV[0] + A2 * DV[1] + A3 * DV[2]) * DR2I
                FCM = [A1 * DR3I, A2 * DR3I, A3 * DR3I]
                FCMD = [(DV[0] - A1 * DRDV) * DR3I, (DV[1] - A2 * DRDV) * DR3I, (DV[2] - A3 * DRDV) * DR3I]
                comp = 0
                while True:                 # label 20
                    FP, FPD = [0.0] * 6, [0.0] * 6
                    for half, (xc, vc) in enumerate(((x1, v1), (x2, v2))):
                        dr2 = 0.0
                        drdv = 0.0
                        dx = [0.0] * 3
                        dv = [0.0] * 3
                        for L in range(3):
                            dx[L] = xk[comp][L] - xc[L]
                            dv[L] = vk[comp][L] - vc[L]
                            dr2 = dr2 + dx[L] ** 2
                            drdv = drdv + dx[L] * dv[L]
                        dr2i = 1.0 / dr2
                        dr3i = bk[comp] * dr2i * np.sqrt(dr2i)
                        drdv = 3.0 * drdv * dr2i
                        for L in range(3):
                            FP[L + 3 * half] = dx[L] * dr3i
                            FPD[L + 3 * half] = (dv[L] - dx[L] * drdv) * dr3i
                    for L in range(3):
                        firr[L] = firr[L] + ((b1 * FP[L] + b2 * FP[L + 3]) / m[I] - FCM[L])
                        fd[L] = fd[L] + ((b1 * FPD[L] + b2 * FPD[L + 3]) / m[I] - FCMD[L])
                    if K == -1 and comp == 0:   # the perturber's second component, no c.m. term
                        FCM = [0.0, 0.0, 0.0]
                        FCMD = [0.0, 0.0, 0.0]
                        comp = 1
                        continue
                    break
        else:
            # CMFIRR_UCOR(I, NNB0, LIST(1,I), FIRR, FD): the c.m. neighbours
            # sit at the end of the ascending list
            klist = row[1:1 + nnb0] - 1
            nnb2 = nnb0                     # the list up to its last single
            while nnb2 >= 1 and klist[nnb2 - 1] >= N:
                nnb2 -= 1
            for J in klist[nnb2:]:
                if not pert(J):             # unperturbed binary: a single particle
                    continue
                q = slot[J]
                A1 = xp[J][0] - xp[I][0]
                A2 = xp[J][1] - xp[I][1]
                A3 = xp[J][2] - xp[I][2]
                RIJ2 = A1 * A1 + A2 * A2 + A3 * A3
                DV = [vp[J][0] - vp[I][0], vp[J][1] - vp[I][1], vp[J][2] - vp[I][2]]
                DR2I = 1.0 / RIJ2
                DR3I = m[J] * DR2I * np.sqrt(DR2I)
                DRDV = 3.0 * (A1 * DV[0] + A2 * DV[1] + A3 * DV[2]) * DR2I
                FCM = [A1 * DR3I, A2 * DR3I, A3 * DR3I]
                FCMD = [(DV[0] - A1 * DRDV) * DR3I, (DV[1] - A2 * DRDV) * DR3I, (DV[2] - A3 * DRDV) * DR3I]
                FP, FPD = [0.0] * 6, [0.0] * 6
                for half in range(2):
                    dr2 = 0.0
                    drdv = 0.0
                    dx = [0.0] * 3
                    dv = [0.0] * 3
                    for L in range(3):
                        dx[L] = S["xk"][q][half][L] - xp[I][L]
                        dv[L] = S["vk"][q][half][L] - vp[I][L]
                        dr2 = dr2 + dx[L] ** 2
                        drdv = drdv + dx[L] * dv[L]
                    dr2i = 1.0 / dr2
                    dr3i = S["mk"][q][half] * dr2i * np.sqrt(dr2i)
                    drdv = 3.0 * drdv * dr2i
                    for L in range(3):
                        FP[L + 3 * half] = dx[L] * dr3i
                        FPD[L + 3 * half] = (dv[L] - dx[L] * drdv) * dr3i
                for L in range(3):
                    firr[L] = firr[L] + (FP[L] + FP[L + 3] - FCM[L])
                    fd[L] = fd[L] + (FPD[L] + FPD[L + 3] - FCMD[L])
        out_a.append(firr)
        out_j.append(fd)
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


@pytest.mark.parametrize("seed", [11, 14])
def test_oracle_corrections_equal_the_reference_routines(orc, seed):
    """The oracle's corrections against CMFIRR_COR / CMFIRR_UCOR restated
    statement by statement (their control flow and operation order): the
    same values, bit for bit.  The system has perturbers that are perturbed
    pairs themselves (CMFIRR_COR's second pass, GO TO 20), unperturbed c.m.
    neighbours (skipped by CMFIRR_UCOR) and bodies whose lists end in c.m.
    bodies only."""
    S = _system(seed)
    ca, cj = _oracle_corrections(orc, S)
    ra, rj = _reference_routines(S)
    assert np.abs(ra).max() > 0
    np.testing.assert_array_equal(ca, ra)
    np.testing.assert_array_equal(cj, rj)


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
