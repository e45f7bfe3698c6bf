"""Seeded synthetic star-cluster initial conditions in Henon units.

These stand in for the reference's own generators (Plummer in
``setup.F:58-101``, the Kroupa 2001 IMF of ``imfbd.f:46-60``, binaries of
``binpop.F``, Henon scaling of ``scale.F``) and for King models, which the
reference only reads from ``dat.10`` (``data.F:36-47``).  They are written from
the published models, not from the reference code:

* Plummer (1911) sphere sampled as in Aarseth, Henon & Wielen (1974):
  r from the inverted cumulative mass, |v| by von Neumann rejection on
  q^2 (1-q^2)^3.5;
* King (1966) lowered-isothermal model: the dimensionless Poisson equation is
  integrated from W(0) = W0 outwards, radii are drawn from the cumulative mass
  and speeds by rejection from v^2 (exp(W - v^2/2) - 1);
* Kroupa (2001) broken power law (alpha = 0.3/1.3/2.3 below/above
  0.08 and 0.5 Msun) sampled by inverse CDF per segment;
* binaries: pairs drawn from the IMF enter as one centre-of-mass body; the
  internal semi-major axis (log-uniform) and eccentricity (f(e) = 2e) are
  returned for the host's KS bookkeeping only;
* scaling to G = M = 1, E = -1/4 at virial ratio Q = 0.5 uses the model's
  analytic potential energy (exact in expectation; no O(N^2) sum).

Neighbour radii follow the local number density so that a particle sees
about ``nnbopt`` neighbours, the state the Ahmad-Cohen rule drives RS to
(``regcor_gpu.F:131-238``); ``dtr`` (STEPR) is a power of two of the order of
the neighbour-sphere crossing time.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Cluster:
    mass: np.ndarray           # (n,)
    pos: np.ndarray            # (n, 3)
    vel: np.ndarray            # (n, 3)
    rs: np.ndarray             # (n,) neighbour radius RS
    dtr: np.ndarray            # (n,) regular step STEPR
    model: str = ""
    npairs: int = 0            # binaries folded into c.m. bodies
    binary_a_au: np.ndarray = field(default_factory=lambda: np.zeros(0))
    binary_e: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])

    def h2(self, m_flag: int = 0) -> np.ndarray:
        """Per-i neighbour criterion as util_gpu.F:46-51 packs it."""
        h2 = self.rs ** 2
        if m_flag:
            h2 = h2 / self.mass.mean()  # RS^2 / BODYM
        return h2


# ---------------------------------------------------------------------------
# IMF
# ---------------------------------------------------------------------------
def kroupa_imf(n: int, rng: np.random.Generator, mlo: float = 0.08, mhi: float = 100.0,
               ) -> np.ndarray:
    """Kroupa (2001) masses in Msun over [mlo, mhi]."""
    breaks = [0.01, 0.08, 0.5, 1e9]
    alphas = [0.3, 1.3, 2.3]
    # segment weights from the integral of m^-alpha with continuity factors
    segs = []
    k = 1.0
    for s in range(3):
        a, b = max(breaks[s], mlo), min(breaks[s + 1], mhi)
        if s > 0:
            k *= breaks[s] ** (alphas[s] - alphas[s - 1])
        if a >= b:
            segs.append((a, b, alphas[s], 0.0))
            continue
        al = alphas[s]
        w = k * (b ** (1 - al) - a ** (1 - al)) / (1 - al)
        segs.append((a, b, al, w))
    w = np.array([s[3] for s in segs])
    w = w / w.sum()
    which = rng.choice(3, size=n, p=w)
    u = rng.random(n)
    m = np.empty(n)
    for s, (a, b, al, _) in enumerate(segs):
        sel = which == s
        if not sel.any():
            continue
        e = 1 - al
        m[sel] = (a ** e + u[sel] * (b ** e - a ** e)) ** (1.0 / e)
    return m


# ---------------------------------------------------------------------------
# Plummer
# ---------------------------------------------------------------------------
def _iso(rng: np.random.Generator, r: np.ndarray) -> np.ndarray:
    n = r.shape[0]
    z = 1.0 - 2.0 * rng.random(n)
    ph = 2.0 * np.pi * rng.random(n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * s * np.cos(ph), r * s * np.sin(ph), r * z], axis=1)


def _plummer_unit(n: int, rng: np.random.Generator) -> tuple[np.ndarray, np.ndarray]:
    """Plummer sphere with a = 1, G = M = 1 (not yet in Henon units)."""
    r = np.empty(0)
    while r.shape[0] < n:
        x = rng.random(2 * n)
        x = x[x > 1e-10]
        rr = (x ** (-2.0 / 3.0) - 1.0) ** -0.5
        r = np.concatenate([r, rr[rr <= 10.0]])
    r = r[:n]
    q = np.empty(0)
    while q.shape[0] < n:
        a = rng.random(3 * n)
        b = rng.random(3 * n)
        ok = 0.1 * b <= a * a * (1.0 - a * a) ** 3.5
        q = np.concatenate([q, a[ok]])
    q = q[:n]
    vesc = np.sqrt(2.0) * (1.0 + r * r) ** -0.25
    return _iso(rng, r), _iso(rng, q * vesc)


def plummer(n: int, seed: int = 43532, imf: bool = False, nnbopt: int = 50,
            smax: float = 0.125) -> Cluster:
    rng = np.random.default_rng(seed)
    pos, vel = _plummer_unit(n, rng)
    if imf:
        m = kroupa_imf(n, rng)
        m = m / m.sum()
    else:
        m = np.full(n, 1.0 / n)
    pos -= (m[:, None] * pos).sum(0)
    vel -= (m[:, None] * vel).sum(0)
    # Plummer a = 1 has W = -3 pi / 32 (G = M = 1); Henon: W = -1/2, K = 1/4.
    sx = 3.0 * np.pi / 16.0
    pos *= sx
    vel /= np.sqrt(sx)
    rho_of_r = lambda rr: (3.0 / (4.0 * np.pi * sx ** 3)) * (1 + (rr / sx) ** 2) ** -2.5
    sig_of_r = lambda rr: np.sqrt((1.0 / sx) / 6.0 / np.sqrt(1 + (rr / sx) ** 2))
    rs, dtr = _radii_steps(pos, m, rho_of_r, sig_of_r, nnbopt, smax)
    return Cluster(m, pos, vel, rs, dtr, model=f"plummer{'-kroupa' if imf else ''}")


# ---------------------------------------------------------------------------
# King (1966)
# ---------------------------------------------------------------------------
def _king_density(w: np.ndarray) -> np.ndarray:
    """Dimensionless King density rho(W)/rho_1 with sigma = 1."""
    from scipy.special import erf
    w = np.maximum(w, 0.0)
    return np.exp(w) * erf(np.sqrt(w)) - np.sqrt(4.0 * w / np.pi) * (1.0 + 2.0 * w / 3.0)


def king_profile(w0: float, npts: int = 20000):
    """Integrate W'' + 2 W'/r = -9 rho(W)/rho(W0) from r = 0 to W = 0.

    Returns radius grid (units of the King radius r0), W, density rho/rho0 and
    enclosed mass (arbitrary units)."""
    from scipy.integrate import solve_ivp
    rho0 = _king_density(np.array([w0]))[0]

    def rhs(r, y):
        w, dw = y
        rho = _king_density(np.array([w]))[0] / rho0
        if r == 0.0:
            return [dw, -3.0 * rho]
        return [dw, -9.0 * rho - 2.0 * dw / r]

    def hit_zero(r, y):
        return y[0]
    hit_zero.terminal = True
    r_start = 1e-6
    y0 = [w0 - 1.5 * r_start ** 2, -3.0 * r_start]
    sol = solve_ivp(rhs, [r_start, 1e4], y0, events=hit_zero, rtol=1e-10, atol=1e-12,
                    dense_output=True, max_step=0.01)
    rt = sol.t_events[0][0] if sol.t_events[0].size else sol.t[-1]
    r = np.linspace(0.0, rt, npts)
    r[0] = 0.0
    w = np.empty_like(r)
    w[0] = w0
    w[1:] = sol.sol(np.maximum(r[1:], r_start))[0]
    w = np.maximum(w, 0.0)
    rho = _king_density(w) / rho0
    # enclosed mass by trapezoid of 4 pi r^2 rho
    dm = 4.0 * np.pi * r * r * rho
    mass = np.concatenate([[0.0], np.cumsum(0.5 * (dm[1:] + dm[:-1]) * np.diff(r))])
    return r, w, rho, mass


def king(n: int, w0: float = 6.0, seed: int = 20260, imf: bool = True,
         binary_fraction: float = 0.0, nnbopt: int = 50, smax: float = 0.125) -> Cluster:
    """King W0 model with n stars; a fraction of n (binary_fraction * n pairs)
    is folded into centre-of-mass bodies, giving n - npairs bodies."""
    rng = np.random.default_rng(seed)
    npairs = int(round(binary_fraction * n))
    nb = n - npairs
    r, w, rho, mcum = king_profile(w0)
    # radii by inverse cumulative mass
    u = rng.random(nb) * mcum[-1]
    ri = np.interp(u, mcum, r)
    wi = np.interp(ri, r, w)
    # speeds: p(v) ~ v^2 (exp(W - v^2/2) - 1), 0 <= v < sqrt(2W); sigma = 1
    v = np.zeros(nb)
    todo = np.arange(nb)
    while todo.size:
        vmax = np.sqrt(2.0 * wi[todo])
        x = rng.random(todo.size) * vmax
        fx = x * x * (np.exp(wi[todo] - 0.5 * x * x) - 1.0)
        # bound of the density on [0, vmax]: evaluate on a coarse grid per point
        g = np.linspace(0.0, 1.0, 33)[None, :] * vmax[:, None]
        fb = (g * g * (np.exp(wi[todo][:, None] - 0.5 * g * g) - 1.0)).max(axis=1) * 1.05 + 1e-300
        ok = rng.random(todo.size) * fb <= fx
        v[todo[ok]] = x[ok]
        todo = todo[~ok]
    pos = _iso(rng, ri)
    vel = _iso(rng, v)
    # masses: single stars and binary c.m. bodies (two IMF draws)
    if imf:
        m = kroupa_imf(nb + npairs, rng)
        mc = m[:nb].copy()
        mc[:npairs] += m[nb:]
    else:
        mc = np.ones(nb)
        mc[:npairs] = 2.0
    mc = mc / mc.sum()
    pos -= (mc[:, None] * pos).sum(0)
    vel -= (mc[:, None] * vel).sum(0)
    # Model units: sigma = 1, King radius r0 = 1, rho0 = 1, so that
    # 4 pi G rho0 = 9 (the scaling of W'' + 2W'/r = -9 rho/rho0).
    g = 9.0 / (4.0 * np.pi)
    mtot = mcum[-1]
    dm = np.diff(mcum)
    rm = 0.5 * (r[1:] + r[:-1])
    mm = 0.5 * (mcum[1:] + mcum[:-1])
    wpot = -g * np.sum(mm * dm / np.maximum(rm, 1e-12))   # W = -G int M(r) dM / r
    # Henon units: G = M = 1 and W = -1/2, i.e. virial radius 1.
    rv = g * mtot * mtot / (2.0 * abs(wpot))
    vu = np.sqrt(g * mtot / rv)
    pos /= rv
    vel /= vu
    rr = r / rv
    rho_h = rho / mtot * rv ** 3                  # mass fraction per Henon volume
    sig_h = np.sqrt(_king_vsq(w) / 3.0) / vu      # 1-D dispersion
    rho_of_r = lambda q: np.interp(q, rr, rho_h, right=rho_h[-1])
    sig_of_r = lambda q: np.interp(q, rr, sig_h, right=sig_h[-1])
    rs, dtr = _radii_steps(pos, mc, rho_of_r, sig_of_r, nnbopt, smax)
    a_au = np.exp(rng.uniform(np.log(0.005), np.log(50.0), npairs))
    ecc = np.sqrt(rng.random(npairs))
    return Cluster(mc, pos, vel, rs, dtr, model=f"king-w0={w0:g}", npairs=npairs,
                   binary_a_au=a_au, binary_e=ecc)


def _king_vsq(w: np.ndarray) -> np.ndarray:
    """Mean v^2 of the lowered Maxwellian at depth W (sigma = 1)."""
    from scipy.special import erf
    w = np.maximum(w, 1e-12)
    s = np.sqrt(w)
    # moments of v^2 (e^{W - v^2/2} - 1) on [0, sqrt(2W)]
    e = np.exp(w)
    m2 = e * (np.sqrt(np.pi / 2) * erf(s)) - np.sqrt(2 * w) * (1.0) - (2 * w) ** 1.5 / 3.0
    m4 = e * (3 * np.sqrt(np.pi / 2) * erf(s)) - np.sqrt(2 * w) * (3.0 + 2 * w) \
        - (2 * w) ** 2.5 / 5.0
    return np.where(m2 > 0, m4 / np.maximum(m2, 1e-300), 0.0)


def _radii_steps(pos, mass, rho_of_r, sig_of_r, nnbopt, smax):
    """RS = distance to the nnbopt-th nearest body (the radius the Ahmad-Cohen
    rule converges to) and STEPR from the RS crossing time."""
    from scipy.spatial import cKDTree
    n = pos.shape[0]
    r = np.sqrt((pos * pos).sum(1))
    k = min(nnbopt + 1, n)                     # +1: the query returns the body itself
    dist, _ = cKDTree(pos).query(pos, k=[k], workers=-1)
    rs = dist[:, 0] * (1.0 + 1e-9)
    sig = np.maximum(sig_of_r(r), 1e-6)
    t = np.maximum(0.25 * rs / sig, 1e-300)   # (coincident bodies: rs = 0)
    k = np.ceil(np.log2(np.maximum(smax / t, 1.0)))
    dtr = smax / 2.0 ** k
    return rs, dtr


def ensemble(nclusters: int = 256, nmin: int = 512, nmax: int = 8192, seed: int = 7,
             nnbopt: int = 50) -> list[Cluster]:
    """Independent Plummer clusters, N log-uniform in [nmin, nmax], own seeds."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(nmin), np.log(nmax), nclusters)).astype(int)
    return [plummer(int(nk), seed=int(seed * 1000 + c), imf=True, nnbopt=nnbopt)
            for c, nk in enumerate(ns)]


def predicted_distance_check(c: Cluster) -> float:
    """Fraction of bodies farther than 10 Henon lengths (diagnostic)."""
    return float((np.sqrt((c.pos ** 2).sum(1)) > 10).mean())
