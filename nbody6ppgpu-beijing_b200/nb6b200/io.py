"""The reference's initial-condition file formats (unit 10) and a writer.

* NBODY format, KZ(22) = 2, 6, 9, 10 (data.F:36-41): one body per record,
  ``BODY X Y Z VX VY VZ``, list-directed (blanks or commas, Fortran ``D``
  exponents allowed).
* TREE format, KZ(22) = 3, 7 (data.F:50-66): ``N``, two header records, N
  masses, N position triples, N velocity triples.

``write_nbody`` writes the NBODY format (what ``fort.10`` holds when the
reference is asked to write its initial conditions), so a run of this
package can be fed back to the reference.  ``to_henon`` rescales to Henon
units (G = M = 1, E = -1/4) at a given virial ratio, as scale.F does for
KZ(22) inputs without their own scaling.
"""
from __future__ import annotations

import numpy as np


def _tokens(path):
    with open(path) as f:
        for line in f:
            line = line.split("!")[0].replace(",", " ")
            for tok in line.split():
                yield tok


def _num(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def read_nbody(path, n: int | None = None):
    """(mass, pos, vel) from an NBODY-format file (all records, or the first
    n as data.F reads N of them)."""
    vals = np.array([_num(t) for t in _tokens(path)], dtype=np.float64)
    if vals.size % 7:
        raise ValueError(f"{path}: {vals.size} numbers is not a multiple of 7")
    rec = vals.reshape(-1, 7)
    if n is not None:
        if rec.shape[0] < n:
            raise ValueError(f"{path}: {rec.shape[0]} bodies, {n} requested")
        rec = rec[:n]
    return rec[:, 0].copy(), rec[:, 1:4].copy(), rec[:, 4:7].copy()


def read_tree(path):
    """(mass, pos, vel) from a TREE-format file."""
    with open(path) as f:
        lines = [ln for ln in f if ln.strip()]
    n = int(_num(lines[0].split()[0]))
    body = lines[3:]
    vals = np.array([_num(t) for ln in body for t in ln.replace(",", " ").split()], dtype=np.float64)
    if vals.size < 7 * n:
        raise ValueError(f"{path}: expected {7 * n} numbers after the header, found {vals.size}")
    m = vals[:n]
    pos = vals[n:4 * n].reshape(n, 3)
    vel = vals[4 * n:7 * n].reshape(n, 3)
    return m.copy(), pos.copy(), vel.copy()


def write_nbody(path, mass, pos, vel) -> None:
    """NBODY format, full double precision."""
    rec = np.column_stack([np.asarray(mass, dtype=np.float64), np.asarray(pos, dtype=np.float64).reshape(-1, 3),
                           np.asarray(vel, dtype=np.float64).reshape(-1, 3)])
    np.savetxt(path, rec, fmt="%.17e")


def potential_energy(mass, pos, block: int = 2048) -> float:
    """W = -sum_{i<j} m_i m_j / r_ij (FP64, blocked direct sum on the host)."""
    m = np.asarray(mass, dtype=np.float64)
    x = np.asarray(pos, dtype=np.float64)
    w = 0.0
    for a in range(0, len(m), block):
        d = x[a:a + block, None, :] - x[None, :, :]
        r = np.sqrt((d * d).sum(-1))
        idx = np.arange(a, min(a + block, len(m)))
        r[np.arange(len(idx)), idx] = np.inf
        w -= 0.5 * float((m[a:a + block, None] * m[None, :] / r).sum())
    return w


def to_henon(mass, pos, vel, q_vir: float = 0.5):
    """Total mass 1, centre of mass at rest at the origin, kinetic energy
    q_vir |W| and total energy -1/4 (scale.F)."""
    m = np.asarray(mass, dtype=np.float64) / float(np.sum(mass))
    x = np.asarray(pos, dtype=np.float64).copy()
    v = np.asarray(vel, dtype=np.float64).copy()
    x -= (m[:, None] * x).sum(0)
    v -= (m[:, None] * v).sum(0)
    w = potential_energy(m, x)
    k = 0.5 * float((m * (v * v).sum(1)).sum())
    if k > 0:
        v *= np.sqrt(q_vir * abs(w) / k)
    e = (q_vir - 1.0) * abs(w)           # after the velocity scaling
    s = e / -0.25                        # r -> r s, v -> v / sqrt(s) gives E / s
    return m, x * s, v / np.sqrt(s)
