"""ctypes access to the parity checkers (TEST INFRASTRUCTURE ONLY).

* :func:`fp64` -- the FP64 C restatement (``oracle/liboracle.so``) of the
  reference's force loops, see ``nb6_oracle.h`` for the cited lines.
* :func:`ref_lib` -- the reference's own CPU force libraries
  (``oracle/_ref/libref_{reg,pot,irr}_avx.so``) compiled from their sources by
  ``oracle/Makefile``.  Each is loaded RTLD_LOCAL and was linked -Bsymbolic,
  so its ``gpunb_*`` / ``gpupot_`` / ``irr_simd_*`` never bind to the
  product's symbols of the same name.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product path never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)


def build(ref: bool = True) -> None:
    """Run oracle/Makefile (the reference libraries only if their sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


_FP64 = None


def fp64():
    global _FP64
    if _FP64 is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        lib = C.CDLL(ORACLE_SO, mode=C.RTLD_LOCAL)
        lib.orc_regf.restype = C.c_long
        lib.orc_pot.restype = None
        lib.orc_predict.restype = None
        lib.orc_firr.restype = None
        _FP64 = lib
    return _FP64


def ref_path(name: str) -> str:
    """name in {"reg", "pot", "irr"} (the AVX CPU libraries),
    "gpunb_velocity" or "gpupot_gpu" (the reference's CUDA libraries)."""
    if name in ("gpunb_velocity", "gpupot_gpu"):
        return os.path.join(REF_DIR, f"libref_{name}.so")
    return os.path.join(REF_DIR, f"libref_{name}_avx.so")


def ref_available(name: str) -> bool:
    return os.path.exists(ref_path(name))


def ref_lib(name: str) -> C.CDLL:
    """name in {"reg", "pot", "irr"}."""
    p = ref_path(name)
    if not os.path.exists(p):
        raise FileNotFoundError(p)
    return C.CDLL(p, mode=C.RTLD_LOCAL)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def regf(mj, xj, vj, h2, dtr, xi, vi, lmax, nnbmax, m_flag=0):
    """FP64 regular force (gpunb_regf_ semantics).  Returns acc, jrk, pot, list."""
    mj, xj, vj = _f(mj), _f(xj), _f(vj)
    h2, dtr, xi, vi = _f(h2), _f(dtr), _f(xi), _f(vi)
    nj, ni = mj.shape[0], h2.shape[0]
    acc = np.zeros((ni, 3))
    jrk = np.zeros((ni, 3))
    pot = np.zeros(ni)
    lst = np.zeros((ni, lmax), dtype=np.int32)
    fp64().orc_regf(int(nj), mj.ctypes.data_as(_d), xj.ctypes.data_as(_d), vj.ctypes.data_as(_d),
                    int(ni), h2.ctypes.data_as(_d), dtr.ctypes.data_as(_d),
                    xi.ctypes.data_as(_d), vi.ctypes.data_as(_d), int(lmax), int(nnbmax),
                    int(m_flag),
                    acc.ctypes.data_as(_d), jrk.ctypes.data_as(_d), pot.ctypes.data_as(_d),
                    lst.ctypes.data_as(_i))
    return acc, jrk, pot, lst


def pot(m, x, istart=1, ni=None):
    m, x = _f(m), _f(x)
    n = m.shape[0]
    if ni is None:
        ni = n - istart + 1
    out = np.zeros(int(ni))
    fp64().orc_pot(int(n), m.ctypes.data_as(_d), x.ctypes.data_as(_d), int(istart), int(ni),
                   out.ctypes.data_as(_d))
    return out


def predict(time, t0, x0, x0dot, f, fdot):
    t0, x0, x0dot, f, fdot = _f(t0), _f(x0), _f(x0dot), _f(f), _f(fdot)
    n = t0.shape[0]
    x = np.zeros((n, 3))
    xd = np.zeros((n, 3))
    fp64().orc_predict(int(n), C.c_double(float(time)), t0.ctypes.data_as(_d), x0.ctypes.data_as(_d),
                       x0dot.ctypes.data_as(_d), f.ctypes.data_as(_d), fdot.ctypes.data_as(_d),
                       x.ctypes.data_as(_d), xd.ctypes.data_as(_d))
    return x, xd


def firr(ti, addr, x0, v0, acc2, jrk6, mass, t0, lists):
    """lists: (nmax, lmax) int32 rows [nnb, 1-based j...]; addr 1-based."""
    x0, v0, acc2, jrk6, mass, t0 = map(_f, (x0, v0, acc2, jrk6, mass, t0))
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    addr = np.ascontiguousarray(addr, dtype=np.int32)
    nmax, lmax = lists.shape
    ni = addr.shape[0]
    acc = np.zeros((ni, 3))
    jrk = np.zeros((ni, 3))
    nnbid = np.zeros(ni, dtype=np.int32)
    fp64().orc_firr(C.c_double(float(ti)), int(ni), addr.ctypes.data_as(_i), int(nmax),
                    x0.ctypes.data_as(_d),
                    v0.ctypes.data_as(_d), acc2.ctypes.data_as(_d), jrk6.ctypes.data_as(_d),
                    mass.ctypes.data_as(_d), t0.ctypes.data_as(_d), lists.ctypes.data_as(_i),
                    int(lmax), acc.ctypes.data_as(_d), jrk.ctypes.data_as(_d),
                    nnbid.ctypes.data_as(_i))
    return acc, jrk, nnbid


def ks_cmcorr(ti, addr, x0, v0, acc2, jrk6, mass, t0, lists, slot, xk, vk, mk, pofs, plist, acc, jrk):
    """acc, jrk of the active bodies addr (1-based) plus the KS c.m.
    corrections of cmfirr_cor.f / cmfirr_ucor.f (returned as new arrays).
    slot[a-1] = perturbed pair of c.m. body a or -1; xk, vk (npair, 2, 3),
    mk (npair, 2); pofs (npair+1), plist 1-based perturbers."""
    x0, v0, acc2, jrk6, mass, t0 = map(_f, (x0, v0, acc2, jrk6, mass, t0))
    lists = np.ascontiguousarray(lists, dtype=np.int32)
    addr = np.ascontiguousarray(addr, dtype=np.int32)
    slot = np.ascontiguousarray(slot, dtype=np.int32)
    xk = np.ascontiguousarray(xk, dtype=np.float64).reshape(-1, 6)
    vk = np.ascontiguousarray(vk, dtype=np.float64).reshape(-1, 6)
    mk = np.ascontiguousarray(mk, dtype=np.float64).reshape(-1, 2)
    pofs = np.ascontiguousarray(pofs, dtype=np.int32)
    plist = np.ascontiguousarray(plist, dtype=np.int32)
    if plist.size == 0:
        plist = np.zeros(1, dtype=np.int32)
    if xk.size == 0:
        xk, vk, mk = np.zeros((1, 6)), np.zeros((1, 6)), np.zeros((1, 2))
    acc = np.array(acc, dtype=np.float64, order="C")
    jrk = np.array(jrk, dtype=np.float64, order="C")
    lmax = lists.shape[1]
    fp64().orc_ks_cmcorr(C.c_double(float(ti)), int(addr.shape[0]), addr.ctypes.data_as(_i),
                         x0.ctypes.data_as(_d), v0.ctypes.data_as(_d), acc2.ctypes.data_as(_d),
                         jrk6.ctypes.data_as(_d), mass.ctypes.data_as(_d), t0.ctypes.data_as(_d),
                         lists.ctypes.data_as(_i), int(lmax), slot.ctypes.data_as(_i),
                         xk.ctypes.data_as(_d), vk.ctypes.data_as(_d), mk.ctypes.data_as(_d),
                         pofs.ctypes.data_as(_i), plist.ctypes.data_as(_i),
                         acc.ctypes.data_as(_d), jrk.ctypes.data_as(_d))
    return acc, jrk


def ac_radius(kz39, nnbopt, nnbmax, adj, nnb, nnb0, dtr, xi, vi, rs, xnb=None, vnb=None):
    """Ahmad-Cohen radius rule (regcor_gpu.F:19-238).  adj = (RDENS[3],
    RSCALE, RC2, RSFAC, BODYM).  Returns (new rs, dfirr, dfd)."""
    nnb = np.ascontiguousarray(nnb, dtype=np.int32)
    n = nnb.shape[0]
    nnb0 = np.ascontiguousarray(nnb0, dtype=np.int32)
    dtr, xi, vi = _f(np.broadcast_to(dtr, (n,))), _f(xi).reshape(n, 3), _f(vi).reshape(n, 3)
    xnb = np.zeros((n, 3, 3)) if xnb is None else _f(xnb).reshape(n, 3, 3)
    vnb = np.zeros((n, 3, 3)) if vnb is None else _f(vnb).reshape(n, 3, 3)
    adj = _f(adj).reshape(7)
    out = _f(rs).reshape(n).copy()
    dfirr = np.zeros((n, 3))
    dfd = np.zeros((n, 3))
    fp64().orc_ac_radius(int(n), int(kz39), int(nnbopt), int(nnbmax), adj.ctypes.data_as(_d),
                         nnb.ctypes.data_as(_i), nnb0.ctypes.data_as(_i), dtr.ctypes.data_as(_d),
                         xi.ctypes.data_as(_d), vi.ctypes.data_as(_d), xnb.ctypes.data_as(_d),
                         vnb.ctypes.data_as(_d), out.ctypes.data_as(_d), dfirr.ctypes.data_as(_d),
                         dfd.ctypes.data_as(_d))
    return out, dfirr, dfd


def ac_shrink(kz39, nnbopt, nnbmax, nnb_neg, rs):
    """Overflow shrink of RS (util_gpu.F:69-100)."""
    nnb_neg = np.ascontiguousarray(nnb_neg, dtype=np.int32)
    out = _f(rs).reshape(-1).copy()
    fp64().orc_ac_shrink(int(out.shape[0]), int(kz39), int(nnbopt), int(nnbmax),
                         nnb_neg.ctypes.data_as(_i), out.ctypes.data_as(_d))
    return out
