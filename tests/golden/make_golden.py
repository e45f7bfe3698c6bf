"""Generate the golden fixtures from the reference's own CPU force libraries.

    python tests/golden/make_golden.py

The reference tree ships no test vectors, so the fixtures are produced by
executing its libraries -- ``reg.avx.cpp`` (gpunb_*), ``pot.avx.cpp``
(gpupot_) and ``irr.avx.cpp`` (irr_simd_*), compiled from their sources by
``oracle/Makefile`` into ``oracle/_ref`` -- on seeded synthetic inputs from
``nb6b200.ics``.  Each ``.npz`` holds the inputs and the reference outputs.
The FP64 oracle is pinned against these files (tests/test_oracle_pin.py) and
the CUDA library is checked against both.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
os.environ.setdefault("OMP_NUM_THREADS", str(min(32, os.cpu_count() or 1)))
sys.path[:0] = [os.path.join(ROOT, "nbody6ppgpu-beijing_b200"), os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from nb6b200 import ics  # noqa: E402
from nb6b200.abi import ForceLib  # noqa: E402


def reg_case(name, cl, isel, lmax, nnbmax, m_flag):
    lib = ForceLib(oracle.ref_lib("reg"), "ref-reg-avx")
    lib.gpunb_open(cl.n + 10, 0)
    lib.gpunb_send(cl.mass, cl.pos, cl.vel)
    h2 = cl.h2(m_flag)[isel]
    acc, jrk, pot, lst = lib.gpunb_regf(h2, cl.dtr[isel], cl.pos[isel], cl.vel[isel], lmax,
                                        nnbmax, m_flag)
    lib.gpunb_close()
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), mj=cl.mass, xj=cl.pos, vj=cl.vel,
                        isel=isel, h2=h2, dtr=cl.dtr[isel], xi=cl.pos[isel],
                        vi=cl.vel[isel], lmax=lmax, nnbmax=nnbmax, m_flag=m_flag,
                        acc=acc, jrk=jrk, pot=pot, list=lst)
    nn = lst[:, 0]
    print(f"{name}: ni={len(isel)} nj={cl.n} nnb mean={nn[nn >= 0].mean() if (nn >= 0).any() else 0:.1f} "
          f"overflow={int((nn < 0).sum())}")


def pot_case(name, cl, istart, ni):
    lib = ForceLib(oracle.ref_lib("pot"), "ref-pot-avx")
    pot = lib.gpupot(cl.mass, cl.pos, istart=istart, ni=ni, absolute_output=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), m=cl.mass, x=cl.pos,
                        istart=istart, ni=ni, pot=pot)
    print(f"{name}: n={cl.n} istart={istart} ni={ni}")


def irr_case(name, cl, seed):
    rng = np.random.default_rng(seed)
    n = cl.n
    lmax = 601
    # F = a/2 and FDOT = adot/6 from the FP64 full force (neighbours included)
    # h2 tiny: only the self pair (r2 = 0) counts as a neighbour
    h2 = np.full(n, 1e-30)
    acc, jrk, _, _ = oracle.regf(cl.mass, cl.pos, cl.vel, h2, np.zeros(n), cl.pos, cl.vel, 8, 6)
    f2 = 0.5 * acc
    fd6 = jrk / 6.0
    t0 = -rng.integers(0, 8, n) / 1024.0          # last-step times on the block grid
    ti = 1.0 / 512.0
    # neighbour lists from the FP64 regular rule, self removed, 1-based
    _, _, _, lst = oracle.regf(cl.mass, cl.pos, cl.vel, cl.rs ** 2, cl.dtr, cl.pos, cl.vel,
                               lmax, lmax - 1, 0)
    lists = np.zeros((n, lmax), dtype=np.int32)
    for i in range(n):
        k = int(lst[i, 0])
        ids = [j + 1 for j in lst[i, 1:1 + k] if j != i][: lmax - 1]
        if i == 5:
            ids = []                                  # an empty list
        lists[i, 0] = len(ids)
        lists[i, 1:1 + len(ids)] = ids
    addr = np.sort(rng.choice(n, size=min(300, n), replace=False) + 1).astype(np.int32)
    addr[0] = 6                                       # include the empty-list particle
    addr = np.unique(addr)
    lib = ForceLib(oracle.ref_lib("irr"), "ref-irr-avx")
    lib.irr_open(n, lmax, 0)
    lib.irr_set_jp_all(cl.pos, cl.vel, f2, fd6, cl.mass, t0)
    for i in range(n):
        lib.irr_set_list(i + 1, lists[i])
    a, j, nnbid = lib.irr_firr_vec(ti, addr)
    lib.irr_close(0)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), x0=cl.pos, v0=cl.vel, acc2=f2,
                        jrk6=fd6, mass=cl.mass, t0=t0, ti=ti, lists=lists, addr=addr,
                        acc=a, jrk=j, nnbid=nnbid)
    print(f"{name}: n={n} ni={len(addr)} mean nnb={lists[:, 0].mean():.1f}")


def main():
    for lib in ("reg", "pot", "irr"):
        if not oracle.ref_available(lib):
            oracle.build(ref=True)
    c1 = ics.plummer(1024, seed=43532, imf=False, nnbopt=50)
    reg_case("reg_plummer1k", c1, np.arange(1024), lmax=512, nnbmax=400, m_flag=0)
    reg_case("reg_plummer1k_overflow", c1, np.arange(1024), lmax=96, nnbmax=64, m_flag=0)
    c2 = ics.plummer(2000, seed=7, imf=True, nnbopt=50)
    isel = np.sort(np.random.default_rng(3).choice(2000, size=777, replace=False))
    reg_case("reg_kroupa2k_mflag", c2, isel, lmax=512, nnbmax=400, m_flag=1)
    pot_case("pot_plummer1k", c1, 1, 1024)
    pot_case("pot_kroupa2k_partial", c2, 101, 333)
    irr_case("irr_plummer1k", c1, seed=11)


if __name__ == "__main__":
    main()
