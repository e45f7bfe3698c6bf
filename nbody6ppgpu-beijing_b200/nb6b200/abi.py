"""ctypes mirror of the reference's Fortran-callable force ABI.

The reference's driver calls (``util_gpu.F:59``, ``fpoly0.F:31,79,131,381``,
``energy.F:33``, ``intgrt.F:533,1229``) pass every argument by pointer and
arrays in Fortran column-major order, i.e. ``X(3,N)`` is C ``double[N][3]``.
:class:`ForceLib` binds those symbols on any shared object that exports them
-- this package's ``libnb6b200.so`` or, in the tests, the reference's own CPU
libraries -- and offers numpy-level calls with the reference's argument
meaning:

* ``gpunb_open(nbmax, irank)``, ``gpunb_send(m, x, v)``,
  ``gpunb_regf(h2, dtr, xi, vi, lmax, nnbmax, m_flag)`` ->
  ``(acc, jrk, pot, list)`` (``gpunb.velocity.cu:905-940``);
* ``gpupot(irank, istart, ni, m, x)`` -> ``pot`` (``gpupot.gpu.cu:116-127``);
* ``irr_simd_open/set_jp/set_list/firr_vec/close``
  (``irr.avx.cpp:568-606``).

Nothing here computes forces; it only marshals arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_d)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_i)


def _f64(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        out = out.reshape(shape)
    return out


def _ci(v: int):
    return C.byref(C.c_int(int(v)))


def _cd(v: float):
    return C.byref(C.c_double(float(v)))


class ForceLib:
    """Numpy-level calls onto a shared object exporting the reference ABI."""

    # Pad i-arrays to a multiple of 4: the reference AVX library reads four
    # i-particles at a time (reg.avx.cpp:204-226), past ni for ragged ni.
    IPAD = 4

    def __init__(self, lib: C.CDLL, name: str = "lib"):
        self.lib = lib
        self.name = name
        self.has_gpunb = hasattr(lib, "gpunb_regf_")
        self.has_gpupot = hasattr(lib, "gpupot_")
        self.has_irr = hasattr(lib, "irr_simd_firr_vec_")
        for fn in ("gpunb_open_", "gpunb_close_", "gpunb_send_", "gpunb_regf_",
                   "gpunb_profile_", "gpunb_devinit_", "gpupot_", "irr_simd_open_",
                   "irr_simd_close_", "irr_simd_set_jp_", "irr_simd_set_list_",
                   "irr_simd_firr_vec_", "irr_simd_profile_", "nb6_regf_seg_",
                   "nb6_irr_predict_send_"):
            if hasattr(lib, fn):
                getattr(lib, fn).restype = None

    # ------------------------------------------------------------------ gpunb
    def gpunb_open(self, nbmax: int, irank: int = 0) -> None:
        self.lib.gpunb_open_(_ci(nbmax), _ci(irank))

    def gpunb_close(self) -> None:
        self.lib.gpunb_close_()

    def gpunb_profile(self, irank: int = 0) -> None:
        self.lib.gpunb_profile_(_ci(irank))

    def gpunb_send(self, m, x, v) -> None:
        m = _f64(m)
        n = m.shape[0]
        x = _f64(x, (n, 3))
        v = _f64(v, (n, 3))
        self.lib.gpunb_send_(_ci(n), _dp(m), _dp(x), _dp(v))

    def gpunb_regf(self, h2, dtr, xi, vi, lmax: int, nnbmax: int, m_flag: int = 0):
        h2 = _f64(h2)
        ni = h2.shape[0]
        pad = (-ni) % self.IPAD
        npad = ni + pad

        def padv(a, cols=None):
            a = _f64(a, (ni,) if cols is None else (ni, cols))
            if pad == 0:
                return np.ascontiguousarray(a)
            shape = (npad,) if cols is None else (npad, cols)
            out = np.zeros(shape)
            out[:ni] = a
            return out

        h2p, dtrp = padv(h2), padv(dtr)
        xip, vip = padv(xi, 3), padv(vi, 3)
        acc = np.zeros((npad, 3))
        jrk = np.zeros((npad, 3))
        pot = np.zeros(npad)
        lst = np.zeros((npad, lmax), dtype=np.int32)
        self.lib.gpunb_regf_(_ci(ni), _dp(h2p), _dp(dtrp), _dp(xip), _dp(vip), _dp(acc),
                             _dp(jrk), _dp(pot), _ci(lmax), _ci(nnbmax), _ip(lst), _ci(m_flag))
        return acc[:ni], jrk[:ni], pot[:ni], lst[:ni]

    def regf_seg(self, h2, dtr, xi, vi, iseg, seg_j0, lmax: int, nnbmax: int, m_flag: int = 0):
        """nb6_regf_seg_ (this package's extension; no reference counterpart):
        gpunb_regf for an ensemble of clusters sent together.  Segment c is
        j range [seg_j0[c], seg_j0[c+1]) of the last send; i-particle k
        belongs to segment iseg[k] (non-decreasing).  List ids come back
        relative to the segment's first j."""
        h2 = _f64(h2)
        ni = h2.shape[0]
        iseg = np.ascontiguousarray(iseg, dtype=np.int32)
        seg_j0 = np.ascontiguousarray(seg_j0, dtype=np.int32)
        nseg = seg_j0.shape[0] - 1
        dtr = _f64(dtr, (ni,))
        xi = _f64(xi, (ni, 3))
        vi = _f64(vi, (ni, 3))
        acc = np.zeros((ni, 3))
        jrk = np.zeros((ni, 3))
        pot = np.zeros(ni)
        lst = np.zeros((ni, lmax), dtype=np.int32)
        self.lib.nb6_regf_seg_(_ci(ni), _ip(iseg), _dp(h2), _dp(dtr), _dp(xi), _dp(vi), _dp(acc),
                               _dp(jrk), _dp(pot), _ci(lmax), _ci(nnbmax), _ip(lst), _ci(m_flag),
                               _ci(nseg), _ip(seg_j0))
        return acc, jrk, pot, lst

    # ----------------------------------------------------------------- gpupot
    def gpupot(self, m, x, istart: int = 1, ni: int | None = None, irank: int = 0,
               absolute_output: bool = False) -> np.ndarray:
        """pot[k] = potential at particle istart-1+k (the GPU library's and
        energy_mpi.F:216's convention).  The reference's CPU pot.avx.cpp
        writes pot[istart-1+k] instead (pot.avx.cpp:343); pass
        absolute_output=True for that library."""
        m = _f64(m)
        n = m.shape[0]
        x = _f64(x, (n, 3))
        if ni is None:
            ni = n - (istart - 1)
        off = (istart - 1) if absolute_output else 0
        # The AVX library writes 8 i at a time (pot.avx.cpp:296-343); pad by 8.
        pot = np.zeros(off + ni + 8)
        self.lib.gpupot_(_ci(irank), _ci(istart), _ci(ni), _ci(n), _dp(m), _dp(x), _dp(pot))
        return pot[off:off + ni].copy()

    # -------------------------------------------------------------- irregular
    def irr_open(self, nmax: int, lmax: int, rank: int = 0) -> None:
        self.lib.irr_simd_open_(_ci(nmax), _ci(lmax), _ci(rank))

    def irr_close(self, rank: int = 0) -> None:
        self.lib.irr_simd_close_(_ci(rank))

    def irr_profile(self, rank: int = 0) -> None:
        self.lib.irr_simd_profile_(_ci(rank))

    def irr_set_jp(self, addr: int, pos, vel, acc2, jrk6, mass: float, time: float) -> None:
        """addr is 1-based (Fortran particle index)."""
        p = _f64(pos, (3,))
        v = _f64(vel, (3,))
        a = _f64(acc2, (3,))
        j = _f64(jrk6, (3,))
        self.lib.irr_simd_set_jp_(_ci(addr), _dp(p), _dp(v), _dp(a), _dp(j), _cd(mass), _cd(time))

    def irr_set_jp_all(self, pos, vel, acc2, jrk6, mass, time, first: int = 1) -> None:
        pos = _f64(pos)
        n = pos.shape[0]
        vel, acc2, jrk6 = _f64(vel), _f64(acc2), _f64(jrk6)
        mass, time = _f64(mass), _f64(time)
        fn = self.lib.irr_simd_set_jp_
        for k in range(n):
            fn(_ci(first + k), _dp(pos[k]), _dp(vel[k]), _dp(acc2[k]), _dp(jrk6[k]),
               C.byref(C.c_double(mass[k])), C.byref(C.c_double(time[k])))

    def irr_predict_send(self, t: float, addr0, count) -> None:
        """nb6_irr_predict_send_ (extension): the gpunb j set made on the
        device from the resident irregular records predicted to t; segment s
        is count[s] records from 1-based address addr0[s]."""
        addr0 = np.ascontiguousarray(addr0, dtype=np.int32)
        count = np.ascontiguousarray(count, dtype=np.int32)
        self.lib.nb6_irr_predict_send_(_cd(t), _ci(addr0.shape[0]), _ip(addr0), _ip(count))

    def irr_set_list(self, addr: int, nblist) -> None:
        """nblist = [nnb, j1, ..., jnnb] with 1-based j (Fortran LIST(1,I)).

        The reference reads ids in blocks of 8 (irr.avx.cpp:468-489), so the
        row handed over is padded to a multiple of 8 past nnb."""
        row = np.asarray(nblist, dtype=np.int32)
        nnb = int(row[0])
        padded = np.zeros(1 + max(8, ((nnb + 7) // 8) * 8), dtype=np.int32)
        padded[: row.shape[0]] = row[: padded.shape[0]]
        self.lib.irr_simd_set_list_(_ci(addr), _ip(padded))

    # ------------------------------------------ device correctors and clock
    def hermite_open(self, eta_i: float, smax: float, dtmin: float) -> None:
        """nb6_hermite_open_ (extension): the per-body Hermite state on the
        device, after irr_open."""
        self.lib.nb6_hermite_open_(_cd(eta_i), _cd(smax), _cd(dtmin))

    def hermite_set_all(self, fi, fidot, fr, frdot, step, t0r, stepr, rs, first: int = 1) -> None:
        """nb6_hermite_set_ for bodies first, first+1, ... (1-based)."""
        fi, fidot, fr, frdot = _f64(fi), _f64(fidot), _f64(fr), _f64(frdot)
        step, t0r, stepr, rs = _f64(step), _f64(t0r), _f64(stepr), _f64(rs)
        fn = self.lib.nb6_hermite_set_
        for k in range(fi.shape[0]):
            fn(_ci(first + k), _dp(fi[k]), _dp(fidot[k]), _dp(fr[k]), _dp(frdot[k]),
               C.byref(C.c_double(step[k])), C.byref(C.c_double(t0r[k])),
               C.byref(C.c_double(stepr[k])), C.byref(C.c_double(rs[k])))

    def hermite_get(self, a0: int, n: int) -> np.ndarray:
        """nb6_hermite_get_: rows (n, 32) of the resident state."""
        out = np.zeros((max(n, 1), 32))
        self.lib.nb6_hermite_get_(_ci(a0), _ci(n), _dp(out))
        return out[:n]

    def irr_correct(self, time: float, addr) -> np.ndarray:
        """nb6_irr_correct_: corrector rows (ni, 24) of the bodies addr."""
        addr = np.ascontiguousarray(addr, dtype=np.int32)
        out = np.zeros((max(addr.shape[0], 1), 24))
        self.lib.nb6_irr_correct_(_cd(time), _ci(addr.shape[0]), _ip(addr), _dp(out))
        return out[:addr.shape[0]]

    def regf_correct(self, time: float, addr, iseg, seg_j0, seg_a0, h2, dtr, rs, xi, vi, lmax: int,
                     nnbmax: int, m_flag: int, prm) -> np.ndarray:
        """nb6_regf_correct_ (extension): regular force and regular corrector
        of the bodies addr (1-based, grouped by segment iseg) on the device,
        after irr_predict_send; rows (ni, 32)."""
        addr = np.ascontiguousarray(addr, dtype=np.int32)
        ni = addr.shape[0]
        iseg = np.ascontiguousarray(iseg, dtype=np.int32)
        seg_j0 = np.ascontiguousarray(seg_j0, dtype=np.int32)
        seg_a0 = np.ascontiguousarray(seg_a0, dtype=np.int32)
        h2, dtr, rs = _f64(h2), _f64(dtr), _f64(rs)
        xi, vi = _f64(xi, (ni, 3)), _f64(vi, (ni, 3))
        prm = _f64(prm)
        out = np.zeros((max(ni, 1), 32))
        self.lib.nb6_regf_correct_(_cd(time), _ci(ni), _ip(addr), _ip(iseg), _ci(seg_a0.shape[0]),
                                   _ip(seg_j0), _ip(seg_a0), _dp(h2), _dp(dtr), _dp(rs), _dp(xi), _dp(vi),
                                   _ci(lmax), _ci(nnbmax), _ci(m_flag), _dp(prm), _dp(out))
        return out[:ni]

    def hermite_adjust(self, nb_flag: int, a0, par) -> None:
        """nb6_hermite_adjust_ (extension): the Ahmad-Cohen rule's form and
        per-cluster quantities (RDENS[3], RSCALE, RC2, RSFAC, BODYM, 0) for
        the device regular corrector; cluster c = addresses [a0[c], a0[c+1])."""
        a0 = np.ascontiguousarray(a0, dtype=np.int32)
        par = _f64(par).reshape(-1)
        ncl = a0.shape[0] - 1
        self.lib.nb6_hermite_adjust_(_ci(nb_flag), _ci(ncl), _ip(a0), _dp(par if par.size else np.zeros(8)))

    def lists_get(self, addr, ls: int) -> np.ndarray:
        """nb6_irr_lists_get_ (extension): resident neighbour rows (n, ls),
        [nnb, 1-based ids], of the bodies addr (1-based)."""
        addr = np.ascontiguousarray(addr, dtype=np.int32)
        n = addr.shape[0]
        out = np.zeros((max(n, 1), ls), dtype=np.int32)
        self.lib.nb6_irr_lists_get_(_ci(n), _ip(addr if n else np.zeros(1, np.int32)), _ci(ls), _ip(out))
        return out[:n]

    def blocks_run(self, tlimit: float, max_blocks: int) -> dict:
        """nb6_blocks_run_: blocks of irregular steps on the device."""
        reason, nact = C.c_int(0), C.c_int(0)
        nb, nirr = C.c_longlong(0), C.c_longlong(0)
        tb = C.c_double(0.0)
        self.lib.nb6_blocks_run_(_cd(tlimit), _ci(max_blocks), C.byref(reason), C.byref(nb), C.byref(nirr),
                                 C.byref(tb), C.byref(nact))
        return {"reason": reason.value, "blocks": nb.value, "irr_steps": nirr.value, "tblock": tb.value,
                "nact": nact.value}

    def blocks_mode(self, persistent: bool) -> None:
        """nb6_blocks_mode_: 1 one persistent launch per nb6_blocks_run_ call,
        0 (the default) a graph of two launches per block (same results)."""
        self.lib.nb6_blocks_mode_(_ci(1 if persistent else 0))

    def blocks_active(self, nmax: int) -> tuple[np.ndarray, np.ndarray]:
        """nb6_blocks_active_: the last block's active bodies (1-based) and
        corrector rows."""
        addr = np.zeros(max(nmax, 1), dtype=np.int32)
        rows = np.zeros((max(nmax, 1), 24))
        na = C.c_int(0)
        self.lib.nb6_blocks_active_(C.byref(na), _ip(addr), _dp(rows))
        return addr[:na.value], rows[:na.value]

    def blocks_regular(self, nmax: int) -> tuple[np.ndarray, np.ndarray]:
        """nb6_blocks_regular_: the last block's regular-due bodies
        (ascending, 1-based) with x0, v0."""
        addr = np.zeros(max(nmax, 1), dtype=np.int32)
        xv = np.zeros((max(nmax, 1), 6))
        nr = C.c_int(0)
        self.lib.nb6_blocks_regular_(C.byref(nr), _ip(addr), _dp(xv))
        return addr[:nr.value], xv[:nr.value]

    def ks_set(self, cm, xk, vk, mk, pofs, plist) -> None:
        """nb6_ks_set_ (extension): the perturbed KS pairs whose components
        the irregular force resolves from now on.  cm: 1-based c.m.
        addresses (npair); xk, vk: (npair, 2, 3) component positions and
        velocities at the coming irregular calls' time; mk: (npair, 2);
        pofs (npair + 1, pofs[0] = 0) and plist (1-based) the perturber
        lists.  An empty cm clears the table."""
        cm = np.ascontiguousarray(cm, dtype=np.int32).reshape(-1)
        npair = cm.shape[0]
        xk = _f64(np.reshape(xk, (-1, 6)) if npair else np.zeros((1, 6)))
        vk = _f64(np.reshape(vk, (-1, 6)) if npair else np.zeros((1, 6)))
        mk = _f64(np.reshape(mk, (-1, 2)) if npair else np.zeros((1, 2)))
        pofs = np.ascontiguousarray(pofs if npair else [0], dtype=np.int32)
        plist = np.ascontiguousarray(plist, dtype=np.int32).reshape(-1)
        if plist.size == 0:
            plist = np.zeros(1, dtype=np.int32)
        cmp = cm if npair else np.zeros(1, dtype=np.int32)
        self.lib.nb6_ks_set_(_ci(npair), _ip(cmp), _dp(xk), _dp(vk), _dp(mk), _ip(pofs), _ip(plist))

    def irr_firr_vec(self, ti: float, addr, out=None) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """irr_simd_firr_vec_: (acc, jrk, nnbid) of the bodies addr (1-based).
        out: optional (acc (ni, 3), jrk (ni, 3), nnbid (ni,) int32) arrays to
        fill, as a Fortran caller passes its own static arrays."""
        addr = np.ascontiguousarray(addr, dtype=np.int32)
        ni = addr.shape[0]
        if out is None:
            acc = np.zeros((max(ni, 1), 3))
            jrk = np.zeros((max(ni, 1), 3))
            nnbid = np.zeros(max(ni, 1), dtype=np.int32)
        else:
            acc, jrk, nnbid = out
            assert acc.dtype == np.float64 and jrk.dtype == np.float64 and nnbid.dtype == np.int32
            assert acc.flags.c_contiguous and jrk.flags.c_contiguous and nnbid.flags.c_contiguous
            assert acc.shape[0] >= ni and jrk.shape[0] >= ni and nnbid.shape[0] >= ni
        self.lib.irr_simd_firr_vec_(_cd(ti), _ci(ni), _ip(addr), _dp(acc), _dp(jrk), _ip(nnbid))
        return acc[:ni], jrk[:ni], nnbid[:ni]
