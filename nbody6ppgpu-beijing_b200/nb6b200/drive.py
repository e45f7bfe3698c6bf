"""ctypes front end of the C++ block-step driver (libnb6drive.so).

``run(backend, cluster, ...)`` integrates a cluster of single stars with the
Hermite / Ahmad-Cohen block-step scheme of the reference (see
``driver/blockstep.cpp``) on a force backend given as shared-object paths:

* ``backend_paths("nb6b200")``  -- this package's libnb6b200.so for all three
  libraries;
* any other mapping {"reg": path, "irr": path, "pot": path}, e.g. the
  reference's own CPU libraries, so both run under the identical driver.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER_LIB = os.path.join(PKG_ROOT, "libnb6drive.so")


class Params(C.Structure):
    _fields_ = [("eta_i", C.c_double), ("eta_r", C.c_double), ("smax", C.c_double),
                ("dtmin", C.c_double), ("tcrit", C.c_double), ("dt_out", C.c_double),
                ("rs0", C.c_double), ("nnbopt", C.c_int), ("nnbmax", C.c_int),
                ("lmax", C.c_int), ("m_flag", C.c_int), ("chunk", C.c_int),
                ("max_blocks", C.c_longlong)]


class Stats(C.Structure):
    _fields_ = [("blocks", C.c_longlong), ("irr_steps", C.c_longlong),
                ("reg_steps", C.c_longlong), ("reg_calls", C.c_longlong),
                ("overflow_retries", C.c_longlong), ("nb_sum", C.c_longlong),
                ("reg_pairs", C.c_longlong), ("wall_reg", C.c_double),
                ("wall_irr", C.c_double), ("wall_total", C.c_double),
                ("t_end", C.c_double), ("nout", C.c_int)]


@dataclass
class RunResult:
    times: np.ndarray
    ekin: np.ndarray
    epot: np.ndarray
    etot: np.ndarray
    x: np.ndarray
    v: np.ndarray
    stats: dict

    @property
    def de_max(self) -> float:
        """max |E(t) - E(0)| / |E(0)| over the outputs."""
        return float(np.max(np.abs(self.etot - self.etot[0])) / abs(self.etot[0]))


_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(DRIVER_LIB):
            raise RuntimeError(f"{DRIVER_LIB} missing: run nbody6ppgpu-beijing_b200/build.py")
        _LIB = C.CDLL(DRIVER_LIB, mode=C.RTLD_LOCAL)
        _LIB.nb6drive_run.restype = C.c_int
    return _LIB


def backend_paths(name: str = "nb6b200") -> dict:
    if name == "nb6b200":
        from . import LIB_PATH
        return {"reg": LIB_PATH, "irr": LIB_PATH, "pot": LIB_PATH}
    raise ValueError(name)


def run(backend: dict, mass, pos, vel, *, tcrit=1.0, eta_i=0.02, eta_r=0.03, smax=0.125,
        dtmin=2.0 ** -24, dt_out=0.125, rs0=0.3, nnbopt=50, nnbmax=400, lmax=512, m_flag=0,
        chunk=1024, max_blocks=10_000_000) -> RunResult:
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    x = np.ascontiguousarray(pos, dtype=np.float64).reshape(n, 3).copy()
    v = np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 3).copy()
    p = Params(eta_i, eta_r, smax, dtmin, tcrit, dt_out, rs0, nnbopt, nnbmax, lmax, m_flag,
               chunk, max_blocks)
    nout_max = int(tcrit / dt_out) + 4
    eout = np.zeros((nout_max, 4))
    st = Stats()
    dp = C.POINTER(C.c_double)
    rc = _lib().nb6drive_run(backend["reg"].encode(), backend["irr"].encode(),
                             backend["pot"].encode(), C.c_int(n), mass.ctypes.data_as(dp),
                             x.ctypes.data_as(dp), v.ctypes.data_as(dp), C.byref(p),
                             eout.ctypes.data_as(dp), C.c_int(nout_max), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"nb6drive_run failed with code {rc}")
    k = st.nout
    stats = {f: getattr(st, f) for f, _ in Stats._fields_}
    return RunResult(eout[:k, 0], eout[:k, 1], eout[:k, 2], eout[:k, 3], x, v, stats)
