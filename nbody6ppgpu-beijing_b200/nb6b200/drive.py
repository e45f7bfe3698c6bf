"""ctypes front end of the C++ block-step driver (libnb6drive.so).

``run(backend, cluster, ...)`` integrates a cluster of single stars with the
Hermite / Ahmad-Cohen block-step scheme of the reference (see
``driver/blockstep.cpp``), and ``run_ensemble(backend, clusters, ...)`` an
ensemble of independent clusters with every force kind issued once per block
for all of them (``driver/ensemble.cpp``), on a force backend given as
shared-object paths:

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
                ("max_blocks", C.c_longlong), ("mlp_mode", C.c_int), ("mlp_pad", C.c_int),
                ("samples", C.POINTER(C.c_float)), ("sample_cap", C.c_longlong),
                ("rs_init", C.POINTER(C.c_double)), ("dev_corrector", C.c_int),
                ("seg_single", C.c_int), ("nb_flag", C.c_int), ("dt_adj", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("blocks", C.c_longlong), ("irr_steps", C.c_longlong),
                ("reg_steps", C.c_longlong), ("reg_calls", C.c_longlong),
                ("overflow_retries", C.c_longlong), ("nb_sum", C.c_longlong),
                ("reg_pairs", C.c_longlong), ("wall_reg", C.c_double),
                ("wall_irr", C.c_double), ("wall_total", C.c_double),
                ("t_end", C.c_double), ("nout", C.c_int), ("nsamples", C.c_longlong),
                ("mlp_used", C.c_longlong), ("mlp_fallback", C.c_longlong),
                ("nb_absdev", C.c_double)]


@dataclass
class RunResult:
    times: np.ndarray
    ekin: np.ndarray
    epot: np.ndarray
    etot: np.ndarray
    x: np.ndarray
    v: np.ndarray
    stats: dict
    samples: np.ndarray | None = None   # [nsamples, 6] (mlp_mode 1)

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
        _LIB.nb6drive_ensemble.restype = C.c_int
        _LIB.nb6drive_ac_radius.restype = None
        _LIB.nb6drive_ac_shrink.restype = None
        _LIB.nb6drive_core.restype = None
    return _LIB


def backend_paths(name: str = "nb6b200") -> dict:
    if name == "nb6b200":
        from . import LIB_PATH
        return {"reg": LIB_PATH, "irr": LIB_PATH, "pot": LIB_PATH}
    raise ValueError(name)


def _mlp_fields(p: "Params", mlp_mode: int, sample_cap: int):
    """Fill the learned-radius fields; returns the sample buffer (or None)."""
    p.mlp_mode = mlp_mode
    p.mlp_pad = 0
    buf = None
    if mlp_mode == 1 and sample_cap > 0:
        buf = np.zeros((sample_cap, 6), dtype=np.float32)
        p.samples = buf.ctypes.data_as(C.POINTER(C.c_float))
        p.sample_cap = sample_cap
    else:
        p.samples = C.POINTER(C.c_float)()
        p.sample_cap = 0
    return buf


def _rs_field(p: "Params", rs_init, n: int):
    if rs_init is None:
        p.rs_init = C.POINTER(C.c_double)()
        return None
    arr = np.ascontiguousarray(rs_init, dtype=np.float64)
    assert arr.shape == (n,)
    p.rs_init = arr.ctypes.data_as(C.POINTER(C.c_double))
    return arr


def run(backend: dict, mass, pos, vel, *, tcrit=1.0, eta_i=0.02, eta_r=0.03, smax=0.125,
        dtmin=2.0 ** -24, dt_out=0.125, rs0=0.3, nnbopt=50, nnbmax=400, lmax=512, m_flag=0,
        chunk=1024, max_blocks=10_000_000, mlp_mode=0, sample_cap=0, rs_init=None,
        nb_flag=1, dt_adj=1.0) -> RunResult:
    """mlp_mode: 0 Ahmad-Cohen radii; 1 Ahmad-Cohen and log up to sample_cap
    (features, target) samples into RunResult.samples; 2 the library's learned
    proposals (nb6b200.mlp.enable(True) first), Ahmad-Cohen as fallback.
    rs_init: initial neighbour radii per body (default RS0 sqrt(1 + r^2)).
    nb_flag: form of the Ahmad-Cohen rule, NB_FLAG of regcor_gpu.F:22 (1,
    the reference's default KZ(39) = 0 or 2: density-centre distances; 0:
    KZ(39) = 1 or 3).  dt_adj: DTADJ, the interval at which the rule's
    quantities (density centre, core and half-mass radius, RSFAC) are
    refreshed (at the first energy output at or after each multiple)."""
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    x = np.ascontiguousarray(pos, dtype=np.float64).reshape(n, 3).copy()
    v = np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 3).copy()
    p = Params(eta_i, eta_r, smax, dtmin, tcrit, dt_out, rs0, nnbopt, nnbmax, lmax, m_flag,
               chunk, max_blocks)
    buf = _mlp_fields(p, mlp_mode, sample_cap)
    p.nb_flag = int(nb_flag)
    p.dt_adj = float(dt_adj)
    rs_arr = _rs_field(p, rs_init, n)
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
    samples = buf[:st.nsamples].copy() if buf is not None else None
    return RunResult(eout[:k, 0], eout[:k, 1], eout[:k, 2], eout[:k, 3], x, v, stats, samples)


@dataclass
class EnsembleResult:
    times: np.ndarray      # [nout]
    energy: np.ndarray     # [nout, ncl, 3]: kinetic, potential, total
    x: list                # per cluster [n_c, 3]
    v: list
    stats: dict
    samples: np.ndarray | None = None

    @property
    def de_max(self) -> np.ndarray:
        """max_t |E_c(t) - E_c(0)| / |E_c(0)| per cluster."""
        e = self.energy[:, :, 2]
        return np.max(np.abs(e - e[0]), axis=0) / np.abs(e[0])


def run_ensemble(backend: dict, clusters, *, batched=True, tcrit=1.0, eta_i=0.02, eta_r=0.03,
                 smax=0.125, dtmin=2.0 ** -24, dt_out=0.125, rs0=0.3, nnbopt=50, nnbmax=400,
                 lmax=512, m_flag=0, chunk=1024, max_blocks=100_000_000, mlp_mode=0,
                 sample_cap=0, rs_init=None, rs_from_clusters=False,
                 dev_corrector=True, seg_single=False, nb_flag=1, dt_adj=1.0) -> EnsembleResult:
    """clusters: sequence of (mass, pos, vel) (or objects with .mass/.pos/.vel),
    each in its own Henon units.  batched=False issues the regular force per
    cluster (what running each alone does); the result is then identical to
    ``run`` on each cluster with a deterministic backend.  rs_init (all
    bodies) or rs_from_clusters=True (each cluster's .rs) sets the initial
    neighbour radii.  dev_corrector (batched mode): 1 (True) runs the
    irregular corrector on the device (nb6_irr_correct_), 2 the regular
    corrector there too (nb6_regf_correct_), 3 the block clock too
    (nb6_blocks_run_: runs of irregular blocks without the host); the
    result is the same bit for
    bit (with mlp_mode 2 up to the last bit of exp on the device) when
    seg_single is set: blocks whose regular bodies are all in one cluster
    then take the segmented call too, as the device regular corrector
    always does (otherwise they take gpunb_regf_, whose sums round
    differently)."""
    parts = [(c.mass, c.pos, c.vel) if hasattr(c, "mass") else c for c in clusters]
    counts = np.array([len(p[0]) for p in parts], dtype=np.int32)
    ncl = len(parts)
    mass = np.ascontiguousarray(np.concatenate([p[0] for p in parts]), dtype=np.float64)
    x = np.ascontiguousarray(np.concatenate([np.reshape(p[1], (-1, 3)) for p in parts]), dtype=np.float64)
    v = np.ascontiguousarray(np.concatenate([np.reshape(p[2], (-1, 3)) for p in parts]), dtype=np.float64)
    p = Params(eta_i, eta_r, smax, dtmin, tcrit, dt_out, rs0, nnbopt, nnbmax, lmax, m_flag,
               chunk, max_blocks)
    buf = _mlp_fields(p, mlp_mode, sample_cap)
    p.dev_corrector = int(dev_corrector)
    p.seg_single = 1 if seg_single else 0
    p.nb_flag = int(nb_flag)
    p.dt_adj = float(dt_adj)
    if rs_init is None and all(hasattr(c, "rs") for c in clusters) and rs_from_clusters:
        rs_init = np.concatenate([c.rs for c in clusters])
    rs_arr = _rs_field(p, rs_init, len(mass))
    nout_max = int(tcrit / dt_out) + 4
    tout = np.zeros(nout_max)
    eout = np.zeros((nout_max, ncl, 3))
    st = Stats()
    dp = C.POINTER(C.c_double)
    rc = _lib().nb6drive_ensemble(backend["reg"].encode(), backend["irr"].encode(),
                                  backend["pot"].encode(), C.c_int(ncl),
                                  counts.ctypes.data_as(C.POINTER(C.c_int)), mass.ctypes.data_as(dp),
                                  x.ctypes.data_as(dp), v.ctypes.data_as(dp), C.byref(p),
                                  C.c_int(1 if batched else 0), tout.ctypes.data_as(dp),
                                  eout.ctypes.data_as(dp), C.c_int(nout_max), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"nb6drive_ensemble failed with code {rc}")
    k = st.nout
    stats = {f: getattr(st, f) for f, _ in Stats._fields_}
    off = np.concatenate([[0], np.cumsum(counts)])
    xs = [x[off[c]:off[c + 1]] for c in range(ncl)]
    vs = [v[off[c]:off[c + 1]] for c in range(ncl)]
    samples = buf[:st.nsamples].copy() if buf is not None else None
    return EnsembleResult(tout[:k], eout[:k], xs, vs, stats, samples)
