"""Single force calls on fixed synthetic workloads, for timing and for
profiler captures of one kernel at a time.

    python -m nb6b200.probe_calls seg [--active 0.1] [--reps 2]
    python -m nb6b200.probe_calls jpar [--ni 64] [--reps 6]
    python -m nb6b200.probe_calls irr [--reps 2]

(run from ``nbody6ppgpu-beijing_b200/``; prints one JSON line with the
kernel's device time from the library's CUDA events):

* ``seg``: ``nb6_regf_seg_`` (``regf_seg_kernel``) on 64 Plummer clusters
  (Kroupa IMF, N log-uniform 512-8192, 160,011 bodies), a random fraction
  of the bodies active, radii at NNBOPT = 50;
* ``jpar``: ``gpunb_regf_`` with ``ni`` bodies of a Plummer N = 262,144 (the
  j-parallel kernel for ni < 128);
* ``irr``: ``irr_simd_firr_vec_`` (``irr_kernel``) for 65,536 bodies of a
  Plummer N = 262,144 with lists of the 64 nearest bodies.

Each runs the call ``reps`` times (the first a warm-up that also uploads
the state) and reports the last call.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import ics, load


def seg(active: float, reps: int) -> dict:
    from .ensemble_bench import make_clusters
    lib = load()
    cls = make_clusters(64)
    m = np.concatenate([c.mass for c in cls])
    x = np.concatenate([c.pos for c in cls])
    v = np.concatenate([c.vel for c in cls])
    rs = np.concatenate([c.rs for c in cls])
    dtr = np.concatenate([c.dtr for c in cls])
    cnt = np.array([c.n for c in cls])
    seg_j0 = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int32)
    iseg = np.repeat(np.arange(64), cnt).astype(np.int32)
    n = len(m)
    sel = np.sort(np.random.default_rng(1).choice(n, max(1, int(n * active)), replace=False))
    lib.gpunb_open(n + 10, 0)
    try:
        lib.gpunb_send(m, x, v)
        for _ in range(reps):
            lib.regf_seg(rs[sel] ** 2, dtr[sel], x[sel], v[sel], iseg[sel], seg_j0, 512, 400, 0)
        ms = float(lib.lib.nb6_regf_last_kernel_ms_())
    finally:
        lib.gpunb_close()
    pairs = float(cnt[iseg[sel]].sum())
    return {"call": "seg", "bodies": n, "active": int(len(sel)), "kernel_ms": ms, "pairs_per_s": pairs / (ms * 1e-3)}


def jpar(ni: int, reps: int) -> dict:
    lib = load()
    p = ics.plummer(262144, seed=5)
    sel = np.arange(1000, 1000 + ni)
    lib.gpunb_open(p.n + 10, 0)
    try:
        lib.gpunb_send(p.mass, p.pos, p.vel)
        for _ in range(reps):
            lib.gpunb_regf(p.rs[sel] ** 2, p.dtr[sel], p.pos[sel], p.vel[sel], 512, 400, 0)
        ms = float(lib.lib.nb6_regf_last_kernel_ms_())
    finally:
        lib.gpunb_close()
    return {"call": "jpar", "ni": ni, "nj": p.n, "kernel_ms": ms, "pairs_per_s": ni * p.n / (ms * 1e-3)}


def irr(reps: int) -> dict:
    from scipy.spatial import cKDTree
    lib = load()
    p = ics.plummer(262144, seed=9)
    n = p.n
    _, idx = cKDTree(p.pos).query(p.pos, k=65)
    rng = np.random.default_rng(2)
    f = rng.normal(size=(n, 3)) * 0.05
    lib.irr_open(n, 128, 0)
    try:
        lib.irr_set_jp_all(p.pos, p.vel, f, f * 0.2, p.mass, -rng.integers(0, 8, n) / 4096.0)
        for i in range(n):
            lib.irr_set_list(i + 1, np.concatenate([[64], np.sort(idx[i, 1:]) + 1]))
        addr = np.sort(rng.choice(n, 65536, replace=False)).astype(np.int32) + 1
        out = (np.zeros((65536, 3)), np.zeros((65536, 3)), np.zeros(65536, np.int32))
        for _ in range(reps):
            lib.irr_firr_vec(1.0 / 2048, addr, out)
        ms = float(lib.lib.nb6_irr_last_kernel_ms_())
    finally:
        lib.irr_close(0)
    pairs = 65536 * 64
    return {"call": "irr", "active": 65536, "list_pairs": pairs, "kernel_ms": ms,
            "gbs_algorithmic": 132.0 * pairs / (ms * 1e-3) / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("call", choices=["seg", "jpar", "irr"])
    ap.add_argument("--active", type=float, default=0.1)
    ap.add_argument("--ni", type=int, default=64)
    ap.add_argument("--reps", type=int, default=2)
    a = ap.parse_args(argv)
    if a.call == "seg":
        out = seg(a.active, a.reps)
    elif a.call == "jpar":
        out = jpar(a.ni, a.reps)
    else:
        out = irr(a.reps)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
