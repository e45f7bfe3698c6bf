"""Batched ensemble vs each cluster alone (the plain method), same GPU.

    python -m nb6b200.ensemble_bench --clusters 256 --tcrit 1.0 [--alone-sample 32] [--mlp]
        [--dev-corrector 3]

(run from ``nbody6ppgpu-beijing_b200/``).  The ensemble is the batched
driver (one irregular and one segmented regular call per block for all
clusters; --dev-corrector 1 runs the irregular corrector on the device, 2
both correctors, 3 the block clock too); "alone" integrates each cluster with the single-cluster driver
and the reference ABI calls.  With --alone-sample k only k clusters, spread
over the size range, are run alone and their wall time is scaled by the
ensemble's total pair count over theirs (stated in the output).  Prints one
JSON line: N-body time per wall second for both, and per-cluster energy
errors.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import drive, ics


def make_clusters(k: int, seed: int = 2026, nmin: int = 512, nmax: int = 8192):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), k)).astype(int)
    return [ics.plummer(int(n), seed=seed + 17 * c, imf=True) for c, n in enumerate(sizes)]


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--clusters", type=int, default=256)
    ap.add_argument("--tcrit", type=float, default=1.0)
    ap.add_argument("--alone-sample", type=int, default=0, help="0 = all clusters alone")
    ap.add_argument("--mlp", action="store_true",
                    help="learned radii: train on samples from plain runs of 16 other clusters "
                         "of the same distribution, then run the ensemble with the proposals")
    ap.add_argument("--dev-corrector", type=int, default=3, choices=(0, 1, 2, 3))
    a = ap.parse_args(argv)
    ours = drive.backend_paths("nb6b200")
    cls = make_clusters(a.clusters)
    sizes = np.array([c.n for c in cls])
    train = None
    if a.mlp:
        from . import learn, mlp
        t = time.perf_counter()
        samples = learn.collect(make_clusters(16, seed=77), a.tcrit)
        hist = learn.fit(samples, epochs=15)
        train = {"samples": int(len(samples)), "loss": [float(hist[0]), float(hist[-1])],
                 "wall_s": time.perf_counter() - t}
        mlp.enable(True)
    t = time.perf_counter()
    ens = drive.run_ensemble(ours, cls, batched=True, tcrit=a.tcrit, dt_out=min(a.tcrit, 0.25),
                             mlp_mode=2 if a.mlp else 0, dev_corrector=a.dev_corrector)
    wall_ens = time.perf_counter() - t
    if a.mlp:
        mlp.enable(False)
    order = np.argsort(sizes)
    pick = order if a.alone_sample <= 0 else order[np.linspace(0, len(cls) - 1, a.alone_sample).astype(int)]
    worst = int(np.argmax(ens.de_max))  # always compared alone as well
    if worst not in set(int(c) for c in pick):
        pick = np.append(pick, worst)
    de_alone, wall_alone, reg_alone, irr_alone = {}, 0.0, 0.0, 0.0
    for c in pick:
        cl = cls[c]
        t = time.perf_counter()
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=a.tcrit, dt_out=min(a.tcrit, 0.25))
        wall_alone += time.perf_counter() - t
        reg_alone += r.stats["wall_reg"]
        irr_alone += r.stats["wall_irr"]
        de_alone[int(c)] = r.de_max
    scale = float((sizes.astype(float) ** 2).sum() / (sizes[pick].astype(float) ** 2).sum())
    wall_alone_all = wall_alone * scale
    de_e = ens.de_max
    ratio = np.array([de_e[c] / de_alone[c] for c in de_alone])
    out = {
        "workload": f"{a.clusters} Plummer clusters, Kroupa IMF, N log-uniform 512-8192, total {int(sizes.sum())}",
        "tcrit": a.tcrit,
        "dev_corrector": a.dev_corrector,
        "ensemble_wall_s": wall_ens,
        "alone_wall_s": wall_alone_all,
        "alone_clusters_run": int(len(pick)),
        "alone_scale": scale,
        "nbody_time_per_wall_s": {"ensemble": a.tcrit / wall_ens, "alone": a.tcrit / wall_alone_all},
        "speedup": wall_alone_all / wall_ens,
        "dE_ensemble_median": float(np.median(de_e)),
        "dE_ensemble_max": float(np.max(de_e)),
        "dE_ensemble_p99": float(np.percentile(de_e, 99)),
        "worst_cluster": {"n": int(sizes[worst]), "dE_ensemble": float(de_e[worst]),
                          "dE_alone": float(de_alone[worst])},
        "dE_ratio_ensemble_over_alone_median": float(np.median(ratio)),
        "dE_ratio_p90": float(np.percentile(ratio, 90)),
        "dE_ratio_max": float(np.max(ratio)),
        "dE_alone_at_max_ratio": float(list(de_alone.values())[int(np.argmax(ratio))]),
        "ensemble_stats": {k: ens.stats[k] for k in ("blocks", "irr_steps", "reg_steps", "reg_calls",
                                                      "overflow_retries", "wall_reg", "wall_irr")},
        "alone_force_call_wall_s": {"reg": reg_alone * scale, "irr": irr_alone * scale},
        "learned_radius": None if train is None else {
            "training": train, "used": ens.stats["mlp_used"], "fallback": ens.stats["mlp_fallback"],
            "nnb_absdev_mean": ens.stats["nb_absdev"] / max(ens.stats["reg_steps"], 1)},
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
