"""The learned neighbour radius end to end: collect samples from plain
Ahmad-Cohen runs, train the model on the GPU, and compare a run that uses
its proposals with a plain run.

    python -m nb6b200.learn --n-train 131072 --n-eval 1048576 --tcrit 0.0078125

(run from ``nbody6ppgpu-beijing_b200/``; prints one JSON line).  A sample is
(features of a particle at one regular step, log(RS* / RS)) where RS* is the
radius that would have given NNBOPT neighbours at its next regular step; see
``mlp.py`` and the library's mlp.cuh for the features.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import drive, ics, mlp


def collect(clusters, tcrit, sample_cap=2_000_000, rs_ics=False, **kw) -> np.ndarray:
    """Samples [k, 6] from plain (Ahmad-Cohen) runs of the clusters on
    libnb6b200, one ensemble run for all of them.  rs_ics: start from the
    clusters' own radii (distance to the NNBOPT-th neighbour) instead of the
    RS0 rule."""
    ours = drive.backend_paths("nb6b200")
    r = drive.run_ensemble(ours, clusters, batched=True, tcrit=tcrit, mlp_mode=1,
                           sample_cap=sample_cap, dt_out=min(tcrit, 0.125),
                           rs_from_clusters=rs_ics, **kw)
    return r.samples


def fit(samples, epochs=15, batch=1024, lr=2e-3, seed=0) -> np.ndarray:
    """Fresh model trained on the samples; returns the loss history."""
    x = samples[:, :5]
    y = samples[:, 5]
    mlp.init(seed)
    return mlp.train(x, y, epochs=epochs, batch=batch, lr=lr, seed=seed)


def _summary(stats, de, tcrit):
    steps = max(stats["reg_steps"], 1)
    return {"nnb_mean": stats["nb_sum"] / steps, "nnb_absdev_mean": stats["nb_absdev"] / steps,
            "overflow_retries": stats["overflow_retries"], "reg_calls": stats["reg_calls"],
            "reg_steps": stats["reg_steps"], "irr_steps": stats["irr_steps"],
            "reg_irr_ratio": stats["reg_steps"] / max(stats["irr_steps"], 1),
            "wall_s": stats["wall_total"], "wall_per_nbody_time": stats["wall_total"] / tcrit,
            "dE": float(de), "mlp_used": stats["mlp_used"], "mlp_fallback": stats["mlp_fallback"]}


def compare(cl, tcrit, plain_method=True, rs_ics=False, dev_corrector=3, **kw) -> dict:
    """One cluster three ways, with the current model for the learned arm:
    the plain GPU method (single-cluster driver: host prediction, gpunb_send_
    per regular block, host correctors, Ahmad-Cohen radii); the batched
    driver (j set predicted on the device; with dev_corrector = 2 both
    correctors on the device too, with 3 the block clock as well) with
    Ahmad-Cohen radii; and the batched
    driver with the learned radii.  Wall times are the drivers' own (block
    loop and energies, not the start-up)."""
    ours = drive.backend_paths("nb6b200")
    dt_out = min(tcrit, 0.125)          # at least one energy after the start
    rs = cl.rs if rs_ics else None
    out = {}
    if plain_method:
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=tcrit, mlp_mode=0, dt_out=dt_out,
                      rs_init=rs, **kw)
        out["plain"] = _summary(r.stats, r.de_max, tcrit)
    r = drive.run_ensemble(ours, [cl], batched=True, tcrit=tcrit, mlp_mode=0, dt_out=dt_out,
                           rs_init=rs, dev_corrector=dev_corrector, **kw)
    out["batched"] = _summary(r.stats, r.de_max[0], tcrit)
    mlp.enable(True)
    try:
        r = drive.run_ensemble(ours, [cl], batched=True, tcrit=tcrit, mlp_mode=2, dt_out=dt_out,
                               rs_init=rs, dev_corrector=dev_corrector, **kw)
    finally:
        mlp.enable(False)
    out["learned"] = _summary(r.stats, r.de_max[0], tcrit)
    base = out.get("plain", out["batched"])
    key = "plain" if plain_method else "batched"
    out["speedup_learned_vs_" + key] = base["wall_s"] / out["learned"]["wall_s"]
    out["speedup_batched_vs_" + key] = base["wall_s"] / out["batched"]["wall_s"]
    out["dev_corrector"] = dev_corrector
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=16384)
    ap.add_argument("--n-eval", type=int, default=16384)
    ap.add_argument("--train-clusters", type=int, default=2)
    ap.add_argument("--tcrit", type=float, default=0.25, help="length of the evaluation runs")
    ap.add_argument("--train-tcrit", type=float, default=None, help="length of the sampling runs")
    ap.add_argument("--epochs", type=int, default=15)
    ap.add_argument("--model", choices=["plummer", "king"], default="king")
    ap.add_argument("--no-plain", action="store_true", help="skip the single-cluster plain arm")
    ap.add_argument("--save", default=None, help="write the trained model (.npy)")
    ap.add_argument("--rs-ics", action="store_true",
                    help="initial radii from the clusters (NNBOPT-th neighbour) instead of RS0")
    a = ap.parse_args(argv)
    if a.model == "king":
        def make(n, s):
            return ics.king(n, w0=6.0, seed=s, imf=True, binary_fraction=0.05)
    else:
        def make(n, s):
            return ics.plummer(n, seed=s, imf=True)
    train_cls = [make(a.n_train, 100 + k) for k in range(a.train_clusters)]
    samples = collect(train_cls, a.train_tcrit or a.tcrit, rs_ics=a.rs_ics)
    hist = fit(samples, epochs=a.epochs)
    if a.save:
        np.save(a.save, mlp.get_model())
    res = compare(make(a.n_eval, 999), a.tcrit, plain_method=not a.no_plain, rs_ics=a.rs_ics)
    res.update({"n_train": a.n_train, "n_eval": a.n_eval, "samples": int(len(samples)),
                "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1]),
                "tcrit": a.tcrit, "model": a.model, "rs_ics": a.rs_ics})
    print(json.dumps(res))


if __name__ == "__main__":
    main()
