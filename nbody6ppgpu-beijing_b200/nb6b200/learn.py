"""The learned neighbour radius end to end: collect samples from plain
Ahmad-Cohen runs, train the model on the GPU, and compare a run that uses
its proposals with a plain run.

    python -m nb6b200.learn --n-train 131072 --n-eval 131072 --tcrit 0.25

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


def collect(clusters, tcrit, sample_cap=2_000_000, **kw) -> np.ndarray:
    """Samples [k, 6] from plain runs (libnb6b200 backend) of the clusters."""
    out = []
    ours = drive.backend_paths("nb6b200")
    for cl in clusters:
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=tcrit, mlp_mode=1,
                      sample_cap=sample_cap, dt_out=max(tcrit, 0.125), **kw)
        out.append(r.samples)
    return np.concatenate(out)


def fit(samples, epochs=15, batch=1024, lr=2e-3, seed=0) -> np.ndarray:
    """Fresh model trained on the samples; returns the loss history."""
    x = samples[:, :5]
    y = samples[:, 5]
    mlp.init(seed)
    return mlp.train(x, y, epochs=epochs, batch=batch, lr=lr, seed=seed)


def compare(cl, tcrit, **kw) -> dict:
    """Plain and learned runs of one cluster with the current model."""
    ours = drive.backend_paths("nb6b200")
    plain = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=tcrit, mlp_mode=0,
                      dt_out=max(tcrit, 0.125), **kw)
    mlp.enable(True)
    try:
        learned = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=tcrit, mlp_mode=2,
                            dt_out=max(tcrit, 0.125), **kw)
    finally:
        mlp.enable(False)

    def summary(r):
        s = r.stats
        steps = max(s["reg_steps"], 1)
        return {"nnb_mean": s["nb_sum"] / steps, "nnb_absdev_mean": s["nb_absdev"] / steps,
                "overflow_retries": s["overflow_retries"], "reg_calls": s["reg_calls"],
                "reg_steps": s["reg_steps"], "irr_steps": s["irr_steps"],
                "reg_irr_ratio": s["reg_steps"] / max(s["irr_steps"], 1),
                "wall_s": s["wall_total"], "wall_per_nbody_time": s["wall_total"] / tcrit,
                "dE": r.de_max, "mlp_used": s["mlp_used"], "mlp_fallback": s["mlp_fallback"]}

    return {"plain": summary(plain), "learned": summary(learned)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=16384)
    ap.add_argument("--n-eval", type=int, default=16384)
    ap.add_argument("--train-clusters", type=int, default=2)
    ap.add_argument("--tcrit", type=float, default=0.25)
    ap.add_argument("--epochs", type=int, default=15)
    ap.add_argument("--model", choices=["plummer", "king"], default="king")
    a = ap.parse_args(argv)
    make = (lambda n, s: ics.king(n, w0=6.0, seed=s, imf=True)) if a.model == "king" else \
        (lambda n, s: ics.plummer(n, seed=s, imf=True))
    train_cls = [make(a.n_train, 100 + k) for k in range(a.train_clusters)]
    samples = collect(train_cls, a.tcrit)
    hist = fit(samples, epochs=a.epochs)
    res = compare(make(a.n_eval, 999), a.tcrit)
    res.update({"n_train": a.n_train, "n_eval": a.n_eval, "samples": int(len(samples)),
                "loss_first_epoch": float(hist[0]), "loss_last_epoch": float(hist[-1]),
                "tcrit": a.tcrit, "model": a.model})
    print(json.dumps(res))


if __name__ == "__main__":
    main()
