#!/usr/bin/env python
"""Benchmark: regular force + jerk + neighbour list, pair interactions/s at N=1M.

Workload (one "step" = one full regular evaluation, as FPOLY0 does it,
fpoly0.F:100-206): a King W0=6 cluster of N = 1,048,576 stars with a Kroupa
IMF and 5% primordial binaries entering as centre-of-mass bodies
(996,147 bodies), seeded synthetic data.  Every body is an i-particle against
all bodies as j, issued in calls of 1024 i (util_gpu.F:7,33-60), NNBMAX = 400,
LMAX = 512, neighbour radii at NNBOPT = 50.

Reported on one JSON line (rank 0):
  value      pairs/s with inputs resident in HBM (nb6_regf_device_), CUDA
             events on the library stream, L2 flushed between timed steps;
  e2e        the same metric through gpunb_send_ + gpunb_regf_ with host
             buffers, all host<->device copies inside the timed region;
  roofline   the force kernel against the FP32 FMA pipe: 60 flops per pair
             (the reference's convention, gpunb.velocity.cu:895) over the
             kernel's own CUDA-event time, peak = measured FP32 FMA rate;
  cpu_baseline  the reference's own reg.avx.cpp (oracle/_ref) on the host
             cores, bounded sample of the same workload;
  err_vs_fp64   force/jerk/potential error against the FP64 oracle on a
             sample of i-particles;
  gpupot, irregular, predictor   the N^2 potential, the irregular force and
             the Hermite predictor on the same bodies, each against its own
             roofline (MUFU rate, HBM bandwidth).

--impl reference runs the reference's CPU library (the timed CPU arm).
Multi-GPU (torchrun, --gpus N): every rank evaluates its own cluster of the
same size (independent clusters, weak scaling), no data-path collective.
cpu_baseline, err_vs_fp64 and the irregular, predictor, end-to-end driver
and reference-GPU legs run at N = 1 only (on rank 0); at N > 1 the line
carries the scaled regular-force figures alone.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "nbody6ppgpu-beijing_b200"), os.path.join(ROOT, "oracle")]
os.environ.setdefault("OMP_NUM_THREADS", str(min(32, os.cpu_count() or 1)))

import numpy as np  # noqa: E402

METRIC = "Regular force+jerk+nbr pair interactions/s at N=1M"
FLOPS_PER_PAIR = 60          # gpunb.velocity.cu:895, reg.avx.cpp:343
# DRAM bytes (read + write) per launch of the headline force kernel,
# regf_x2_kernel<1> with 1024 i x 996,147 j over the Morton-ordered j set
# (tile-relative far operands included), from one ncu capture of that
# launch: dram__bytes_read.sum 69.58 MB + dram__bytes_write.sum 3.45 MB.
NCU_TRAFFIC_PER_LAUNCH = 69.58e6 + 3.45e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1048576, help="stars (before folding binaries)")
    ap.add_argument("--chunk", type=int, default=1024)
    ap.add_argument("--nnbmax", type=int, default=400)
    ap.add_argument("--lmax", type=int, default=512)
    ap.add_argument("--m-flag", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip timing the reference's CUDA library (oracle/_ref) on the same workload")
    ap.add_argument("--no-pot", action="store_true", help="skip the N^2 potential leg")
    ap.add_argument("--no-irr", action="store_true", help="skip the irregular-force leg")
    ap.add_argument("--no-pred", action="store_true", help="skip the Hermite predictor leg")
    ap.add_argument("--no-err", action="store_true", help="skip the error check against the FP64 oracle")
    ap.add_argument("--no-northstar", action="store_true",
                    help="skip the config 3/4 driver leg (plain GPU method vs batched device form)")
    ap.add_argument("--ns-t3", type=float, default=1.0 / 64, help="config 3 end time")
    ap.add_argument("--ns-t4", type=float, default=1.0, help="config 4 end time")
    ap.add_argument("--ns-clusters", type=int, default=256)
    ap.add_argument("--ns-alone", type=int, default=8, help="config 4 clusters run alone")
    ap.add_argument("--seed", type=int, default=20260)
    return ap.parse_args()


def workload(n: int, seed: int):
    path = f"/tmp/nb6_king_w6_n{n}_s{seed}.npz"
    if os.path.exists(path):
        d = np.load(path)
        return d["m"], d["x"], d["v"], d["rs"], d["dtr"]
    from nb6b200 import ics
    c = ics.king(n, w0=6.0, seed=seed, imf=True, binary_fraction=0.05, nnbopt=50)
    try:
        np.savez(path, m=c.mass, x=c.pos, v=c.vel, rs=c.rs, dtr=c.dtr)
    except OSError:
        pass
    return c.mass, c.pos, c.vel, c.rs, c.dtr


class Clocks:
    """nvidia-smi sampling during the timed region (the recipe's clocks line)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, pw, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [q.strip() for q in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
                pw.append(float(p[3]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if p[5 + k].lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s, w in zip(sm, pw) if w > 0.3 * max(pw)] or sm
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": float(max(pw)), "sm_mhz_min": float(min(sm))}


def reduce_max(value: float, pg, device=None) -> float:
    """The maximum of value over all ranks (the slowest rank's time); the
    value itself on one rank."""
    if pg is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, pairs_per_step: float, steps: int, total_ms_max: float) -> float:
    """Pairs per second of the whole job: every rank runs its own replica of
    the workload (weak scaling), timed by the slowest rank."""
    return world * pairs_per_step * steps / (total_ms_max * 1e-3)


def bench_config(args, n: int, world: int) -> dict:
    """The workload description shared by both arms' JSON lines."""
    return {"workload": f"king-w0=6 N={args.n} ({n} c.m. bodies), full regular "
                        f"evaluation in {args.chunk}-i calls",
            "n_bodies": n, "chunk": args.chunk, "calls_per_step": (n + args.chunk - 1) // args.chunk,
            "nnbopt": 50, "nnbmax": args.nnbmax, "lmax": args.lmax,
            "m_flag": args.m_flag, "parallelism": f"replicas x{world}",
            "l2": "flushed (256 MiB write) between timed steps"}


def cpu_model() -> str:
    """The host CPU's model name (lscpu), for the CPU baselines."""
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=20).stdout
        for ln in out.splitlines():
            if ln.startswith("Model name:"):
                return ln.split(":", 1)[1].strip()
    except (OSError, subprocess.SubprocessError):
        pass
    return "unknown"


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference_rate(m, x, v, rs, dtr, args, seconds: float, max_calls: int | None = None):
    """Time the reference's reg.avx.cpp gpunb_regf_ on the host cores over a
    bounded sample of 1024-i calls of the same workload."""
    import oracle
    from nb6b200.abi import ForceLib
    if not oracle.ref_available("reg"):
        oracle.build(ref=True)
    lib = ForceLib(oracle.ref_lib("reg"), "ref-reg-avx")
    n = m.shape[0]
    lib.gpunb_open(n + 10, 0)
    lib.gpunb_send(m, x, v)
    h2 = rs ** 2 if not args.m_flag else rs ** 2 / m.mean()
    pairs, t_used, calls = 0, 0.0, 0
    rng = np.random.default_rng(1)
    starts = rng.permutation(n // args.chunk) * args.chunk
    for s in starts:
        sl = slice(s, min(n, s + args.chunk))
        t0 = time.perf_counter()
        lib.gpunb_regf(h2[sl], dtr[sl], x[sl], v[sl], args.lmax, args.nnbmax, args.m_flag)
        t_used += time.perf_counter() - t0
        pairs += (sl.stop - sl.start) * n
        calls += 1
        if t_used >= seconds or (max_calls and calls >= max_calls):
            break
    lib.gpunb_close()
    threads = int(os.environ.get("OMP_NUM_THREADS", "1"))
    return pairs / t_used, threads, calls, t_used


def reference_gpu_rate(m, x, v, rs, dtr, args, seconds: float):
    """The reference's own CUDA regular-force library (gpunb.velocity.cu,
    built for sm_100a into oracle/_ref) on the same workload, through its C
    ABI with host buffers: gpunb_send_ once, then the 1024-i gpunb_regf_
    calls in order (synchronous calls, wall clock), a bounded sample.
    Returns None when the library was not built."""
    import oracle
    from nb6b200.abi import ForceLib
    if not oracle.ref_available("gpunb_velocity"):
        return None
    lib = ForceLib(oracle.ref_lib("gpunb_velocity"), "ref-gpunb-velocity")
    n = m.shape[0]
    h2 = rs ** 2 if not args.m_flag else rs ** 2 / m.mean()
    lib.gpunb_open(n + 10, 0)
    t0 = time.perf_counter()
    lib.gpunb_send(m, x, v)
    t_send = time.perf_counter() - t0
    chunks = [(s, min(n, s + args.chunk)) for s in range(0, n, args.chunk)]
    for s, e in chunks[:2]:                                   # warm-up
        lib.gpunb_regf(h2[s:e], dtr[s:e], x[s:e], v[s:e], args.lmax, args.nnbmax, args.m_flag)
    pairs, t_used, calls = 0.0, 0.0, 0
    for s, e in chunks:
        t0 = time.perf_counter()
        lib.gpunb_regf(h2[s:e], dtr[s:e], x[s:e], v[s:e], args.lmax, args.nnbmax, args.m_flag)
        t_used += time.perf_counter() - t0
        pairs += (e - s) * float(n)
        calls += 1
        if t_used >= seconds:
            break
    lib.gpunb_close()
    return {"value": pairs / t_used, "unit": "pairs/s", "calls": calls,
            "send_s": t_send,
            "kind": "the reference's CUDA library gpunb.velocity.cu built for sm_100a "
                    "(oracle/_ref), through its C ABI with host buffers: compare with e2e",
            "sample": f"{calls} calls x {args.chunk} i x {n} j of the same workload, {t_used:.1f} s"}


def mufu_peak_per_s() -> float:
    """Nominal MUFU (rsqrt) rate: 16 results per SM per clock (the CUDA
    throughput table's figure for reciprocal square root) x SMs x the GPU's
    maximum SM clock."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = 1965.0
    try:
        import subprocess
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm", "--format=csv,noheader,nounits",
                              "-i", "0"], capture_output=True, text=True, timeout=20).stdout.strip()
        mhz = float(out.splitlines()[0])
    except Exception:
        pass
    return 16.0 * sms * mhz * 1e6


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s) of this pool's B200s, else the
    earlier fallback measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def predictor_leg(lib, m, x, v, flush_l2, reps: int = 10):
    """The Hermite j predictor (xbpredall.F:48-62) over every body, state
    resident in HBM (nb6_state_set_, nb6_predict_device_): 104 bytes read
    (T0, X0, X0DOT, F, FDOT) and 48 written (X, XDOT) per body, HBM-bound.
    Kernel time from the library's CUDA events, L2 flushed before each
    launch; the prediction checked against the FP64 oracle's."""
    import oracle
    raw = lib.lib
    n = m.shape[0]
    rng = np.random.default_rng(11)
    a = {"body": m, "t0": -rng.integers(0, 64, n) / 8192.0, "x0": x, "x0dot": v,
         "f": rng.normal(size=(n, 3)) * 0.3, "fdot": rng.normal(size=(n, 3)) * 0.1}
    a = {k: np.ascontiguousarray(val, dtype=np.float64) for k, val in a.items()}
    dp = C.POINTER(C.c_double)
    t = C.c_double(1.0 / 1024)
    ms = []
    raw.nb6_state_open_(C.byref(C.c_int(n)))
    try:
        raw.nb6_state_set_(C.byref(C.c_int(n)), *(a[k].ctypes.data_as(dp)
                                                  for k in ("body", "t0", "x0", "x0dot", "f", "fdot")))
        dx, dv = dp(), dp()
        for _ in range(3):
            raw.nb6_predict_device_(C.byref(t), C.byref(dx), C.byref(dv))
        for _ in range(reps):
            flush_l2()
            raw.nb6_predict_device_(C.byref(t), C.byref(dx), C.byref(dv))
            ms.append(float(raw.nb6_predict_last_kernel_ms_()))
        xs, xds = np.zeros((n, 3)), np.zeros((n, 3))
        raw.nb6_predict_(C.byref(t), xs.ctypes.data_as(dp), xds.ctypes.data_as(dp))
    finally:
        raw.nb6_state_close_()
    ox, oxd = oracle.predict(t.value, a["t0"], a["x0"], a["x0dot"], a["f"], a["fdot"])
    k_ms = float(np.median(ms))
    gbs = 152.0 * n / (k_ms * 1e-3) / 1e9
    hbm, src = hbm_peak()
    return {"bodies": n, "kernel_ms": k_ms, "bytes_per_body": 152, "gbs_algorithmic": gbs,
            "frac_hbm": gbs / hbm, "hbm_peak_gbs": hbm, "hbm_peak_source": src,
            "x_diff_vs_oracle_max_over_extent": float(np.max(np.abs(xs - ox)) / np.max(np.abs(ox))),
            "timing": f"median of {reps} launches, CUDA events on the library stream, "
                      "L2 flushed (256 MiB write) before each"}


def irregular_leg(lib, m, x, v, h2, dtr, args, nsample: int = 65536):
    """Irregular force + jerk + nearest neighbour over lists of ~NNBOPT,
    this library vs the reference's irr.avx.cpp, same inputs."""
    import oracle
    from nb6b200.abi import ForceLib
    n = m.shape[0]
    ns = min(nsample, n)
    lmax = args.lmax
    rows = np.zeros((ns, lmax), dtype=np.int32)
    for s in range(0, ns, args.chunk):
        e = min(ns, s + args.chunk)
        _, _, _, lst = lib.gpunb_regf(h2[s:e], dtr[s:e], x[s:e], v[s:e], lmax, args.nnbmax, args.m_flag)
        for r in range(e - s):
            k = int(lst[r, 0])
            ids = lst[r, 1:1 + max(k, 0)]
            ids = ids[ids != s + r][: lmax - 1] + 1       # 1-based, self removed
            rows[s + r, 0] = len(ids)
            rows[s + r, 1:1 + len(ids)] = ids
    zeros = np.zeros((n, 3))
    t0 = np.zeros(n)
    addr = np.arange(1, ns + 1, dtype=np.int32)
    pairs = float(rows[:, 0].sum())
    out = {"sample_i": ns, "list_pairs": int(pairs), "nnb_mean": pairs / ns}

    def run(flib, name, reps):
        flib.irr_open(n, lmax, 0)
        flib.irr_set_jp_all(x, v, zeros, zeros, m, t0)
        for i in range(ns):
            flib.irr_set_list(i + 1, rows[i])
        # the caller's own result arrays (a Fortran caller's static FIRR,
        # FD and neighbour-id arrays), reused call after call
        out = (np.zeros((ns, 3)), np.zeros((ns, 3)), np.zeros(ns, dtype=np.int32))
        flib.irr_firr_vec(0.0, addr, out)          # uploads the staged state
        t = time.perf_counter()
        for _ in range(reps):
            res = flib.irr_firr_vec(0.0, addr, out)
        dt = (time.perf_counter() - t) / reps
        res = tuple(a.copy() for a in res)
        flib.irr_close(0)
        return res, dt

    import ctypes as C
    # the kernel over every body in one launch (the roofline figure), then
    # the default call: four launches whose results are copied into the
    # caller's arrays while the later ones run (the call time)
    lib.lib.nb6_irr_tune_(C.byref(C.c_int(1)))
    run(lib, "libnb6b200", 5)
    k_ms = float(lib.lib.nb6_irr_last_kernel_ms_())
    lib.lib.nb6_irr_tune_(C.byref(C.c_int(0)))
    ours, t_ours = run(lib, "libnb6b200", 5)
    span_ms = float(lib.lib.nb6_irr_last_kernel_ms_())
    if not oracle.ref_available("irr"):
        oracle.build(ref=True)
    ref, t_ref = run(ForceLib(oracle.ref_lib("irr"), "ref-irr-avx"), "irr.avx", 2)
    a_o, a_r = ours[0], ref[0]
    rel = np.sqrt(((a_o - a_r) ** 2).sum(1) / np.maximum((a_r ** 2).sum(1), 1e-300))
    if k_ms:
        # 128-byte FP64 record + 4-byte id per list pair (HBM-bound gathers)
        out["kernel_ms"] = k_ms
        out["kernel_pairs_per_s"] = pairs / (k_ms * 1e-3)
        out["kernel_gbs_algorithmic"] = 132.0 * pairs / (k_ms * 1e-3) / 1e9
        hbm, src = hbm_peak()
        out["kernel_frac_hbm"] = out["kernel_gbs_algorithmic"] / hbm
        out["hbm_peak_gbs"] = hbm
        out["hbm_peak_source"] = src
        out["kernel_launch"] = "one launch over every body"
        out["call_launches_span_ms"] = span_ms
    out.update({"pairs_per_s": pairs / t_ours, "ms_per_call": 1e3 * t_ours,
                "cpu_reference_pairs_per_s": pairs / t_ref,
                "cpu_reference_threads": int(os.environ.get("OMP_NUM_THREADS", "1")),
                "acc_rel_diff_vs_reference_max": float(rel.max()),
                "nnbid_equal_fraction": float(np.mean(ours[2] == ref[2])),
                "timing": "wall clock around the synchronous irr_simd_firr_vec_ call (state "
                          "already uploaded)"})
    return out


def tuned_table():
    """The regular-force autotuner's choices in this process, as
    "log2 N_active/log2 N_j/m_flag: variant" strings."""
    import ctypes as C
    from nb6b200 import load_cdll
    lib = load_cdll()
    n, cap = C.c_int(0), C.c_int(256)
    buf = (C.c_int * (4 * 256))()
    lib.nb6_regf_tuned_(C.byref(n), C.byref(cap), buf)
    return [f"{buf[4 * k]}/{buf[4 * k + 1]}/{buf[4 * k + 2]}: {buf[4 * k + 3]}" for k in range(min(n.value, 256))]


def northstar_leg(m, x, v, rs, args):
    """N-body time per wall second of the block-step drivers on this GPU,
    the plain GPU method against the batched, device-resident form:

    config 3  the bench's King W0=6 cluster (N = 1M, 5% binaries as c.m.
              bodies), radii from its NNBOPT-th neighbour, to T = args.ns_t3:
              plain = the single-cluster driver (host prediction and
              gpunb_send_ per regular block, host correctors, 1024-i
              gpunb_regf_ calls, util_gpu.F); batched = the ensemble driver
              with the j set predicted, both correctors and the block clock
              on the device (dev_corrector 3);
    config 4  args.ns_clusters Plummer clusters (Kroupa IMF, N log-uniform
              512-8192) to T = args.ns_t4 as one batched ensemble, against
              each cluster run alone with the plain method, measured on
              args.ns_alone clusters spread over the size range and scaled
              by the ensemble's total N^2 over theirs.

    Wall times are the drivers' own (block loop and energy outputs; the
    start-up evaluation is reported beside them).  Energy errors are the
    largest |E(t) - E(0)| / |E(0)| over the outputs, per cluster."""
    from nb6b200 import drive
    from nb6b200.ensemble_bench import make_clusters
    ours = drive.backend_paths("nb6b200")
    out = {}
    t3 = args.ns_t3
    t = time.perf_counter()
    plain = drive.run(ours, m, x, v, tcrit=t3, dt_out=t3, rs_init=rs)
    t_plain = time.perf_counter() - t
    t = time.perf_counter()
    batch = drive.run_ensemble(ours, [(m, x, v)], batched=True, tcrit=t3, dt_out=t3, rs_init=rs,
                               dev_corrector=3)
    t_batch = time.perf_counter() - t
    wp, wb = plain.stats["wall_total"], batch.stats["wall_total"]
    out["config3"] = {
        "workload": f"king-w0=6 N={args.n} ({m.shape[0]} c.m. bodies) to T = {t3}",
        "plain": {"wall_s": wp, "wall_with_startup_s": t_plain, "nbody_time_per_wall_s": t3 / wp,
                  "dE": plain.de_max, "reg_calls": plain.stats["reg_calls"],
                  "reg_steps": plain.stats["reg_steps"], "irr_steps": plain.stats["irr_steps"]},
        "batched_device": {"wall_s": wb, "wall_with_startup_s": t_batch, "nbody_time_per_wall_s": t3 / wb,
                           "dE": float(batch.de_max[0]), "reg_calls": batch.stats["reg_calls"],
                           "reg_steps": batch.stats["reg_steps"], "irr_steps": batch.stats["irr_steps"],
                           "wall_block_runs_s": batch.stats["wall_irr"],
                           "wall_regular_s": batch.stats["wall_reg"]},
        "speedup": wp / wb,
        "autotuner": tuned_table(),
        "dE_ratio_batched_over_plain": float(batch.de_max[0]) / plain.de_max if plain.de_max > 0 else None}
    cls = make_clusters(args.ns_clusters)
    sizes = np.array([c.n for c in cls])
    t4 = args.ns_t4
    dt_out = min(t4, 0.25)
    t = time.perf_counter()
    ens = drive.run_ensemble(ours, cls, batched=True, tcrit=t4, dt_out=dt_out, dev_corrector=3)
    t_ens = time.perf_counter() - t
    order = np.argsort(sizes)
    pick = order[np.linspace(0, len(cls) - 1, min(args.ns_alone, len(cls))).astype(int)]
    w_alone, ratios = 0.0, []
    for c in pick:
        cl = cls[c]
        r = drive.run(ours, cl.mass, cl.pos, cl.vel, tcrit=t4, dt_out=dt_out)
        w_alone += r.stats["wall_total"]
        ratios.append(float(ens.de_max[c]) / r.de_max if r.de_max > 0 else float("nan"))
    scale = float((sizes.astype(float) ** 2).sum() / (sizes[pick].astype(float) ** 2).sum())
    we = ens.stats["wall_total"]
    out["config4"] = {
        "workload": f"{len(cls)} Plummer clusters, Kroupa IMF, N log-uniform 512-8192, "
                    f"total {int(sizes.sum())} bodies, to T = {t4}",
        "ensemble": {"wall_s": we, "wall_with_startup_s": t_ens, "nbody_time_per_wall_s": t4 / we,
                     "dE_median": float(np.median(ens.de_max)), "dE_p90": float(np.percentile(ens.de_max, 90))},
        "alone": {"clusters_run": int(len(pick)), "wall_s_measured": w_alone, "scale_sum_n2": scale,
                  "wall_s": w_alone * scale, "nbody_time_per_wall_s": t4 / (w_alone * scale)},
        "speedup": w_alone * scale / we,
        "dE_ratio_ensemble_over_alone": {"median": float(np.nanmedian(ratios)),
                                         "max": float(np.nanmax(ratios)), "clusters": len(ratios)}}
    return out


def _rel(a, b):
    """Per-row relative error |a - b| / |b| (vector rows or scalars)."""
    if a.ndim == 1:
        return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    return np.sqrt(((a - b) ** 2).sum(1) / np.maximum((b ** 2).sum(1), 1e-300))


def fp64_error_leg(lib, m, x, v, h2, dtr, args, ncalls: int = 16, ncore: int = 2):
    """Force, jerk and potential error against the FP64 oracle over many
    calls of the timed shape: `ncalls` of the step's 1024-i calls, evenly
    spaced over the call sequence (the bodies are in random radial order, so
    each is a sample of the whole cluster), plus `ncore` calls of the bodies
    nearest the centre -- the King core, where the near field is densest
    and the regular force of a body cancels most.  Every i of every call is
    checked; lists are compared row for row."""
    import oracle
    n = m.shape[0]
    chunks = [(s, min(n, s + args.chunk)) for s in range(0, n, args.chunk)]
    picks = sorted(set(np.linspace(0, len(chunks) - 1, min(ncalls, len(chunks))).astype(int).tolist()))
    calls = [("timed", np.arange(*chunks[k])) for k in picks]
    centre = (m[:, None] * x).sum(0) / m.sum()
    byr = np.argsort(((x - centre) ** 2).sum(1), kind="stable")
    for c in range(ncore):
        calls.append(("core", np.sort(byr[c * args.chunk:(c + 1) * args.chunk])))
    ea, ej, ep, core_a, core_j = [], [], [], [], []
    rows_differ, nnb, t_orc = 0, [], 0.0
    for kind, idx in calls:
        a_g, j_g, p_g, l_g = lib.gpunb_regf(h2[idx], dtr[idx], x[idx], v[idx], args.lmax,
                                            args.nnbmax, args.m_flag)
        t0 = time.perf_counter()
        a_o, j_o, p_o, l_o = oracle.regf(m, x, v, h2[idx], dtr[idx], x[idx], v[idx],
                                         args.lmax, args.nnbmax, args.m_flag)
        t_orc += time.perf_counter() - t0
        rows_differ += int(np.sum(np.any(l_g != l_o, axis=1)))
        ok = l_o[:, 0] >= 0
        ra, rj, rp = _rel(a_g, a_o)[ok], _rel(j_g, j_o)[ok], _rel(p_g, p_o)[ok]
        ea.append(ra)
        ej.append(rj)
        ep.append(rp)
        nnb.append(l_o[ok, 0])
        if kind == "core":
            core_a.append(ra)
            core_j.append(rj)
    ea, ej, ep = np.concatenate(ea), np.concatenate(ej), np.concatenate(ep)
    core_a, core_j = np.concatenate(core_a), np.concatenate(core_j)

    def q(e, p):
        return float(np.quantile(e, p))
    return {"calls": len(calls), "timed_calls_checked": len(picks), "core_calls": ncore,
            "sample_i": int(ea.size),
            "core_radius_max": float(np.sqrt(((x[byr[ncore * args.chunk - 1]] - centre) ** 2).sum())),
            "acc_rel_max": float(ea.max()), "acc_rel_p999": q(ea, 0.999),
            "acc_rel_median": q(ea, 0.5),
            "jrk_rel_max": float(ej.max()), "jrk_rel_p999": q(ej, 0.999),
            "jrk_rel_median": q(ej, 0.5),
            "pot_rel_max": float(ep.max()), "pot_rel_p999": q(ep, 0.999),
            "core_acc_rel_max": float(core_a.max()), "core_jrk_rel_max": float(core_j.max()),
            "rows_acc_above_1e-6": int(np.sum(ea > 1e-6)),
            "lists_identical": rows_differ == 0, "list_rows_differing": rows_differ,
            "nnb_mean": float(np.concatenate(nnb).mean()),
            "oracle_s": t_orc}


def run_reference(args):
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return 0
    m, x, v, rs, dtr = workload(args.n, args.seed)
    n = m.shape[0]
    # each step: a bounded sample of the workload (a few seconds of CPU)
    _, threads, _, t1 = cpu_reference_rate(m, x, v, rs, dtr, args, seconds=0.0, max_calls=1)
    calls = max(1, int(2.0 / max(t1, 1e-3)))
    for _ in range(args.warmup):
        cpu_reference_rate(m, x, v, rs, dtr, args, seconds=1e9, max_calls=1)
    rates, times = [], []
    for _ in range(args.steps):
        r, threads, c, t = cpu_reference_rate(m, x, v, rs, dtr, args, seconds=1e9, max_calls=calls)
        rates.append(r)
        times.append(t)
    value = float(np.sum([r * t for r, t in zip(rates, times)]) / np.sum(times))
    sample = (f"{calls} of the step's {(n + args.chunk - 1) // args.chunk} calls (random ones) x "
              f"{args.chunk} i x {n} j per timed step, reg.avx.cpp gpunb_regf_; the rate is "
              f"pairs over the time of those calls")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic King W0=6 (seeded), Kroupa IMF 0.08-100 Msun, 5% binaries "
                "as c.m. bodies, Henon units",
        "config": bench_config(args, n, args.gpus),
        "sample": sample,
        "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": threads,
                         "cpu": cpu_model(), "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    world, rank, local = dist_setup(args)
    os.environ["NB_GPU_DEVICE"] = str(local)
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist

    import nb6b200
    lib = nb6b200.load()
    raw = lib.lib
    m, x, v, rs, dtr = workload(args.n, args.seed + 7919 * rank)
    n = m.shape[0]
    h2 = rs ** 2 if not args.m_flag else rs ** 2 / m.mean()
    lib.gpunb_open(n + 10, 0)
    lib.gpunb_send(m, x, v)
    stream = torch.cuda.ExternalStream(raw.nb6_stream_())
    dev = torch.device("cuda", local)
    d_h2 = torch.tensor(h2, dtype=torch.float64, device=dev)
    d_dtr = torch.tensor(dtr, dtype=torch.float64, device=dev)
    d_x = torch.tensor(x, dtype=torch.float64, device=dev).contiguous()
    d_v = torch.tensor(v, dtype=torch.float64, device=dev).contiguous()
    torch.cuda.synchronize()
    chunks = [(s, min(n, s + args.chunk)) for s in range(0, n, args.chunk)]
    ci = C.c_int
    lmax, nnbmax, mflag = ci(args.lmax), ci(args.nnbmax), ci(args.m_flag)

    def dev_step():
        for s, e in chunks:
            raw.nb6_regf_device_(C.byref(ci(e - s)), C.c_void_p(d_h2.data_ptr() + 8 * s),
                                 C.c_void_p(d_dtr.data_ptr() + 8 * s),
                                 C.c_void_p(d_x.data_ptr() + 24 * s),
                                 C.c_void_p(d_v.data_ptr() + 24 * s),
                                 C.byref(lmax), C.byref(nnbmax), C.byref(mflag))

    flush_buf = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush_l2():
        with torch.cuda.stream(stream):
            flush_buf.fill_(1.0)
        stream.synchronize()

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    # warm-up
    for _ in range(args.warmup):
        dev_step()
    raw.nb6_sync_()
    peak_tf = float(raw.nb6_fp32_peak_probe_(C.byref(ci(20000))))

    # kernel-only launch time of the force kernel (live CUDA events on the
    # library stream around regf_kernel alone), over a sample of full calls
    kms = []
    for s, e in chunks[: min(64, len(chunks))]:
        raw.nb6_regf_device_(C.byref(ci(e - s)), C.c_void_p(d_h2.data_ptr() + 8 * s),
                             C.c_void_p(d_dtr.data_ptr() + 8 * s),
                             C.c_void_p(d_x.data_ptr() + 24 * s),
                             C.c_void_p(d_v.data_ptr() + 24 * s),
                             C.byref(lmax), C.byref(nnbmax), C.byref(mflag))
        kms.append(float(raw.nb6_regf_last_kernel_ms_()))
    geom = (ci * 3)()
    raw.nb6_regf_last_geometry_(geom)
    kernel_ms = float(np.median(kms))

    # timed region: K steps, L2 flushed between steps, events on the library stream
    clocks = Clocks(local)
    step_ms = []
    clocks.start()
    for _ in range(args.steps):
        flush_l2()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dev_step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    barrier()
    clk = clocks.stop()
    ms = float(np.mean(step_ms))
    total_ms = reduce_max(float(np.sum(step_ms)), pg, dev)
    pairs_step = float(n) * float(n)
    value = whole_job_rate(world, pairs_step, args.steps, total_ms)

    # e2e through the C ABI with host buffers: gpunb_send_ + gpunb_regf_ calls
    e2e = None
    if not args.no_e2e:
        lst = np.zeros((args.chunk, args.lmax), dtype=np.int32)
        acc = np.zeros((args.chunk, 3))
        jrk = np.zeros((args.chunk, 3))
        pot = np.zeros(args.chunk)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)

        def e2e_step():
            lib.gpunb_send(m, x, v)
            for s, e in chunks:
                raw.gpunb_regf_(C.byref(ci(e - s)), h2[s:e].ctypes.data_as(dp),
                                dtr[s:e].ctypes.data_as(dp), x[s:e].ctypes.data_as(dp),
                                v[s:e].ctypes.data_as(dp), acc.ctypes.data_as(dp),
                                jrk.ctypes.data_as(dp), pot.ctypes.data_as(dp), C.byref(lmax),
                                C.byref(nnbmax), lst.ctypes.data_as(ip), C.byref(mflag))
        e2e_step()
        barrier()
        t0 = time.perf_counter()
        e2e_steps = max(1, min(args.steps, 2))
        for _ in range(e2e_steps):
            e2e_step()
        e2e_s = reduce_max((time.perf_counter() - t0) / e2e_steps, pg, dev)
        # bytes moved per step: the j set (m, x, v) and the i data up; the
        # force rows (8 doubles) and each list row's count + ids down (the
        # library writes only the used part of a row into pinned memory);
        # the ids are counted from the neighbour lists of the last call
        nnb_last = np.abs(lst[: chunks[-1][1] - chunks[-1][0], 0]).astype(float)
        ids_per_i = float(nnb_last.mean()) + 1.0
        e2e = {"value": world * pairs_step / e2e_s, "unit": "pairs/s",
               "h2d_bytes_per_step": int(n * (8 + 24 + 24) + n * 64),
               "d2h_bytes_per_step": int(n * 64 + n * ids_per_i * 4),
               "steps": e2e_steps, "timing": "wall clock around synchronous ABI calls"}

    # the N^2 potential of the same cluster (GPUPOT, energy.F:33): device
    # time on the library stream of the whole call after the upload (the
    # spatial order, the kernel and the sums), 27 flops per pair
    # (pot.avx.cpp:123-135); accuracy of that call's result on a contiguous
    # sample of 64 i against the FP64 oracle
    pot = None
    if not args.no_pot:
        d_m = torch.tensor(m, dtype=torch.float64, device=dev)
        outp = C.POINTER(C.c_double)()
        for _ in range(2):
            raw.nb6_pot_device_(C.byref(ci(1)), C.byref(ci(n)), C.byref(ci(n)),
                                C.c_void_p(d_m.data_ptr()), C.c_void_p(d_x.data_ptr()), C.byref(outp))
        pot_ms = float(raw.nb6_pot_last_kernel_ms_())
        pot = {"pairs_per_s": float(n) * n / (pot_ms * 1e-3), "kernel_ms": pot_ms,
               "note": "the ordered far loop issues 7 FP32 lane operations and one MUFU "
                       "rsqrt per pair, so the MUFU pipe bounds it: the fraction below is "
                       "rsqrt results per second against the nominal MUFU rate",
               # one rsqrt per pair against the nominal 16 MUFU results per SM
               # per clock at the GPU's maximum SM clock
               "frac_mufu_peak": float(n) * n / (pot_ms * 1e-3) / mufu_peak_per_s()}
        if rank == 0 and world == 1:
            import oracle
            i0 = int(np.random.default_rng(9).integers(1, n - 64))
            po = oracle.pot(m, x, i0, 64)
            t0 = time.perf_counter()
            pg_full = lib.gpupot(m, x)                      # the whole-set call, as timed
            pot["e2e_s"] = time.perf_counter() - t0         # through gpupot_ with host arrays
            pg_ = pg_full[i0 - 1:i0 - 1 + 64]
            pot["rel_err_max_sample64"] = float(np.max(np.abs(pg_ / po - 1)))
            # the reference's own CUDA potential (gpupot.gpu.cu built for
            # sm_100a), same call with host arrays, when it was built
            if not args.no_ref_gpu and oracle.ref_available("gpupot_gpu"):
                from nb6b200.abi import ForceLib
                rlib = ForceLib(oracle.ref_lib("gpupot_gpu"), "ref-gpupot-gpu")
                rlib.gpupot(m[:4096], x[:4096])             # warm-up (context, module)
                t0 = time.perf_counter()
                pr_ = rlib.gpupot(m, x)
                pot["reference_gpu_s"] = time.perf_counter() - t0
                pot["reference_gpu_rel_diff_max"] = float(np.max(np.abs(pr_ / pg_full - 1)))
        del d_m

    # the irregular path on the same cluster: neighbour lists of a sample
    # of bodies from this library's regular call, every body's state in the
    # irregular store, one irr_simd_firr_vec_ over the sample; 60 flops per
    # list pair (irr.avx.cpp:411).  The reference's irr.avx.cpp runs the
    # identical calls on the host cores.
    # the diagnostic legs below run on rank 0 of a one-GPU run only: with N
    # replicas they would only hold the other GPUs while rank 0 works alone
    solo = rank == 0 and world == 1
    irr = None
    if not args.no_irr and solo:
        irr = irregular_leg(lib, m, x, v, h2, dtr, args)

    # the Hermite predictor over the same bodies (rank 0)
    pred = None
    if not args.no_pred and solo:
        pred = predictor_leg(lib, m, x, v, flush_l2)

    # accuracy against the FP64 oracle on calls of the timed shape (chunks of
    # 1024 i, so the same tuned kernel and its far-tile path run; rank 0)
    err = None
    cpu = None
    if solo:
        if not args.no_err:
            err = fp64_error_leg(lib, m, x, v, h2, dtr, args)
        if not args.no_cpu_baseline:
            rate, threads, calls, t_used = cpu_reference_rate(m, x, v, rs, dtr, args,
                                                              seconds=args.cpu_seconds)
            cpu = {"value": rate, "unit": "pairs/s", "cores": threads, "cpu": cpu_model(),
                   "kind": "reference",
                   "sample": f"{calls} calls x {args.chunk} i x {n} j of the same workload, "
                             f"reg.avx.cpp gpunb_regf_ (oracle/_ref), {t_used:.1f} s"}

    lib.gpunb_close()
    # configs 3 and 4 end to end: the plain GPU method against the batched,
    # device-resident drivers (rank 0)
    ns = None
    if solo and not args.no_northstar:
        ns_clk = Clocks(local)
        ns_clk.start()
        ns = northstar_leg(m, x, v, rs, args)
        ns["clocks"] = ns_clk.stop()
    # the reference's own GPU code on this GPU, same workload (rank 0)
    ref_gpu = None
    if solo and not args.no_ref_gpu:
        ref_gpu = reference_gpu_rate(m, x, v, rs, dtr, args, seconds=5.0)
    achieved = FLOPS_PER_PAIR * args.chunk * n / (kernel_ms * 1e-3) / 1e12
    nominal = 2 * 128 * 148 * (clk.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
            "frac": achieved / peak_tf if peak_tf else None,
            "traffic": NCU_TRAFFIC_PER_LAUNCH,
            "kernel": {11: "regf_x2_kernel<1>", 12: "regf_x2_kernel<2>", 13: "regf_x2_kernel<1,f64dx>",
                       1: "regf_kernel<1>", 2: "regf_kernel<2>", 4: "regf_kernel<4>"}.get(
                           geom[0], f"regf_jpar_kernel<{-geom[0]}>"),
            "kernel_ms_per_launch": kernel_ms,
            "flops_per_launch": FLOPS_PER_PAIR * args.chunk * n,
            "algorithmic_bytes_per_launch": 48 * n + 64 * args.chunk,
            "peak_source": "measured: FFMA probe kernel in the library, same process "
                           "(MEASURED_PEAKS.json carries no FP32 figure)",
            "frac_of_nominal_fp32": achieved / nominal,
            "geometry": {"i_per_thread": geom[0], "i_tiles": geom[1], "j_slices": geom[2]}}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic King W0=6 (seeded), Kroupa IMF 0.08-100 Msun, 5% binaries "
                    "as c.m. bodies, Henon units",
            "config": bench_config(args, n, world),
            # per call: force kernel + finalize, plus the active-set order
            # when the j set is spatially ordered (>= 32768 bodies)
            "gpu_launches": int(args.steps * len(chunks) * (3 if n >= 32768 else 2)),
            "clocks": clk, "roofline": roof, "e2e": e2e, "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "err_vs_fp64": err,
            "gpupot": pot,
            "irregular": irr,
            "predictor": pred,
            "northstar": ns,
            "pct_fp32_peak": 100.0 * FLOPS_PER_PAIR * pairs_step / (ms * 1e-3) / 1e12 / peak_tf,
        }
        print(json.dumps(out), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
