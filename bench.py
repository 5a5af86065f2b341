#!/usr/bin/env python
"""Benchmark: reduced columns/s of the engine on the 64^3 lower-star workload.

Workload (one "step" = one full reduction, init passes to sorted pairs): the
lower-star filtration of the Freudenthal triangulation of a 64^3 grid (all
vertices, edges, triangles and tetrahedra: 6,573,043 columns, 18,646,740
non-zeros) whose vertex values are seeded Gaussian white noise smoothed by a
Gaussian of sigma = 2 voxels (float32); ties broken by dimension then
lexicographic vertex order; int32 indices; model 1 (high-dimension guided
clearing, max_iteration 10), ss_block_size 102400, growth 1.05.  Synthetic,
seeded data stands in for the reference's input files.

  value  = columns / device time with the matrix already resident in HBM
           (CUDA events on the launching stream, L2 flushed between steps)
  e2e    = the same metric through the C ABI from pinned host buffers,
           host->device copy of the matrix and device->host copy of the pairs
           and essential classes inside the timed region
  --impl reference: the CPU restatement of the reference's reduction (the
           reference's own CPU path, phat-highclear, cannot be built: its PHAT
           library headers are not part of the reference tree), timed on the
           host on the same workload.

Multi-GPU: one process per GPU (torchrun); a single reduction does not shard,
so every rank reduces its own replica of the workload (request-level weak
scaling, no collective on the data path); value = total columns / max time.

Extra keys (rank 0, after the timed legs; --no-extra skips them):
  rips2000  2,000-point Rips, model 0, reference default parameters (e2e)
  vr100k    100,000-point Rips, model 3, max_iteration 100 (collapse +
            guided clearing), with the reduction's roofline
  batched   512 uneven Rips complexes reduced as one batch (autotuned) vs the
            same 512 one at a time with the reference's default parameters
  served    a seeded Poisson request stream through the serving loop vs a
            serial one-at-a-time loop: columns/s and p50/p95/p99 latency
Every leg checks its pairs (against the oracle, or against the plain path
whose pairs are checked against the oracle on a sample).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
import threading

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
# 32 hardware work queues for the engine's side streams, before any CUDA context
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
sys.path.insert(0, ROOT)

GRID, SIGMA, SEED = 64, 2.0, 2
MODEL, MAX_ITER, SS, GROWTH, QUEUE, L1, L2 = 1, 10, 102400, 1.05, 65536, 32, 8192
METRIC, UNIT = "reduced_columns_per_s", "columns/s"


def workload_config(n, nnz):
    return {"workload": f"lower-star Freudenthal {GRID}^3, sigma {SIGMA}, model {MODEL}, max_iteration {MAX_ITER}, "
                        f"ss_block_size {SS}, growth {GROWTH}",
            "ncols": n, "nnz": nnz, "grid": GRID, "sigma": SIGMA, "seed": SEED, "model": MODEL,
            "max_iteration": MAX_ITER, "ss_block_size": SS, "growth": GROWTH, "queue_size": QUEUE,
            "level1_capacity": L1, "level2_capacity": L2, "dualize": 0, "index": "int32", "values": "float32",
            "l2": "flushed between steps (256 MiB write); inputs (149 MB) also exceed L2",
            "hw_queues": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS")}


def dist_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """SM clock and throttle-reason sampling during the timed region.

    NVML is read every 5 ms from a thread (a timed region of ~100 ms gets ~20
    samples); without NVML, nvidia-smi is polled every 200 ms instead.  Only
    reads: no clock or other GPU setting is touched.
    """

    _NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device):
        self.sm, self.mx, self.reasons = [], 0.0, set()
        self.p = self.thread = None
        self.done = threading.Event()
        try:
            import pynvml

            pynvml.nvmlInit()
            try:
                import torch

                uuid = str(torch.cuda.get_device_properties(device).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + uuid if not uuid.startswith("GPU-") else uuid)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            bits = dict(zip(self._NAMES, (pynvml.nvmlClocksEventReasonHwSlowdown,
                                          pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                                          pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                                          pynvml.nvmlClocksEventReasonSwPowerCap)))
            first = threading.Event()

            def run():
                while True:
                    try:
                        self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.reasons.update(n for n, b in bits.items() if r & b)
                    except Exception:
                        pass
                    first.set()
                    if self.done.wait(0.005):
                        return

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            first.wait(2.0)
            return
        except Exception:
            self.thread = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.thread is not None:
            self.done.set()
            self.thread.join(timeout=5)
            return self._summary("nvml")
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                self.sm.append(float(parts[1]))
                self.mx = max(self.mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(self._NAMES, parts[5:9]):
                if v.lower() == "active":
                    self.reasons.add(nm)
        os.unlink(self.f.name)
        return self._summary("nvidia-smi")

    def _summary(self, source):
        if not self.sm:
            return None
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.mx, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": source}


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0}, "fallback"


def load_traffic():
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except (OSError, ValueError):
        return {}


def oracle_run(m):
    oracle = oracle_module()

    t = time.perf_counter()
    r = oracle.reduce(m, model=MODEL, max_iteration=MAX_ITER)
    return time.perf_counter() - t, r


def reference_arm(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    # the input is built with numpy (same sizes and value distribution as the
    # engine's generator), so this arm loads none of the engine's libraries
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lowerstar_np

    class _M:
        pass

    m = _M()
    m.dims, m.col_ptr, m.rows = lowerstar_np.lowerstar(GRID, SIGMA, SEED)
    m.ncols, m.nnz = int(m.dims.shape[0]), int(m.rows.shape[0])
    for _ in range(args.warmup):
        oracle_run(m)
    times = []
    for _ in range(args.steps):
        dt, r = oracle_run(m)
        times.append(dt)
    total = sum(times)
    value = m.ncols * len(times) / total
    sample = (f"full workload ({m.ncols} columns, built with numpy: oracle/lowerstar_np.py) per step, "
              f"single-threaded C++ restatement (oracle/sspp_oracle.cpp)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": workload_config(m.ncols, m.nnz),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ extra legs
# Each returns a dict added to the JSON line under its own key.  Host timers
# (time.perf_counter) bracket whole calls that end with the results in host
# memory, so these are end-to-end numbers through the public API.

def _timed(fn):
    t = time.perf_counter()
    out = fn()
    return time.perf_counter() - t, out


def leg_rips2000(steps):
    """2,000 points in [0,1]^3, radius 0.08, dim <= 3, model 0 (reference defaults)."""
    from specseqplusplus_b200 import Engine, Params, gen

    m = gen.rips(2000, 3, 1, 0.08, 3)
    p = Params()
    with Engine(0) as e:
        for _ in range(3):
            e.load_csc(m)
            e.reduce(p)
        ts = []
        for _ in range(max(steps, 5)):
            dt, _ = _timed(lambda: (e.load_csc(m), e.reduce(p), e.pairs(), e.essentials()))
            ts.append(dt)
        pr = e.pairs()
    ref = oracle_module().reduce(m)
    return {"workload": "Rips 2000 pts [0,1]^3 r 0.08 dim<=3, model 0, reference default parameters",
            "ncols": m.ncols, "cols_per_s_e2e": m.ncols / statistics.median(ts), "ms_e2e": 1000 * statistics.median(ts),
            "pairs_exact": bool(np.array_equal(pr, ref.pairs))}


def leg_vr100k(steps, peak):
    """100,000 points, radius 0.016, dim <= 3, model 3 (collapse + guided clearing, max_iteration 100)."""
    import torch

    from specseqplusplus_b200 import Engine, Params, gen

    m = gen.rips(100000, 3, 7, 0.016, 3)
    p = Params(model=3, max_iteration=100, queue_size=65536, level1_capacity=100, level2_capacity=250)
    dev = torch.device("cuda", 0)
    d = [torch.from_numpy(x).to(dev) for x in (m.dims, m.col_ptr, m.rows)]
    stream = torch.cuda.current_stream(dev)
    with Engine(0, profile=1) as e:
        e.load_csc_device(m.ncols, d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr())
        for _ in range(3):
            e.reduce(p, stream=stream.cuda_stream)
        dev_ms, host_ms, red_ms = [], [], []
        for _ in range(max(steps, 5)):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            a.record(stream)
            e.reduce(p, stream=stream.cuda_stream)
            b.record(stream)
            torch.cuda.synchronize()
            host_ms.append(1000 * (time.perf_counter() - t0))
            dev_ms.append(a.elapsed_time(b))
            st = e.stats()
            red_ms.append(st["light_gpu_ms"] + st["heavy_gpu_ms"])
        pr, es = e.pairs(), e.essentials()
        st = e.stats()
    ref = oracle_module().reduce(m, model=3, max_iteration=100)
    exact = bool(np.array_equal(pr, ref.pairs) and np.array_equal(es, ref.essential))
    rms = statistics.median(red_ms)
    ach = ref.stats["add_bytes"] / (rms / 1000) / 1e9 if rms > 0 else None
    return {"workload": "Rips 100k pts [0,1]^3 r 0.016 dim<=3, model 3, max_iteration 100, queue 65536, L1/L2 100/250",
            "ncols": m.ncols, "nnz": m.nnz, "cols_per_s": m.ncols / (statistics.median(host_ms) / 1000),
            "device_ms": statistics.median(dev_ms), "host_ms": statistics.median(host_ms),
            "collapse_dropped": st["collapse_dropped"], "highclear_cleared": st["highclear_cleared"],
            "reduction_gpu_ms": rms, "additions": st["additions"],
            "roofline": {"bound": "hbm", "kernel": "reduction", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": (ach / peak) if ach else None, "algorithmic_bytes": ref.stats["add_bytes"],
                         "note": "about 1 MB of input: latency-bound, not bandwidth-bound"},
            "pairs_exact": exact}


def leg_batched(steps):
    """512 Rips complexes (200-5,000 points log-uniform, half 2-D dim<=2, half 3-D dim<=3, mean degree 8-40),
    reduced together (one block-diagonal reduction, autotuned) vs one at a time."""
    from specseqplusplus_b200 import Engine, Params, workloads

    mats, _ = workloads.batch_of_rips(512)
    N = sum(m.ncols for m in mats)
    # autotune 2: launch parameters and the choice between the boundary matrix
    # and dualization mode 2 (the pairs are the same either way)
    p_auto, p_ref = Params(autotune=2), Params()
    with Engine(0) as e:
        for _ in range(10):  # the autotuner tries its candidates on this size class first
            e.load_batch(mats)
            e.reduce(p_auto)
            e.batch_results()
        ts = []
        for _ in range(max(steps, 3)):
            dt, res = _timed(lambda: (e.load_batch(mats), e.reduce(p_auto), e.batch_results())[2])
            ts.append(dt)
        chosen = e.params()

    def one_at_a_time(p, reps):
        with Engine(0) as e1:
            for m in mats:  # warm-up (and, with autotune, the per-class trials)
                for _ in range(reps):
                    e1.load_csc(m)
                    e1.reduce(p)
            out = []
            t = time.perf_counter()
            for m in mats:
                e1.load_csc(m)
                e1.reduce(p)
                out.append((e1.pairs(), e1.essentials()))
            return time.perf_counter() - t, out

    t_ref, plain = one_at_a_time(p_ref, 1)
    t_auto, _ = one_at_a_time(p_auto, 9)
    same = all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(res, plain))
    orc = oracle_module()
    sample = list(range(0, len(mats), 32))
    exact = all(np.array_equal(res[i][0], orc.reduce(mats[i]).pairs) for i in sample)
    tb = statistics.median(ts)
    return {"workload": "512 Rips complexes, 200-5000 pts log-uniform, half 2-D (dim<=2) half 3-D (dim<=3), "
                        "mean degree U[8,40], per-instance seeds",
            "ncols": N, "batched_cols_per_s": N / tb, "batched_ms": 1000 * tb,
            "plain_cols_per_s": N / t_ref, "plain_ms": 1000 * t_ref,
            "plain_autotuned_cols_per_s": N / t_auto,
            "speedup_vs_plain": t_ref / tb, "speedup_vs_plain_autotuned": t_auto / tb,
            "batched_params": {"level1_capacity": chosen.level1_capacity, "level2_capacity": chosen.level2_capacity,
                               "ss_block_size": chosen.ss_block_size, "growth": chosen.growth,
                               "heavy_threads": chosen.heavy_threads, "dualize": chosen.dualize, "autotune": 2},
            "plain_params": "reference defaults (level capacities 1000/8000, ss_block_size 102400, growth 1.05, "
                            "queue_size 65536)",
            "pairs_equal_plain_all": bool(same), "pairs_exact_oracle_sample": bool(exact),
            "oracle_sample": f"{len(sample)} of {len(mats)} instances (every 32nd)"}


def leg_served(count=48, rates=(100.0, None), workers=3):
    """Poisson request stream (Rips 300-20,000 pts 2-D/3-D degree 8-40; lower-star 16^3-96^3 sigma 1-3):
    the serving loop (3 workers, autotune 2, continuous batching) vs a serial one-at-a-time loop with the
    reference's default parameters."""
    from specseqplusplus_b200 import Engine, Params, Server, workloads

    stream = workloads.serving_stream(count, 1.0, seed=5)
    mats = [m for _, _, m, _ in stream]
    gaps = np.diff([0.0] + [a for a, _, _, _ in stream])
    N = sum(m.ncols for m in mats)
    warm = [m for _, _, m, _ in workloads.serving_stream(16, 1.0, seed=99)]
    out = {"workload": f"{count} requests, Poisson arrivals (seeded); 75% Rips 300-20000 pts (2-D/3-D, degree "
                       f"8-40, dim<=3), 25% lower-star 16^3-96^3 sigma 1-3",
           "ncols": N, "max_request_cols": max(m.ncols for m in mats), "rates": []}
    plain_results = None
    for rate in rates:
        arrivals = np.cumsum(gaps / rate) if rate else np.zeros(count)

        def plain(p):
            with Engine(0) as e:
                for _ in range(2):
                    for m in warm:
                        e.load_csc(m)
                        e.reduce(p)
                lat, res = [], []
                t0 = time.perf_counter()
                for a, m in zip(arrivals, mats):
                    now = time.perf_counter() - t0
                    if now < a:
                        time.sleep(a - now)
                    e.load_csc(m)
                    e.reduce(p)
                    res.append((e.pairs(), e.essentials()))
                    lat.append(1000 * (time.perf_counter() - t0 - a))
                return N / (time.perf_counter() - t0 - arrivals[0]), np.percentile(lat, [50, 95, 99]), res

        cp, lp, pres = plain(Params())
        if plain_results is None:
            plain_results = pres
        with Server(Params(autotune=2), workers=workers) as srv:
            for _ in range(3):
                ids = [srv.submit(m, copy=False) for m in warm]
                for i in ids:
                    srv.wait(i)
                    srv.release(i)
            srv.reset_stats()
            ids = []
            t0 = time.perf_counter()
            for a, m in zip(arrivals, mats):
                now = time.perf_counter() - t0
                if now < a:
                    time.sleep(a - now)
                ids.append(srv.submit(m, copy=False))
            for i in ids:
                srv.wait(i)
            st = srv.stats()
            same = all(np.array_equal(srv.pairs(i), r[0]) and np.array_equal(srv.essentials(i), r[1])
                       for i, r in zip(ids, plain_results))
        out["rates"].append({"rate_per_s": rate if rate else "all at once",
                             "served_cols_per_s": st["cols_per_s"], "served_p50_ms": st["p50_ms"],
                             "served_p95_ms": st["p95_ms"], "served_p99_ms": st["p99_ms"],
                             "served_mean_batch": st["mean_batch_requests"],
                             "plain_cols_per_s": cp, "plain_p50_ms": float(lp[0]), "plain_p95_ms": float(lp[1]),
                             "plain_p99_ms": float(lp[2]), "speedup_vs_plain": st["cols_per_s"] / cp,
                             "served_phase_s": {"load": st["load_s"], "reduce": st["reduce_s"],
                                                "results": st["results_s"]},
                             "results_equal_plain": bool(same)})
    # the serial loop's results (which every served result equals) against the
    # oracle on a sample: every 6th request by size, up to 5 M columns each
    orc = oracle_module()
    by_size = sorted(range(count), key=lambda i: mats[i].ncols)
    sample = [i for i in by_size[::6] if mats[i].ncols <= 5_000_000]
    out["plain_vs_oracle"] = {"sample": f"{len(sample)} of {count} requests (every 6th by size, <= 5 M columns)",
                              "exact": bool(all(np.array_equal(plain_results[i][0], r.pairs) and
                                                np.array_equal(plain_results[i][1], r.essential)
                                                for i, r in ((i, orc.reduce(mats[i])) for i in sample)))}
    out["workers"] = workers
    out["built"] = served_built(stream, N, plain_results, workers)
    return out


def served_built(stream, N, want, workers=3):
    """The same requests given as point clouds and fields (the complexes are built on the device), all at
    once: the server against a serial one-at-a-time loop of device build + reduction."""
    from specseqplusplus_b200 import Engine, Params, Server, gen

    inputs = []
    for _, kind, _, d in stream:
        if kind == "rips":
            inputs.append(("r", gen.points(d["npts"], d["space_dim"], d["seed"]), d["radius"],
                           2 if d["space_dim"] == 2 else 3))
        else:
            inputs.append(("l", gen.field(d["grid"], d["sigma"], d["seed"]), None, 3))

    def load(e, x):
        if x[0] == "r":
            e.load_rips(x[1], x[2], x[3])
        else:
            e.load_lowerstar(x[1], x[3])

    with Engine(0) as e:
        for x in inputs[:8]:
            load(e, x)
            e.reduce(Params())
        lat, res = [], []
        t0 = time.perf_counter()
        for x in inputs:
            load(e, x)
            e.reduce(Params())
            res.append((e.pairs(), e.essentials()))
            lat.append(1000 * (time.perf_counter() - t0))
        plain = N / (time.perf_counter() - t0)
    with Server(Params(autotune=2), workers=workers) as srv:
        for _ in range(2):
            ids = [srv.submit_rips(x[1], x[2], x[3], copy=False) if x[0] == "r" else
                   srv.submit_lowerstar(x[1], x[3], copy=False) for x in inputs[:16]]
            for i in ids:
                srv.wait(i)
                srv.release(i)
        srv.reset_stats()
        ids = [srv.submit_rips(x[1], x[2], x[3], copy=False) if x[0] == "r" else
               srv.submit_lowerstar(x[1], x[3], copy=False) for x in inputs]
        for i in ids:
            srv.wait(i)
        st = srv.stats()
        same = all(np.array_equal(srv.pairs(i), w[0]) and np.array_equal(srv.essentials(i), w[1])
                   for i, w in zip(ids, want))
    same = same and all(np.array_equal(r[0], w[0]) and np.array_equal(r[1], w[1]) for r, w in zip(res, want))
    lp = np.percentile(lat, [50, 99])
    return {"workload": "the same requests as point clouds and fields, all at once; complexes built on the device",
            "served_cols_per_s": st["cols_per_s"], "served_p50_ms": st["p50_ms"], "served_p99_ms": st["p99_ms"],
            "plain_cols_per_s": plain, "plain_p50_ms": float(lp[0]), "plain_p99_ms": float(lp[1]),
            "speedup_vs_plain": st["cols_per_s"] / plain, "results_equal_boundary_matrix_path": bool(same)}


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    return oracle


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=GRID, help="smaller grid for profiling runs (default 64)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer leg (profiling runs)")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched, served, 2000-point Rips and 100k-point VR legs")
    ap.add_argument("--only", choices=["vr100k"],
                    help="profiling runs: run one extra leg alone and print its JSON")
    args = ap.parse_args()
    if args.grid != GRID:
        globals()["GRID"] = args.grid
    if args.impl == "reference":
        return reference_arm(args)
    if args.only == "vr100k":
        peak = float(load_peaks()[0].get("hbm_gbs", 6650.0))
        print(json.dumps({"vr100k": leg_vr100k(args.steps, peak), "profiling_run": True}))
        return 0

    import numpy as np
    import torch

    from specseqplusplus_b200 import Engine, Params, gen

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    m = gen.lowerstar(GRID, SIGMA, SEED)
    n, nnz = m.ncols, m.nnz
    p = Params(model=MODEL, max_iteration=MAX_ITER, ss_block_size=SS, growth=GROWTH, queue_size=QUEUE,
               level1_capacity=L1, level2_capacity=L2)
    dev = torch.device("cuda", local)
    d_dims = torch.from_numpy(m.dims).to(dev)
    d_colptr = torch.from_numpy(m.col_ptr).to(dev)
    d_rows = torch.from_numpy(m.rows).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---------------------------------------------------------- device-resident
    eng = Engine(local, profile=1)
    eng.load_csc_device(n, d_dims.data_ptr(), d_colptr.data_ptr(), d_rows.data_ptr())
    for _ in range(args.warmup):
        eng.reduce(p, stream=sh)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    per_step, phases, launches = [], {"init_gpu_ms": 0.0, "light_gpu_ms": 0.0, "heavy_gpu_ms": 0.0,
                                      "pairs_gpu_ms": 0.0}, 0
    light_launches = heavy_launches = 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.reduce(p, stream=sh)
        b.record(stream)
        torch.cuda.synchronize()
        per_step.append(a.elapsed_time(b))
        st = eng.stats()
        for k in phases:
            phases[k] += st[k]
        launches += st["launches"]
        light_launches += st["light_launches"]
        heavy_launches += st["heavy_launches"]
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    total_ms = sum(per_step)
    st = eng.stats()
    dev_pairs = eng.pairs()
    dev_ess = eng.essentials()
    eng.close()

    # ---------------------------------------------------------------- e2e
    if args.no_e2e:
        print(json.dumps({"metric": METRIC, "value": n * args.steps / (total_ms / 1000), "unit": UNIT,
                          "ms_per_step": total_ms / args.steps, "phases": {k: v / args.steps for k, v in phases.items()},
                          "profiling_run": True, "grid": GRID}), flush=True)
        return 0
    h_dims = torch.from_numpy(m.dims).pin_memory()
    h_colptr = torch.from_numpy(m.col_ptr).pin_memory()
    h_rows = torch.from_numpy(m.rows).pin_memory()
    out_pairs = torch.empty(2 * n, dtype=torch.int64).pin_memory()
    out_ess = torch.empty(n, dtype=torch.int64).pin_memory()
    hm = gen.BoundaryMatrix(h_dims.numpy(), h_colptr.numpy(), h_rows.numpy())
    e2 = Engine(local)
    for _ in range(max(1, args.warmup)):
        e2.load_csc(hm)
        e2.reduce(p)
        e2.pairs(out_pairs.numpy())
        e2.essentials(out_ess.numpy())
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e2.load_csc(hm)
        e2.reduce(p)
        pr = e2.pairs(out_pairs.numpy())
        es = e2.essentials(out_ess.numpy())
        e2e_ms.append(1000 * (time.perf_counter() - t0))
    h2d = 4 * n + 8 * (n + 1) + 4 * nnz
    d2h = 16 * len(pr) + 8 * len(es)
    ok_e2e = np.array_equal(pr, dev_pairs) and np.array_equal(es, dev_ess)
    e2.close()

    # --------------------------------------------------------- max over ranks
    tot = torch.tensor([total_ms, sum(e2e_ms)], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(tot, op=dist.ReduceOp.MAX)
    total_ms, e2e_total = float(tot[0]), float(tot[1])
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    value = world * n * args.steps / (total_ms / 1000)
    e2e_value = world * n * args.steps / (e2e_total / 1000)

    # roofline of the dominant device phase (algorithmic bytes per step)
    peaks, peak_kind = load_peaks()
    peak = float(peaks.get("hbm_gbs", 6650.0))
    cpu = None
    alg_add_bytes = None
    if not args.no_cpu_baseline:
        dt, r = oracle_run(m)
        alg_add_bytes = r.stats["add_bytes"]
        assert np.array_equal(dev_pairs, r.pairs) and np.array_equal(dev_ess, r.essential), "parity failure"
        cpu = {"value": n / dt, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"full workload ({n} columns), one run, single-threaded C++ restatement"}
    ph = {k: v / args.steps for k, v in phases.items()}
    init_bytes = 16 * nnz + 8 * n           # CSC read three times and written once, pivot + low tables
    # the heavy-tier launches overlap each other on side streams, so the
    # reduction's device time is the step's event time less the phases that
    # run alone on the main stream (init passes, pair extraction)
    red_ms = min(ph["light_gpu_ms"] + ph["heavy_gpu_ms"],
                 total_ms / args.steps - ph["init_gpu_ms"] - ph["pairs_gpu_ms"])
    candidates = {"init_passes": (ph["init_gpu_ms"], init_bytes),
                  "reduction": (red_ms, alg_add_bytes if alg_add_bytes is not None else None)}
    dom = max(candidates, key=lambda k: candidates[k][0])
    dom_ms, dom_bytes = candidates[dom]
    traffic = load_traffic().get(dom)
    roof = None
    if dom_bytes is not None and dom_ms > 0:
        achieved = dom_bytes / (dom_ms / 1000) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": dom, "peak_kind": peak_kind,
                "algorithmic_bytes_per_step": dom_bytes, "device_ms_per_step": dom_ms}
    init_roof = None
    if ph["init_gpu_ms"] > 0:
        ia = init_bytes / (ph["init_gpu_ms"] / 1000) / 1e9
        init_roof = {"bound": "hbm", "achieved": ia, "peak": peak, "unit": "GB/s", "frac": ia / peak,
                     "algorithmic_bytes_per_step": init_bytes, "device_ms_per_step": ph["init_gpu_ms"]}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": workload_config(n, nnz),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / args.steps, "pairs_match_device_run": bool(ok_e2e)},
            "gpu_launches": launches,
            "phases_ms_per_step": ph,
            "launches_per_step": {"total": launches // args.steps, "light": light_launches // args.steps,
                                  "heavy": heavy_launches // args.steps},
            "roofline": roof, "roofline_init": init_roof, "cpu_baseline": cpu, "clocks": clk,
            "stats": {k: st[k] for k in ("active_after_init", "apparent_pairs", "cleared_init", "highclear_cleared",
                                         "additions", "displaced", "ss_steps", "npairs", "nessential")}}
    if not args.no_extra:
        line["rips2000"] = leg_rips2000(args.steps)
        line["vr100k"] = leg_vr100k(args.steps, peak)
        line["batched"] = leg_batched(args.steps)
        line["served"] = leg_served()
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
