"""Benchmark: UMAP fit of 1,000,000 x 64 rows on B200, and the learned
transform surrogate against the plain transform (one JSON line).

Fit workload: the 50-component anisotropic Gaussian mixture (seed 11, means
~N(0, 5^2), per-dim std ~U(0.5, 2)), n_neighbors=15, exact kNN, spectral
init, 200 SGD epochs, 2-D output.  One step = one complete fit.

  value   seconds per fit with the rows already resident in HBM
          (umapb_fit_transform_device), device-timed with CUDA events;
  e2e     seconds per fit through the public API (Umap.fit_transform) from
          pinned host memory: host->device copy of the rows and
          device->host copy of the embedding inside the timed region.

Transform workload ("transform" object): fit 200,000 x 128 rows of a
20-component mixture (means ~N(0, 4^2), unit variance, seed 5), train the
surrogate (BF16 MLP 128-512-512-2, GELU, Adam 1e-3, batch 4096, 20 epochs),
then embed 1,000,000 query rows of the same mixture (seed 6) through the
surrogate with its gate and plain fallback, and through the plain transform
(kNN to the training rows + SGD refine); rows/s device-resident and end to
end from pinned host memory, trustworthiness@15 of both on 10,000 queries.

--impl reference times the CPU restatement of the reference's path (the
oracle) on all host cores.  Its exact kNN is timed directly on the full
matrix: each step searches a fixed block of 2,000 query rows against all
1,000,000 rows and scales by the query count only (the rows searched and their
memory traffic are those of the real fit).  The other stages (graph, spectral
init, SGD) are timed once per run by oracle fits of the first 25,000 and
50,000 rows; each stage is extrapolated to 1,000,000 rows along the power law
through its two times (the fitted exponent is reported).  Multi-GPU runs are
replicas: every rank fits its own copy and the step time is the maximum over
ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fit s @1M×64 TC vs FP32 kNN; transform rows/s MLP vs plain at equal trust@15"
N_ROWS, N_DIM, K, EPOCHS = 1_000_000, 64, 15, 200
PROFILED_FITS = 3  # instrumented fits after the timed region, for the stage breakdown
# DRAM bytes of one first-pass tc_knn_kernel launch on the headline fit (ncu, 1M x 64):
# 166.41 GB read + 13.57 GB written in 194.9 ms.
KNN_DRAM_BYTES_1M = 179_980_000_000
KNN_BLOCK = 2_000               # query rows of the CPU kNN block (against all N_ROWS)
CAL_SIZES = (25_000, 50_000)   # rows of the two CPU fits that time the other stages
T_FIT, T_QUERY, T_DIM = 200_000, 1_000_000, 128
T_SAMPLE = 2_000  # queries of the CPU transform baseline


def pool_reserved_gb(lib) -> float:
    """GB the device's stream-ordered memory pool holds mapped right now."""
    from umapers_b200 import _lib

    reserved, used = ctypes.c_int64(0), ctypes.c_int64(0)
    _lib.check(lib.umapb_pool_bytes(ctypes.byref(reserved), ctypes.byref(used)))
    return round(reserved.value / 1e9, 3)


def peaks() -> dict:
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        p = json.loads(path.read_text())
        return {"hbm_gbs": p["hbm_gbs"], "bf16_tflops": p["bf16_tflops"],
                "bf16_tflops_sustained": p.get("bf16_tflops_sustained", p["bf16_tflops"]),
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []
        self.others: set[str] = set()
        self.load: list[float] = []

    def _other_processes(self) -> None:
        """Compute processes other than this one on the device (they share its
        SMs), and the host's 1-minute load average (a loaded host delays the
        launches and synchronisations between stages)."""
        try:
            self.load.append(round(os.getloadavg()[0], 2))
        except OSError:
            pass
        try:
            out = subprocess.run(["nvidia-smi", f"--id={self.device}",
                                  "--query-compute-apps=pid", "--format=csv,noheader"],
                                 capture_output=True, text=True, timeout=10).stdout
        except (OSError, subprocess.TimeoutExpired):
            return
        me = str(os.getpid())
        self.others |= {ln.strip() for ln in out.splitlines() if ln.strip() and ln.strip() != me}

    def __enter__(self):
        self._other_processes()
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self._other_processes()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm),
                "other_processes": len(self.others), "host_load_1min": self.load,
                "host_cpus": os.cpu_count()}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_calibrate(x: np.ndarray, threads: int) -> dict:
    """Oracle fits of the first 25,000 and 50,000 rows: per stage other than
    the kNN (graph, spectral init, SGD) the two times, the exponent of the
    power law through them and its value at N_ROWS."""
    import math

    from oracle import oracle

    oracle.set_threads(threads)
    runs = {}
    for n in CAL_SIZES:
        _, runs[n] = oracle.fit_transform(x[:n].copy(), return_stats=True, n_neighbors=K,
                                          n_epochs=EPOCHS, use_approximate_knn=0)
    n1, n2 = CAL_SIZES
    out = {}
    for stage in ("graph_sec", "init_sec", "sgd_sec"):
        t1, t2 = float(runs[n1][stage]), float(runs[n2][stage])
        alpha = math.log(max(t2, 1e-9) / max(t1, 1e-9)) / math.log(n2 / n1)
        out[stage] = {"sec": [round(t1, 3), round(t2, 3)], "exponent": round(alpha, 3),
                      "at_n": round(t2 * (N_ROWS / n2) ** alpha, 2)}
    return out


def cpu_knn_block(x: np.ndarray, threads: int) -> float:
    """The oracle's exact kNN of the first KNN_BLOCK rows against all rows of
    x, scaled by the query count to all N_ROWS queries."""
    from oracle import oracle

    oracle.set_threads(threads)
    rows = np.arange(KNN_BLOCK, dtype=np.int64)
    t0 = time.perf_counter()
    oracle.exact_knn_rows(x, rows, K)
    return (time.perf_counter() - t0) * x.shape[0] / KNN_BLOCK


def cpu_sample_note(cal: dict) -> str:
    return (f"exact kNN: oracle search of {KNN_BLOCK} query rows against all {N_ROWS} rows "
            f"(the full 256 MB matrix), scaled by the query count; graph / spectral init / SGD: "
            f"oracle fits of {CAL_SIZES[0]} and {CAL_SIZES[1]} rows, each stage extrapolated "
            f"to {N_ROWS} rows along the power law through its two times "
            + json.dumps(cal))


def run_reference(args) -> None:
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from umapers_b200 import workloads

    threads = os.cpu_count() or 1
    x = workloads.anisotropic_mixture(N_ROWS, N_DIM, 50, seed=11)
    cal = cpu_calibrate(x, threads)
    rest = sum(v["at_n"] for v in cal.values())
    for _ in range(args.warmup):
        cpu_knn_block(x, threads)
    knn = [cpu_knn_block(x, threads) for _ in range(args.steps)]
    value = float(np.mean(knn)) + rest
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(value * 1000, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic: 50-component anisotropic Gaussian mixture, seed 11",
        "config": {"workload": f"fit {N_ROWS} x {N_DIM}, k={K}, exact kNN, spectral init, "
                               f"{EPOCHS} epochs, 2-D; each step: the exact kNN of a "
                               f"{KNN_BLOCK}-row query block against all {N_ROWS} rows",
                   "parallelism": "host cores",
                   "knn_sec_at_n": round(float(np.mean(knn)), 2),
                   "other_stages_sec_at_n": round(rest, 2)},
        "cpu_baseline": {
            "value": round(value, 3), "unit": "s", "cores": threads, "kind": "port",
            "sample": cpu_sample_note(cal),
        },
        "e2e": {"value": round(value, 3), "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_gpu(args) -> None:
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from umapers import Umap
    from umapers_b200 import _lib, diagnostics, workloads

    lib = _lib.load()
    x = workloads.anisotropic_mixture(N_ROWS, N_DIM, 50, seed=11)
    x_dev = torch.from_numpy(x).cuda()
    out_dev = torch.empty((N_ROWS, 2), dtype=torch.float32, device="cuda")

    model = Umap(n_neighbors=K, n_epochs=EPOCHS, ann_mode="exact", knn_backend=args.knn_backend)
    handle = model._core._handle
    timings = _lib.Timings()
    info = _lib.FitInfo()

    def device_step(profiled: bool = False) -> float:
        # timed steps make the call a user makes (no stage timings: with them the
        # engine waits for the device at every stage boundary and counts the
        # sampled edges in every epoch); profiled fits run after the timed region
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        _lib.check(lib.umapb_fit_transform_device(
            handle, x_dev.data_ptr(), N_ROWS, N_DIM, out_dev.data_ptr(),
            ctypes.byref(timings) if profiled else None, ctypes.byref(info) if profiled else None))
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / 1000.0

    x_pinned = torch.from_numpy(x).pin_memory().numpy()
    out_pinned = torch.empty((N_ROWS, 2), dtype=torch.float32).pin_memory().numpy()

    def e2e_step() -> float:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        model.fit_transform(x_pinned, out=out_pinned)
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / 1000.0

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    for _ in range(args.warmup):
        device_step()
    pool0 = pool_reserved_gb(lib)
    launches0 = lib.umapb_kernel_launches()
    barrier()
    sampler = ClockSampler(local)
    with sampler:
        dev_times, pool = [], []
        for _ in range(args.steps):
            dev_times.append(device_step())
            pool.append(pool_reserved_gb(lib))
        barrier()
        launches = (lib.umapb_kernel_launches() - launches0) // max(args.steps, 1)
        for _ in range(args.warmup):  # the host path's own warm-up (pinned staging, pool)
            e2e_step()
        e2e_times = [e2e_step() for _ in range(args.steps)]
        barrier()
    # profiled fits (stage timings, kernel event times, sample counts), untimed
    knn_sec, sgd_sec, stage, waits, sgd_kernel, prof_times = [], [], [], [], [], []
    for _ in range(PROFILED_FITS):
        prof_times.append(device_step(profiled=True))
        knn_sec.append(info.knn_kernel_sec)
        sgd_kernel.append(info.sgd_kernel_sec)
        waits.append((info.stage_wait_sec, info.stage_host_sec))
        sgd_sec.append(timings.optimize_sec)
        stage.append({f: getattr(timings, f) for f in _lib.TIMING_FIELDS})
    value = max_over_ranks(float(np.mean(dev_times)))
    e2e = max_over_ranks(float(np.mean(e2e_times)))
    emb = out_dev.cpu().numpy()
    transform = None if args.skip_transform else transform_leg(args, lib, local)
    extra = None if args.skip_transform else knn_legs(args, lib, x)

    if rank == 0:
        pk = peaks()
        n_fallback = int(info.knn_fallback_rows)
        backend = {1: "tensor", 2: "plain"}.get(info.knn_backend_used, "unknown")
        knn_t = float(np.mean(knn_sec))
        # the epochs' own event time (the optimize stage also holds the schedule's
        # setup and period sort)
        sgd_t = float(np.mean(sgd_kernel)) if min(sgd_kernel) > 0 else float(np.mean(sgd_sec))
        flops = 2.0 * N_ROWS * N_ROWS * N_DIM
        samples = float(info.sgd_edge_samples)
        # per sampled edge: head+tail read (16 B) and written (16 B), 5 negative
        # rows read (40 B), schedule state eps/next/next_neg (20 B); per edge
        # per epoch the epoch_of_next_sample read (4 B)
        sgd_bytes = samples * (16 + 16 + 40 + 20) + info.n_edges * EPOCHS * 4
        roof_knn = {
            "kernel": "exact kNN distance tiles + fused top-k (" + backend + ")",
            "bound": "tensor",
            "achieved": round(flops / knn_t / 1e12, 2),
            "peak": pk["bf16_tflops_sustained"],
            "unit": "TFLOP/s",
            "frac": round(flops / knn_t / 1e12 / pk["bf16_tflops_sustained"], 4),
            # DRAM bytes read + written by the first-pass launch at this size, from one ncu
            # capture (dram__bytes_read.sum + dram__bytes_write.sum, one pass, -c 1)
            "traffic": KNN_DRAM_BYTES_1M,
            "note": "algorithmic 2*N*N*D flop per fit; peak = sustained bf16 ("
                    + pk["source"] + "); traffic = DRAM bytes of the first-pass launch (ncu): "
                    "the 160 MB candidate operand streamed past L2 by each wave of query groups, "
                    "and the lists",
        }
        roof_sgd = {
            "kernel": "sgd_epoch_2d (200 launches)",
            "bound": "hbm",
            "achieved": round(sgd_bytes / sgd_t / 1e9, 1),
            "peak": pk["hbm_gbs"],
            "unit": "GB/s",
            "frac": round(sgd_bytes / sgd_t / 1e9 / pk["hbm_gbs"], 4),
            "traffic": None,
            "note": "algorithmic bytes of the sampled edges over the 200 epoch launches' CUDA-event "
                    "time; peak = measured HBM copy (" + pk["source"] + ")",
        }
        # spectral init: 256 products of the normalised adjacency with an
        # N x 20 FP32 block (row_ptr/tails/weights read, 80 B gathered per
        # edge, the block read and written) and a CholQR2 (4 passes over the
        # block) after every 4th product
        init_t = float(np.mean([st["init_sec"] for st in stage]))
        spec_bytes = 256 * (info.n_edges * (4 + 4 + 80) + N_ROWS * 80 * 2) + 64 * N_ROWS * 80 * 4
        roof_spec = {
            "kernel": "spmm_kernel + CholQR2 (spectral init stage)",
            "bound": "hbm",
            "achieved": round(spec_bytes / init_t / 1e9, 1),
            "peak": pk["hbm_gbs"],
            "unit": "GB/s",
            "frac": round(spec_bytes / init_t / 1e9 / pk["hbm_gbs"], 4),
            "traffic": None,
            "note": "algorithmic bytes of 256 block products and 64 CholQR2 over the whole "
                    "init stage time; peak = measured HBM copy (" + pk["source"] + ")",
        }
        dominant = roof_knn if knn_t >= sgd_t else roof_sgd
        q = diagnostics.quality(x, emb, sample=10_000, seed=11)
        line = {
            "metric": METRIC,
            "value": round(value, 4),
            "unit": "s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(value * 1000, 2),
            "higher_is_better": False,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "fp16->f32 (kNN tiles), f32" if backend == "tensor" else "f32",
            "data": "synthetic: 50-component anisotropic Gaussian mixture, seed 11",
            "config": {
                "workload": f"fit {N_ROWS} x {N_DIM}, k={K}, exact kNN ({backend}), spectral "
                            f"init, {EPOCHS} epochs, 2-D",
                "parallelism": f"replicas x{world}",
                "l2": "inputs (256 MB) larger than L2 (126 MB); no flush",
                "knn_fallback_rows": n_fallback,
                "graph_components": int(info.n_components_graph),
                "n_edges": int(info.n_edges),
            },
            "e2e": {"value": round(e2e, 4), "unit": "s",
                    "h2d_bytes_per_step": int(x.nbytes), "d2h_bytes_per_step": int(emb.nbytes)},
            "gpu_launches": int(launches),
            "roofline": dominant,
            "rooflines": {"knn": roof_knn, "sgd": roof_sgd, "spectral": roof_spec},
            "stages_sec": {k: round(float(np.mean([s[k] for s in stage])), 4)
                           for k in ("knn_sec", "smooth_knn_sec", "membership_sec", "symmetrize_sec",
                                     "prune_sec", "init_sec",
                                     "optimize_sec", "total_sec")},
            "quality": {k: round(v, 4) for k, v in q.items()},
            "clocks": sampler.summary(),
            # per timed step: its time, and the memory pool's mapped size after it
            "step_sec": [round(t, 4) for t in dev_times],
            "step_sec_median": round(float(np.median(dev_times)), 4),
            # the profiled fits after the timed region (stages_sec, the rooflines and
            # the step_* lists below come from them): their time with instrumentation
            "profiled_fit_sec": [round(t, 4) for t in prof_times],
            "step_stages_sec": [[round(st[k], 4) for k in ("knn_sec", "membership_sec",
                                                             "symmetrize_sec", "prune_sec",
                                                             "init_sec", "optimize_sec")]
                                for st in stage],
            # the tensor kNN kernel alone, CUDA events on the engine's stream: a
            # step whose kNN stage is long while this stays flat lost its time
            # outside the kernel
            "step_knn_kernel_sec": [round(t, 4) for t in knn_sec],
            # the 200 layout epochs alone (CUDA events around the epoch loop)
            "step_sgd_kernel_sec": [round(t, 4) for t in sgd_kernel],
            # per step: host time waiting for the device at the stage
            # boundaries, and the rest (host work and launches); a slow step
            # whose wait grew lost its time on the device
            "step_wait_host_sec": [[round(a, 4), round(b, 4)] for a, b in waits],
            "pool_reserved_gb": [pool0] + pool,
        }
        if transform is not None:
            line["transform"] = transform
        if extra is not None:
            line["knn_configs"] = extra
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            cal = cpu_calibrate(x, threads)
            v = cpu_knn_block(x, threads) + sum(c["at_n"] for c in cal.values())
            line["cpu_baseline"] = {
                "value": round(v, 2), "unit": "s", "cores": threads, "kind": "port",
                "sample": cpu_sample_note(cal),
            }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def sparse_leg(args, lib) -> dict:
    """CSR input: 200,000 x 2,000 rows at about 20 stored values per row,
    LogNormal(0, 1) values, cosine, k = 30.  The exact sparse kNN through the
    host API (upload, index build, kernel, download), a complete fit from the
    CSR rows, bit-exact agreement with the oracle on 200 sampled rows, and the
    oracle's time for those rows on all host cores."""
    from oracle import oracle
    from umapers import Umap
    from umapers_b200 import _lib, workloads

    xs = workloads.sparse_lognormal_csr(200_000, 2000, 20, seed=3)
    n, d, k = xs.shape[0], xs.shape[1], 30
    ip = np.ascontiguousarray(xs.indptr, np.int64)
    ix = np.ascontiguousarray(xs.indices, np.int64)
    dv = np.ascontiguousarray(xs.data, np.float32)
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    t_knn = float("inf")
    for _ in range(2):
        t0 = time.perf_counter()
        _lib.check(lib.umapb_knn_csr(ip.ctypes.data, ix.ctypes.data, dv.ctypes.data, n, d, k, 2,
                                     idx.ctypes.data, dist.ctypes.data))
        t_knn = min(t_knn, time.perf_counter() - t0)
    m = Umap(n_neighbors=k, metric="cosine", n_epochs=EPOCHS, random_seed=3)
    m.fit_transform(xs)
    t0 = time.perf_counter()
    m.fit_transform(xs)
    t_fit = time.perf_counter() - t0
    # NN-descent on the CSR rows (10 iterations, 30 candidates, as configured)
    # and a fit that takes it (an explicit approximate request)
    ni = np.empty((n, k), np.int64)
    nd = np.empty((n, k), np.float32)
    ran, n_eval, nd_ksec = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_double(0.0)
    t_nd = float("inf")
    for _ in range(2):
        t0 = time.perf_counter()
        _lib.check(lib.umapb_nndescent_csr(ip.ctypes.data, ix.ctypes.data, dv.ctypes.data, n, d,
                                           k, 2, 30, 10, 3 ^ 0xC0FEFEED1234ABCD, ni.ctypes.data,
                                           nd.ctypes.data, ctypes.byref(ran),
                                           ctypes.byref(n_eval), ctypes.byref(nd_ksec)))
        t_nd = min(t_nd, time.perf_counter() - t0)
    samp = np.random.default_rng(30).choice(n, 2000, replace=False)
    nd_recall = float(np.mean([len(set(ni[r]) & set(idx[r])) / k for r in samp]))
    ma = Umap(n_neighbors=k, metric="cosine", n_epochs=EPOCHS, random_seed=3,
              ann_mode="approximate", approx_knn_candidates=30, approx_knn_iters=10)
    ma.fit_transform(xs)
    t0 = time.perf_counter()
    ma.fit_transform(xs)
    t_fit_nd = time.perf_counter() - t0
    rows = np.random.default_rng(3).choice(n, 200, replace=False)
    oracle.set_threads(os.cpu_count() or 1)
    t0 = time.perf_counter()
    oi, od = oracle.csr_knn_rows(xs, rows, k, "cosine")
    t_cpu = time.perf_counter() - t0
    exact = bool(np.array_equal(oi, idx[rows]) and
                 np.array_equal(od.view(np.uint32), dist[rows].view(np.uint32)))
    return {"knn_s": round(t_knn, 4), "fit_s": round(t_fit, 4), "nnz": int(xs.nnz),
            "nndescent": {"knn_s": round(t_nd, 4), "kernel_s": round(nd_ksec.value, 4),
                          "iters": int(ran.value), "candidates_evaluated": int(n_eval.value),
                          "recall_at_30_vs_exact": round(nd_recall, 4),
                          "fit_s": round(t_fit_nd, 4),
                          "note": "umapb_nndescent_csr, 30 candidates, 10 iterations; recall "
                                  "against the exact sparse kNN on 2,000 sampled rows; the fit "
                                  "is Umap(ann_mode='approximate') on the CSR rows"},
            "bit_exact_on_sample": exact,
            "cpu_knn_s_extrapolated": round(t_cpu * n / rows.shape[0], 1),
            "cpu_cores": os.cpu_count(),
            "note": "exact sparse kNN and NN-descent on CSR rows (the reference has no sparse "
                    "NN-descent and rejects densMAP for sparse input); host API, 200 epochs; the "
                    "CPU figure is the oracle on 200 rows scaled to all rows"}


def knn_legs(args, lib, x: np.ndarray) -> dict:
    """The exact-kNN precision path at 20,000 x 192 (tensor vs plain, same
    result) and NN-descent (10 iterations, 30 candidates) at the fit's size."""
    from umapers import Umap
    from umapers_b200 import _lib, diagnostics, workloads

    out = {}
    xp = workloads.isotropic_mixture(20_000, 192, 10, 4.0, seed=7)
    res, times = {}, {}
    for backend, code in (("tensor", 1), ("plain", 2)):
        idx = np.empty((xp.shape[0], K), np.int64)
        dist = np.empty((xp.shape[0], K), np.float32)
        fb = ctypes.c_int64(0)
        best = float("inf")
        for _ in range(max(args.warmup, 1) + 2):
            t0 = time.perf_counter()
            _lib.check(lib.umapb_knn_exact(xp.ctypes.data, xp.shape[0], 192, K, 0, code,
                                           idx.ctypes.data, dist.ctypes.data, ctypes.byref(fb)))
            best = min(best, time.perf_counter() - t0)
        res[backend], times[backend] = (idx, dist, fb.value), best
    fits = {}
    for backend in ("tensor", "plain"):
        m = Umap(n_neighbors=K, n_epochs=EPOCHS, ann_mode="exact", knn_backend=backend)
        m.fit_transform(xp)
        t0 = time.perf_counter()
        emb = m.fit_transform(xp)
        fits[backend] = (time.perf_counter() - t0, diagnostics.quality(xp, emb, sample=None))
    out["precision_20000x192"] = {
        "knn_s_tensor": round(times["tensor"], 4), "knn_s_plain": round(times["plain"], 4),
        "identical_indices": bool(np.array_equal(res["tensor"][0], res["plain"][0])),
        "identical_distances": bool(np.array_equal(res["tensor"][1], res["plain"][1])),
        "fallback_rows": int(res["tensor"][2]),
        "fit_s_tensor": round(fits["tensor"][0], 4), "fit_s_plain": round(fits["plain"][0], 4),
        "trust15_tensor": round(fits["tensor"][1]["trustworthiness"], 4),
        "trust15_plain": round(fits["plain"][1]["trustworthiness"], 4),
        "note": "host API, 10-component mixture (means ~N(0, 4^2)), seed 7, k=15",
    }
    n = x.shape[0]
    ni = np.empty((n, K), np.int64)
    nd = np.empty((n, K), np.float32)
    ran = ctypes.c_int64(0)
    n_eval = ctypes.c_int64(0)
    nd_ksec = ctypes.c_double(0.0)
    seed = 42 ^ 0xC0FEFEED1234ABCD
    t_nd, k_nd = float("inf"), float("inf")
    for _ in range(2):
        t0 = time.perf_counter()
        _lib.check(lib.umapb_nndescent(x.ctypes.data, n, x.shape[1], K, 0, 30, 10, seed,
                                       ni.ctypes.data, nd.ctypes.data, ctypes.byref(ran),
                                       ctypes.byref(n_eval), ctypes.byref(nd_ksec)))
        t_nd = min(t_nd, time.perf_counter() - t0)
        k_nd = min(k_nd, nd_ksec.value)
    # gathered candidate rows (D x 4 B each) plus, per list pass, the k-entry
    # lists read and written (index + distance, 8 B each)
    nd_bytes = n_eval.value * x.shape[1] * 4 + (ran.value + 1) * n * K * 8 * 2
    ei = np.empty((n, K), np.int64)
    ed = np.empty((n, K), np.float32)
    _lib.check(lib.umapb_knn_exact(x.ctypes.data, n, x.shape[1], K, 0, 1, ei.ctypes.data,
                                   ed.ctypes.data, None))
    rows = np.random.default_rng(3).choice(n, 2000, replace=False)
    recall = float(np.mean([len(set(ni[r]) & set(ei[r])) / K for r in rows]))
    # the fit's ratio to the plain FP32 CUDA-core path: its exact kNN (the same
    # sets as the tensor path's, checked in full) and one fit on it
    pi = np.empty((n, K), np.int64)
    pd = np.empty((n, K), np.float32)
    t0 = time.perf_counter()
    _lib.check(lib.umapb_knn_exact(x.ctypes.data, n, x.shape[1], K, 0, 2, pi.ctypes.data,
                                   pd.ctypes.data, None))
    t_plain_knn = time.perf_counter() - t0
    mp = Umap(n_neighbors=K, n_epochs=EPOCHS, ann_mode="exact", knn_backend="plain")
    t0 = time.perf_counter()
    emb_p = mp.fit_transform(x)
    t_plain_fit = time.perf_counter() - t0
    qp = diagnostics.quality(x, emb_p, sample=10_000, seed=11)
    out["plain_1m_x64"] = {
        "knn_s_plain": round(t_plain_knn, 3), "fit_s_plain": round(t_plain_fit, 3),
        "identical_indices": bool(np.array_equal(pi, ei)),
        "identical_distances": bool(np.array_equal(pd, ed)),
        "trust15_plain": round(qp["trustworthiness"], 4),
        "note": "host API from a host array (the 256 MB upload inside), one fit; compare with "
                "the headline's e2e and quality"}
    out["sparse_cosine_200000x2000"] = sparse_leg(args, lib)
    pk = peaks()
    out["nndescent_1m_x64"] = {
        "knn_s": round(t_nd, 4), "kernel_s": round(k_nd, 4), "iters": int(ran.value),
        "recall_at_15": round(recall, 4), "candidates_evaluated": int(n_eval.value),
        "roofline": {"kernel": "nd_init_kernel + nd_iter_kernel", "bound": "hbm",
                     "achieved": round(nd_bytes / k_nd / 1e9, 1), "peak": pk["hbm_gbs"],
                     "unit": "GB/s", "frac": round(nd_bytes / k_nd / 1e9 / pk["hbm_gbs"], 4),
                     "traffic": None,
                     "note": "algorithmic bytes: evaluated candidates x D x 4 B + k-lists read "
                             "and written per pass, over the kernels' CUDA-event time"},
        "note": "host API (includes the 256 MB upload), max_candidates=30, n_iters=10; recall "
                "against the exact neighbours on 2,000 rows"}
    return out


def transform_leg(args, lib, device: int) -> dict:
    """Surrogate transform against the plain transform on 1M queries."""
    import torch

    from umapers import Umap
    from umapers_b200 import _lib, diagnostics, workloads

    fit, query = workloads.transform_mixture(T_FIT, T_QUERY, T_DIM)
    model = Umap(n_neighbors=K, random_seed=5, ann_mode="exact")
    model.fit(fit)
    t0 = time.perf_counter()
    info = model.fit_surrogate()
    train_wall = time.perf_counter() - t0
    handle = model._core._handle
    q_dev = torch.from_numpy(query).cuda()
    out_sur = torch.empty((T_QUERY, 2), dtype=torch.float32, device="cuda")
    out_plain = torch.empty_like(out_sur)
    q_pin_t = torch.from_numpy(query).pin_memory()
    q_pinned = q_pin_t.numpy()
    h_out = torch.empty((T_QUERY, 2), dtype=torch.float32).pin_memory().numpy()
    n_fb = ctypes.c_int64(0)

    def dev(surrogate: bool) -> float:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        if surrogate:
            _lib.check(lib.umapb_surrogate_transform_device(
                handle, q_dev.data_ptr(), T_QUERY, T_DIM, 1, out_sur.data_ptr(), None,
                ctypes.byref(n_fb)))
        else:
            _lib.check(lib.umapb_transform_device(handle, q_dev.data_ptr(), T_QUERY, T_DIM,
                                                  out_plain.data_ptr()))
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / 1000.0

    def e2e(surrogate: bool) -> float:
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        model.transform(q_pinned, out=h_out, method="surrogate" if surrogate else "plain")
        stop.record()
        torch.cuda.synchronize()
        return start.elapsed_time(stop) / 1000.0

    for _ in range(args.warmup):
        dev(True)
        dev(False)
        e2e(True)
        e2e(False)
    launches0 = lib.umapb_kernel_launches()
    sampler = ClockSampler(device)
    with sampler:
        t_sur = [dev(True) for _ in range(args.steps)]
        sur_launches = (lib.umapb_kernel_launches() - launches0) // max(args.steps, 1)
        t_plain = [dev(False) for _ in range(args.steps)]
        e_sur = [e2e(True) for _ in range(args.steps)]
        e_plain = [e2e(False) for _ in range(args.steps)]
    # the upload alone: the pinned query block copied to the device (bounds e2e)
    h2d = []
    for _ in range(3):
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        start.record()
        q_dev.copy_(q_pin_t, non_blocking=True)
        stop.record()
        torch.cuda.synchronize()
        h2d.append(start.elapsed_time(stop) / 1000.0)
    ts, tp = float(np.mean(t_sur)), float(np.mean(t_plain))
    es, ep = float(np.mean(e_sur)), float(np.mean(e_plain))
    sur, plain = out_sur.cpu().numpy(), out_plain.cpu().numpy()
    q_s = diagnostics.quality(query, sur, sample=10_000, seed=6)
    q_p = diagnostics.quality(query, plain, sample=10_000, seed=6)
    # per query row: standardise (read 128 f32), two hidden GEMMs, the head
    # and the nearest-anchor GEMM of the gate
    H, C = 512, int(info["n_anchors"])
    flop_row = 2.0 * (T_DIM * H + H * H + H * 2 + T_DIM * C)
    pk = peaks()
    achieved = flop_row * T_QUERY / ts / 1e12
    out = {
        "metric": "transform rows/s, 1,000,000 queries (surrogate with gate + plain fallback)",
        "value": round(T_QUERY / ts, 1),
        "unit": "rows/s",
        "higher_is_better": True,
        "e2e": {"value": round(T_QUERY / es, 1), "unit": "rows/s",
                "h2d_bytes_per_step": int(query.nbytes), "d2h_bytes_per_step": int(sur.nbytes)},
        "plain": {"value": round(T_QUERY / tp, 1), "e2e": round(T_QUERY / ep, 1),
                  "unit": "rows/s"},
        "speedup_device": round(tp / ts, 2),
        "speedup_e2e": round(ep / es, 2),
        "fallback_rows": int(n_fb.value),
        "step_sec": {"surrogate": [round(v, 5) for v in t_sur],
                     "plain": [round(v, 5) for v in t_plain],
                     "surrogate_e2e": [round(v, 5) for v in e_sur],
                     "plain_e2e": [round(v, 5) for v in e_plain]},
        "h2d_upload": {"bytes": int(q_pin_t.numel() * 4), "sec": [round(v, 5) for v in h2d],
                       "gbs": round(q_pin_t.numel() * 4 / float(np.median(h2d)) / 1e9, 1)},
        "quality": {"surrogate_trust15": round(q_s["trustworthiness"], 4),
                    "plain_trust15": round(q_p["trustworthiness"], 4),
                    "surrogate_knn_pres": round(q_s["knn_preservation"], 4),
                    "plain_knn_pres": round(q_p["knn_preservation"], 4)},
        "training": {"wall_s": round(train_wall, 3),
                     **{k: (round(v, 4) if isinstance(v, float) else v) for k, v in info.items()}},
        "gpu_launches": int(sur_launches),
        "roofline": {
            "kernel": "surrogate inference (standardise, 3 tcgen05 GEMMs, head, gate)",
            "bound": "tensor", "achieved": round(achieved, 2), "peak": pk["bf16_tflops"],
            "unit": "TFLOP/s", "frac": round(achieved / pk["bf16_tflops"], 4), "traffic": None,
            "note": f"{flop_row:.0f} flop per row; peak = burst bf16 ({pk['source']})"},
        # the same call against HBM: per query the FP32 row read (T_DIM x 4 B), the 2-D output
        # written (8 B) and its gate flag (1 B), over the device-resident call's time
        "roofline_hbm": {
            "kernel": "surrogate transform (whole device-resident call)", "bound": "hbm",
            "achieved": round(T_QUERY * (T_DIM * 4 + 8 + 1) / ts / 1e9, 1),
            "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": round(T_QUERY * (T_DIM * 4 + 8 + 1) / ts / 1e9 / pk["hbm_gbs"], 4),
            "traffic": None,
            "note": f"{T_DIM * 4 + 9} B per query; peak = measured HBM copy ({pk['source']})"},
        "config": {"workload": f"fit {T_FIT} x {T_DIM} (20-component mixture, seed 5), "
                               f"{T_QUERY} queries (seed 6), k={K}, 2-D",
                   "surrogate": "MLP 128-512-512-2 GELU, BF16 GEMMs / FP32 master, Adam 1e-3, "
                                "batch 4096, 20 epochs"},
        "clocks": sampler.summary(),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle

        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        a, b = model._core.ab_params
        t0 = time.perf_counter()
        oracle.transform(fit, model.embedding_, query[:T_SAMPLE], a, b, n_neighbors=K,
                         n_epochs=30, random_seed=5)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {
            "value": round(T_SAMPLE / dt, 1), "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"oracle plain transform of {T_SAMPLE} of the queries (30 epochs, the "
                      f"count a 1M-row request uses) against the {T_FIT}-row fit"}
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--knn-backend", default="auto", choices=["auto", "tensor", "plain"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-transform", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
