"""Benchmark of the graph-diffusion hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full diffusion of the dense block):
  500,000 cells from the seeded 10-component 50-D mixture, k=30 kNN (FP32 on
  the device; a harness input, not timed), Gaussian adaptive-sigma weights,
  (W+W^T)/2, row-normalised CSR; X0 500,000 x 64 FP32 ~ N(0,1); 16 diffusion
  steps. Inputs are resident in HBM when the timed region starts and the L2 is
  flushed (256 MiB write) before every timed step.

Reported (one JSON line on rank 0):
  value      algorithmic HBM GB/s of the FP32 plain diffusion, whole job
             (B_step = nnz*(4+4) + (n+1)*4 + 2*n*F*4 bytes per SpMM step)
  forms      BF16 / FP16 storage forms (GB/s, speed-up vs FP32, error vs FP64)
  e2e        the same metric through scl_diffusion_diffuse_matrix with host
             buffers (pinned), including all host<->device copies
  roofline   dominant kernel (SpMM) vs the measured HBM copy bandwidth
  cpu_baseline  scl-core's own CPU diffuse_matrix (oracle/_ref) on the host

--impl reference times scl-core's CPU implementation of the same workload on
the host cores and prints the same line with "impl": "reference".
Multi-GPU (torchrun): every rank runs an independent replica (weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "scl-core_b200"))

N_CELLS, K_NN, N_FEAT, N_STEPS = 500_000, 30, 64, 16
METRIC = "diffusion HBM GB/s & fwd+bwd ms (500k cells,k=30,64 cols) BF16 vs FP32 plain"


def step_bytes(n, nnz, F, s_idx=4, s_val=4, s_x=4):
    return nnz * (s_idx + s_val) + (n + 1) * 4 + 2 * n * F * s_x


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---- clocks sampling -----------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int, uuid: str = None):
        self.gpu = gpu_index
        self.uuid = uuid
        self.samples = []
        self.source = None
        self._stop = threading.Event()
        self._t = None

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        if self.uuid:
            try:
                return pynvml, pynvml.nvmlDeviceGetHandleByUUID(self.uuid)
            except Exception:
                pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _run_nvml(self, nv, h):
        """Read-only NVML queries every 10 ms (the same fields nvidia-smi prints)."""
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.samples.append([str(self.gpu), str(sm), str(mx), f"{pw:.1f}", hex(r)]
                                    + ["Active" if r & b else "Not Active" for b in bits])
            except Exception:
                pass
            self._stop.wait(0.01)

    def _run(self):
        try:
            nv, h = self._nvml_handle()
            self.source = "nvml 10 ms"
            return self._run_nvml(nv, h)
        except Exception:
            self.source = "nvidia-smi 200 ms"
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples), "source": self.source}


def gpu_uuid(torch, device):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(device).uuid)
    except Exception:
        return None


# ---- inputs ------------------------------------------------------------------------
def synthetic_module():
    """scl-core_b200/scl/synthetic.py loaded on its own (NumPy / torch only), so
    that the reference arm never imports this repository's package or loads
    its libraries."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("scl_synthetic_inputs", ROOT / "scl-core_b200" / "scl" / "synthetic.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def native_knn(scl, pts, k):
    """kNN of the rows of `pts` through this library's scl_knn (the drop-in
    neighbors ABI, host buffers): (idx int32 [n, k], dist float32 [n, k]) as
    NumPy arrays, and the wall time in seconds."""
    pts = np.ascontiguousarray(pts, dtype=np.float32)
    n, d = pts.shape
    ip = np.arange(0, (n + 1) * d, d, dtype=np.int64)
    if ip[-1] < 2**31:
        ip = ip.astype(np.int32)
    m = scl.CsrMatrix.wrap(ip, np.tile(np.arange(d, dtype=np.int32), n), pts.reshape(-1), (n, d))
    t0 = time.perf_counter()
    norms = scl.neighbors.compute_norms(m)
    idx, dist = scl.neighbors.knn(m, k, norms)
    dt = time.perf_counter() - t0
    del m
    return idx.astype(np.int32, copy=False), dist.astype(np.float32, copy=False), dt


def native_graph(torch, scl, n, k, seed, stream=None, normalize=True):
    """Seeded mixture -> scl_knn -> Gaussian weights and (W+W^T)/2 -> row
    normalisation, all through this library: (GpuGraph, info dict)."""
    syn = synthetic_module()
    pts = syn.mixture(n, seed=seed)
    ki, kd, t_knn = native_knn(scl, pts, k)
    del pts
    s = stream if stream is not None else torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kit, kdt = torch.from_numpy(ki).cuda(), torch.from_numpy(kd).cuda()
    a.record(s)
    g = scl.gpu.GpuGraph.from_knn(kit, kdt, stream=s)
    if normalize:
        g.normalize(symmetric=False, stream=s)
    b.record(s)
    b.synchronize()
    return g, {"knn_s": round(t_knn, 3), "build_ms": round(a.elapsed_time(b), 3)}


def flush_l2(torch, buf):
    buf.add_(1.0)


def timed_calls(torch, fn, steps, warmup, flush_buf, stream):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush_l2(torch, flush_buf)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        times.append(a.elapsed_time(b))
    return times


# ---- CPU baseline (scl-core's own implementation) ---------------------------------------
def reference_diffusion(R, ip, ind, P, X0, steps, reps=1):
    """scl-core's own diffuse_matrix (oracle/_ref, all host threads) on the given
    graph and block: (result of the last rep, seconds per rep list)."""
    out, ts = None, []
    for _ in range(reps):
        t0 = time.perf_counter()
        out = R.diffuse_matrix(ip, ind, P, X0, steps)
        ts.append(time.perf_counter() - t0)
    return out, ts


def host_cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def workload_config(world):
    """The config dict both arms print (the workload's definition, not its
    generated graph: nnz is reported beside it)."""
    return {"workload": "diffusion 500k cells k=30 64 cols 16 steps (FP32 plain, row-normalised)",
            "cells": N_CELLS, "k": K_NN, "features": N_FEAT, "diffusion_steps": N_STEPS,
            "graph": "seeded 10-component 50-D mixture (seed 0), Gaussian adaptive-sigma weights, (W+W^T)/2",
            "x0": "N(0,1) FP32, torch generator seed 1 + rank",
            "l2": "GPU arm: flushed (256 MiB write) before every timed step",
            "parallelism": f"replicas x{world}"}


def profiled_traffic(name):
    """DRAM bytes per launch recorded from an ncu capture in profiles/<name>.md
    (`dram_bytes_per_launch: N`), or None."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return int(line.split(":", 1)[1])
    return None


def event_ms(torch, fn, stream, reps, warmup, flush_buf=None):
    """Median CUDA-event time of fn() on `stream` (L2 flushed before each rep when flush_buf is given)."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        if flush_buf is not None:
            flush_l2(torch, flush_buf)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def bench_backward(torch, scl, device, stream, reps, warmup, flush):
    """Differentiation form: 200,000 cells, k=30, X0 200,000 x 32 FP32, 8 steps,
    L = sum((X_8 - Y)^2), checkpoint every 4. Forward = the checkpointed
    diffusion; forward+backward adds the loss gradient and the backward pass
    (dL/dX0 and dL/dW through the row normalisation)."""
    import scl.autograd  # noqa: F401

    n, k, F, T, every = 200_000, 30, 32, 8, 4
    g, _ = native_graph(torch, scl, n, k, seed=0, stream=stream)
    gen = torch.Generator(device=device).manual_seed(7)
    X0 = torch.randn((n, F), device=device, generator=gen)
    Yt = torch.randn((n, F), device=device, generator=gen)
    ck = torch.empty((g.checkpoint_slots(T, every), n, F), device=device)
    XT = torch.empty_like(X0)

    def fwd():
        g.diffuse_checkpointed(X0, T, every, out=XT, checkpoints=ck, stream=stream)

    def fwd_bwd():
        g.diffuse_checkpointed(X0, T, every, out=XT, checkpoints=ck, stream=stream)
        dY = 2.0 * (XT - Yt)
        g.diffuse_backward(X0, ck, dY, T, every, need_dW=True, stream=stream)

    t_f = event_ms(torch, fwd, stream, reps, warmup, flush)
    t_fb = event_ms(torch, fwd_bwd, stream, reps, warmup, flush)
    nnz = g.shape[2]
    g.close()
    return {"workload": "200k cells k=30 32 cols 8 steps, checkpoint every 4, L=sum((X_8-Y)^2), dL/dX0 + dL/dW",
            "cells": n, "nnz": nnz, "fwd_ms": round(t_f, 4), "fwd_bwd_ms": round(t_fb, 4),
            "fwd_bwd_over_fwd": round(t_fb / t_f, 3)}


def bench_impute(torch, scl, device, reps, warmup, with_reference=True):
    """MAGIC imputation through the drop-in C ABI (scl_impute_magic, host
    buffers in and out, pinned): 100,000 cells, Gaussian kNN affinity (k=15,
    (W+W^T)/2, not normalised: MAGIC normalises its rows itself), a sparse
    expression matrix of 100,000 x 1,000 at 5 % density (seeded, values in
    [0, 1)), t = 3. The same call on scl-core's own CPU implementation
    (oracle/_ref, all host threads) is timed once beside it and its output
    compared with the GPU's bit for bit."""
    import ctypes

    import scipy.sparse as sp

    n, k, G, t = 100_000, 15, 1000, 3
    g, _ = native_graph(torch, scl, n, k, seed=11, normalize=False)
    ip, ind, W = g.export()
    g.close()
    Xs = sp.random(n, G, density=0.05, random_state=12, format="csr", dtype=np.float32)
    Xs.sort_indices()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    x_arr = (pin(Xs.indptr.astype(np.int32)), pin(Xs.indices.astype(np.int32)), pin(Xs.data))
    t_arr = (pin(ip.astype(np.int32)), pin(ind.astype(np.int32)), pin(W.astype(np.float32)))
    M = scl.CsrMatrix.wrap(*x_arr, (n, G))
    A = scl.CsrMatrix.wrap(*t_arr, (n, n))
    out = torch.empty((n, G), dtype=torch.float32).pin_memory().numpy()
    lib = M.lib
    P = out.ctypes.data_as(ctypes.POINTER(lib.real_type))
    ts = []
    for it in range(warmup + reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = lib.scl_impute_magic(M.handle, A.handle, n, G, t, P)
        dt = time.perf_counter() - t0
        if rc != 0:
            raise RuntimeError(f"scl_impute_magic failed: {rc}")
        if it >= warmup:
            ts.append(dt)
    st = scl.diffusion.last_stats(lib)
    res = {"workload": "MAGIC imputation, 100k cells, kNN affinity k=15, 1,000 genes at 5% density, t=3, "
                       "host buffers through scl_impute_magic",
           "cells": n, "genes": G, "expr_nnz": int(Xs.nnz), "graph_nnz": int(ind.size), "t": t,
           "e2e_ms": round(1e3 * float(np.median(ts)), 3), "device_ms": round(float(st["device_ms"]), 3),
           "h2d_bytes": int(st["h2d_bytes"]), "d2h_bytes": int(st["d2h_bytes"])}
    if with_reference:
        try:
            from oracle import ref

            R = ref.RefLib("f32_i32")
            t0 = time.perf_counter()
            want = R.impute("magic", (Xs.indptr, Xs.indices, Xs.data), (n, G), True, (ip, ind, W), n, G, t)
            rdt = time.perf_counter() - t0
            res.update({"reference_cpu_ms": round(1e3 * rdt, 1), "reference_cores": os.cpu_count(),
                        "reference_lib": R.path.name, "e2e_speedup_vs_reference": round(rdt / float(np.median(ts)), 2),
                        "bit_identical_to_reference": bool(np.array_equal(want.view(np.uint32),
                                                                          out.view(np.uint32)))})
        except Exception as e:  # informational; never fail the run on it
            res["reference_cpu_ms"] = f"unavailable: {e}"
    del M, A
    return res


def bench_knn(torch, scl, reps, warmup, with_reference=True):
    """Brute-force kNN through the drop-in C ABI (scl_knn, host buffers): the
    seeded 10-component 50-D mixture at 50,000 cells, k = 30 (the graph
    build's first step), with norms from scl_neighbors_compute_norms. Beside
    it, scl-core's own scl_knn (oracle/_ref, all host threads) on the first
    10,000 cells, and the GPU on the same 10,000 cells with the reference's
    norms, whose output must equal the reference's bit for bit."""
    def wrap_dense(P):
        n, d = P.shape
        ip = np.arange(0, (n + 1) * d, d, dtype=np.int32)
        ind = np.tile(np.arange(d, dtype=np.int32), n)
        return scl.CsrMatrix.wrap(ip, ind, np.ascontiguousarray(P.reshape(-1)), (n, d)), (ip, ind)

    n, k = 50_000, 30
    pts = scl.synthetic.mixture(n, seed=21).astype(np.float32)
    m, _ = wrap_dense(pts)
    norms = scl.neighbors.compute_norms(m)
    ts = []
    for it in range(warmup + reps):
        t0 = time.perf_counter()
        gi, gd = scl.neighbors.knn(m, k, norms)
        if it >= warmup:
            ts.append(time.perf_counter() - t0)
    st = scl.diffusion.last_stats(m.lib)
    res = {"workload": "brute-force kNN, 50k cells x 50 features (mixture), k=30, host buffers through scl_knn",
           "cells": n, "features": int(pts.shape[1]), "k": k, "e2e_ms": round(1e3 * float(np.median(ts)), 3),
           "device_ms": round(float(st["device_ms"]), 3),
           "distance_evaluations_per_s": round(n * (n - 1) / (st["device_ms"] * 1e-3), 1)}
    # the same search with every distance on CUDA cores: the tensor-core filter must give the same bits
    prev = scl.neighbors.set_kernel(1, m)
    try:
        ci, cd = scl.neighbors.knn(m, k, norms)
        sc = scl.diffusion.last_stats(m.lib)
    finally:
        scl.neighbors.set_kernel(prev, m)
    res.update({"kernel": "tensor cores (k_knn_tc)", "cuda_core_kernel_device_ms": round(float(sc["device_ms"]), 3),
                "bit_identical_to_cuda_core_kernel": bool(np.array_equal(ci, gi) and
                                                          np.array_equal(cd.view(np.uint32), gd.view(np.uint32)))})
    if with_reference:
        try:
            from oracle import ref

            R = ref.RefLib("f32_i32")
            ns = 10_000
            sub = np.ascontiguousarray(pts[:ns])
            ms, (ip, ind) = wrap_dense(sub)
            t0 = time.perf_counter()
            ri, rd, rn = R.knn(ip, ind, sub.reshape(-1), sub.shape, k)
            rdt = time.perf_counter() - t0
            t0 = time.perf_counter()
            si, sd = scl.neighbors.knn(ms, k, rn)
            gdt = time.perf_counter() - t0
            res.update({"sample_cells": ns, "reference_cpu_ms": round(1e3 * rdt, 1),
                        "reference_cores": os.cpu_count(), "gpu_e2e_ms_on_sample": round(1e3 * gdt, 3),
                        "e2e_speedup_vs_reference": round(rdt / gdt, 2),
                        "bit_identical_to_reference": bool(np.array_equal(si, ri) and
                                                           np.array_equal(sd.view(np.uint32), rd.view(np.uint32)))})
        except Exception as e:  # informational; never fail the run on it
            res["reference_cpu_ms"] = f"unavailable: {e}"
    return res


def bench_batched(torch, scl, device, stream, reps, warmup, rank=0, world=1, dist=None, check_reference=True):
    """Batched form: 64 graphs, cell counts log-uniform in [2,000, 100,000]
    (seed 0), each its own 10-component mixture, k=15, row-normalised FP32,
    16-column blocks, 8 steps: one persistent CUDA-graph launch (autotuned
    schedule) against 64 sequential scl_gpu_diffuse calls. With N ranks the
    graphs are sharded by longest-processing-time on nnz*F*T (no collective
    in the data path) and the times are the max over ranks."""
    from scl import sharding

    rng = np.random.default_rng(0)
    sizes_all = np.exp(rng.uniform(np.log(2000), np.log(100_000), 64)).astype(int)
    mine = sharding.shard_for_rank([float(n) for n in sizes_all], rank, world)
    sizes = [(b, sizes_all[b]) for b in mine]
    graphs = []
    for b, n in sizes:
        g, _ = native_graph(torch, scl, int(n), 15, seed=100 + b, stream=stream)
        graphs.append(g)
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    F, T = 16, 8
    batch = scl.gpu.GpuBatch(graphs, F, T, stream=stream)
    X0 = torch.randn((batch.n_rows, F), device=device, generator=torch.Generator(device=device).manual_seed(3))
    Y = torch.empty_like(X0)
    sched = batch.autotune(X0, Y, reps=3, stream=stream)
    t_b = event_ms(torch, lambda: batch.solve(X0, out=Y, stream=stream), stream, reps, warmup)
    code, _ = batch.status(stream)
    offs = batch.row_offsets
    Ys = torch.empty_like(X0)
    views = [(X0[offs[i]:offs[i + 1]], Ys[offs[i]:offs[i + 1]]) for i in range(len(graphs))]

    def seq():
        for g, (xi, yi) in zip(graphs, views):
            g.diffuse(xi, T, out=yi, stream=stream)

    t_s = event_ms(torch, seq, stream, reps, warmup)
    same = bool(torch.equal(Y, Ys))
    nnz = batch.nnz_total
    # every graph's batched result against scl-core's own diffuse_matrix
    # (oracle/_ref, host threads) on the same graph and block, outside the timing
    ref_same = None
    if check_reference:
        try:
            from oracle import ref

            R = ref.RefLib("f32_i32")
            Xh, Yh = X0.cpu().numpy(), Y.cpu().numpy()
            ref_same = True
            for i, g in enumerate(graphs):
                ip, ind, P = g.export()
                want, _ = reference_diffusion(R, ip, ind, P, Xh[offs[i]:offs[i + 1]], T)
                ref_same &= bool(np.array_equal(want.view(np.uint32), Yh[offs[i]:offs[i + 1]].view(np.uint32)))
        except Exception as e:  # informational; never fail the run on it
            ref_same = f"unavailable: {e}"
    batch.close()
    for g in graphs:
        g.close()
    if dist is not None:
        tt = torch.tensor([t_b, t_s], device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_b, t_s = float(tt[0]), float(tt[1])
    return {"workload": "64 graphs, cells log-uniform [2k, 100k], k=15, 16 cols, 8 steps, FP32",
            "graphs": 64, "graphs_this_rank": len(mine), "cells_this_rank": int(offs[-1]),
            "nnz_this_rank": int(nnz), "sharding": f"LPT over {world} rank(s), no data-path collective",
            "batched_ms": round(t_b, 4), "sequential_ms": round(t_s, 4), "speedup": round(t_s / t_b, 3),
            "bit_identical_to_sequential": same, "bit_identical_to_reference": ref_same, "status": code,
            "schedule": sched}


def run_reference_arm(args, warmup):
    """scl-core's own CPU diffusion (oracle/_ref f32_i32, all host threads) on
    this workload, through its C ABI the way its Python wrapper drives it.
    Rank 0 alone runs; nothing of this repository's package or libraries is
    imported or loaded. The graph is built on the host from kNN lists computed
    with torch (an input generator, untimed), Gaussian weights and (W+W^T)/2
    in NumPy / SciPy, then scl-core's own
    scl_diffusion_compute_transition_matrix. One step = one full 16-step
    diffusion of the 500k x 64 block, as in the GPU arm."""
    import scipy.sparse as sp
    import torch

    from oracle import ref

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    local = int(os.environ.get("LOCAL_RANK", "0"))
    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    syn = synthetic_module()
    t0 = time.time()
    pts = syn.mixture(N_CELLS, seed=0)
    ki, kd = syn.knn_device(pts, K_NN, device=device, block=2048)
    ki, kd = ki.cpu().numpy(), kd.cpu().numpy()
    del pts
    torch.cuda.empty_cache()
    # sigma_i = distance to the k-th neighbour (floored at 1e-10), w = exp(-(d/sigma_i)^2), (W + W^T)/2
    sigma = np.maximum(kd.max(axis=1), np.float32(1e-10)).astype(np.float32)
    w = np.exp(-np.square(kd / sigma[:, None])).astype(np.float32)
    A = sp.csr_matrix((w.reshape(-1), ki.reshape(-1).astype(np.int64), np.arange(0, N_CELLS * K_NN + 1, K_NN)),
                      shape=(N_CELLS, N_CELLS))
    S = ((A + A.T) * np.float32(0.5)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    ip, ind, W = S.indptr, S.indices, S.data.astype(np.float32)
    t_inputs = time.time() - t0
    R = ref.RefLib("f32_i32")
    t0 = time.perf_counter()
    P = R.transition(ip, ind, W, N_CELLS)
    t_tr = time.perf_counter() - t0
    gen = torch.Generator(device=device).manual_seed(1)
    X0 = torch.randn((N_CELLS, N_FEAT), device=device, dtype=torch.float32, generator=gen).cpu().numpy()
    nnz = int(ind.size)
    _, tw = reference_diffusion(R, ip, ind, P, X0, N_STEPS, reps=warmup)
    _, ts = reference_diffusion(R, ip, ind, P, X0, N_STEPS, reps=args.steps)
    t = float(np.mean(ts))
    gbs = step_bytes(N_CELLS, nnz, N_FEAT) * N_STEPS / t / 1e9
    cores = host_cores()
    line = {"impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": warmup, "ms_per_step": round(1e3 * t, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 10-component 50-D mixture; kNN lists from torch on the device, untimed)",
            "config": workload_config(world),
            "graph": {"nnz": nnz, "inputs_s": round(t_inputs, 2)},
            "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": cores, "kind": "reference",
                             "sample": f"scl_diffusion_diffuse_matrix ({R.path.name}, scl-core compiled) on the full "
                                       f"500k graph, all 16 steps per sample, {cpu_model()}"},
            "transition_ms_cpu": round(1e3 * t_tr, 3),
            "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---- named profiling cases --------------------------------------------------------------------
CASES = {
    "spmm": "diffusion steps through scl_gpu_diffuse (--storage, --plan, --no-reorder)",
    "backward": "checkpointed forward + backward of L = sum((X_T - Y)^2) (--every)",
    "knn": "brute-force kNN of the mixture through scl_knn (host buffers)",
    "ppr": "personalized PageRank from cell 0 through the drop-in ABI",
    "dpt": "diffusion pseudotime from cell 0 through the drop-in ABI",
    "e2e": "scl_diffusion_diffuse_matrix with pinned host buffers",
}


def run_case(args):
    """One named workload, for ncu captures and sweeps: the seeded mixture graph
    built natively (scl_knn, weights, (W+W^T)/2, row normalisation), then the
    case's calls; prints one line with a checksum.

        python bench.py --case spmm --cells 500000 --features 64 --case-steps 4 [--storage bf16]
    """
    import torch

    import scl

    steps = max(args.case_steps, 1)
    if args.case == "knn":
        syn = synthetic_module()
        pts = syn.mixture(args.cells, seed=21).astype(np.float32)[:, : args.features]
        for _ in range(steps):
            idx, dist, _ = native_knn(scl, pts, args.k)
        print(f"cells={pts.shape[0]} features={pts.shape[1]} k={args.k} "
              f"checksum={float(dist[np.isfinite(dist)].sum()):.6e}")
        return
    g, info = native_graph(torch, scl, args.cells, args.k, seed=0)
    n, _, nnz = g.shape
    if args.case in ("ppr", "dpt", "e2e"):
        ip, ind, P = g.export()
        m = scl.CsrMatrix.wrap(ip.astype(np.int32), ind, P, (n, n))
        if args.case == "ppr":
            for _ in range(steps):
                out = scl.diffusion.personalized_pagerank(m, 0)
        elif args.case == "dpt":
            for _ in range(steps):
                out = scl.diffusion.compute_dpt(m, 0)
        else:
            X0 = torch.randn((n, args.features)).numpy()
            for _ in range(steps):
                out = torch.from_numpy(X0).pin_memory().numpy()
                scl.diffusion.diffuse_matrix(m, out, N_STEPS)
        print(f"case={args.case} cells={n} nnz={nnz} checksum={float(np.sum(out, dtype=np.float64)):.6e}")
        return
    if args.case == "backward":
        gen = torch.Generator(device="cuda").manual_seed(7)
        X0 = torch.randn((n, args.features), device="cuda", generator=gen)
        Yt = torch.randn((n, args.features), device="cuda", generator=gen)
        XT, ck = g.diffuse_checkpointed(X0, steps, args.every)
        dX, dW = g.diffuse_backward(X0, ck, 2.0 * (XT - Yt), steps, args.every)
        torch.cuda.synchronize()
        print(f"case=backward cells={n} nnz={nnz} features={args.features} steps={steps} every={args.every} "
              f"loss={float(((XT - Yt) ** 2).sum()):.6e} |dX|={float(dX.norm()):.6e} |dW|={float(dW.norm()):.6e}")
        return
    if not args.no_reorder:
        g.reorder(1)
    dt = {"bf16": torch.bfloat16, "f16": torch.float16}.get(args.storage)
    if dt is not None:
        g.set_storage(dt)
    if args.plan:
        grp, vec, kind, stage = (int(x) for x in args.plan.split(","))
        g.set_plan(args.features, grp, vec, kind, stage)
    X = torch.randn((n, args.features), device="cuda")
    if dt is not None:
        X = X.to(dt)
    Y = g.diffuse(X, steps)
    torch.cuda.synchronize()
    print(f"case=spmm cells={n} nnz={nnz} features={args.features} steps={steps} storage={args.storage} "
          f"reorder={not args.no_reorder} build_ms={info['build_ms']:.2f} checksum={float(Y.float().sum()):.6e}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", default=None, choices=sorted(CASES),
                    help="run one named profiling case instead of the benchmark (see run_case)")
    ap.add_argument("--cells", type=int, default=200_000, help="--case: cells")
    ap.add_argument("--k", type=int, default=30, help="--case: neighbours")
    ap.add_argument("--features", type=int, default=64, help="--case: columns")
    ap.add_argument("--case-steps", type=int, default=3, help="--case: diffusion steps / repetitions")
    ap.add_argument("--every", type=int, default=4, help="--case backward: checkpoint interval")
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16"], help="--case spmm: storage")
    ap.add_argument("--no-reorder", action="store_true", help="--case spmm: no locality reordering")
    ap.add_argument("--plan", default="", help="--case spmm: group,vec,kind,stage launch shape")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the BF16/FP16 forms")
    ap.add_argument("--no-backward", action="store_true", help="skip the forward+backward configuration")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched configuration")
    ap.add_argument("--no-impute", action="store_true", help="skip the MAGIC imputation configuration")
    ap.add_argument("--no-walks", action="store_true", help="skip the personalized PageRank configuration")
    ap.add_argument("--no-knn", action="store_true", help="skip the kNN configuration")
    args = ap.parse_args()
    warmup = max(3, args.warmup)
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference_arm(args, warmup)

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = f"cuda:{local}"
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device(device))

    import scl

    stream = torch.cuda.current_stream()

    # ---- graph from features, natively: scl_knn -> weights / (W+W^T)/2 -> row normalisation ----
    g, build = native_graph(torch, scl, N_CELLS, K_NN, seed=0, stream=stream, normalize=False)
    ip, ind, W = g.export()  # pre-normalisation weights, for the FP64 checks
    bt0 = torch.cuda.Event(enable_timing=True)
    bt1 = torch.cuda.Event(enable_timing=True)
    bt0.record(stream)
    g.normalize(symmetric=False, stream=stream)
    bt1.record(stream)
    bt1.synchronize()
    build["normalize_ms"] = round(bt0.elapsed_time(bt1), 3)
    # locality reordering, a one-off per graph
    bt0.record(stream)
    g.reorder(1, stream=stream)
    bt1.record(stream)
    bt1.synchronize()
    build["reorder_ms"] = round(bt0.elapsed_time(bt1), 3)
    _, build["reorder_cc_rounds"] = g.reorder_info()
    n, _, nnz = g.shape
    F, T = N_FEAT, N_STEPS
    tuned = g.autotune(F, reps=3, stream=stream)  # one-off: fastest bit-identical launch shape
    floor_ms = g.gather_floor(F, reps=5, stream=stream)  # gathers only, same rows and order
    B32 = step_bytes(n, nnz, F)
    B16 = step_bytes(n, nnz, F, s_val=2, s_x=2)
    gen = torch.Generator(device=device).manual_seed(1 + rank)
    X0 = torch.randn((n, F), device=device, dtype=torch.float32, generator=gen)
    Y = torch.empty_like(X0)
    flush = torch.empty(64 * 1024 * 1024, device=device, dtype=torch.float32)

    def run_f32():
        g.diffuse(X0, T, out=Y, stream=stream)

    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local, gpu_uuid(torch, device)) as clk:
        times = timed_calls(torch, run_f32, args.steps, warmup, flush, stream)
    torch.cuda.synchronize()
    t_ms = float(np.mean(times))
    if dist is not None:
        tt = torch.tensor([t_ms], device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = world * B32 * T / (t_ms * 1e-3) / 1e9
    per_launch_ms = t_ms / T
    peak, peak_kind = load_peaks()
    achieved = B32 / (per_launch_ms * 1e-3) / 1e9
    _, _, Pm = g.export()

    # ---- FP64 on the device (same weights, FP64 transition) and the precision forms -------
    forms = {}
    fp64 = {}
    if rank == 0 and not args.no_forms:
        g64 = scl.gpu.GpuGraph.from_csr(ip, ind, W.astype(np.float64), (n, n), variant="f64_i64")
        g64.normalize(symmetric=False)
        g64.reorder(1)
        Y64 = g64.diffuse(X0.double(), T)
        e32 = scl.gpu.residual_fp64(Y, Y64, rel_floor=1e-3)
        forms["f32"] = {"gbs": round(value / world, 2), "ms": round(t_ms, 4), "rel_fro_err_vs_fp64": e32["rel_fro"],
                        "max_rel_err_vs_fp64": e32["max_rel"]}
        for name, tdt in (("bf16", torch.bfloat16), ("f16", torch.float16)):
            g.set_storage(tdt, stream=stream)
            tuned_l = g.autotune(F, reps=3, stream=stream)  # fastest bit-identical shape for this storage
            Xl = X0.to(tdt)
            Yl = torch.empty((n, F), device=device, dtype=torch.float32)

            def run_l():
                g.diffuse(Xl, T, out=Yl, stream=stream)

            tl = float(np.mean(timed_calls(torch, run_l, args.steps, warmup, flush, stream)))
            el = scl.gpu.residual_fp64(Yl, Y64, rel_floor=1e-3)
            # per-step errors vs FP64 (16-bit iterates against FP64 iterates), reduced in FP64 on the device
            step_err = []
            Xs, X64s = Xl, X0.double()
            for _ in range(T):
                Xs = g.diffuse(Xs, 1, out_dtype=tdt)
                X64s = g64.diffuse(X64s, 1)
                step_err.append(scl.gpu.residual_fp64(Xs, X64s, rel_floor=1e-3)["rel_fro"])
            forms[name] = {"gbs": round(B16 * T / (tl * 1e-3) / 1e9, 2), "ms": round(tl, 4),
                           "plan": {"kind": tuned_l["kind"], "stage": tuned_l["stage"]},
                           "speedup_vs_f32": round(t_ms / tl, 3), "rel_fro_err_vs_fp64": round(el["rel_fro"], 8),
                           "max_rel_err_vs_fp64": round(el["max_rel"], 6),
                           "per_step_rel_fro_err": [round(e, 6) for e in step_err]}
            del Xs, X64s
        g.set_storage(torch.float32, stream=stream)
        g64.close()
        # FP64 pinned to scl-core's own f64 build (transition + diffusion on the same weights and block)
        if world == 1 and not args.no_cpu_baseline:
            try:
                from oracle import ref

                R64 = ref.RefLib("f64_i64")
                P64r = R64.transition(ip, ind, W.astype(np.float64), n)
                Y64r, t64 = reference_diffusion(R64, ip, ind, P64r, X0.double().cpu().numpy(), T)
                fp64 = {"gpu_fp64_bit_identical_to_reference_f64": bool(np.array_equal(
                            Y64.cpu().numpy().view(np.uint64), Y64r.view(np.uint64))),
                        "reference_f64_s": round(t64[0], 2)}
                e32r = scl.gpu.residual_fp64(Y, torch.from_numpy(Y64r).to(device), rel_floor=1e-3)
                fp64["f32_rel_fro_err_vs_reference_f64"] = e32r["rel_fro"]
                fp64["f32_max_rel_err_vs_reference_f64"] = e32r["max_rel"]
                del Y64r, P64r
            except Exception as e:  # informational; never fail the run on it
                fp64 = {"reference_f64": f"unavailable: {e}"}
        del Y64

    # ---- differentiation and batched forms (each rank runs its own replica) ---------------
    fwd_bwd = None
    if not args.no_backward:
        fwd_bwd = bench_backward(torch, scl, device, stream, args.steps, warmup, flush)
    batched = None
    if not args.no_batched:
        batched = bench_batched(torch, scl, device, stream, args.steps, warmup, rank, world, dist,
                                check_reference=(rank == 0 and not args.no_cpu_baseline))

    impute = None
    if rank == 0 and not args.no_impute:
        impute = bench_impute(torch, scl, device, min(args.steps, 3), 1, with_reference=not args.no_cpu_baseline)
    knn = None
    if rank == 0 and not args.no_knn:
        knn = bench_knn(torch, scl, min(args.steps, 3), 1, with_reference=not args.no_cpu_baseline)
        knn["graph_500k_scl_knn_s"] = build["knn_s"]

    # ---- end to end through the drop-in C ABI with pinned host buffers --------------------
    e2e = None
    walks = None
    if not args.no_e2e:
        Xh = torch.empty((n, F), dtype=torch.float32).pin_memory()
        iph = torch.from_numpy(ip.astype(np.int32)).pin_memory()
        indh = torch.from_numpy(ind).pin_memory()
        Ph = torch.from_numpy(Pm).pin_memory()
        X0h = X0.cpu().numpy()
        m = scl.CsrMatrix.wrap(iph.numpy(), indh.numpy(), Ph.numpy(), (n, n))
        Xn = Xh.numpy()
        et = []
        for it in range(warmup + args.steps):
            Xn[...] = X0h
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            scl.diffusion.diffuse_matrix(m, Xn, T)
            dt = time.perf_counter() - t0
            if it >= warmup:
                et.append(dt)
        st = scl.diffusion.last_stats(m.lib)
        e_s = float(np.mean(et))
        if dist is not None:
            tt = torch.tensor([e_s], device=device)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e_s = float(tt.item())
        e2e = {"value": round(world * B32 * T / e_s / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": int(st["h2d_bytes"]), "d2h_bytes_per_step": int(st["d2h_bytes"]),
               "ms_per_step": round(1e3 * e_s, 3), "device_ms": round(float(st["device_ms"]), 3),
               "api": "scl_diffusion_diffuse_matrix (libscl_f32_i32.so)",
               "bit_exact_vs_device_path": bool(np.array_equal(Xn.view(np.uint32),
                                                               Y.cpu().numpy().view(np.uint32)))}
        # context, not the headline: the same call with the graph kept on the device between calls
        # (scl_diffusion_gpu_attach), so each call moves only the dense block
        scl.diffusion.attach(m)
        at = []
        for it in range(warmup + args.steps):
            Xn[...] = X0h
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            scl.diffusion.diffuse_matrix(m, Xn, T)
            if it >= warmup:
                at.append(time.perf_counter() - t0)
        sa = scl.diffusion.last_stats(m.lib)
        scl.diffusion.detach(m)
        e2e["graph_attached"] = {"ms_per_step": round(1e3 * float(np.mean(at)), 3),
                                 "h2d_bytes_per_step": int(sa["h2d_bytes"]),
                                 "d2h_bytes_per_step": int(sa["d2h_bytes"]),
                                 "bit_exact_vs_device_path": bool(np.array_equal(Xn.view(np.uint32),
                                                                                 Y.cpu().numpy().view(np.uint32)))}
        # personalized PageRank on the same graph and host handle (scl_diffusion_personalized_pagerank,
        # alpha 0.85, tol 1e-6 on the L1 change, at most 100 steps), beside scl-core's own build
        if rank == 0 and not args.no_walks:
            walks = {"workload": "personalized PageRank, 500k cells k=30 row-normalised graph, seed 0, "
                                 "alpha 0.85, tol 1e-6, max 100 steps, host buffers"}
            pt = []
            for it in range(warmup + args.steps):
                t0 = time.perf_counter()
                pr = scl.diffusion.personalized_pagerank(m, 0)
                if it >= warmup:
                    pt.append(time.perf_counter() - t0)
            st = scl.diffusion.last_stats(m.lib)
            walks.update({"e2e_ms": round(1e3 * float(np.median(pt)), 3), "device_ms": round(st["device_ms"], 3),
                          "h2d_bytes": int(st["h2d_bytes"]), "d2h_bytes": int(st["d2h_bytes"])})
            if not args.no_cpu_baseline:
                try:
                    from oracle import ref

                    R = ref.RefLib("f32_i32")
                    t0 = time.perf_counter()
                    want = R.walk("ppr", ip, ind, Pm, n, seed=0, alpha=0.85, max_iter=100, tol=1e-6)
                    rdt = time.perf_counter() - t0
                    walks.update({"reference_cpu_ms": round(1e3 * rdt, 1), "reference_cores": host_cores(),
                                  "e2e_speedup_vs_reference": round(rdt / float(np.median(pt)), 2),
                                  "max_rel_diff_vs_reference": float(np.max(np.abs(pr - want) /
                                                                            np.maximum(np.abs(want), 1e-30)))})
                except Exception as e:  # informational; never fail the run on it
                    walks["reference_cpu_ms"] = f"unavailable: {e}"
        del m

    # ---- CPU baseline and full-size parity (rank 0, N=1): scl-core's own diffuse_matrix on the
    # same P and the same X0 as the device run; the device result must equal it bit for bit ----------
    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref

            R = ref.RefLib("f32_i32")
            want, ts = reference_diffusion(R, ip, ind, Pm, X0.cpu().numpy(), T, reps=3)
            dt = float(np.median(ts))
            cpu = {"value": round(B32 * T / dt / 1e9, 3), "unit": "GB/s", "cores": host_cores(), "kind": "reference",
                   "sample": f"scl_diffusion_diffuse_matrix (scl-core compiled, {R.path.name}) on the full 500k "
                             f"graph and the device run's X0, all 16 steps, median of 3 ({dt:.2f} s), {cpu_model()}"}
            parity = {"bit_identical_to_reference": bool(np.array_equal(want.view(np.uint32),
                                                                        Y.cpu().numpy().view(np.uint32))),
                      "reference": f"{R.path.name} diffuse_matrix, same P and X0, 16 steps"}
            # transition: this library's FP64-degree normalisation vs scl-core's f32 compute_transition_matrix
            Pr = R.transition(ip, ind, W, n)
            du = np.abs(Pm.view(np.int32).astype(np.int64) - Pr.view(np.int32).astype(np.int64))
            parity["transition_max_ulp_vs_reference_f32"] = int(du.max())
        except Exception as e:  # the baseline is informational; never fail the run on it
            cpu = {"value": None, "unit": "GB/s", "cores": host_cores(), "kind": "reference",
                   "sample": f"unavailable: {e}"}
    if parity is not None:
        parity.update(fp64)

    if rank == 0:
        summary = {
            "f32_ms": round(t_ms, 4), "f32_frac_of_gather_floor": round(floor_ms / per_launch_ms, 4),
            "bit_identical_to_reference": parity.get("bit_identical_to_reference") if parity else None,
            "bf16_speedup": forms.get("bf16", {}).get("speedup_vs_f32"),
            "bf16_rel_fro_err": forms.get("bf16", {}).get("rel_fro_err_vs_fp64"),
            "f16_speedup": forms.get("f16", {}).get("speedup_vs_f32"),
            "f16_rel_fro_err": forms.get("f16", {}).get("rel_fro_err_vs_fp64"),
            "fwd_bwd_over_fwd": fwd_bwd["fwd_bwd_over_fwd"] if fwd_bwd else None,
            "batched_speedup": batched["speedup"] if batched else None,
            "batched_bit_identical_to_reference": batched.get("bit_identical_to_reference") if batched else None,
            "e2e_ms": e2e["ms_per_step"] if e2e else None,
        }
        # the ncu capture of the plan the autotuner picked (kind 12: multi-row, kind 4: warp per row)
        traffic_profile = "spmm_rows16_f32_500k" if tuned["kind"] == 12 else "spmm_row_f32_500k"
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": warmup, "ms_per_step": round(t_ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 10-component 50-D mixture; kNN by this library's scl_knn, untimed)",
            "config": workload_config(world),
            "graph": {"nnz": nnz, "bytes_per_spmm_step": B32, **build},
            "gpu_launches": args.steps * (T + 1),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": profiled_traffic(traffic_profile),
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                           f"profiles/{traffic_profile}.md", "peak_kind": peak_kind,
                         "kernel": f"SpMM plan kind {tuned['kind']} stage {tuned['stage']}",
                         "per_launch_ms": round(per_launch_ms, 5),
                         "gather_floor_ms": round(floor_ms, 5),
                         "frac_of_gather_floor": round(floor_ms / per_launch_ms, 4),
                         "gather_floor_note": "time of a kernel that only gathers the same 256-byte X rows "
                                              "in the same order at full occupancy (scl_gpu_graph_gather_floor)"},
            "parity": parity,
            "forms": forms,
            "fwd_bwd_ms": fwd_bwd["fwd_bwd_ms"] if fwd_bwd else None,
            "fwd_bwd": fwd_bwd,
            "batched": batched,
            "impute": impute,
            "walks": walks,
            "knn": knn,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "summary": summary,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
