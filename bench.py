#!/usr/bin/env python
"""Benchmark of the raptr reconstruction hot path on B200.

Workload (default): the full ePET configuration -- 70^3 voxels of 2 mm,
180 angles x 13^4 crystal pairs = 5,140,980 channels, 1000 Monte Carlo rays
per channel, a two-sphere + five-rod phantom with 1e8 Poisson counts, 50
MLEM iterations from a uniform image.  Data are synthetic (seeded).

One step = one whole reconstruction job from the measurement resident in
HBM: system-matrix build for all channels (CSR), its transpose (CSC), the
FP64 sensitivity image, and 50 MLEM iterations.  The reported metric is MLEM
iterations per second of that job (50 / job time), so the matrix build is
inside the timed region (the reference rebuilds the matrix in every
iteration, src/tests/reco.cu:230-252); matrix_build_s and the resident
per-iteration rate are reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl raptr|reference]

With N > 1 (torchrun, one rank per GPU) the channel rows are sharded over
the ranks (strong scaling of the same job); each iteration all-reduces the
N-voxel back projection over NCCL, as the reference does over MPI
(src/tests/reco.cu:237-281).

--impl reference times the reference's own CPU algorithm (candidate search,
per-candidate mean intersection length over all rays, CSR SpMVs; built from
the reference sources into oracle/_ref) on a bounded channel sample on all
host cores, extrapolated by channel count to the same job.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from raptr_b200 import config as cfg  # noqa: E402

SEED = 1251
MEAS_SEED = 20240

# DRAM bytes per matrix entry of one launch, from an ncu capture of the
# profile case (`python -m raptr_b200.profile_case --rows 300000 --forms`:
# rows 0..299,999 of the full workload, 191,091,787 entries):
# (dram__bytes_read.sum + dram__bytes_write.sum) / entries.  The roofline's `traffic` scales them by
# the entries of the timed matrix (traffic grows with the entries).
TRAFFIC_BYTES_PER_ENTRY = {
    # column-slab profile case (x slabs 33-36, full-length columns)
    "mlem_back_kernel": (3.020836e9 + 5.886464e6) / 371438029,
    # row profile case (rows 0..299,999, full rows)
    "mlem_forward_kernel": (1.539569e9 + 4.874752e6) / 191091787,
}


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["raptr", "reference"], default="raptr")
    p.add_argument("--workload", choices=list(cfg.WORKLOADS), default="full")
    p.add_argument("--cpu-sample-s", type=float, default=12.0, help="CPU seconds for the cpu_baseline sample")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-forms", action="store_true", help="skip the FP16 / batched / serving forms")
    return p.parse_args()


def workload(name):
    w = dict(cfg.WORKLOADS[name])
    w["name"] = name
    return w


def config_of(w, n_gpus):
    g = w["geom"]
    return {
        "workload": f"ePET {g.grid_n[0]}^3 x {g.grid_d[0] * 1e3:g} mm, {g.na} angles x 13^4 crystal pairs = "
                    f"{g.n_channels} channels, {w['nrays']} rays/channel, {w['counts']:.0e} counts, "
                    f"{w['niter']} MLEM iterations",
        "voxels": g.n_voxels,
        "channels": g.n_channels,
        "rays_per_channel": w["nrays"],
        "counts": w["counts"],
        "iterations": w["niter"],
        "parallelism": f"row-shard x{n_gpus}" if n_gpus > 1 else "single GPU",
        "l2": "inputs larger than L2 (system matrix ~30 GB CSR + ~30 GB CSC)",
        "phantom": "background 0.1, sphere r15 mm 1.0, sphere r8 mm at +20 mm x 4.0" +
                   (", 5 rods r2-6 mm 2.0" if w["rods"] else ""),
    }


def metric_name(w):
    g = w["geom"]
    return (f"MLEM iterations/s, whole job incl. system-matrix build ({g.grid_n[0]}^3 voxels, "
            f"{g.n_channels / 1e6:.2f}M channels, {w['nrays']} rays)")


# ---------------------------------------------------------------------------
# Clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # the memory clock and HBM temperature, from a second process so that a
    # field a driver does not know costs only these: the HBM-bound passes
    # run ~5 % apart on different boxes at the same SM clock
    EXTRA = "clocks.mem,clocks.max.mem,temperature.memory"

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = self.proc_extra = None
        self.t0 = self.t1 = None

    def _spawn(self, fields):
        try:
            return subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 self.gpu_id], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            return None

    @staticmethod
    def _collect(proc):
        if proc is None:
            return ""
        proc.terminate()
        try:
            out, _ = proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            proc.kill()
            out, _ = proc.communicate()
        return out

    def start(self):
        self.proc = self._spawn(self.FIELDS)
        self.proc_extra = self._spawn(self.EXTRA)

    def stop(self):
        extra_out = self._collect(self.proc_extra)
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        out = self._collect(self.proc)
        sm, smax, reasons, power = [], [], set(), []
        extra = {"mem_mhz": [], "mem_max_mhz": [], "hbm_temp_c": []}
        for line in extra_out.splitlines():
            for k, v in zip(extra, (x.strip() for x in line.split(","))):
                try:
                    extra[k].append(float(v))
                except ValueError:  # "N/A" on parts that do not report it
                    pass
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        loaded = [s for s, p in zip(sm, power) if p > 0.25 * max(power)] or sm
        rec = {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
               "samples": len(sm), "power_w_max": max(power)}
        if extra["mem_mhz"]:
            rec["mem_mhz"] = statistics.median(extra["mem_mhz"])
        if extra["mem_max_mhz"]:
            rec["mem_max_mhz"] = max(extra["mem_max_mhz"])
        if extra["hbm_temp_c"]:
            rec["hbm_temp_c_max"] = max(extra["hbm_temp_c"])
        return rec


def gpu_id_for(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:  # noqa: BLE001
        return str(dev)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "of measured"
    return 6650.0, "of fallback"


# ---------------------------------------------------------------------------
# CPU baselines (reference harness or oracle port)
# ---------------------------------------------------------------------------

def cpu_reference_sample(w, budget_s: float, threads: int):
    """Times the reference algorithm on a channel sample (all host threads):
    candidates by getWorkqueue, each element the mean over all rays of
    intersectionLength, then the two CSR SpMVs of an iteration over the
    sample's rows (the reference's COO keeps every candidate).  Returns
    (per-channel build seconds, per-entry SpMV seconds, entries per channel,
    kind, channels sampled, threads)."""
    import ctypes as C

    from oracle import oracle as O

    g = w["geom"]
    nrays = w["nrays"]
    kind = "reference" if O.ref_available() else "port"
    rng = np.random.Generator(np.random.PCG64(99))
    sample = rng.permutation(g.n_channels).astype(np.int32)
    og = O.to_ogeom(g)
    per_call = 2

    def run_ref(chs):
        U = O.ray_uniforms_batch(SEED, chs, nrays)
        cap = int(len(chs) * 40000)
        oc = np.zeros(cap, np.int32)
        ov = np.zeros(cap, np.int32)
        oval = np.zeros(cap, np.float32)
        n = O.ref().ref_sysmat(C.byref(og), chs, len(chs), nrays, U, cap, oc, ov, oval)
        return int(n), oc[:n], ov[:n], oval[:n]

    def run_port(chs):
        rp, col, val = O.sysmat(g, chs, nrays, SEED, method=0, keep_zeros=True, nthreads=1)
        return int(col.size), np.repeat(chs, np.diff(rp)), col, val

    fn = run_ref if kind == "reference" else run_port
    done, entries, t0 = 0, 0, time.perf_counter()
    rows_c, rows_v, rows_val = [], [], []
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while time.perf_counter() - t0 < budget_s:
            chunk = [sample[done + i * per_call: done + (i + 1) * per_call] for i in range(threads)]
            for n, oc, ov, oval in ex.map(fn, chunk):
                entries += n
                if len(rows_c) < 64:
                    rows_c.append(oc)
                    rows_v.append(ov)
                    rows_val.append(oval)
            done += threads * per_call
    t_build = time.perf_counter() - t0
    # SpMV cost per entry on the sampled rows (single thread, scaled by threads)
    cnl = np.concatenate(rows_c)
    col = np.concatenate(rows_v).astype(np.int32)
    val = np.concatenate(rows_val).astype(np.float32)
    _, inv = np.unique(cnl, return_inverse=True)
    order = np.lexsort((col, inv))
    rows = inv[order].astype(np.int32)
    rp = O.coo2csr(rows, int(rows.max()) + 1)
    x = np.ones(g.n_voxels, np.float32)
    t1 = time.perf_counter()
    reps = 0
    while time.perf_counter() - t1 < 0.5:
        ycol = O.spmv(0, rp.size - 1, g.n_voxels, rp, col[order], val[order], x)
        O.spmv(1, rp.size - 1, g.n_voxels, rp, col[order], val[order], ycol)
        reps += 1
    t_spmv_entry = (time.perf_counter() - t1) / reps / max(col.size, 1) / 2 / threads
    return t_build * threads / done, t_spmv_entry, entries / done, kind, done, threads


def cpu_job_rate(w, budget_s, threads):
    """MLEM iterations/s of the reference's job on the host cores: every
    iteration rebuilds the matrix of all measured channels and runs two
    SpMVs over it (src/tests/reco.cu:230-281)."""
    g = w["geom"]
    per_ch, per_entry, ent_per_ch, kind, nsamp, thr = cpu_reference_sample(w, budget_s, threads)
    t_build = per_ch * g.n_channels / thr
    t_spmv = 2 * per_entry * ent_per_ch * g.n_channels
    t_iter = t_build + t_spmv
    return {
        "value": 1.0 / t_iter,
        "unit": "MLEM iterations/s",
        "cores": thr,
        "kind": kind,
        "sample": f"{nsamp} random channels x {w['nrays']} rays on {thr} threads ({budget_s:.0f} s), "
                  f"extrapolated by channel count to {g.n_channels} channels; one iteration = rebuild "
                  f"({t_build:.3g} s) + 2 SpMVs over {ent_per_ch:.0f} entries/channel ({t_spmv:.3g} s)",
        "matrix_build_s": t_build,
    }


# ---------------------------------------------------------------------------
# The GPU job
# ---------------------------------------------------------------------------

def synth_measurement(R, torch, ctx, w, lst, dist=None):
    """Seeded Poisson measurement of the phantom through the system matrix
    (setup, not timed).  Each rank projects its own rows; the expected counts
    are gathered so that every rank draws the same measurement."""
    g = w["geom"]
    A = ctx.build(lst, w["nrays"], SEED)
    xt = torch.from_numpy(cfg.phantom(g, w["rods"])).cuda()
    lam = R.spmv(R.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt)
    del A
    gc.collect()
    if dist is not None:
        world = dist.get_world_size()
        sizes = [(r + 1) * g.n_channels // world - r * g.n_channels // world for r in range(world)]
        parts = [torch.empty(n, device="cuda") for n in sizes]
        dist.all_gather(parts, lam)
        lam = torch.cat(parts)
    torch.cuda.synchronize()
    return cfg.poisson_measurement(lam.cpu().numpy(), w["counts"], MEAS_SEED)


def run_job(R, torch, ctx, w, lst, y_dev, dist=None):
    """One reconstruction job; returns per-phase device times (ms) and the
    device time of every forward and back pass of its iterations (CUDA
    events between the passes, on the stream they are launched on: stream
    launches, which run the iterations as fast as one CUDA graph of them)."""
    g = w["geom"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    ev[0].record()
    A = ctx.build(lst, w["nrays"], SEED)
    ev[1].record()
    A.transpose()
    ev[2].record()
    if dist is None:
        s64, s = R.sensitivity(A)
    else:
        from raptr_b200.distributed import GpuShardOps, ShardedMLEM

        sharded = ShardedMLEM(GpuShardOps(A), dist)
        s = sharded.sensitivity()
    ev[3].record()
    x = torch.full((g.n_voxels,), np.float32(1.0 / g.n_voxels), device="cuda")
    kt = None
    if dist is None:
        kt = ctx.mlem(A, y_dev, s, x, w["niter"], use_graph=False, kernel_times=True)
    else:
        ops = sharded.ops
        kev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(w["niter"])]
        for it in range(w["niter"]):  # ShardedMLEM.iterate, with events around the two passes
            kev[it][0].record()
            e = ops.forward(y_dev, x)
            kev[it][1].record()
            c = ops.back(e)
            kev[it][2].record()
            dist.all_reduce(c)
            ops.update(x, c, s)
        torch.cuda.synchronize()
        kt = np.array([[k[0].elapsed_time(k[1]), k[1].elapsed_time(k[2])] for k in kev])
    ev[4].record()
    torch.cuda.synchronize()
    t = [ev[i].elapsed_time(ev[i + 1]) for i in range(4)]
    info = {"nnz": A.nnz, "m": A.m}
    del A  # freed by reference count (its blocks go back to the library's cache)
    return {"build_ms": t[0], "transpose_ms": t[1], "sens_ms": t[2], "mlem_ms": t[3], "job_ms": sum(t),
            "kernel_ms": kt, "x": x, **info}


def precision_report(R, torch, ctx, w, lst, y_dev, peak):
    """The FP16-matrix form (plain: 6 bytes per entry; delta-coded: 4) beside
    the FP32 one, all against the FP64 iteration on the same matrix:
    relative L2 and max error of the image after 10 / 25 / 50 iterations,
    iteration rates (CUDA graph) and the roofline of the FP16 passes."""
    g = w["geom"]
    n = g.n_voxels
    A = ctx.build(lst, w["nrays"], SEED)
    A.transpose()
    A.to_half()
    A.to_packed()
    nnz, m = A.nnz, A.m
    pwords, twords = A.pword.numel(), A.tword.numel()
    s64, s32 = R.sensitivity(A)
    h64, h32 = R.sensitivity_half(A)
    marks = [c for c in (10, 25, 50) if c <= w["niter"]] or [w["niter"]]
    x64 = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    x32 = torch.full((n,), np.float32(1.0 / n), device="cuda")
    x16 = torch.full((n,), np.float32(1.0 / n), device="cuda")
    xpk = torch.full((n,), np.float32(1.0 / n), device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    errs = {"fp32": {}, "fp16": {}, "fp16_delta": {}}
    ms = {"fp32": 0.0, "fp16": 0.0, "fp16_delta": 0.0}
    kt16 = []
    done = 0
    for mark in marks:
        k = mark - done
        ctx.mlem_f64(A, y_dev, s64 / s64.sum(), x64, k)
        ev[0].record()
        ctx.mlem(A, y_dev, s32, x32, k, use_graph=True)
        ev[1].record()
        ctx.mlem_half(A, y_dev, h32, x16, k, use_graph=True)
        ev[2].record()
        ctx.mlem_packed(A, y_dev, h32, xpk, k, use_graph=True)
        ev[3].record()
        torch.cuda.synchronize()
        ms["fp32"] += ev[0].elapsed_time(ev[1])
        ms["fp16"] += ev[1].elapsed_time(ev[2])
        ms["fp16_delta"] += ev[2].elapsed_time(ev[3])
        ref = x64
        for name, x in (("fp32", x32), ("fp16", x16), ("fp16_delta", xpk)):
            d = x.double() - ref
            errs[name][str(mark)] = {"rel_l2": float(d.norm() / ref.norm()),
                                     "max_rel": float(d.abs().max() / ref.abs().max())}
        done = mark
    # per-pass device times of the FP16 iteration (no graph, events between passes)
    kt16 = ctx.mlem_half(A, y_dev, h32, x16.clone(), 5, use_graph=False, kernel_times=True)
    fwd_ms, back_ms = float(kt16[:, 0].mean()), float(kt16[:, 1].mean())
    fwd_b = nnz * 6 + (m + 1) * 8 + m * 4 * 4 + n * 4
    back_b = nnz * 6 + (n + 1) * 8 + 3 * n * 4 + m * 4
    ktp = ctx.mlem_packed(A, y_dev, h32, xpk.clone(), 5, use_graph=False, kernel_times=True)
    pf_ms, pb_ms = float(ktp[:, 0].mean()), float(ktp[:, 1].mean())
    # words (4 bytes per entry, plus the steps above 65535 and the padding),
    # quad offsets and anchors, then the vectors as for the plain form
    pf_b = pwords * 4 + (m + 1) * 8 + m * 4 + m * 4 * 4 + n * 4
    pb_b = twords * 4 + (n + 1) * 8 + n * 4 + 3 * n * 4 + m * 4

    def line(b, t):
        return {"achieved": round(b / t / 1e6, 1), "frac": round(b / t / 1e6 / peak, 4), "ms": round(t, 4)}

    out = {
        "iterations": done,
        "iters_per_s": {k: done / (v / 1e3) for k, v in ms.items()},
        "speedup_fp16_vs_fp32": ms["fp32"] / ms["fp16"],
        "speedup_fp16_delta_vs_fp32": ms["fp32"] / ms["fp16_delta"],
        "error_vs_fp64": errs,
        "matrix_bytes_per_entry": {"fp32": 8, "fp16": 6, "fp16_delta": round(4 * (pwords + twords) / (2 * nnz), 4)},
        "roofline_fp16": {
            "mlem_forward_half_kernel": line(fwd_b, fwd_ms),
            "mlem_back_half_kernel": line(back_b, back_ms),
            "mlem_forward_packed_kernel": line(pf_b, pf_ms),
            "mlem_back_packed_kernel": line(pb_b, pb_ms),
        },
        "reference": "FP64 vectors and accumulation over the FP32 matrix (raptr_mlem_f64, GPU)",
    }
    del A
    gc.collect()
    return out


def batch_report(R, torch, ctx, w, lst, plain_iters_per_s, peak, n_frames=64, niter=None):
    """The batched dynamic-PET form: n_frames frames sharing the matrix,
    activity x_true * exp(-k_j f) with per-voxel washout rates k ~ U[0.01,
    0.1] per frame, counts per frame log-uniform in [1e5, 1e8], solved
    together with the FP16 matrix (frame tile from the autotuner, CUDA-graph
    iterations).  Reports frame-iterations per second against the plain
    FP32 single-frame rate, and frame 0's image against the FP64 iteration."""
    g = w["geom"]
    n = g.n_voxels
    niter = niter or w["niter"]
    A = ctx.build(lst, w["nrays"], SEED)
    A.to_half()
    rng = np.random.default_rng(SEED + 64)
    rates = torch.from_numpy(rng.uniform(0.01, 0.1, n).astype(np.float32)).cuda()
    counts = 10.0 ** rng.uniform(5, 8, n_frames)
    xt = torch.from_numpy(cfg.phantom(g, rods=w.get("rods", False)).astype(np.float32)).cuda()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(SEED + 65)
    Y = torch.empty((A.m, n_frames), dtype=torch.float32, device="cuda")
    for f in range(n_frames):
        lam = R.spmv(R.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, (xt * torch.exp(-rates * f)).contiguous())
        Y[:, f] = torch.poisson(lam * (counts[f] / float(lam.double().sum())), generator=gen)
    h64, s16 = R.sensitivity_half(A)
    X = torch.full((n, n_frames), np.float32(1.0 / n), device="cuda")
    best, tile_ms = ctx.batch_autotune(A, Y, s16, X)
    kt = ctx.mlem_batch(A, Y, s16, X.clone(), 3, frame_tile=best, use_graph=False, kernel_times=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record()
    ctx.mlem_batch(A, Y, s16, X, niter, frame_tile=best, use_graph=True)
    ev[1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    rate = n_frames * niter / (ms / 1e3)
    # frame 0 against the FP64 iteration on its own
    s64, _ = R.sensitivity(A)
    x64 = torch.full((n,), 1.0 / n, dtype=torch.float64, device="cuda")
    ctx.mlem_f64(A, Y[:, 0].contiguous(), s64 / s64.sum(), x64, niter)
    d = X[:, 0].double() - x64
    fwd_ms, back_ms = float(kt[:, 0].mean()), float(kt[:, 1].mean())
    nnz, m = A.nnz, A.m
    out = {
        "frames": n_frames, "iterations": niter, "matrix": "fp16 (row-scaled), transpose in channel order",
        "frame_tile": best, "autotune_ms_per_iteration": {str(k): round(v, 3) for k, v in tile_ms.items()},
        "frame_iterations_per_s": rate, "ms_per_iteration_all_frames": ms / niter,
        "speedup_vs_plain_fp32_single_frame": rate / plain_iters_per_s,
        "passes_ms": {"forward": round(fwd_ms, 3), "back": round(back_ms, 3)},
        "matrix_gb_per_s": {"forward": round(nnz * 6 * (n_frames // best) / fwd_ms / 1e6, 1),
                            "back": round(nnz * 6 * (n_frames // best) / back_ms / 1e6, 1)},
        "gathered_gb_per_s": {"forward": round(nnz * n_frames * 4 / fwd_ms / 1e6, 1),
                              "back": round(nnz * n_frames * 4 / back_ms / 1e6, 1)},
        "frame0_vs_fp64": {"rel_l2": float(d.norm() / x64.norm()), "max_rel": float(d.abs().max() / x64.abs().max())},
        "data": "seeded per-voxel washout rates and log-uniform counts; Poisson via a seeded CUDA generator",
    }
    del A, Y, X
    gc.collect()
    torch.cuda.empty_cache()
    return out


def streamed_report(R, torch, ctx, w, lst, y_dev, fraction=0.25, niter=3):
    """The single-GPU form of the reference's chunked reconstruction
    (src/tests/reco.cu:226-275): raptr_mlem_stream with a resident budget of
    `fraction` of the full CSR's bytes, so that the other rows are rebuilt
    in every iteration; the sensitivity is computed in its first
    iteration.  Reports the steady iteration rate beside the resident one."""
    g = w["geom"]
    nnz_est = 3732681385 if g == cfg.FULL else None
    if nnz_est is None:
        A = ctx.build(lst, w["nrays"], SEED)
        nnz_est = A.nnz
        del A
        gc.collect()
    csr_bytes = nnz_est * 8 + (lst.numel() + 1) * 8
    budget = int(fraction * csr_bytes)
    x = torch.full((g.n_voxels,), np.float32(1.0 / g.n_voxels), device="cuda")
    st = ctx.mlem_stream(lst, w["nrays"], SEED, y_dev, None, x, niter, budget)
    return {"resident_budget_bytes": budget, "resident_fraction_of_csr": fraction, "iterations": niter,
            "resident_rows": st["resident_rows"], "streamed_rows": st["streamed_rows"],
            "first_iteration_ms": round(st["first_iter_ms"], 1), "iteration_ms": round(st["iter_ms"], 1),
            "mlem_iters_per_s": 1e3 / st["iter_ms"] if st["iter_ms"] > 0 else None,
            "note": "rows beyond the budget are rebuilt (rays walked again) and projected from the build's "
                    "staging in every iteration; the first iteration builds every row and the sensitivity"}


def serving_report(R, torch, rate_hz=20.0, window_s=8.0, budget_gb=120, seed=SEED + 500):
    """The serving form: Poisson arrivals at rate_hz for window_s seconds of
    reconstructions drawn from three geometries (40^3 x 2 mm / 5 angles,
    70^3 x 2 mm / 180 angles, 100^3 x 1.5 mm / 60 angles), counts
    log-uniform in [1e5, 1e8], iterations uniform in {10, 25, 50, 100}.
    Matrices are built by the server on first use (warmed before the
    window); latency is the server's submit-to-result time per request."""
    rng = np.random.default_rng(seed)
    kinds = [("small", cfg.WORKLOADS["small"]), ("full", cfg.WORKLOADS["full"]), ("fine", cfg.WORKLOADS["fine"])]
    per_kind = 6
    meas = {}
    t_syn = time.perf_counter()
    for name, w in kinds:
        g = w["geom"]
        ctx = R.Context(g, 0)
        lst = torch.arange(g.n_channels, dtype=torch.int32, device="cuda")
        A = ctx.build(lst, w["nrays"], SEED)
        xt = torch.from_numpy(cfg.phantom(g, w.get("rods", False))).cuda()
        lam = R.spmv(R.OP_N, A.m, A.n, A.row_ptr, A.col, A.val, xt)
        del A, ctx
        gc.collect()
        lam = lam / lam.double().sum().float()
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed + len(meas))
        meas[name] = []
        for _ in range(per_kind):
            counts = float(10 ** rng.uniform(5, 8))
            meas[name].append((counts, torch.poisson(lam * counts, generator=gen).cpu().numpy()))
        del lam
        torch.cuda.empty_cache()
    t_syn = time.perf_counter() - t_syn
    srv = R.Server(0, hbm_budget_bytes=int(budget_gb) << 30)
    warm = {}
    for name, w in sorted(kinds, key=lambda kv: -kv[1]["geom"].n_channels):
        g = w["geom"]
        rid = srv.submit(g, meas[name][0][1], 10, w["nrays"], SEED)
        _, st = srv.wait(rid, g.n_voxels)
        warm[name] = st["total_ms"]
    # arrivals
    n_req = rng.poisson(rate_hz * window_s)
    gaps = rng.exponential(1.0 / rate_hz, n_req)
    picks = rng.integers(0, len(kinds), n_req)
    which = rng.integers(0, per_kind, n_req)
    iters = rng.choice([10, 25, 50, 100], n_req)
    t0 = time.perf_counter()
    sub = []
    t_next = 0.0
    for i in range(n_req):
        t_next += gaps[i]
        dt = t0 + t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        name, w = kinds[int(picks[i])]
        counts, y = meas[name][int(which[i])]
        sub.append((name, w["geom"], int(iters[i]), srv.submit(w["geom"], y, int(iters[i]), w["nrays"], SEED)))
    results = []
    for name, g, it, rid in sub:
        _, st = srv.wait(rid, g.n_voxels)
        results.append((name, it, st))
    t_end = time.perf_counter()
    stats = srv.stats()
    srv.close()
    lat = np.array([st["total_ms"] for _, _, st in results])
    run = np.array([st["run_ms"] for _, _, st in results])
    frame_iters = sum(it for _, it, _ in results)
    by = {}
    for name, _ in kinds:
        l = np.array([st["total_ms"] for n_, _, st in results if n_ == name])
        if l.size:
            by[name] = {"requests": int(l.size), "p50_ms": float(np.percentile(l, 50)),
                        "p99_ms": float(np.percentile(l, 99))}
    return {
        "offered_req_per_s": rate_hz, "window_s": window_s, "requests": int(n_req),
        "completed_req_per_s": n_req / (t_end - t0), "frame_iterations_per_s": frame_iters / (t_end - t0),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p95": float(np.percentile(lat, 95)),
                       "p99": float(np.percentile(lat, 99)), "max": float(lat.max())},
        "run_ms": {"p50": float(np.percentile(run, 50)), "p99": float(np.percentile(run, 99))},
        "by_geometry": by, "warm_first_request_ms": warm,
        "server": {k: stats[k] for k in ("builds", "evictions", "batch_steps", "iterations")},
        "largest_batch": int(max(st["frames_max"] for _, _, st in results)),
        "hbm_budget_gb": budget_gb, "synthesis_s": t_syn,
        "accuracy": "batched FP16 iteration; equal alone and in the mix and within 1e-3 of FP64 (tests/test_gpu_server.py)",
    }


def main():
    args = parse_args()
    w = workload(args.workload)
    g = w["geom"]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    n_gpus = max(args.gpus, world)

    if args.impl == "reference":
        if rank != 0:
            return
        threads = os.cpu_count() or 1
        vals = []
        per_step_budget = max(4.0, 90.0 / max(args.steps + args.warmup, 1))
        for i in range(args.warmup + args.steps):
            r = cpu_job_rate(w, per_step_budget, threads)
            if i >= args.warmup:
                vals.append(r)
        v = statistics.mean(x["value"] for x in vals)
        base = vals[-1]
        out = {"metric": metric_name(w), "value": v, "unit": "MLEM iterations/s", "n_gpus": n_gpus,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * w["niter"] / v,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded ray sample of the same geometry)", "config": config_of(w, 1),
               "impl": "reference",
               "cpu_baseline": {"value": v, "unit": "MLEM iterations/s", "cores": base["cores"], "kind": base["kind"],
                                "sample": base["sample"]},
               "e2e": {"value": v, "unit": "MLEM iterations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
               "matrix_build_s": statistics.mean(x["matrix_build_s"] for x in vals)}
        print(json.dumps(out))
        return

    import torch

    import raptr_b200 as R

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as td

        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                              device_id=torch.device("cuda", local_rank))
        dist = td
    else:
        torch.cuda.set_device(local_rank)
    dev = torch.cuda.current_device()
    ctx = R.Context(g, dev)
    all_ch = np.arange(g.n_channels, dtype=np.int32)
    lo = rank * g.n_channels // world
    hi = (rank + 1) * g.n_channels // world
    lst = torch.from_numpy(all_ch[lo:hi]).cuda()
    y_full = synth_measurement(R, torch, ctx, w, lst, dist)
    y_dev = torch.from_numpy(y_full[lo:hi]).cuda()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        run_job(R, torch, ctx, w, lst, y_dev, dist)
    sampler = ClockSampler(gpu_id_for(torch, dev))
    sampler.start()
    launches0 = R.kernel_launches()
    barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("raptr_timed_steps")
    t_start.record()
    steps = [run_job(R, torch, ctx, w, lst, y_dev, dist) for _ in range(args.steps)]
    t_end.record()
    torch.cuda.nvtx.range_pop()
    barrier()
    launches = R.kernel_launches() - launches0
    clocks = sampler.stop()
    gc.collect()
    total_ms = t_start.elapsed_time(t_end)
    if dist is not None:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t)
    phase_keys = ("build_ms", "transpose_ms", "sens_ms", "mlem_ms")
    phases_per_step = [{k: round(s[k], 3) for k in phase_keys} for s in steps]
    phase = {k: statistics.mean(s[k] for s in steps) for k in phase_keys}
    if dist is not None:
        t = torch.tensor([phase[k] for k in sorted(phase)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        phase = dict(zip(sorted(phase), t.tolist()))
    ms_per_step = total_ms / args.steps
    value = w["niter"] / (ms_per_step / 1e3)
    nnz = steps[-1]["nnz"]
    m = steps[-1]["m"]
    if dist is not None:
        t = torch.tensor([nnz], dtype=torch.int64, device="cuda")
        dist.all_reduce(t)
        nnz_total = int(t)
    else:
        nnz_total = nnz

    out = {"metric": metric_name(w), "value": value, "unit": "MLEM iterations/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
           "scaling": "strong", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic (seeded phantom, Poisson counts, Philox rays)", "config": config_of(w, world),
           "matrix_build_s": phase["build_ms"] / 1e3,
           "phases_ms": {k: round(v, 3) for k, v in phase.items()}, "phases_ms_per_step": phases_per_step,
           "resident_mlem_iters_per_s": w["niter"] / (phase["mlem_ms"] / 1e3),
           "nnz": nnz_total, "gpu_launches": int(launches), "clocks": clocks}

    if rank == 0:
        # Roofline of the HBM-bound MLEM passes, from the per-kernel device
        # times of the timed steps.
        peak, peak_kind = measured_peaks()
        kts = np.concatenate([s["kernel_ms"] for s in steps if s["kernel_ms"] is not None])
        if np.all(np.isfinite(kts)):
            fwd_ms, back_ms = float(kts[:, 0].mean()), float(kts[:, 1].mean())
            n = g.n_voxels
            fwd_bytes = nnz * 8 + (m + 1) * 8 + m * 4 + m * 4 + n * 4
            back_bytes = nnz * 8 + (n + 1) * 8 + 3 * n * 4 + m * 4
            r_f = fwd_bytes / (fwd_ms / 1e3) / 1e9
            r_b = back_bytes / (back_ms / 1e3) / 1e9
            dom = ("mlem_back_kernel", r_b, back_bytes, back_ms) if back_ms >= fwd_ms else \
                ("mlem_forward_kernel", r_f, fwd_bytes, fwd_ms)
            out["roofline"] = {"bound": "hbm", "kernel": dom[0], "achieved": round(dom[1], 1), "peak": peak,
                               "unit": "GB/s", "frac": round(dom[1] / peak, 4), "peak_source": peak_kind,
                               "traffic": int(TRAFFIC_BYTES_PER_ENTRY[dom[0]] * nnz),
                               "traffic_source": "ncu DRAM bytes per entry of the kernel's profile case x entries",
                               "algorithmic_bytes": int(dom[2]), "launch_ms": round(dom[3], 4)}
            out["roofline_all"] = {
                "mlem_forward_kernel": {"achieved": round(r_f, 1), "frac": round(r_f / peak, 4),
                                        "bytes": int(fwd_bytes), "ms": round(fwd_ms, 4)},
                "mlem_back_kernel": {"achieved": round(r_b, 1), "frac": round(r_b / peak, 4),
                                     "bytes": int(back_bytes), "ms": round(back_ms, 4)},
            }
        out["build_throughput"] = {"rays_per_s": g.n_channels * w["nrays"] / (phase["build_ms"] / 1e3),
                                   "entries_per_s": nnz_total / (phase["build_ms"] / 1e3)}

    # End to end through the public C ABI from host buffers (rank 0, N=1).
    if not args.no_e2e and world == 1:
        times, sts, st = [], [], None
        R.reco_host(g, y_full, w["nrays"], SEED, w["niter"], device=dev)  # warm-up, untimed
        for _ in range(max(1, min(args.steps, 3))):
            t0 = time.perf_counter()
            x_h, st = R.reco_host(g, y_full, w["nrays"], SEED, w["niter"], device=dev)
            times.append(time.perf_counter() - t0)
            sts.append(st)
        e2e_s = statistics.mean(times)
        out["e2e"] = {"value": w["niter"] / e2e_s, "unit": "MLEM iterations/s",
                      "h2d_bytes_per_step": int(st["h2d_bytes"]), "d2h_bytes_per_step": int(st["d2h_bytes"]),
                      "wall_s": e2e_s, "build_ms": st["build_ms"], "iter_ms": st["iter_ms"],
                      "phases_ms": {k: round(st[k], 3) for k in ("setup_ms", "inputs_ms", "build_ms", "transpose_ms",
                                                                 "sens_ms", "iter_ms", "output_ms", "release_ms",
                                                                 "wall_ms")},
                      "calls": [{"wall_s": round(t, 4),
                                 **{k: round(c[k], 3) for k in ("build_ms", "transpose_ms", "sens_ms", "iter_ms",
                                                                "release_ms", "wall_ms")}}
                                for t, c in zip(times, sts)],
                      "streamed_rows": int(st["streamed_rows"])}
    if rank == 0 and world == 1 and not args.no_forms:
        peak, _ = measured_peaks()
        out["forms"] = {"precision": precision_report(R, torch, ctx, w, lst, y_dev, peak)}
        out["forms"]["batched"] = batch_report(R, torch, ctx, w, lst, out["resident_mlem_iters_per_s"], peak)
        out["forms"]["streamed"] = streamed_report(R, torch, ctx, w, lst, y_dev)
        del lst, y_dev
        gc.collect()
        torch.cuda.empty_cache()
        out["forms"]["serving"] = {"offered_20_per_s": serving_report(R, torch, rate_hz=20.0, window_s=30.0),
                                   "offered_8_per_s": serving_report(R, torch, rate_hz=8.0, window_s=20.0)}
    if rank == 0 and world == 1:
        out["cpu_baseline"] = {k: v for k, v in cpu_job_rate(w, args.cpu_sample_s, os.cpu_count() or 1).items()
                               if k != "matrix_build_s"}
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
