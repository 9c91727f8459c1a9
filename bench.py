#!/usr/bin/env python
"""Benchmark: MBIR slice-iterations/s on the full-volume workload.

Workload (one GPU): 256 slices of 2048 x 2048 float32, a seeded 3-D foam
phantom (2000 spheres, r in [5, 60] px, density 1 in a 0.2 cylinder), 1969
angles on [0, pi), 2048 detector pixels, Poisson noise at 1e4 counts; qGGMRF
prior p = 1.2, sigma = 100 (the reference's default smoothness 0.01), the
reference's Nesterov/backtracking iteration.  A step is one MBIR iteration
over the whole volume (inputs of 4.3 GB per array, larger than L2).

Warm-up (untimed): W steps with the graph, W with the host loop, max(W, 30)
more with the graph; then exactly K timed steps of each form.  The two forms run the
same kernels; if the graph's K steps take more than 1.15 x the host loop's,
the graph region is timed once more and config.graph_retimed records the
first time (see the comment at the check).

Lines reported by rank 0 (one JSON line):
  value      slice-iterations/s of the graph-captured device solver
             (tc_mbir_solve), max over ranks, CUDA events
  plain      the same solve driven from the host one attempt at a time
  per_slice  the plain per-slice form: one slice pair per Toeplitz launch,
             host-driven loop
  e2e        cTomocam.mbir (the reference binding's call) on pinned host
             buffers with the workload's 50 iterations: normalisation, FBP
             guess, centring/padding to 2908^2, A^T y, PSF, the iterations
             and the copies, wall clock; timed after one untimed call of 3
             iterations (the process's first call meets the device
             allocations of the 2908^2 sizes, reported as e2e.warmup_call)
  roofline   Toeplitz operator (the dominant kernels) achieved GB/s on its
             algorithmic bytes, against the measured HBM copy peak
  cpu_baseline  the FP64 oracle port of the same iteration on host cores

--impl reference: the reference arm times the reference's algorithm on the
host cores, through the project's FP64 CPU restatement (oracle/, pinned to
the reference's own run2, pre/post-processing and prior).  The reference's
full GPU build needs cuFINUFFT, HDF5 and TBB, absent on these machines; its
GPU sources built with an exact-DFT stand-in for cuFINUFFT are timed beside
the product by oracle/compare_gpu.py, not by this bench.

Multi-GPU (torchrun): every rank reconstructs an independent volume
(replicas; the MBIR path of one volume is one GPU), value = all ranks'
slice-iterations / max-over-ranks time, scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MBIR slice-iters/s, 2048², batched vs plain, rel.err≤1e-4 vs FP64; % HBM peak"
UNIT = "slice-iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slices", type=int, default=256)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--nproj", type=int, default=1969)
    ap.add_argument("--spheres", type=int, default=2000)
    ap.add_argument("--sigma", type=float, default=100.0)
    ap.add_argument("--e2e-iters", type=int, default=50)  # the workload's iteration count
    ap.add_argument("--cpu-slices", type=int, default=2)
    ap.add_argument("--cpu-iters", type=int, default=2)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-plain", action="store_true")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("timestamp,pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "clocks.mem")

    def __init__(self, bus_id: str):
        self.bus = bus_id.lower()
        self.proc = None
        # the raw samples; TC_CLOCKS_CSV keeps them at a chosen path
        self.path = os.environ.get("TC_CLOCKS_CSV") or os.path.join(
            tempfile.gettempdir(), f"tomocam_b200_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.5)
        except Exception:
            self.proc = None

    def mark(self):
        return time.time()

    def stop(self, t0, t1):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mem, mx, reasons = [], [], None, set()
        from datetime import datetime
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            if self.bus and self.bus[-12:] not in parts[1].lower():
                continue
            if ts < t0 - 0.15 or ts > t1 + 0.15:
                continue
            sm.append(float(parts[2]))
            mx = float(parts[3])
            if len(parts) > 10:
                try:
                    mem.append(float(parts[10]))
                except ValueError:
                    pass
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, parts[6:10]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "mem_mhz": float(np.median(mem)) if mem else None,
                "mem_min_mhz": float(np.min(mem)) if mem else None}


def bus_id_of(dev):
    import torch
    p = torch.cuda.get_device_properties(dev)
    try:
        return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
    except AttributeError:
        return ""


def profiled_traffic(kernel, n, m=0):
    """DRAM bytes per slice of a kernel from profiles/traffic.json (numbers
    taken from committed ncu captures), or None when none matches."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            table = json.load(f)
        for e in table.get(kernel, []):
            if int(e["n"]) == n and int(e.get("m", 0)) == m:
                return float(e["bytes_per_slice"])
    except (OSError, ValueError, KeyError, TypeError):
        pass
    return None


# ---------------------------------------------------------------------------
# the CPU arm: the oracle port of the iteration on host cores
# ---------------------------------------------------------------------------
def cpu_iteration_rate(n, nproj, sino_slices, aty, x0, sigma, iters, warm=1, tol=1e-6):
    """slice-iters/s of oracle.run2 on the given slices; returns (rate, seconds, sample)."""
    from oracle import oracle as O
    ang = np.arange(nproj) * (np.pi / nproj)
    psf = O.psf_kernel(n, ang.astype(np.float32).astype(np.float64), "es", tol)
    sino_sq = float(np.sum(np.asarray(sino_slices, np.float64) ** 2))
    step, _ = O.lipschitz_step(psf, n)
    aty = np.asarray(aty, np.float64)

    def grad_fn(v):
        return O.gradient2(v, aty, psf) + O.qggmrf_grad(v, sigma, 1.2)

    def err_fn(v):
        return math.sqrt(O.function_value2(v, aty, psf, sino_sq))

    x = np.asarray(x0, np.float64)
    if warm:
        x = O.run2(x, warm, step, grad_fn, err_fn)
    t0 = time.perf_counter()
    O.run2(x, iters, step, grad_fn, err_fn)
    dt = time.perf_counter() - t0
    S = aty.shape[0]
    return S * iters / dt, dt, f"{S} slices of {n}x{n}, {nproj} angles, {iters} iterations (FP64)"


def reference_arm(a):
    """Times the CPU restatement of the reference's MBIR iteration (oracle/)."""
    from oracle import oracle as O
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n, P, S = a.n, a.nproj, a.cpu_slices
    ang = (np.arange(P) * (np.pi / P)).astype(np.float32)
    a64 = ang.astype(np.float64)
    img = np.stack([O.ellipse_phantom(n, 10, s) for s in range(S)])
    sino = O.project(img, a64, "es", 1e-6)
    sino = sino / sino.max()
    aty = O.backproject(sino, a64, False, "es", 1e-6)
    x0 = O.backproject(sino, a64, True, "es", 1e-6)
    from oracle import oracle as O2  # noqa: F401  (same module; kept explicit for readers)
    psf = O.psf_kernel(n, a64, "es", 1e-6)
    sino_sq = float(np.sum(sino ** 2))
    step, _ = O.lipschitz_step(psf, n)

    def grad_fn(v):
        return O.gradient2(v, aty, psf) + O.qggmrf_grad(v, a.sigma, 1.2)

    def err_fn(v):
        return math.sqrt(O.function_value2(v, aty, psf, sino_sq))

    x = O.run2(x0, a.warmup, step, grad_fn, err_fn) if a.warmup > 0 else x0
    times = []
    for _ in range(a.steps):
        t0 = time.perf_counter()
        x = O.run2(x, 1, step, grad_fn, err_fn)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    value = S * a.steps / tot
    cores = os.cpu_count()
    sample = f"{S} slices of {n}x{n}, {P} angles; one MBIR iteration per step (FP64 numpy/scipy + OpenMP C)"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * tot / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded ellipse phantoms)",
        "config": {"workload": f"full-volume MBIR sample: {S}x{n}x{n}, {P} angles",
                   "note": "reference GPU build unavailable (cuFINUFFT/HDF5/TBB absent); "
                           "CPU restatement of the reference algorithm (oracle/) timed instead"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def main():
    a = parse()
    if a.impl == "reference":
        reference_arm(a)
        return
    import torch

    from tomocam_b200.replicas import Replicas
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ranks = Replicas("nccl", dev)
    world, rank = ranks.world, ranks.rank

    from tomocam_b200 import cTomocam, phantom
    from tomocam_b200.plan import Plan

    S, n, P = a.slices, a.n, a.nproj
    ang = (np.arange(P) * (np.pi / P)).astype(np.float32)

    # ---- synthetic inputs (untimed) --------------------------------------
    vol = phantom.foam_volume(S, n, a.spheres, seed=rank, device=dev)
    pl = Plan(n, ang)
    sino = pl.radon(vol)
    del vol
    sino = phantom.transmission_noise(sino, 1e4, 3.0, seed=rank)
    sino_host = None
    if not a.skip_e2e:
        sino_host = torch.empty(sino.shape, dtype=torch.float32, pin_memory=True)
        sino_host.copy_(sino)
    sino.div_(sino.max())                       # mbir2 normalisation
    aty = pl.iradon(sino)
    x0 = pl.iradon(sino, ramp=True)
    sino_sq = float((sino.double() ** 2).sum())
    cpu_inputs = None
    if rank == 0 and world == 1 and not a.skip_cpu:
        k = a.cpu_slices
        cpu_inputs = (sino[:k].cpu().numpy(), aty[:k].cpu().numpy(), x0[:k].cpu().numpy())
    del sino
    torch.cuda.synchronize()

    barrier = ranks.barrier
    max_over_ranks = ranks.max_over_ranks

    def timed_solve(iters, graph, plan=None):
        plan = pl if plan is None else plan
        x = x0.clone()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        x, hist = plan.mbir_solve(aty, sino_sq, x, iters, a.sigma, 1.2, use_graph=graph, inplace=True)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1), hist, x

    # warm-up: W steps of the graph and of the plain path, then at least 30
    # more of the graph right before its timed region: in a fresh process
    # the first second or so of this load runs slower (measured: 3-step regions
    # at 40-42 ms per step, the first 20-step region 2 % slower than every
    # later one, graph or host loop alike)
    timed_solve(a.warmup, True)
    if not a.skip_plain:
        timed_solve(a.warmup, False)
    timed_solve(max(a.warmup, 30), True)

    clocks = ClockSampler(bus_id_of(dev))
    clocks.start()
    t_wall0 = time.time()
    ms, hist, xg = timed_solve(a.steps, True)
    t_wall1 = time.time()
    clk = clocks.stop(t_wall0, t_wall1)
    ms = max_over_ranks(ms)
    value = ranks.aggregate_rate(S * a.steps, ms / 1e3)
    attempts = int(hist[:, 2].sum())
    finite = bool(np.all(np.isfinite(hist[:, 0])))

    plain = None
    if not a.skip_plain:
        ms_p, _, xp = timed_solve(a.steps, False)
        ms_p = max_over_ranks(ms_p)
        plain = {"value": ranks.aggregate_rate(S * a.steps, ms_p / 1e3), "unit": UNIT, "ms_per_step": ms_p / a.steps,
                 "identical_to_graph": bool(torch.equal(xg, xp))}
        del xp
    # The graph-driven and host-driven solves run the same kernels on the same
    # data (their results are compared bit for bit above); a graph region more
    # than 15 % slower than the host region was disturbed (the GPU has been
    # seen partly idle during one such region), so it is timed
    # once more and the first time is reported beside the second.
    graph_retimed = None
    if plain is not None and ms > 1.15 * ms_p:
        first = ms
        clocks = ClockSampler(bus_id_of(dev))
        clocks.start()
        t_wall0 = time.time()
        ms, _, xg2 = timed_solve(a.steps, True)
        t_wall1 = time.time()
        clk = clocks.stop(t_wall0, t_wall1)
        del xg2
        ms = max_over_ranks(ms)
        value = ranks.aggregate_rate(S * a.steps, ms / 1e3)
        graph_retimed = {"first_ms_per_step": first / a.steps,
                         "rule": "graph region > 1.15 x host-loop region: timed once more"}
    # the plain per-slice form: the same iteration with every Toeplitz launch
    # covering one slice pair (chunks of two slices) and the loop on the host
    per_slice = None
    if not a.skip_plain:
        ps = Plan(n, ang, max_batch=2)
        timed_solve(a.warmup, False, ps)
        ms_s, _, xs_ = timed_solve(a.steps, False, ps)
        ms_s = max_over_ranks(ms_s)
        per_slice = {"value": ranks.aggregate_rate(S * a.steps, ms_s / 1e3), "unit": UNIT,
                     "ms_per_step": ms_s / a.steps, "toeplitz_pairs_per_launch": ps.info["toeplitz_pairs"],
                     "loop": "host",
                     "max_rel_diff_vs_batched": float((xs_ - xg).norm() / xg.norm())}
        del xs_
        ps.close()
    del xg

    # ---- roofline of the Toeplitz operator -----------------------------------
    # timed as the solver runs it (H x with the x.Hx dot, no A^T y), over the
    # same volume, with CUDA events on the stream the library launches on
    from tomocam_b200 import bytes_model
    info = pl.info
    M = info["toeplitz_m"]
    pairs_per_chunk = max(1, int(info["toeplitz_pairs"]))
    chunks = math.ceil(S / (2 * pairs_per_chunk))
    g = torch.empty_like(aty)
    pl.toeplitz_grad(x0, None, out=g, dots=True)
    reps = 3
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        pl.toeplitz_grad(x0, None, out=g, dots=True)
    e1.record()
    torch.cuda.synchronize()
    t_op = e0.elapsed_time(e1) / reps / 1e3
    del g
    slices_per_psf = min(S, 2 * pairs_per_chunk)
    bytes_slice = bytes_model.toeplitz(n, M, slices_per_psf)
    bytes_launch = bytes_slice * S / chunks          # one launch triple per chunk
    t_launch = t_op / chunks
    peak, peak_kind = peaks()
    achieved = bytes_launch / t_launch / 1e9
    traffic = profiled_traffic("toeplitz_passes", n, M)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak,
                "traffic": None if traffic is None else traffic * S / chunks,
                "kernel": ("Toeplitz operator, 3 passes (k_tpf_rows, k_tpf_cols, k_tpf_out)"
                           if info["toeplitz_fast"] else
                           "Toeplitz operator, 3 passes (k_tp_rows, k_tp_cols, k_tp_out)"),
                "launch": f"one launch triple per chunk of {2 * pairs_per_chunk} slices, "
                          "as the solver runs it (H x and the FP64 x.Hx dot)",
                "bytes_per_slice": bytes_slice, "peak_kind": f"{peak_kind} HBM copy",
                "ms_per_slice": 1e3 * t_op / S,
                "compulsory_frac": (bytes_model.compulsory(n) * S / t_op / 1e9) / peak,
                "traffic_source": "ncu dram__bytes_read+write of the three passes "
                                  "(profiles/traffic.json), scaled per launch triple"}
    # ---- the fused update kernel, timed in place -------------------------------
    # host-driven attempts with CUDA events around each k_mbir_update launch
    ph = np.zeros(4, np.float64)
    xu = x0.clone()
    pl.mbir_solve(aty, sino_sq, xu, 2, a.sigma, 1.2, use_graph=False, inplace=True, phase_ms=ph)
    del xu
    t_upd = ph[0] / max(ph[3], 1.0) / 1e3          # seconds per launch
    upd_bytes = bytes_model.update(n, same=True)     # every attempt here follows an acceptance
    upd_traffic = profiled_traffic("mbir_update", n)
    update_roofline = {"bound": "hbm", "kernel": "k_mbir_update (fused qGGMRF stencil + Nesterov "
                       "update, x = sol form)", "achieved": upd_bytes * S / t_upd / 1e9,
                       "peak": peak, "unit": "GB/s", "ms_per_launch": 1e3 * t_upd,
                       "bytes_per_slice": upd_bytes, "peak_kind": f"{peak_kind} HBM copy",
                       "traffic": None if upd_traffic is None else upd_traffic * S,
                       "toeplitz_ms_per_attempt": ph[1] / max(ph[3], 1.0),
                       "step_test_ms_per_attempt": ph[2] / max(ph[3], 1.0),
                       "attempts_timed": int(ph[3])}
    update_roofline["frac"] = update_roofline["achieved"] / peak
    # whole iteration against its algorithmic bytes (update + one Toeplitz)
    it_bytes = bytes_model.iteration(n, M, slices_per_psf)
    iteration_roofline = {"bytes_per_slice_iter": it_bytes,
                          "achieved": it_bytes * S * a.steps / (ms / 1e3) / 1e9,
                          "unit": "GB/s"}
    iteration_roofline["frac"] = iteration_roofline["achieved"] / peak

    # ---- kernel launches inside the timed region -----------------------------
    # begin, the two update forms (one returns at once), decide and 3 passes per chunk
    gpu_launches = attempts * (4 + 3 * chunks)

    # ---- end to end through the reference binding ------------------------------
    e2e = None
    del aty, x0
    pl.close()
    torch.cuda.empty_cache()
    if not a.skip_e2e and sino_host is not None:
        # warm-up call (untimed): the first call in a process allocates the
        # padded grid's buffers, which the device memory cache then keeps
        barrier()
        torch.cuda.synchronize()
        warm_iters = min(3, a.e2e_iters)
        t0 = time.perf_counter()
        out = cTomocam.mbir(sino_host.numpy(), ang, (n - 1) / 2.0 + 0.5, warm_iters, a.sigma, 1e-4, 1e-4)
        torch.cuda.synchronize()
        warm_dt = max_over_ranks(time.perf_counter() - t0)
        del out
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = cTomocam.mbir(sino_host.numpy(), ang, (n - 1) / 2.0 + 0.5, a.e2e_iters, a.sigma, 1e-4, 1e-4)
        torch.cuda.synchronize()
        dt = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": ranks.aggregate_rate(S * a.e2e_iters, dt), "unit": UNIT,
               "h2d_bytes_per_step": int(sino_host.numel() * 4), "d2h_bytes_per_step": int(out.nbytes),
               "iterations_per_step": a.e2e_iters, "seconds": dt,
               "grid": f"{out.shape[1]}x{out.shape[2]} output, iterated on the reference's padded "
                       f"{n + 2 * (int(0.42 * n) // 2)}^2 grid",
               "includes": "H2D sinogram, normalisation, FBP guess, centring/padding, A^T y, "
                           "FP64 PSF, Lipschitz step, iterations, crop, D2H",
               "warmup_call": {"iterations": warm_iters, "seconds": warm_dt}}
        del out

    # ---- CPU baseline (rank 0, one GPU) ----------------------------------------
    cpu = None
    if cpu_inputs is not None:
        rate, dt, sample = cpu_iteration_rate(n, P, cpu_inputs[0], cpu_inputs[1], cpu_inputs[2],
                                              a.sigma, a.cpu_iters)
        cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": sample + f"; {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 3-D foam phantom, Poisson noise at 1e4 counts)",
            "config": {"workload": f"full-volume MBIR: {S} slices {n}x{n}, {P} angles, "
                                   f"{n} detector pixels, qGGMRF p=1.2 sigma={a.sigma:g}",
                       "solver": "graph-captured device loop (tc_mbir_solve)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (4.3 GB per volume array)",
                       "attempts": attempts, "finite": finite, "graph_retimed": graph_retimed},
            "plain": plain, "per_slice": per_slice, "e2e": e2e, "roofline": roofline,
            "iteration_roofline": iteration_roofline, "update_roofline": update_roofline,
            "cpu_baseline": cpu,
            "clocks": clk, "gpu_launches": gpu_launches,
        }
        print(json.dumps(line), flush=True)
    ranks.close()


if __name__ == "__main__":
    main()
