#!/usr/bin/env python
"""Benchmark: 50-PC randomized PCA of a 1,000,000 x 2,000 sparse CSR on B200.

Workload (seeded synthetic stand-in for a census-scale log-normalised HVG
matrix): negative-binomial counts, ~10 % density (~2.1e8 nonzeros),
log1p(1e4 * count / rowsum) values, n_comps=50, n_oversamples=10,
4 power iterations, implicit centring plus per-gene unit-variance scaling
clipped at 10.  One step = one complete PCA (plan run) on the resident matrix.

Headline ``value``: ms per PCA in BF16-mixed precision (values streamed as
BF16, FP32 accumulation, FP64 Gram/Cholesky/SVD); the strict FP32 path is
timed on the same workload alongside (``fp32``) with the singular-value
agreement between the two.  ``e2e``: the same PCA through the one-shot C ABI
call with host (pinned) CSR buffers, upload and embedding download included.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (the path has no collective), one process
per GPU under torchrun; the step time is the max over ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

N_OBS = 1_000_000
N_VARS = 2_000
LOC = -3.0
DISPERSION = 0.3
SEED = 0
N_COMPS = 50
N_OVERSAMPLES = 10
N_POWER = 4
CLIP = 10.0
METRIC = "1M x 2k-gene rPCA (50 PCs) ms per PCA, BF16-mixed (FP32 path alongside)"
FALLBACK_HBM_GBS = 6650.0

# DRAM bytes per stored nonzero of the two product kernels, from one ncu
# capture at 250,000 x 2,000 (profiles/spmm_tc_250k_full.txt:
# dram__bytes_read.sum + dram__bytes_write.sum of one launch / its 57,193,010
# nonzeros).  Traffic grows in proportion to the nonzeros at fixed density, so
# the figure scales to the bench workload.
NCU_TRAFFIC_BYTES_PER_NNZ = {"transpose": 5.210, "forward": 6.134}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n-obs", type=int, default=N_OBS)
    ap.add_argument("--mode", choices=["mixed_bf16", "mixed_f16", "strict_fp32"], default="mixed_bf16")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32 comparison leg")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-rows", type=int, default=None,
                    help="rows of the CPU-baseline sample (default: all rows for ours, 50,000 for --impl reference)")
    ap.add_argument("--no-backward", action="store_true", help="skip the differentiable-PCA leg")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched sub-PCA leg")
    ap.add_argument("--no-stream", action="store_true", help="skip the streamed (out-of-VRAM) leg")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# process group (replicas) helpers
# ---------------------------------------------------------------------------

def dist_setup(backend: str):
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, 0
    from datetime import timedelta

    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=timedelta(seconds=300))
    return dist.get_rank(), world, int(os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(x: float, device=None) -> float:
    """Max of a scalar over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(device=None):
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[3:7]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# algorithmic bytes
# ---------------------------------------------------------------------------

def bytes_of_a(nnz: int, n: int, s_v: int) -> int:
    return nnz * (s_v + 4) + 8 * (n + 1)


def kernel_bytes(stage: str, nnz: int, n: int, g: int, k: int, s_v: int) -> int:
    """Algorithmic bytes of one launch: the matrix once, the tall operand once."""
    a = bytes_of_a(nnz, n, s_v)
    if stage == "forward":     # read A and V, write Y (n x k FP32)
        return a + 4 * g * k + 4 * n * k
    if stage == "transpose":   # read A and Q (n x k FP32), write Z (g x k)
        return a + 4 * n * k + 4 * g * k
    raise ValueError(stage)


def pca_bytes(nnz: int, n: int, k: int, c: int, q: int, s_v: int) -> int:
    """Executed-pass algorithmic bytes of one PCA on the resident matrix.

    (q+1) forward products (read A, write Y) + (q+1) transposed products (read
    A and Q) + (q+2) tall Gram reads + the explicit Q formation (read + write)
    + the embeddings (read Q, write n x c).  Statistics and the value transform
    run once at plan creation and are not part of a step.
    """
    a = bytes_of_a(nnz, n, s_v)
    tall = 4 * n * k
    return ((q + 1) * (a + tall) + (q + 1) * (a + tall) + (q + 2) * tall + 2 * tall
            + tall + 4 * n * c)


# ---------------------------------------------------------------------------
# CPU baseline: the multithreaded C++ restatement of the reference's CPU path
# ---------------------------------------------------------------------------

def cpu_baseline(indptr, indices, values, n_full: int, rows: int, threads: int):
    import numpy as np

    from oracle import build_cpu, rpca

    rows = min(rows, len(indptr) - 1)
    ip = np.ascontiguousarray(indptr[: rows + 1], dtype=np.int64)
    nnz = int(ip[-1])
    ix = np.ascontiguousarray(indices[:nnz])
    vv = np.ascontiguousarray(values[:nnz], dtype=np.float32)
    k = N_COMPS + N_OVERSAMPLES
    om = rpca.gaussian_omega(N_VARS, k, SEED)
    build_cpu.load()
    t0 = time.perf_counter()
    res = build_cpu.run(ip, ix, vv, (rows, N_VARS), N_COMPS, k, N_POWER, om, zero_center=True,
                        scale=True, clip_max=CLIP, threads=threads)
    dt = time.perf_counter() - t0
    return dt * 1e3 * (n_full / rows), nnz, dt, res


SUBSAMPLE_ROWS = 50_000


def precision_report(ours: dict, fp64_full: dict | None, sub_ours: dict, sub_csr) -> dict:
    """Singular-value and principal-angle error of the GPU results against the
    FP64 randomized result on the whole matrix (the C++ restatement, same
    seeded Omega) and against the exact FP64 PCA of a 50,000-cell subsample
    (dense Gram eigendecomposition of the same scaled, clipped, centred
    matrix).  Checker only: nothing here is timed."""
    import numpy as np

    from oracle import rpca

    def cmp(sv, comps, ref_sv, ref_comps):
        sv = np.asarray(sv, dtype=np.float64)
        rel = np.abs(sv - ref_sv) / ref_sv
        a = np.asarray(comps, dtype=np.float64).T
        b = np.asarray(ref_comps, dtype=np.float64).T
        ang = rpca.per_component_angles(a, b)
        return {"sigma_max_rel_err": float(rel.max()), "sigma_max_rel_err_top10": float(rel[:10].max()),
                "angle_max_rad_top10": float(ang[:10].max()),
                "subspace_angle_max_rad_top50": float(rpca.principal_angles(a, b).max())}

    out = {}
    if fp64_full is not None:
        out["vs_fp64_randomized_full"] = {m: cmp(r["sv"], r["comps"], fp64_full["singular_values"],
                                                 fp64_full["components"]) for m, r in ours.items()}
    ip, ix, vv = sub_csr
    n = len(ip) - 1
    csr = rpca.Csr(ip, ix, vv, (n, N_VARS))
    p, _, _, _ = rpca.scale_values(csr, CLIP, True)
    dense = np.zeros((n, N_VARS))
    rows = np.repeat(np.arange(n), np.diff(ip))
    np.add.at(dense, (rows, ix.astype(np.int64)), p)
    dense -= dense.mean(axis=0, keepdims=True)
    lam, vec = np.linalg.eigh(dense.T @ dense)
    order = np.argsort(lam)[::-1][:N_COMPS]
    ex_sv, ex_comps = np.sqrt(np.maximum(lam[order], 0.0)), vec[:, order].T
    out["subsample_vs_exact_fp64"] = {m: cmp(r["sv"], r["comps"], ex_sv, ex_comps) for m, r in sub_ours.items()}
    # the FP64 randomized PCA of the subsample (same Omega) separates the
    # algorithm's own error (q power iterations on a flat spectrum) from the
    # arithmetic's
    from oracle import build_cpu
    sub64 = build_cpu.run(ip, ix, vv, (n, N_VARS), N_COMPS, N_COMPS + N_OVERSAMPLES, N_POWER,
                          rpca.gaussian_omega(N_VARS, N_COMPS + N_OVERSAMPLES, SEED), zero_center=True,
                          scale=True, clip_max=CLIP, threads=os.cpu_count() or 1)
    out["subsample_vs_fp64_randomized"] = {m: cmp(r["sv"], r["comps"], sub64["singular_values"],
                                                  sub64["components"]) for m, r in sub_ours.items()}
    out["subsample_fp64_randomized_vs_exact"] = cmp(sub64["singular_values"], sub64["components"], ex_sv,
                                                    ex_comps)
    out["subsample"] = f"first {n:,} rows of the same matrix ({len(ix):,} nnz); exact PCA by dense FP64 Gram eigh"
    return out


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def base_config(n_obs, nnz, mode, world):
    return {
        "workload": f"randomized PCA of a {n_obs:,} x {N_VARS:,} NB-synthetic CSR "
                    f"(50 PCs, oversample 10, 4 power iterations, centred + unit-variance "
                    f"scaled, clip 10)",
        "n_obs": n_obs, "n_vars": N_VARS, "nnz": nnz,
        "density": round(nnz / (n_obs * N_VARS), 4),
        "n_components": N_COMPS, "n_oversamples": N_OVERSAMPLES,
        "n_power_iterations": N_POWER, "values": mode, "qr_method": "cholesky",
        "generator": f"NB: mu_g~LogNormal({LOC},1.5), s_c~LogNormal(0,0.5), dispersion 0.3, seed {SEED}",
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "l2": "inputs larger than L2 (CSR >> 126 MB); no flush needed",
    }


def run_ours(args):
    import numpy as np
    import torch

    from scx_b200 import accel

    rank, world, local = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n_obs = args.n_obs
    ip, ix, vv = accel.synth_nb_csr_device(n_obs, N_VARS, seed=SEED, loc=LOC,
                                           dispersion=DISPERSION, device=local)
    nnz = int(ix.numel())
    stream = torch.cuda.Stream(device=dev)
    s_v = 4 if args.mode == "strict_fp32" else 2

    def make_plan(mode):
        return accel.Plan(ip, ix, vv, (n_obs, N_VARS), n_components=N_COMPS,
                          n_oversamples=N_OVERSAMPLES, n_power_iterations=N_POWER,
                          zero_center=True, scale=True, clip_max=CLIP, seed=SEED,
                          qr_method="cholesky", math_mode=mode, device=local,
                          stream=stream.cuda_stream)

    def timed(plan, steps, warmup, sample_clocks):
        """The timed steps run as the library runs a repeated plan (the
        recorded graph of the run, replayed); then the same number of steps
        with stage profiling on (plain launches, CUDA events around every
        stage on the plan's stream) give the stage shares and per-kernel
        launch times."""
        emb = torch.empty((n_obs, N_COMPS), dtype=torch.float32, device=dev)
        res = None
        for _ in range(warmup):
            res = plan.run(embeddings_out=emb)
        launches0 = plan.profile()["kernel_launches"]
        barrier(dev)
        torch.cuda.synchronize(dev)
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            res = plan.run(embeddings_out=emb)
        end.record(stream)
        torch.cuda.synchronize(dev)
        clocks = sampler.stop() if sampler else None
        barrier(dev)
        ms = start.elapsed_time(end) / steps
        launches = plan.profile()["kernel_launches"] - launches0  # our kernels in the timed steps
        plan.set_profiling(True)
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(steps):
            plan.run(embeddings_out=emb)
        p1.record(stream)
        torch.cuda.synchronize(dev)
        prof = plan.profile()
        prof["profiled_ms"] = p0.elapsed_time(p1) / steps
        prof["timed_launches"] = launches
        return ms, res, prof, clocks

    plan = make_plan(args.mode)
    k = plan.k
    ms, res, prof, clocks = timed(plan, args.steps, args.warmup, True)
    ms_max = max_over_ranks(ms, dev)
    plan.close()

    out = {
        "metric": METRIC, "value": None, "unit": "ms", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {"mixed_bf16": "bf16", "mixed_f16": "f16", "strict_fp32": "f32"}[args.mode],
        "data": "synthetic (seeded negative-binomial CSR generated on device)",
        "config": base_config(n_obs, nnz, args.mode, world),
    }
    out["ms_per_step"] = round(ms_max, 4)
    out["eig_sweeps"] = int(res.eig_sweeps)
    out["value"] = round(ms_max / world, 4)
    out["value_is"] = ("the job's time per PCA: ms_per_step (the slowest replica's step, one whole PCA per GPU) "
                       f"/ {world} replica(s)")

    # roofline of the dominant kernel, from the live stage timing of the timed region
    peak, peak_kind = measured_hbm_peak()
    stages = prof["stages"]
    dom = max(("forward", "transpose"), key=lambda s: stages[s]["device_ms"])
    launch_ms = stages[dom]["device_ms"] / max(stages[dom]["launches"], 1)
    kb = kernel_bytes(dom, nnz, n_obs, N_VARS, k, s_v)
    achieved = kb / (launch_ms * 1e-3) / 1e9
    traffic = NCU_TRAFFIC_BYTES_PER_NNZ.get(dom)
    out["roofline"] = {
        "bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
        "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
        "traffic": int(traffic * nnz) if traffic else None,
        "algorithmic_bytes_per_launch": kb, "launch_ms": round(launch_ms, 4),
    }
    total_ms = sum(v["device_ms"] for v in stages.values())
    out["stage_share"] = {s: round(v["device_ms"] / total_ms, 4) for s, v in stages.items()
                          if v["launches"]}
    pb = pca_bytes(nnz, n_obs, k, N_COMPS, N_POWER, s_v)
    out["pca_hbm"] = {"algorithmic_bytes": pb, "gbs": round(pb / (ms_max * 1e-3) / 1e9, 1),
                      "frac": round(pb / (ms_max * 1e-3) / 1e9 / peak, 4)}
    out["gpu_launches"] = int(prof["timed_launches"])
    out["profiled_ms_per_step"] = round(prof["profiled_ms"], 4)
    out["clocks"] = clocks
    sv_main = np.asarray(res.singular_values)

    if not args.no_fp32 and args.mode != "strict_fp32":
        p32 = make_plan("strict_fp32")
        ms32, res32, prof32, _ = timed(p32, max(2, args.steps // 2), 2, False)
        ms32 = max_over_ranks(ms32, dev)
        p32.close()
        sv32 = np.asarray(res32.singular_values)
        comps32 = np.asarray(res32.components)
        st32 = prof32["stages"]
        tot32 = sum(v["device_ms"] for v in st32.values())
        kern32 = {}
        for stg in ("forward", "transpose"):
            lm = st32[stg]["device_ms"] / max(st32[stg]["launches"], 1)
            kb32 = kernel_bytes(stg, nnz, n_obs, N_VARS, k, 4)
            kern32[stg] = {"launch_ms": round(lm, 4), "algorithmic_bytes_per_launch": kb32,
                           "gbs": round(kb32 / (lm * 1e-3) / 1e9, 1),
                           "frac": round(kb32 / (lm * 1e-3) / 1e9 / peak, 4)}
        out["fp32"] = {"ms": round(ms32, 4), "speedup_mixed_vs_fp32": round(ms32 / ms_max, 3),
                       "sigma_max_rel_diff_mixed_vs_fp32":
                           float(np.max(np.abs(sv_main - sv32) / sv32)),
                       "stage_share": {s_: round(v["device_ms"] / tot32, 4) for s_, v in st32.items()
                                       if v["launches"]},
                       "kernels": kern32}

    if not args.no_e2e:
        out["e2e"], host_csr = e2e_leg(args, ip, ix, vv, n_obs, local, dev, world)
        out["device_one_shot"] = device_one_shot_leg(args, ip, ix, vv, n_obs, local, dev, stream)
        if not args.no_stream:
            out["streamed"] = streamed_leg(args, host_csr, n_obs, local, res)
    else:
        host_csr = (ip.cpu().numpy(), ix.cpu().numpy(), vv.cpu().numpy())

    if not args.no_backward:
        out["differentiable"] = differentiable_leg(args, local, dev)
    if not args.no_batched:
        out["batched"] = batched_leg(args, local, dev)

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        sample_rows = args.cpu_sample_rows or n_obs
        cpu_ms, sample_nnz, sample_s, fp64 = cpu_baseline(*host_csr, n_obs, sample_rows, threads)
        out["cpu_baseline"] = {
            "value": round(cpu_ms, 1), "unit": "ms", "cores": threads, "kind": "port",
            "sample": (f"the whole matrix ({sample_nnz:,} nnz)" if sample_rows >= n_obs else
                       f"first {sample_rows:,} rows ({sample_nnz:,} nnz) of the same matrix, scaled by "
                       f"rows to {n_obs:,}") +
                      f", FP64 C++ restatement of the reference CPU randomized PCA, {sample_s:.2f} s",
        }
        # precision of the GPU paths against FP64 (config 3): the whole matrix
        # against the FP64 randomized result just computed (same seeded Omega),
        # a 50,000-cell subsample against the exact PCA
        ours = {args.mode: {"sv": res.singular_values, "comps": res.components}}
        extra = [m for m in ("mixed_bf16", "mixed_f16", "strict_fp32") if m != args.mode]
        sub_n = min(SUBSAMPLE_ROWS, n_obs)
        sub_nnz = int(host_csr[0][sub_n])
        sub_csr = (np.ascontiguousarray(host_csr[0][: sub_n + 1]), np.ascontiguousarray(host_csr[1][:sub_nnz]),
                   np.ascontiguousarray(host_csr[2][:sub_nnz]))
        sub_ours = {}
        for m in [args.mode] + extra:
            if m != args.mode and m in ("mixed_f16",):
                pm = make_plan(m)
                rm = pm.run()
                pm.close()
                ours[m] = {"sv": rm.singular_values, "comps": rm.components}
            elif m == "strict_fp32" and "fp32" in out:
                ours[m] = {"sv": sv32, "comps": comps32}
            ps = accel.Plan(ip[: sub_n + 1], ix[:sub_nnz], vv[:sub_nnz], (sub_n, N_VARS), n_components=N_COMPS,
                            n_oversamples=N_OVERSAMPLES, n_power_iterations=N_POWER, zero_center=True,
                            scale=True, clip_max=CLIP, seed=SEED, qr_method="cholesky", math_mode=m,
                            device=local)
            rs = ps.run()
            ps.close()
            sub_ours[m] = {"sv": rs.singular_values, "comps": rs.components}
        out["precision"] = precision_report(ours, fp64, sub_ours, sub_csr)

    if rank == 0:
        print(json.dumps(out), flush=True)
    _finish_dist()


def e2e_leg(args, ip, ix, vv, n_obs, local, dev, world):
    """The PCA through the one-shot C ABI call from pinned host memory to host
    embeddings (upload, validation, statistics, value transform, packing, the
    PCA, download and teardown inside every timed step).  Values go up in the
    precision the mode computes in (BF16 or FP16 for the mixed modes, FP32 for
    the strict mode); indices int32, indptr int64.  Reports the median of the
    library's own per-phase times (device clock on the call's stream) and the
    host-to-device bandwidth of a plain copy of the same pinned bytes measured
    in the same run, which sets the upload phase."""
    import numpy as np
    import torch

    from scx_b200 import accel

    vdt = {"mixed_bf16": torch.bfloat16, "mixed_f16": torch.float16, "strict_fp32": torch.float32}[args.mode]
    h_ip = ip.cpu().pin_memory()
    h_ix = ix.cpu().pin_memory()
    h_vv = vv.to(vdt).cpu().pin_memory()
    h_emb = torch.empty((n_obs, N_COMPS), dtype=torch.float32).pin_memory()
    a_ip, a_ix, a_emb = h_ip.numpy(), h_ix.numpy(), h_emb.numpy()
    a_vv = h_vv if vdt == torch.bfloat16 else h_vv.numpy()

    def one():
        return accel.randomized_pca(a_ip, a_ix, a_vv, (n_obs, N_VARS), n_components=N_COMPS,
                                    n_oversamples=N_OVERSAMPLES, n_power_iterations=N_POWER,
                                    zero_center=True, scale=True, clip_max=CLIP, seed=SEED,
                                    qr_method="cholesky", math_mode=args.mode, device=local,
                                    embeddings_out=a_emb)

    for _ in range(max(2, args.warmup)):
        one()
    steps = max(1, min(10, args.steps))
    phases = []
    per_step = []
    barrier(dev)
    t0 = time.perf_counter()
    for _ in range(steps):
        ts = time.perf_counter()
        one()
        per_step.append((time.perf_counter() - ts) * 1e3)
        phases.append(accel.last_call_phases())
    e2e_ms = (time.perf_counter() - t0) * 1e3 / steps
    e2e_ms = max_over_ranks(e2e_ms, dev)
    h2d = h_ip.numel() * 8 + h_ix.numel() * 4 + h_vv.numel() * h_vv.element_size()
    d2h = a_emb.nbytes + N_COMPS * N_VARS * 4 + N_COMPS * 8 * 3 + N_VARS * 8 * 2
    # plain pinned host-to-device copy of the same bytes, for the upload phase
    d_ix = torch.empty_like(ix)
    d_vv = torch.empty(h_vv.shape, dtype=vdt, device=dev)
    torch.cuda.synchronize(dev)
    cs = torch.cuda.Stream(device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(cs):
        e0.record(cs)
        d_ix.copy_(h_ix, non_blocking=True)
        d_vv.copy_(h_vv, non_blocking=True)
        e1.record(cs)
    torch.cuda.synchronize(dev)
    copy_ms = e0.elapsed_time(e1)
    del d_ix, d_vv
    med = {k: round(statistics.median(p[k] for p in phases), 3) for k in phases[0]}
    out = {"value": round(e2e_ms / world, 3), "unit": "ms", "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "steps": steps,
           "path": "scxpca_randomized (host pinned CSR -> host embeddings)",
           "step_ms": {"min": round(min(per_step), 3), "median": round(statistics.median(per_step), 3),
                       "max": round(max(per_step), 3)},
           "values_on_host": str(vdt).replace("torch.", ""),
           "phases_ms": med,
           "slowest_step_phases_ms": {k: round(v, 3) for k, v in phases[per_step.index(max(per_step))].items()},
           "h2d_copy": {"ms": round(copy_ms, 3),
                        "gbs": round((h_ix.numel() * 4 + h_vv.numel() * h_vv.element_size()) / copy_ms / 1e6, 1)}}
    host_csr = (a_ip, a_ix, vv.cpu().numpy())
    return out, host_csr


STREAM_BUDGET = 2 << 30  # bytes of device memory the streamed leg may use


def streamed_leg(args, host_csr, n_obs, local, res_resident):
    """The same PCA with the matrix left in (pinned) host memory and streamed
    in row shards through every product, the plan held to a 2 GiB device
    budget (the resident plan needs several GB): the out-of-VRAM path.  Times
    the one-shot call (host wall clock) and compares its singular values with
    the resident run's."""
    import numpy as np
    import torch

    from scx_b200 import accel

    h_ip = torch.from_numpy(np.asarray(host_csr[0])).pin_memory()
    h_ix = torch.from_numpy(np.asarray(host_csr[1])).pin_memory()
    # FP32 host values, as the resident plan was built from: the statistics and
    # the value transform then see the same inputs and the singular values
    # differ only by the order of the per-shard partial sums.
    h_vv = torch.from_numpy(np.asarray(host_csr[2], dtype=np.float32)).pin_memory()

    def one():
        return accel.randomized_pca(h_ip.numpy(), h_ix.numpy(), h_vv.numpy(), (n_obs, N_VARS), n_components=N_COMPS,
                                    n_oversamples=N_OVERSAMPLES, n_power_iterations=N_POWER, zero_center=True,
                                    scale=True, clip_max=CLIP, seed=SEED, qr_method="cholesky",
                                    math_mode=args.mode, device=local, device_budget=STREAM_BUDGET)

    one()
    times, r = [], None
    for _ in range(max(1, min(3, args.steps))):
        t0 = time.perf_counter()
        r = one()
        times.append((time.perf_counter() - t0) * 1e3)
    sv = np.asarray(res_resident.singular_values)
    return {"ms": round(statistics.median(times), 2), "steps": len(times), "device_budget_bytes": STREAM_BUDGET,
            "resident_csr": bool(r.resident_csr), "n_shards": int(r.n_shards),
            "sigma_max_rel_diff_vs_resident": float(np.max(np.abs(np.asarray(r.singular_values) - sv) / sv)),
            "values_on_host": "float32",
            "path": "scxpca_randomized on pinned host CSR, streamed in row shards"}


def device_one_shot_leg(args, ip, ix, vv, n_obs, local, dev, stream):
    """Plan creation + run + destruction from the DEVICE CSR (FP32 values, so
    validation, statistics, the value transform and packing all run), timed
    with CUDA events on the plan's stream: the per-matrix set-up that the
    resident headline excludes, counted like-for-like with the reference's
    per-call host work."""
    import torch

    from scx_b200 import accel

    emb = torch.empty((n_obs, N_COMPS), dtype=torch.float32, device=dev)
    times = []
    for i in range(2 + max(1, min(3, args.steps))):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        plan = accel.Plan(ip, ix, vv, (n_obs, N_VARS), n_components=N_COMPS, n_oversamples=N_OVERSAMPLES,
                          n_power_iterations=N_POWER, zero_center=True, scale=True, clip_max=CLIP, seed=SEED,
                          qr_method="cholesky", math_mode=args.mode, device=local, stream=stream.cuda_stream)
        plan.run(embeddings_out=emb)
        plan.close()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i >= 2:
            times.append(e0.elapsed_time(e1))
    return {"ms": round(statistics.median(times), 3), "steps": len(times),
            "path": "scxpca_plan_create + scxpca_plan_run + scxpca_plan_destroy on the device CSR (FP32 values)"}


DIFF_N_OBS = 200_000
CONVERGED_SOLVE = 64
SOLVE_SWEEP = (4, 8, 16, 32)
GRAD_RTOL = 2e-3
PLANTED = dict(rank=50, density=0.1, ratio=0.98, noise=0.3, top=1000.0)


def planted_csr_device(n, g, rank, density, ratio, noise, top, seed, dev):
    """Seeded sparse matrix with a planted rank-`rank` leading spectrum, made
    on the device with torch: the stored entries are a Bernoulli(density) mask;
    their values are those of U diag(top ratio^i) V^T (random orthonormal U, V)
    scaled by 1 / density, plus N(0, noise).  With rank = the number of
    components, the components' subspace is separated from the rest of the
    spectrum, so the scores' derivative is well posed.  Rows sorted by gene."""
    import torch

    gen = torch.Generator(device=dev).manual_seed(seed)
    U = torch.linalg.qr(torch.randn((n, rank), generator=gen, device=dev, dtype=torch.float64))[0]
    V = torch.linalg.qr(torch.randn((g, rank), generator=gen, device=dev, dtype=torch.float64))[0]
    sig = top * ratio ** torch.arange(rank, device=dev, dtype=torch.float64)
    vals = ((U * sig) @ V.T).float() / density
    del U
    vals += noise * torch.randn((n, g), generator=gen, device=dev)
    mask = torch.rand((n, g), generator=gen, device=dev) < density
    rows, cols = mask.nonzero(as_tuple=True)
    v = vals[rows, cols].contiguous()
    del vals, mask
    indptr = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    indptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0)
    return indptr, cols.to(torch.int32).contiguous(), v


def _differentiable_case(args, local, dev, ip, ix, vv, n, g, sweep, time_it):
    """Accuracy sweep of the gradient's CG solve, then (time_it) forward and
    backward timed with CUDA events on the plan's stream."""
    import numpy as np
    import torch

    from scx_b200 import accel

    sums = torch.bincount(ix.long(), weights=vv.double(), minlength=g)
    sq = torch.bincount(ix.long(), weights=vv.double() ** 2, minlength=g)
    mean = sums / n
    std = ((sq - n * mean * mean) / (n - 1)).clamp_min(0).sqrt()
    scale = torch.where(std > 0, 1.0 / std, torch.ones_like(std))
    stream = torch.cuda.Stream(device=dev)
    gen = torch.Generator(device=dev).manual_seed(SEED)
    W = torch.randn((n, N_COMPS), generator=gen, device=dev, dtype=torch.float32)
    plan = accel.Plan(ip, ix, vv, (n, g), n_components=N_COMPS, n_oversamples=N_OVERSAMPLES,
                      n_power_iterations=N_POWER, seed=SEED, qr_method="householder",
                      math_mode="strict_fp32", device=local, stream=stream.cuda_stream,
                      center=mean, gene_scale=scale)
    S = torch.empty((n, N_COMPS), dtype=torch.float32, device=dev)

    def grads(iters):
        r = plan.run(embeddings_out=S)
        with torch.cuda.stream(stream):
            G = 2.0 * W * S
        gv, gc, gs = plan.backward(S, G, iters)
        torch.cuda.synchronize(dev)
        return (gv.double(), gc.double(), gs.double()), r

    def rel(a, b):
        return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))

    ref, r = grads(CONVERGED_SOLVE)
    sv = np.asarray(r.singular_values)
    errs = {}
    for iters in sweep:
        gr, _ = grads(iters)
        errs[iters] = {"values": rel(gr[0], ref[0]), "center": rel(gr[1], ref[1]), "scale": rel(gr[2], ref[2])}
    enough = [i for i in sweep if max(errs[i].values()) <= GRAD_RTOL]
    out = {"nnz": int(ix.numel()),
           "grad_rel_err": {str(i): {k_: float(f"{v:.3e}") for k_, v in e.items()} for i, e in errs.items()},
           "grad_rel_err_reference": f"{CONVERGED_SOLVE} CG steps on the same run",
           "sigma_49_over_sigma_0": float(sv[-1] / sv[0]),
           "solve_reaches_rtol": bool(enough)}
    if time_it:
        solve = enough[0] if enough else sweep[-1]
        fwd_ms, bwd_ms = [], []
        steps = max(2, min(args.steps, 5))
        for i in range(args.warmup + steps):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            plan.run(embeddings_out=S)
            e1.record(stream)
            with torch.cuda.stream(stream):
                G = 2.0 * W * S
            plan.backward(S, G, solve)
            e2.record(stream)
            torch.cuda.synchronize(dev)
            if i >= args.warmup:
                fwd_ms.append(e0.elapsed_time(e1))
                bwd_ms.append(e1.elapsed_time(e2))
        f = statistics.median(fwd_ms)
        b = statistics.median(bwd_ms)
        out.update({"forward_ms": round(f, 3), "backward_ms": round(b, 3), "backward_over_forward": round(b / f, 3),
                    "solve_iterations": solve, "steps": steps})
    plan.close()
    return out


def differentiable_leg(args, local, dev):
    """Forward vs backward of the differentiable scores, FP32, 50 PCs,
    oversample 10, 4 power iterations, centred on the column means and scaled
    by 1 / std (explicit per-gene vectors), loss sum(W * S**2) with W a seeded
    N(0, 1) n x 50 matrix.

    The gradient's conjugate-gradient solve is first checked for accuracy: the
    gradients (values, centre, scale) after 4, 8, 16 and 32 steps against a
    converged solve of 64 steps of the same run; the smallest step count that
    agrees to 2e-3 relative is the one timed.

    Timed on a 200,000 x 2,000 matrix with a planted 50-dimensional leading
    subspace (10 % density): the derivative of the top-50 scores is then well
    posed.  On the 200,000 x 2,000 NB-synthetic CSR the 50th and 51st
    eigenvalues of the scaled matrix nearly coincide (a flat noise spectrum),
    the solve is ill conditioned and does not reach 2e-3 within 32 steps; its
    sweep is reported beside (untimed)."""
    import torch

    from scx_b200 import accel

    n, g = DIFF_N_OBS, N_VARS
    ip, ix, vv = planted_csr_device(n, g, seed=SEED + 2, dev=dev, **PLANTED)
    planted = _differentiable_case(args, local, dev, ip, ix, vv, n, g, SOLVE_SWEEP, True)
    del ip, ix, vv
    torch.cuda.empty_cache()
    ip, ix, vv = accel.synth_nb_csr_device(n, g, seed=SEED + 1, loc=LOC, dispersion=DISPERSION, device=local)
    nb = _differentiable_case(args, local, dev, ip, ix, vv, n, g, (8, 32), False)
    out = {"workload": f"{n:,} x {g:,} CSR with a planted 50-dimensional leading subspace "
                       f"({planted['nnz']:,} nnz, density {PLANTED['density']}, singular values "
                       f"{PLANTED['top']:g} x {PLANTED['ratio']}^i plus N(0, {PLANTED['noise']}) entries), FP32, "
                       "50 PCs, oversample 10, 4 power iterations, loss sum(W * S^2)",
           "grad_rtol": GRAD_RTOL}
    out.update({k: v for k, v in planted.items() if k != "nnz"})
    out["nb_synthetic_untimed"] = {"workload": f"{n:,} x {g:,} NB-synthetic CSR ({nb['nnz']:,} nnz)",
                                   **{k: v for k, v in nb.items() if k != "nnz"}}
    return out


BATCH_CLUSTERS = 256
BATCH_LOC = -3.2  # ~9 % density


def batched_leg(args, local, dev):
    """256 cell clusters (sizes LogNormal(log 4000, 1.0) clipped to [500,
    50,000], seed 0) of 2,000 genes, each cluster from the NB generator with
    its own seed -- its own gene-mean profile -- at ~9 % density, BF16 values;
    a centred 30-PC randomized PCA (oversample 10, 3 power iterations) per
    cluster.  Times one launch of the batch's graph against the 256 plain
    per-cluster launches, both on the device (CUDA events)."""
    import numpy as np
    import torch

    from scx_b200 import accel

    rng = np.random.default_rng(SEED)
    sizes = np.clip(np.round(rng.lognormal(np.log(4000.0), 1.0, BATCH_CLUSTERS)), 500, 50_000).astype(np.int64)
    ips, ixs, vvs, base = [torch.zeros(1, dtype=torch.int64, device=dev)], [], [], 0
    for q, nq in enumerate(sizes):
        ip, ix, vv = accel.synth_nb_csr_device(int(nq), N_VARS, seed=1000 + q, loc=BATCH_LOC,
                                               dispersion=DISPERSION, device=local)
        ips.append(ip[1:] + base)
        base += int(ix.numel())
        ixs.append(ix)
        vvs.append(vv.to(torch.bfloat16))
    ip, ix, vv = torch.cat(ips), torch.cat(ixs), torch.cat(vvs)
    n = int(sizes.sum())
    offs = np.r_[0, np.cumsum(sizes)]
    b = accel.Batch(ip, ix, vv, (n, N_VARS), offs, n_components=30, n_oversamples=10, n_power_iterations=3,
                    seed=SEED, math_mode="mixed_bf16", device=local, branches=0)
    emb = torch.empty((n, 30), dtype=torch.float32, device=dev)
    graph_ms, plain_ms = [], []
    for i in range(2 + max(2, min(args.steps, 3))):
        _, _, sv_g, _, ms = b.run(use_graph=True, embeddings_out=emb, components=False)
        if i >= 2:
            graph_ms.append(ms)
    for i in range(1 + 2):
        _, _, sv_p, _, ms = b.run(use_graph=False, embeddings_out=emb, components=False)
        if i >= 1:
            plain_ms.append(ms)
    out = {"workload": f"{BATCH_CLUSTERS} clusters, {n:,} cells x {N_VARS:,} genes ({int(ix.numel()):,} nnz, "
                       f"{int(ix.numel()) / (n * N_VARS):.3f} density), BF16, 30 PCs, oversample 10, q = 3",
           "cluster_sizes": {"min": int(sizes.min()), "median": int(np.median(sizes)), "max": int(sizes.max())},
           "graph_ms": round(statistics.median(graph_ms), 3), "plain_launches_ms": round(statistics.median(plain_ms), 3),
           "speedup_graph_vs_plain": round(statistics.median(plain_ms) / statistics.median(graph_ms), 3),
           "branches": abs(b.branches), "schedule": "lockstep" if b.lockstep else "segment per branch",
           "graph_nodes": b.graph_nodes,
           "autotune_ms": {(f"lockstep {-k}" if k < 0 else str(k)): round(v, 3) for k, v in b.tuned_ms.items()},
           "sigma_max_rel_diff_graph_vs_plain": float(np.max(np.abs(sv_g - sv_p) / sv_p))}
    b.close()
    # correctness at the timed setting: clusters from smallest to largest
    # against the FP64 randomized PCA (C++ restatement, same seeded Omega) of
    # the same BF16-rounded values
    out["vs_oracle"] = batched_oracle_check(sizes, offs, ip, ix, vv, sv_g)
    return out


BATCH_CHECKED = 8


def batched_oracle_check(sizes, offs, ip, ix, vv, sv):
    import numpy as np

    from oracle import build_cpu, rpca

    order = np.argsort(sizes, kind="stable")
    pick = sorted({int(order[0]), int(order[-1])} |
                  {int(order[i]) for i in np.linspace(0, len(order) - 1, BATCH_CHECKED).round().astype(int)})
    h_ip = ip.cpu().numpy()
    h_ix = ix.cpu().numpy()
    h_vv = vv.float().cpu().numpy()  # the BF16 values the GPU saw, widened exactly
    om = rpca.gaussian_omega(N_VARS, 40, SEED)
    errs = {}
    for q in pick:
        r0, r1 = int(offs[q]), int(offs[q + 1])
        p0, p1 = int(h_ip[r0]), int(h_ip[r1])
        res = build_cpu.run(h_ip[r0:r1 + 1] - p0, h_ix[p0:p1], h_vv[p0:p1], (r1 - r0, N_VARS), 30, 40, 3, om,
                            zero_center=True, threads=os.cpu_count() or 1)
        ref = res["singular_values"]
        errs[str(q)] = {"cells": r1 - r0, "sigma_max_rel_err": float(np.max(np.abs(sv[q] - ref) / ref))}
    return {"clusters": errs, "sigma_max_rel_err": max(e["sigma_max_rel_err"] for e in errs.values()),
            "reference": "FP64 C++ restatement of the reference CPU randomized PCA, same seeded Omega, "
                         "BF16-rounded values"}


def _finish_dist():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()


def run_reference(args):
    """Reference arm: the reference's CPU randomized PCA (its multithreaded C++
    restatement, the Rust reference being unbuildable here) on all host
    cores, on the whole matrix of the GPU arm: the same device generator and
    seed, copied to host memory once before timing.  Warm-up steps run on the
    first 50,000 rows (the CPU has nothing to warm); every timed step is one
    complete PCA of the whole matrix."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import numpy as np
    import torch

    from scx_b200 import accel

    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        ip_d, ix_d, vv_d = accel.synth_nb_csr_device(args.n_obs, N_VARS, seed=SEED, loc=LOC,
                                                     dispersion=DISPERSION, device=local)
        ip, ix, vv = ip_d.cpu().numpy(), ix_d.cpu().numpy(), vv_d.cpu().numpy()
        del ip_d, ix_d, vv_d
        torch.cuda.empty_cache()
        data = "synthetic (seeded negative-binomial CSR generated on device, copied to host before timing)"
    else:  # no device: the host restatement of the generator (a different matrix of the same law)
        from scx_b200.synth import synth_nb_csr
        ip, ix, vv = synth_nb_csr(args.n_obs, N_VARS, seed=SEED, loc=LOC, dispersion=DISPERSION)
        data = "synthetic (seeded negative-binomial CSR, host generator; no device present)"
    nnz = int(ip[-1])
    threads = os.cpu_count() or 1
    warm_rows = min(SUBSAMPLE_ROWS, args.n_obs)
    for _ in range(args.warmup):
        cpu_baseline(ip, ix, vv, warm_rows, warm_rows, threads)
    times = []
    for _ in range(args.steps):
        ms, _, _, _ = cpu_baseline(ip, ix, vv, args.n_obs, args.n_obs, threads)
        times.append(ms)
    value = float(np.mean(times))
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "ms", "impl": "reference",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(value, 1), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": data,
        "config": base_config(args.n_obs, nnz, "f32 input, f64 compute", 1),
        "cpu_baseline": {"value": round(value, 1), "unit": "ms", "cores": threads, "kind": "port",
                         "sample": f"the whole matrix ({args.n_obs:,} rows, {nnz:,} nnz) per timed step; "
                                   f"warm-up on the first {warm_rows:,} rows; reference is Rust (unbuildable "
                                   "here), timed via its FP64 C++ restatement"},
        "e2e": {"value": round(value, 1), "unit": "ms", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
