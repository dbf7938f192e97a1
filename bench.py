#!/usr/bin/env python
"""Benchmark of the sbd tpb selected-CI hot path on B200.

Metric (the reference's headline for this path): H*v det-pairs/s, plus the
Davidson time to a 1e-8 residual in FP64 and in the mixed (FP32-storage,
FP64 defect-correction) form, on the plain-FP64 drop-in workload: L = 58
orbitals, 7 alpha + 7 beta electrons, 8000 x 8000 sampled strings (64M
determinants, 512 MB per FP64 vector), seeded synthetic integrals and strings.

One step = one sigma (S = H C) over the whole workload. `value` times K steps
with C resident in HBM (CUDA events on the launching stream, max over ranks);
C (512 MB) is larger than the 126 MB L2, so no flush is needed between steps.
`e2e` times the same product through the C-ABI call sbdx_sigma with pinned
host buffers, the host->device copy of C and the device->host copy of S inside
every step. `roofline` describes the dominant kernel of the sigma (the
alpha-beta kernel), which gathers from rows staged in shared memory and is
bound by the shared-memory pipe: its conflict-free shared bytes per launch
(one ket and one integral element per alpha-single x beta-single det-pair,
2*s_c*P_ab) over its CUDA-event time, against 128 bytes per clock per SM at
the sampled SM clock. `roofline.hbm` keeps the SpMV byte model (one vector
gather per pair plus the partial-sigma read-modify-write, P_ab*s_c + 16*D)
against the measured HBM copy bandwidth, and the DRAM bytes ncu measured;
`roofline.sigma` gives the model for the whole sigma,
B = P*s_c + D*(2*s_c + s_h) + 4*(connectivity entries) + 8*(na + nb). The CPU baseline is the reference's own
OpenMP mult (compiled in oracle/_ref) on a bounded sample of bra alpha rows.
`mixed_precision` runs the 400 M-determinant workload (2 roots) in FP64 and
mixed precision with energy and 1-RDM errors; `projection` times the
Davidson subspace projection (DMMA tiles on the FP64 tensor pipe) at the
shapes the solvers issue; `summary`, printed last, holds the headline figures.

Multi-GPU (--gpus N under torchrun): one sigma of the same workload split by
alpha-row shards over the N GPUs (sbdx/shard.py: the whole C gathered on every
GPU by NCCL, each GPU evaluating its own rows), strong scaling; value = the
det-pairs of the whole sigma over the slowest rank's step time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "sbd-ykt_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "H·v det-pairs/s and Davidson s to 1e-8 Ha, mixed vs FP64, 1 B200"
UNIT = "det-pairs/s"
WORKLOAD = "cfg2"
WORKLOAD_DESC = "plain FP64 drop-in: L=58, 7a+7b electrons, 8000x8000 strings (64M dets), K=96 integrals"
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "sbd_ref_cli")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-davidson", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU-baseline sample duration")
    ap.add_argument("--davidson-tol", type=float, default=1e-8)
    ap.add_argument("--roots", type=int, default=2, help="roots of the multi-root Davidson runs (0 = skip them)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-subspace runs")
    ap.add_argument("--batch-threads", type=int, default=16)
    ap.add_argument("--diff", default="cfg4", metavar="WORKLOAD",
                    help="workload of the differentiation measurement ('' = skip)")
    ap.add_argument("--diff-entries", type=int, default=4, help="entries checked by central differences")
    ap.add_argument("--stored", default="cfg4", metavar="WORKLOAD",
                    help="workload of the stored-Hamiltonian (method 1) measurement ('' = skip)")
    ap.add_argument("--mixed", default="cfg3", metavar="WORKLOAD",
                    help="workload of the mixed-precision measurement (2 roots, FP64 block solve vs mixed with "
                         "refresh every 4 steps and adaptive; '' = skip)")
    ap.add_argument("--projection-d", type=int, default=None, metavar="D",
                    help="vector length of the projection measurement (default: the workload's; 0 = skip)")
    ap.add_argument("--sharded", action="store_true",
                    help="run the alpha-row-shard path (the N > 1 path) also at N = 1")
    ap.add_argument("--tune", default=None, metavar="SAME,AB",
                    help="fixed sigma launch codes for both precisions instead of the autotuner (profiling runs)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def smem_peak_gbs(sm_mhz: float) -> float:
    """Shared-memory bandwidth of the whole GPU: 128 bytes per clock per SM
    (one 128-byte wavefront per cycle) x SMs x the SM clock sampled during
    the timed region."""
    import torch

    nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    return 128.0 * nsm * sm_mhz * 1e6 / 1e9


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.fh = None

    def start(self):
        try:
            self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.flush()
        with open(self.fh.name) as f:
            rows = [r.strip().split(", ") for r in f if r.strip()]
        os.unlink(self.fh.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
            except ValueError:
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def gpu_index(local: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local < len(ids) and ids[local].strip().isdigit():
            return int(ids[local])
    return local


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_sample(prob, target_s: float, reps: int, threads: int):
    """Run the reference's own mult on a block of bra alpha rows in the middle
    of the sorted alpha list (typical strings; the Aufbau string at row 0 has
    by far the most connections), with all beta rows. The reference's OpenMP
    loop gives each thread its own bra rows, so the block holds a multiple of
    `threads` rows, sized so one run takes about target_s seconds. Returns
    (per-run results, description)."""
    from sbdx import synth

    if not os.path.exists(REF_CLI):
        return None, "reference CPU build not present (oracle/_ref)"
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "problem.bin")
        synth.write_problem_bin(path, prob)

        def run(row0, rows, n):
            out = subprocess.run([REF_CLI, "sigma-sample", path, str(rows), str(n), str(threads), str(row0)],
                                 check=True, capture_output=True, text=True).stdout
            return [json.loads(line) for line in out.splitlines() if line.startswith("{")]

        rows = min(prob.na, threads)
        row0 = max(0, prob.na // 2 - rows // 2)
        cal = run(row0, rows, 1)[0]
        mult = max(1, int(target_s / max(cal["seconds"], 1e-6)))
        rows = min(prob.na, rows * mult)
        row0 = max(0, prob.na // 2 - rows // 2)
        res = run(row0, rows, reps)
    return res, (row0, rows)


def roofline_bytes(prob, dp, s_c: int, s_h: int = 8) -> float:
    conn = dp["Sa"] + dp["Da"] + dp["Sb"] + dp["Db"]
    return dp["offdiag"] * s_c + prob.D * (2 * s_c + s_h) + 4 * conn + 8 * (prob.na + prob.nb)


# CUDA kernel of each sigma phase (alpha-first path) and its ncu summary file
PHASE_KERNELS = {"alpha_same_spin": "sigma_same_v6", "transpose": "phase_split", "beta_same_spin": "sigma_same_v6",
                 "alpha_beta": "sigma_ab_v7", "combine": "combine_phase"}


def ab_smem_bytes(dp, s_c: int) -> float:
    """Shared-memory bytes the alpha-beta kernel must load: per alpha-single x
    beta-single det-pair one element of the staged ket row and one of the
    staged integral row (2 * s_c), at one 128-byte wavefront per 8 lanes of a
    16-byte load, i.e. without bank conflicts."""
    return 2.0 * s_c * dp["alpha_beta"]


def phase_bytes(prob, dp, s_c: int) -> dict:
    """Algorithmic bytes of each sigma phase: one vector gather per nonzero of
    its part of H (the matrix is never stored), plus the streams every
    element of the phase reads or writes once."""
    D = prob.D
    na, nb = prob.na, prob.nb
    return {
        "transpose": 3.0 * D * s_c,                                            # read C, write phi o C and its transpose
        "alpha_same_spin": nb * (dp["Sa"] + dp["Da"]) * s_c + D * (s_c + 16),  # + own row, hii, Y
        "beta_same_spin": na * (dp["Sb"] + dp["Db"]) * s_c + D * 8,           # + Yt
        "alpha_beta": dp["alpha_beta"] * s_c + 16.0 * D,                       # + Y read-modify-write
        "combine": D * (16.0 + s_c),                                           # Y, Yt -> S
    }


def traffic_per_launch(kernel: str, workload: str):
    """DRAM bytes of one launch of `kernel` on `workload` from the committed
    ncu summary profiles/<kernel>_<workload>.md (line 'dram_bytes_per_launch: N')."""
    import re

    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if os.path.exists(path):
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
        if m:
            return float(m.group(1))
    return None


def max_over_ranks(x: float, pg=None, device: str = "cuda") -> float:
    """Maximum of x over all ranks of the process group (x itself at N=1)."""
    if pg is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(pairs_per_step: float, ms_local: float, world: int, pg=None, device: str = "cuda"):
    """Whole-job det-pairs/s when every one of `world` ranks evaluates
    pairs_per_step per step; the job's step time is the slowest rank's."""
    ms = max_over_ranks(ms_local, pg, device)
    return ms, world * pairs_per_step / (ms * 1e-3)


def workload_desc(name: str) -> str:
    from sbdx import synth

    base = name.split("@")[0]
    if base == WORKLOAD and "@" not in name:
        return WORKLOAD_DESC
    if base in synth.CONFIGS:
        L, n, K, Na, Nb = synth.CONFIGS[base][:5]
        scale = float(name.split("@")[1]) if "@" in name else 1.0
        return (f"L={L}, {n}a+{n}b electrons, {Na}x{Nb} strings scaled by {scale:g} "
                f"({round(Na * scale)}x{round(Nb * scale)}), K={K} integrals")
    return name


def load_workload(name: str):
    """'cfg2' or 'cfg2@0.6' (string counts scaled, for small profiling cases)."""
    from sbdx import synth

    if "@" in name:
        base, scale = name.split("@", 1)
        return synth.config(base, float(scale))
    return synth.config(name)


def run_batched(args) -> dict:
    """64 subspaces sharing one Hamiltonian (L=40, 8+8 electrons, Na and Nb
    log-uniform in [200, 4000]), 2 roots each to the Davidson tolerance:
    batched mixed precision (concurrent solves) against the same subspaces
    solved one after another (FP64 and mixed)."""
    import sbdx
    from sbdx import synth

    subs = synth.batched_config()
    p0 = subs[0]
    pairs = []
    for p in subs:  # det-pairs of one sigma of each subspace, from its connectivity lengths
        with sbdx.Context(0) as ctx:
            ctx.load(p)
            ctx.build_connectivity()
            sa, da, _ = ctx.connectivity(0)
            sb, db, _ = ctx.connectivity(1)
            pairs.append(synth.det_pairs(sa, da, sb, db)["total"])
    out = {"workload": "64 subspaces, L=40, 8a+8b electrons, Na, Nb log-uniform in [200, 4000], K=96 integrals",
           "subspaces": len(subs), "dets": int(sum(p.D for p in subs)),
           "dets_min": int(min(p.D for p in subs)), "dets_max": int(max(p.D for p in subs)),
           "nroots": 2, "tol": args.davidson_tol}
    with sbdx.Batch(p0.L, p0.I0, p0.h, p0.eri) as batch:
        for p in subs:
            batch.add(p.alpha, p.beta)
        out["tuning"] = batch.tune()
        runs = {}
        ref_E = None
        for label, prec, threads, graphs in (("sequential_fp64", sbdx.SBDX_FP64, 1, False),
                                             ("sequential_mixed", sbdx.SBDX_FP32, 1, False),
                                             ("batched_fp64", sbdx.SBDX_FP64, args.batch_threads, False),
                                             ("batched_mixed", sbdx.SBDX_FP32, args.batch_threads, False),
                                             ("batched_mixed_graph_steps", sbdx.SBDX_FP32, args.batch_threads, True),
                                             ("sequential_mixed_graph_steps", sbdx.SBDX_FP32, 1, True)):
            batch.set_graph_steps(graphs)
            E, R, infos, sec = batch.solve(nroots=2, max_it=100, max_nb=12, eps=args.davidson_tol, precision=prec,
                                           nthreads=threads)
            if ref_E is None:
                ref_E = E
            nsig = [i.n_sigma + i.n_sigma64 for i in infos]
            t_sub = [i.seconds for i in infos]
            runs[label] = {"seconds": sec, "threads": threads, "converged": int(sum(i.converged for i in infos)),
                           "sigmas": int(sum(nsig)), "max_abs_dE_vs_sequential_fp64": float(np.abs(E - ref_E).max()),
                           "max_residual": float(R.max()),
                           "sigma_det_pairs_per_s": float(sum(n * q for n, q in zip(nsig, pairs)) / sec),
                           "subspace_seconds_median": float(np.median(t_sub)),
                           "subspace_seconds_max": float(np.max(t_sub))}
        batch.set_graph_steps(False)
        out["runs"] = runs
        out["speedup_batched_mixed_vs_sequential_fp64"] = runs["sequential_fp64"]["seconds"] / runs["batched_mixed"]["seconds"]
        out["speedup_batched_mixed_graph_steps_vs_sequential_fp64"] = (
            runs["sequential_fp64"]["seconds"] / runs["batched_mixed_graph_steps"]["seconds"])
    return out


def run_projection(args, hbm: float) -> dict:
    """The Davidson subspace projection on the FP64 tensor pipe
    (sbdx_project_device, DMMA tiles): P = V X^T at the shapes the solvers
    issue, on vectors of `--projection-d` elements (default: the workload's
    determinant count). First one call of each of three shapes (FP64 24 x 2,
    FP32 24 x 2, FP32 62 x 2), so that an ncu capture of the first three
    launches sees three kernels; then, shape by shape, one warm-up call and
    10 timed calls (CUDA events). Bytes: one read of the m + nx vectors; they
    are far larger than L2."""
    import torch

    import sbdx

    D = args.projection_d
    F64, F32 = sbdx.SBDX_FP64, sbdx.SBDX_FP32
    first = [(F64, 24, 2), (F32, 24, 2), (F32, 62, 2)]
    sweep = [(p, m, nx) for p in (F64, F32)
             for m, nx in ((1, 1), (2, 1), (4, 4), (8, 2), (16, 2), (24, 2), (40, 2), (62, 2), (20, 1))]
    out = {"kernel": "project_kernel (mma.sync m8n8k4 f64); m <= 4 with nx = 1: multidot_kernel (CUDA cores)",
           "D": D, "cases": []}
    with sbdx.Context(torch.cuda.current_device()) as ctx:
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)

        def operands(prec, m, nx):
            dt = torch.float64 if prec == F64 else torch.float32
            V = torch.randn(m, D, dtype=dt, device="cuda")
            X = torch.randn(nx, D, dtype=dt, device="cuda")
            P = torch.empty(m * nx, dtype=torch.float64, device="cuda")
            return V, X, P, (lambda: ctx.project_device(prec, V.data_ptr(), D, m, X.data_ptr(), D, nx, D,
                                                         P.data_ptr()))

        for shape in first:
            ops = operands(*shape)
            ops[3]()
            del ops
        for prec, m, nx in sweep:
            V, X, P, call = operands(prec, m, nx)
            call()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(10):
                call()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 10
            gbs = (m + nx) * D * V.element_size() / (ms * 1e-3) / 1e9
            out["cases"].append({"precision": "fp64" if prec == F64 else "fp32", "m": m, "nx": nx,
                                 "ms": ms, "gbs": gbs, "frac_of_hbm": gbs / hbm})
            del V, X, P, call
            torch.cuda.empty_cache()
    return out


def run_stored(args, hbm: float) -> dict:
    """The stored Hamiltonian (method 1, sbdx_build_hamiltonian) on a workload
    whose matrix fits in HBM: build time, element count, the FP64 product
    against the on-the-fly sigma of the same context (CUDA events, 10
    products after 3 warm-up ones; the matrix is far larger than L2). Bytes
    of a product: 12 per stored element (column + value) plus the row
    pointers and three D-vectors (input, diagonal, output)."""
    import torch

    import sbdx
    from sbdx import synth

    w, _, sc = args.stored.partition("@")
    prob = synth.config(w, float(sc) if sc else 1.0)
    with sbdx.Context(torch.cuda.current_device()) as ctx:
        ctx.load(prob)
        ctx.build_connectivity()
        ctx.diag_terms()
        stream = torch.cuda.current_stream()
        ctx.set_stream(stream.cuda_stream)
        C = torch.randn(prob.D, dtype=torch.float64, device="cuda")
        S = torch.empty_like(C)

        def time_sigma(n=10):
            for _ in range(3):
                ctx.sigma_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr())
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(n):
                ctx.sigma_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / n

        ms_fly = time_sigma()
        S_fly = S.clone()
        t0 = time.perf_counter()
        nnz = ctx.build_hamiltonian()
        build_s = time.perf_counter() - t0
        ms_st = time_sigma()
        rel = float((S - S_fly).abs().max() / S_fly.abs().max())
        ctx.release_hamiltonian()
    nbytes = 12 * nnz + 8 * (prob.D + 1) + 24 * prob.D
    gbs = nbytes / (ms_st * 1e-3) / 1e9
    return {"workload": args.stored, "desc": workload_desc(args.stored), "dets": int(prob.D), "elements": nnz,
            "matrix_gb": (12 * nnz + 8 * (prob.D + 1)) / 1e9, "build_seconds": build_s,
            "ms_stored_product": ms_st, "ms_on_the_fly_sigma": ms_fly, "gbs": gbs, "frac_of_hbm": gbs / hbm,
            "max_rel_diff_vs_on_the_fly": rel}


def run_differentiation(args) -> dict:
    """Energy adjoint on the differentiation workload (L=32, 6+6 electrons,
    2000x2000 strings): FP64 forward solve to 1e-10, the backward kernel
    (dE/dh and dE/d(pq|rs) from the 1-/2-RDM of the converged vector, the
    connectivity recomputed) and, on a few seeded entries, central
    differences of the forward solve (step 1e-5) against it."""
    import torch

    import sbdx
    from sbdx import autograd as sag
    from sbdx import synth

    w, _, sc = args.diff.partition("@")
    prob = synth.config(w, float(sc) if sc else 1.0)
    L = prob.L
    out = {"workload": args.diff, "desc": workload_desc(args.diff), "dets": int(prob.D)}
    with sbdx.Context(torch.cuda.current_device()) as ctx:
        ctx.set_strings(prob.alpha, prob.beta)
        h_tri = torch.tensor(sag.tril_pack(prob.h.reshape(L, L)), requires_grad=True)
        eri = torch.tensor(prob.eri, requires_grad=True)
        t0 = time.perf_counter()
        E = sag.energy(ctx, h_tri, eri, L, prob.I0)
        out["forward_seconds"] = time.perf_counter() - t0
        out["energy"] = float(E.detach())
        t0 = time.perf_counter()
        E.backward()
        out["backward_seconds"] = time.perf_counter() - t0
        gh, ge = h_tri.grad.numpy(), eri.grad.numpy()
        rng = np.random.default_rng(9)
        k = max(args.diff_entries, 0)
        picks = [("h", int(i)) for i in rng.choice(len(gh), k // 2, replace=False)]
        nz = np.flatnonzero(np.abs(prob.eri) > 1e-3)
        picks += [("eri", int(i)) for i in rng.choice(nz, k - k // 2, replace=False)]
        worst, step = 0.0, 1e-5
        for kind, i in picks:
            vals = []
            for sgn in (+1, -1):
                ht, et = h_tri.detach().clone(), eri.detach().clone()
                (ht if kind == "h" else et)[i] += sgn * step
                vals.append(float(sag.energy(ctx, ht, et, L, prob.I0)))
            fd = (vals[0] - vals[1]) / (2 * step)
            an = float(gh[i] if kind == "h" else ge[i])
            worst = max(worst, abs(fd - an) / max(1.0, abs(an)))
        out.update({"fd_entries": len(picks), "fd_step": step, "max_rel_err_vs_central_differences": worst})
    return out


def run_mixed(args) -> dict:
    """The mixed-precision workload (L=58, 7+7 electrons, 20000 x 20000
    strings, 400 M determinants): the 2 lowest roots to the Davidson tolerance
    with the FP64 block solver (FP64 corrections) and with the mixed solver
    (FP32-stored corrections, FP32-storage sigmas with FP64 row accumulation,
    FP64 anchors refreshed by exact FP64 sigmas every 4 steps, and with the
    adaptive refresh). Per root: |dE| and the max-abs difference of the 1-RDM
    of the mixed vector against the 1-RDM of the FP64 vector, all on the
    device (the vectors never leave it)."""
    import torch

    import sbdx
    from sbdx import synth

    w, _, sc = args.mixed.partition("@")
    prob = synth.config(w, float(sc) if sc else 1.0)
    out = {"workload": args.mixed, "desc": workload_desc(args.mixed), "dets": int(prob.D), "nroots": 2,
           "tol": args.davidson_tol, "max_nb": 12}
    with sbdx.Context(torch.cuda.current_device()) as ctx:
        ctx.load(prob)
        t0 = time.perf_counter()
        ctx.build_connectivity()
        out["connectivity_seconds"] = time.perf_counter() - t0
        out["tuning"] = ctx.autotune()
        sa, da, _ = ctx.connectivity(0)
        sb, db, _ = ctx.connectivity(1)
        out["det_pairs_per_sigma"] = synth.det_pairs(sa, da, sb, db)["total"]

        def solve(precision, defect_every):
            info, E, R, _ = ctx.davidson_roots(2, max_it=100, max_nb=12, eps=args.davidson_tol, precision=precision,
                                               defect_every=defect_every, to_host=False)
            one = [ctx.rdm_device(ctx.wavefunction_device(r), two=False)[0] for r in range(2)]
            return info, E, R, one

        f64, E64, R64, one64 = solve(sbdx.SBDX_FP64, 0)
        out["fp64"] = {"seconds": f64.seconds, "sigmas": f64.n_sigma64, "energies": E64.tolist(),
                       "residuals": R64.tolist(), "converged": bool(f64.converged)}
        for label, every in (("mixed_every4", 4), ("mixed_adaptive", 0)):
            f32, E32, R32, one32 = solve(sbdx.SBDX_FP32, every)
            out[label] = {"seconds": f32.seconds, "sigmas_fp32": f32.n_sigma, "sigmas_fp64": f32.n_sigma64,
                          "energies": E32.tolist(), "residuals": R32.tolist(), "converged": bool(f32.converged),
                          "dE_vs_fp64": (E32 - E64).tolist(),
                          "rdm1_maxabs_vs_fp64": [float(np.abs(one32[r] - one64[r]).max()) for r in range(2)],
                          "speedup_vs_fp64": f64.seconds / f32.seconds if f32.seconds > 0 else None}
    return out


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    prob = load_workload(args.workload)
    threads = cpu_cores()
    res, rows = reference_sample(prob, target_s=2.0, reps=args.warmup + args.steps, threads=threads)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": rows}))
        return 0
    row0, rows = rows
    timed = res[args.warmup:]
    secs = sum(r["seconds"] for r in timed)
    pairs = sum(r["pairs"] for r in timed)
    value = pairs / secs
    sample = (f"reference mult (chemistry/tpb/mult.h) on bra alpha rows [{row0},{row0 + rows}) of {prob.na} "
              f"(middle of the sorted list), all beta rows, {threads} threads")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / len(timed),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": workload_desc(args.workload),
                   "parallelism": "reference at MPI world size 1, OpenMP threads",
                   "sample_rows": rows},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_sharded(args, rank, world, local):
    """N > 1: one sigma of the workload split over the GPUs by alpha-row
    shards (sbdx/shard.py): each step gathers the whole C on every GPU (one
    NCCL broadcast per rank) and evaluates the rank's rows
    (sbdx_sigma_rows_device). value = det-pairs of the whole sigma / the
    slowest rank's step time (strong scaling: the work is fixed as N grows).
    Also the sharded FP64 Davidson to the tolerance (time to solution)."""
    import torch
    import torch.distributed as dist

    import sbdx
    from sbdx import shard, synth

    torch.cuda.set_device(local)
    if world == 1 and "MASTER_ADDR" not in os.environ:  # --sharded without torchrun
        import socket

        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    comm = shard.Comm(dist.group.WORLD)
    prob = load_workload(args.workload)
    ctx = sbdx.Context(local)
    ctx.load(prob)
    ctx.build_connectivity()
    if args.tune:
        tune = tuple(int(x) for x in args.tune.split(","))
        ctx.set_tuning(*tune)
    else:
        tune = ctx.autotune()
    sa, da, _ = ctx.connectivity(0)
    sb, db, _ = ctx.connectivity(1)
    dp = synth.det_pairs(sa, da, sb, db)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    bounds = shard.partition(shard.row_work(ctx), world)
    a0, a1 = bounds[rank]
    nb = prob.nb
    n_loc = (a1 - a0) * nb
    op = shard.ShardedSigma(ctx, comm, bounds)
    gen = torch.Generator(device="cuda").manual_seed(1234)
    C = torch.randn(prob.D, dtype=torch.float64, device="cuda", generator=gen)
    C_loc = C[a0 * nb:a1 * nb].clone()
    del C
    S_loc = torch.empty_like(C_loc)

    def barrier():
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        op(C_loc, S_loc)
    barrier()
    sampler = ClockSampler(gpu_index(local))
    sampler.start()
    launches0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        op(C_loc, S_loc)
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    launches = ctx.launches - launches0
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist)
    value = dp["total"] / (ms * 1e-3)
    # end to end: the rank's rows from pinned host memory and back, every step
    hC = C_loc.cpu().pin_memory()
    hS = torch.empty(n_loc, dtype=torch.float64).pin_memory()
    barrier()
    n_e2e = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(n_e2e):
        C_loc.copy_(hC, non_blocking=True)
        op(C_loc, S_loc)
        hS.copy_(S_loc, non_blocking=True)
        stream.synchronize()
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(max(e0.elapsed_time(e1) / n_e2e, 1e3 * (time.perf_counter() - t0) / n_e2e), dist)
    # per-phase durations of this rank's row-range product (events between its
    # kernels; every rank takes the same collective steps)
    ctx.set_profiling(True)
    for _ in range(max(2, min(args.steps, 5))):
        op(C_loc, S_loc)
    ncalls, phases = ctx.phase_times()
    ctx.set_profiling(False)
    phases = {k: v / max(ncalls, 1) for k, v in phases.items()}
    dav = None
    if not args.no_davidson:
        hii = torch.from_numpy(ctx.diag_terms()[a0 * nb:a1 * nb]).cuda()
        W0 = torch.zeros(n_loc, dtype=torch.float64, device="cuda")
        if a0 == 0 and n_loc > 0:
            W0[0] = 1.0
        E, _, inf = shard.davidson(op, hii, comm, W0, max_it=100, max_nb=12, eps=args.davidson_tol)
        dav = {"tol": args.davidson_tol, "max_nb": 12, "seconds": max_over_ranks(inf["seconds"], dist),
               "sigmas": inf["sigmas"], "energy": E, "residual": inf["residual"], "converged": inf["converged"]}
    hbm, peak_kind = peaks()
    B = roofline_bytes(prob, dp, 8)
    gbs = B / world / (ms * 1e-3) / 1e9
    # the alpha-beta kernel of this rank's shard against the shared-memory
    # pipe, as at N = 1: 16 conflict-free bytes per alpha-beta det-pair
    ab_pairs = float(sa[a0:a1].sum()) * float(sb.sum())
    ab_ms = phases.get("alpha_beta", 0.0)
    smem_peak = smem_peak_gbs((clocks or {}).get("sm_mhz") or 1965.0)
    ab_gbs = 16.0 * ab_pairs / (ab_ms * 1e-3) / 1e9 if ab_ms > 0 else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded integrals and string samples of the stated law)",
        "config": {"workload": args.workload, "desc": workload_desc(args.workload), "dets": prob.D, "na": prob.na,
                   "nb": nb, "norb": prob.L, "det_pairs_per_sigma": dp["total"],
                   "parallelism": f"alpha-row shards x{world} (whole C gathered per step)",
                   "shards": bounds, "tuning": {"same_vec": tune[0], "ab_rows": tune[1]},
                   "l2": f"inputs larger than L2 (C = {8 * prob.D / 1e6:.0f} MB > 126 MB), no flush"},
        "roofline": {"bound": "smem", "achieved": ab_gbs, "peak": smem_peak, "unit": "GB/s",
                     "frac": ab_gbs / smem_peak if ab_gbs else None, "traffic": None,
                     "kernel": "sigma_ab_v7", "phase": "alpha_beta", "shard": [a0, a1],
                     "ms_per_launch": ab_ms, "smem_bytes_per_launch": 16.0 * ab_pairs,
                     "peak_kind": "128 B/clk/SM x SMs x sampled SM clock (rank 0's shard)",
                     "phases": phases,
                     "hbm": {"model": "whole sigma of a row shard (SpMV byte model / N per GPU)", "gbs": gbs,
                             "model_frac": gbs / hbm, "peak_gbs": hbm, "peak_kind": peak_kind}},
        "e2e": {"value": dp["total"] / (ms_e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 8 * prob.D,
                "d2h_bytes_per_step": 8 * prob.D, "ms_per_step": ms_e2e},
        "gpu_launches": launches,
        "clocks": clocks,
        "davidson_sharded": dav,
        "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(line))
    del op
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def run_ours(args, rank, world, local):
    import torch

    import sbdx
    from sbdx import synth

    if world > 1 or args.sharded:
        return run_sharded(args, rank, world, local)
    torch.cuda.set_device(local)
    pg = None
    prob = load_workload(args.workload)
    ctx = sbdx.Context(local)
    ctx.load(prob)
    ctx.build_connectivity()
    if args.tune:
        tune = tuple(int(x) for x in args.tune.split(","))
        ctx.set_tuning(*tune)
    else:
        tune = ctx.autotune()
    sa, da, _ = ctx.connectivity(0)
    sb, db, _ = ctx.connectivity(1)
    dp = synth.det_pairs(sa, da, sb, db)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    D = prob.D
    gen = torch.Generator(device="cuda").manual_seed(1234 + rank)
    C = torch.randn(D, dtype=torch.float64, device="cuda", generator=gen)
    S = torch.empty_like(C)

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    def max_over_ranks_(x: float) -> float:
        return max_over_ranks(x, pg)

    # ---- device-resident FP64 sigma (value) --------------------------------------
    for _ in range(args.warmup):
        ctx.sigma_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr())
    barrier()
    sampler = ClockSampler(gpu_index(local))
    sampler.start()
    launches0 = ctx.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ctx.sigma_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr())
    e1.record(stream)
    barrier()
    clocks = sampler.stop()
    launches = ctx.launches - launches0
    ms, value = replica_throughput(dp["total"], e0.elapsed_time(e1) / args.steps, world, pg)

    # ---- per-phase durations (events between the sigma's kernels) ---------------
    ctx.set_profiling(True)
    nprof = max(2, min(args.steps, 5))
    for _ in range(nprof):
        ctx.sigma_device(sbdx.SBDX_FP64, C.data_ptr(), S.data_ptr())
    ncalls, phases = ctx.phase_times()
    ctx.set_profiling(False)
    phases = {k: v / ncalls for k, v in phases.items()}
    dominant = max(phases, key=phases.get)

    # ---- FP32-storage sigma ---------------------------------------------------
    C32, S32 = C.float(), torch.empty(D, dtype=torch.float32, device="cuda")
    for _ in range(2):
        ctx.sigma_device(sbdx.SBDX_FP32, C32.data_ptr(), S32.data_ptr())
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        ctx.sigma_device(sbdx.SBDX_FP32, C32.data_ptr(), S32.data_ptr())
    e1.record(stream)
    barrier()
    ms32 = max_over_ranks_(e0.elapsed_time(e1) / args.steps)
    ctx.set_profiling(True)
    for _ in range(nprof):
        ctx.sigma_device(sbdx.SBDX_FP32, C32.data_ptr(), S32.data_ptr())
    ncalls32, phases32 = ctx.phase_times()
    ctx.set_profiling(False)
    phases32 = {k: v / ncalls32 for k, v in phases32.items()}
    del C32, S32

    # ---- end to end through the C-ABI with pinned host buffers --------------------
    hC = C.cpu().pin_memory()
    hS = torch.empty(D, dtype=torch.float64).pin_memory()
    ctx.sigma_host_ptr(hC.data_ptr(), hS.data_ptr())
    barrier()
    n_e2e = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(n_e2e):
        ctx.sigma_host_ptr(hC.data_ptr(), hS.data_ptr())
    e1.record(stream)
    barrier()
    wall_e2e = (time.perf_counter() - t0) / n_e2e
    ms_e2e = max_over_ranks_(max(e0.elapsed_time(e1) / n_e2e, 1e3 * wall_e2e))
    e2e_value = world * dp["total"] / (ms_e2e * 1e-3)
    del hC, hS

    # ---- Davidson to 1e-8: FP64 vs mixed -------------------------------------------
    dav = None
    if not args.no_davidson:
        del S
        torch.cuda.empty_cache()
        i64, _ = ctx.davidson(max_it=100, max_nb=12, eps=args.davidson_tol)
        i32, _ = ctx.davidson(max_it=100, max_nb=12, eps=args.davidson_tol, precision=sbdx.SBDX_FP32)
        dav = {"tol": args.davidson_tol, "max_nb": 12,
               "fp64": {"seconds": i64.seconds, "sigmas": i64.n_sigma, "energy": i64.energy, "residual": i64.residual,
                        "converged": bool(i64.converged)},
               "mixed": {"seconds": i32.seconds, "sigmas_fp32": i32.n_sigma, "sigmas_fp64": i32.n_sigma64,
                         "energy": i32.energy, "residual": i32.residual, "converged": bool(i32.converged),
                         "dE_vs_fp64": i32.energy - i64.energy},
               "speedup_mixed_vs_fp64": i64.seconds / i32.seconds if i32.seconds > 0 else None}
        # the mixed solver's algorithm (Olsen-Davidson, FP64 anchor, thick restart)
        # with FP64 corrections: separates the algorithmic gain from the precision gain
        ib, Eb, rb, _ = ctx.davidson_roots(1, max_it=100, max_nb=12, eps=args.davidson_tol)
        dav["fp64_same_algorithm"] = {"seconds": ib.seconds, "sigmas": ib.n_sigma64, "energy": float(Eb[0]),
                                      "residual": float(rb[0]), "converged": bool(ib.converged),
                                      "speedup_mixed_vs_this": ib.seconds / i32.seconds if i32.seconds > 0 else None}
        if args.roots > 1:
            k = args.roots
            f64, E64, r64, _ = ctx.davidson_roots(k, max_it=100, max_nb=12, eps=args.davidson_tol)
            f32, E32, r32, _ = ctx.davidson_roots(k, max_it=100, max_nb=12, eps=args.davidson_tol,
                                                  precision=sbdx.SBDX_FP32)
            dav["roots"] = {"nroots": k,
                            "fp64": {"seconds": f64.seconds, "sigmas": f64.n_sigma64, "energies": E64.tolist(),
                                     "residuals": r64.tolist(), "converged": bool(f64.converged)},
                            "mixed": {"seconds": f32.seconds, "sigmas_fp32": f32.n_sigma, "sigmas_fp64": f32.n_sigma64,
                                      "energies": E32.tolist(), "residuals": r32.tolist(),
                                      "converged": bool(f32.converged),
                                      "dE_vs_fp64": (E32 - E64).tolist()},
                            "speedup_mixed_vs_fp64": f64.seconds / f32.seconds if f32.seconds > 0 else None}

    # ---- mixed precision on the 400 M-determinant workload, 2 roots -----------------
    mixed = None
    if not args.no_davidson and args.mixed and world == 1:
        mixed = run_mixed(args)

    # ---- batched subspaces (64 independent solves sharing one Hamiltonian) ---------
    batched = None
    if not args.no_davidson and not args.no_batched and world == 1:
        batched = run_batched(args)

    # ---- CPU baseline (reference OpenMP mult, bounded sample, rank 0, N=1) -------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = cpu_cores()
        res, rows = reference_sample(prob, target_s=args.cpu_seconds, reps=1, threads=threads)
        if res is not None:
            r = res[0]
            row0, nrows = rows
            cpu = {"value": r["pairs"] / r["seconds"], "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"reference mult (chemistry/tpb/mult.h) on bra alpha rows [{row0},{row0 + nrows}) of "
                             f"{prob.na} (middle of the sorted list), all beta rows: {r['pairs']:.3e} det-pairs "
                             f"in {r['seconds']:.2f} s"}
        else:
            cpu = {"value": None, "unit": UNIT, "cores": threads, "kind": "reference", "sample": rows}

    hbm, peak_kind = peaks()
    stored = None
    if args.stored and world == 1:
        stored = run_stored(args, hbm)
    proj = None
    if args.projection_d is None:
        args.projection_d = int(prob.D)
    if args.projection_d and world == 1:
        proj = run_projection(args, hbm)
    diff = None
    if args.diff and world == 1 and not args.no_davidson:
        diff = run_differentiation(args)
    B = roofline_bytes(prob, dp, 8)
    pb = phase_bytes(prob, dp, 8)
    pb32 = phase_bytes(prob, dp, 4)
    kern = PHASE_KERNELS[dominant]
    if dominant == "alpha_beta" and tune[1] // 10 != 7:
        kern = "sigma_ab_v6"  # codes 61-64: unpacked staged rows
    if dominant in ("alpha_same_spin", "beta_same_spin") and tune[0] // 10 == 3:
        kern = "sigma_same_blk"  # codes 31-38: blocks of 4 bra strings
    # The alpha-beta kernel gathers from rows staged in shared memory; DRAM
    # moves a few percent of the SpMV byte model (profiles/sigma_ab_v7_cfg2.md),
    # so its bound is the shared-memory pipe: frac = conflict-free shared bytes
    # (two 8-byte elements per det-pair) / time / (128 B per clock per SM).
    sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
    smem_peak = smem_peak_gbs(sm_mhz)
    traffic = traffic_per_launch(kern, args.workload)
    t_dom = phases[dominant] * 1e-3
    hbm_model = {"algorithmic_bytes_per_launch": pb[dominant], "gbs": pb[dominant] / t_dom / 1e9,
                 "model_frac": pb[dominant] / t_dom / 1e9 / hbm,
                 "dram_gbs": traffic / t_dom / 1e9 if traffic else None,
                 "dram_frac": traffic / t_dom / 1e9 / hbm if traffic else None, "peak_gbs": hbm,
                 "peak_kind": peak_kind}
    if dominant == "alpha_beta":
        sbytes = ab_smem_bytes(dp, 8)
        achieved = sbytes / t_dom / 1e9
        roofline = {"bound": "smem", "achieved": achieved, "peak": smem_peak, "unit": "GB/s",
                    "frac": achieved / smem_peak, "traffic": traffic, "kernel": kern, "phase": dominant,
                    "smem_bytes_per_launch": sbytes, "ms_per_launch": phases[dominant],
                    "peak_kind": f"128 B/clk/SM x SMs x {sm_mhz:.0f} MHz (sampled)", "hbm": hbm_model}
    else:
        achieved = pb[dominant] / t_dom / 1e9
        roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                    "traffic": traffic, "kernel": kern, "phase": dominant,
                    "algorithmic_bytes_per_launch": pb[dominant], "ms_per_launch": phases[dominant],
                    "peak_kind": peak_kind}
    roofline["phases"] = {k: {"ms": phases[k], "bytes": pb[k], "gbs": pb[k] / (phases[k] * 1e-3) / 1e9,
                              "model_frac": pb[k] / (phases[k] * 1e-3) / 1e9 / hbm} for k in phases}
    roofline["phases"]["alpha_beta"]["smem_frac"] = ab_smem_bytes(dp, 8) / (phases["alpha_beta"] * 1e-3) / 1e9 / smem_peak
    roofline["sigma"] = {"algorithmic_bytes": B, "ms": ms, "gbs": B / (ms * 1e-3) / 1e9,
                         "model_frac": B / (ms * 1e-3) / 1e9 / hbm}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded integrals and string samples of the stated law)",
        "config": {"workload": args.workload, "desc": workload_desc(args.workload), "dets": D, "na": prob.na, "nb": prob.nb,
                   "norb": prob.L, "det_pairs_per_sigma": dp["total"], "parallelism": "one GPU (alpha-row shards x1)",
                   "tuning": {"same_vec": tune[0], "ab_rows": tune[1]},
                   "l2": f"inputs larger than L2 (C = {8 * D / 1e6:.0f} MB > 126 MB), no flush"
                         if 8 * D > 126e6 else "C fits in L2: timings include L2 reuse"},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * D, "d2h_bytes_per_step": 8 * D,
                "ms_per_step": ms_e2e},
        "gpu_launches": launches,
        "clocks": clocks,
        "fp32_sigma": {"value": world * dp["total"] / (ms32 * 1e-3), "ms_per_step": ms32,
                       "phases": {k: {"ms": phases32[k], "gbs": pb32[k] / (phases32[k] * 1e-3) / 1e9}
                                  for k in phases32},
                       "alpha_beta_smem_frac": ab_smem_bytes(dp, 4) / (phases32["alpha_beta"] * 1e-3) / 1e9
                       / smem_peak},
        "davidson": dav,
        "mixed_precision": mixed,
        "batched": batched,
        "stored_hamiltonian": stored,
        "projection": proj,
        "differentiation": diff,
        "cpu_baseline": cpu,
    }
    line["summary"] = summary(line)
    if rank == 0:
        print(json.dumps(line))
    ctx.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def summary(line) -> dict:
    """The headline figures in one short object, printed last on the line."""
    def get(*keys):
        d = line
        for k in keys:
            if not isinstance(d, dict) or d.get(k) is None:
                return None
            d = d[k]
        return d

    out = {"sigma_fp64_ms": line["ms_per_step"], "sigma_fp32_ms": get("fp32_sigma", "ms_per_step"),
           "alpha_beta_smem_frac": get("roofline", "phases", "alpha_beta", "smem_frac"),
           "mixed_vs_fp64_cfg2_1root": get("davidson", "speedup_mixed_vs_fp64"),
           "mixed_vs_fp64_cfg2_2roots": get("davidson", "roots", "speedup_mixed_vs_fp64")}
    m = line.get("mixed_precision")
    if m:
        for lab in ("mixed_every4", "mixed_adaptive"):
            out[f"{lab}_vs_fp64_cfg3_2roots"] = m[lab]["speedup_vs_fp64"]
            out[f"{lab}_cfg3_max_abs_dE"] = max(abs(x) for x in m[lab]["dE_vs_fp64"])
            out[f"{lab}_cfg3_max_rdm1_err"] = max(m[lab]["rdm1_maxabs_vs_fp64"])
    out["batched_mixed_vs_sequential_fp64"] = get("batched", "speedup_batched_mixed_vs_sequential_fp64")
    out["batched_mixed_graph_steps_vs_sequential_fp64"] = get("batched",
                                                              "speedup_batched_mixed_graph_steps_vs_sequential_fp64")
    pr = line.get("projection")
    if pr:
        out["projection_dmma_frac_of_hbm"] = {f"{c['precision']}_m{c['m']}_nx{c['nx']}": round(c["frac_of_hbm"], 3)
                                               for c in pr["cases"] if (c["m"], c["nx"]) in ((24, 2), (62, 2))}
    d = line.get("differentiation")
    if d:
        out["backward_over_forward"] = d["backward_seconds"] / d["forward_seconds"]
        out["backward_fd_rel_err"] = d["max_rel_err_vs_central_differences"]
    return out


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    return run_ours(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
