#!/usr/bin/env python
"""Benchmark of the semi-analytic E_l assembly (pair-integrals/s).

Workload: unit icosphere subdivided 3x (1280 triangles, 3840 unknowns per
step), rho=1, mu=1, lambda=1, dt=0.025, T=1 (Nt=40, L=40 Toeplitz blocks),
7-point outer Gauss-Hammer rule, plain FP64.  One step = assembly of
E_0..E_39 (26.68 M non-null pair-lags on this generated icosphere, 26.14 M on
the reference's sphereUniform_3 mesh; 4.7 GB of output, far larger than L2).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) each rank assembles a row panel of source triangles
(no data-path collective); the job value is all ranks' pair-integrals over
the slowest rank's device time.  ``--impl reference`` times the CPU
restatement of the reference's MATLAB path (the oracle) on the host cores.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "E_l assembly pair-integrals/s (plain FP64 SA, sphere N=1280, L=40, GH7)"
UNIT = "pair-integrals/s"

# FP64 operation census of the SA path (oracle compiled with a counting
# scalar; +,-,*,/,sqrt and each transcendental = 1 flop), on 5000 seeded
# pairs of this workload: flops per non-null pair-lag when every time level
# is evaluated once (the schedule the kernel runs), and under the
# reference's three-instants-per-lag schedule.
FLOPS_PER_PAIR_INTEGRAL = 19_232.0
FLOPS_PER_PAIR_INTEGRAL_REF_SCHEDULE = 53_560.0

# DRAM bytes (read + write) of the dominant kernel, the level pass of the
# two-pass assembly (sa_level_kernel storing F(t_k) of every pair and level):
# ncu on the sphere N=320 case (2,478,740 pair-integrals, one launch) measured
# 11.78 MB read + 105.78 MB written; the writes are the stored levels, which
# grow with the pair-integrals, so a launch's traffic is scaled by the
# pair-integrals it processes.
NCU_LEVEL_PASS_BYTES_N320 = 11.780352e6 + 105.780480e6
NCU_LEVEL_PASS_UNITS_N320 = 2_478_740


KERNEL = "sa_level_kernel (level pass)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=2)
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def physical_gpu(local_rank: int) -> str:
    """The nvidia-smi id (index or UUID) of this rank's device: the
    local_rank-th entry of CUDA_VISIBLE_DEVICES when it is set."""
    ids = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
    return ids[local_rank] if local_rank < len(ids) else str(local_rank)


# --------------------------------------------------------------------------
def fp64_peak_tflops(torch) -> float:
    """Measured FP64 throughput: cuBLAS DGEMM (torch.matmul, float64,
    8192^3, 2 n^3 flops), best of 5."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2 * n ** 3 / best / 1e12


def cpu_baseline(workload, target_s: float = 12.0, nthreads: int = 0):
    """The oracle (C++ restatement of the reference's SA path, the reference's
    three-instants-per-lag schedule) on a seeded sample of non-null pair-lags
    of the same workload, all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O
    m, prm = workload.mesh, workload.params
    L = O.num_blocks(m, prm)
    N = m.numberTriangles
    rng = np.random.default_rng(11)
    ctr, ml = m.center, m.maxL

    def sample(q):
        src = rng.integers(0, N, 4 * q)
        fld = rng.integers(0, N, 4 * q)
        lag = rng.integers(0, L, 4 * q)
        d = np.linalg.norm(ctr[fld] - ctr[src], axis=1)
        ok = ((lag - 1) * prm.velS * prm.dt < d + ml[fld] + ml[src]) & \
             ((lag + 1) * prm.velP * prm.dt >= d - ml[fld] - ml[src])
        return src[ok][:q], fld[ok][:q], lag[ok][:q]
    cores = os.cpu_count() if nthreads <= 0 else nthreads
    s, f, l = sample(20000)
    t0 = time.perf_counter()
    O.assemble_sa_pairs(m, prm, workload.n_gh, s, f, l, nthreads=cores)
    t1 = time.perf_counter()
    q = int(min(5_000_000, max(20000, len(s) * target_s / max(t1 - t0, 1e-3))))
    s, f, l = sample(q)
    t0 = time.perf_counter()
    O.assemble_sa_pairs(m, prm, workload.n_gh, s, f, l, nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": len(s) / dt, "unit": UNIT, "cores": cores, "kind": "port", "seconds": dt, "pairs": len(s),
            "sample": f"{len(s)} seeded non-null (source, field, lag) blocks of the sphere N=1280 GH7 workload, "
                      f"oracle (C++ restatement of BEMenerg_coreSA_calcMatrixSubBlock, 3 instants per lag), "
                      f"{dt:.1f} s"}


def forms(core, problem, torch, w, dm, L, plain_rate):
    """The assembly forms against the plain FP64 assembly: mixed precision on
    the benchmark workload (speed and error of blocks, density, displacement)
    and the batched persistent launch on 64 instances of uneven size (against
    one launch per instance)."""
    def timed(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    n3 = 3 * dm.N
    out = {}

    def mixed_form(n_gh):
        # the sphere of 1280 triangles with outer rule n_gh: assembly times,
        # errors of blocks, density and displacement (256 exterior points x 40
        # times) of the mixed form against FP64; E_0's asymmetry and the
        # density of the Cholesky factorisation of its symmetric part against LU
        buf64 = torch.empty((L, n3, n3), dtype=torch.float64, device="cuda")
        buf32 = torch.empty_like(buf64)
        t64 = timed(lambda: core.assemble_sa(dm, w.params, n_gh, 0, L, out=buf64))
        t32 = timed(lambda: core.assemble_sa(dm, w.params, n_gh, 0, L, out=buf32, prec=core.PREC_MIXED))
        e_rel = float((buf32 - buf64).norm() / buf64.norm())
        del buf32
        E0 = buf64[0]
        asym = float((E0 - E0.t()).norm() / E0.norm())
        b = core.rhs(dm, w.params, n_gh, w.datum)
        phi_ch = core.march(buf64.transpose(1, 2), b, factor=core.FACTOR_CHOLESKY)
        phi64, _ = core.timemarch_sa(dm, w.params, n_gh, w.datum)
        phi32, _ = core.timemarch_sa(dm, w.params, n_gh, w.datum, prec=core.PREC_MIXED)
        u64 = core.pp_sa(dm, w.params, phi64, w.points, w.times)
        u32 = core.pp_sa(dm, w.params, phi32, w.points, w.times)
        res = {"assembly_ms": t32, "fp64_assembly_ms": t64, "speedup": t64 / t32, "blocks_rel_err": e_rel,
               "density_rel_err": float((phi32 - phi64).norm() / phi64.norm()),
               "displacement_rel_err": float((u32 - u64).norm() / u64.norm()),
               "points": int(len(w.points)), "times": int(len(w.times)),
               "e0_asymmetry": asym,
               "cholesky_vs_lu_density_rel": float((phi_ch - phi64).norm() / phi64.norm()),
               "scope": "FP32 edge Gauss-Legendre nodes, FP64 closed forms / moments / marching"}
        del buf64, phi64, phi32, phi_ch
        torch.cuda.empty_cache()
        return res

    out["mixed"] = mixed_form(w.n_gh)
    out["mixed_gh12"] = mixed_form(12)
    out["selector"] = selector_form(core, torch, w, dm, L, timed)
    inst = problem.batch_workload(count=64, seed=4)
    dms = [core.DeviceMesh(m) for _, m, _ in inst]
    prms = [p for _, _, p in inst]
    nlag = [core.num_blocks(d, p) for d, p in zip(dms, prms)]          # all lags of every instance
    outs = [torch.empty((l, 3 * d.N, 3 * d.N), dtype=torch.float64, device="cuda") for d, l in zip(dms, nlag)]
    counts = [core.assemble_sa(d, p, 7, 0, l, out=o, count=True)[1] for d, p, l, o in zip(dms, prms, nlag, outs)]
    plan = core.BatchPlan(dms, prms, 7, nlag=nlag, prec=core.PREC_FP64)
    t_batch = timed(lambda: plan.assemble(outs))
    t_seq = timed(lambda: [core.assemble_sa(d, p, 7, 0, l, out=o) for d, p, l, o in zip(dms, prms, nlag, outs)])
    plan32 = core.BatchPlan(dms, prms, 7, nlag=nlag, prec=core.PREC_MIXED)
    t_b32 = timed(lambda: plan32.assemble(outs))
    info = plan.info()
    out["batched"] = {"instances": len(inst), "N_range": [min(d.N for d in dms), max(d.N for d in dms)],
                      "lags_per_instance": "all (L of each instance)",
                      "output_gb": sum(9 * d.N ** 2 * l * 8 for d, l in zip(dms, nlag)) / 1e9,
                      "pair_integrals": int(sum(counts)),
                      "batch_ms": t_batch, "one_launch_per_instance_ms": t_seq, "speedup": t_seq / t_batch,
                      "batch_mixed_ms": t_b32, "pair_integrals_per_s": sum(counts) / t_batch * 1e3,
                      "schedule": ("persistent launch over all instances" if info["warps_per_block"]
                                   else "one two-pass assembly per instance"),
                      "tile": {"warps_per_block": info["warps_per_block"], "pairs_per_grab": info["pairs_per_grab"]}}
    plan.close(); plan32.close()
    del outs
    torch.cuda.empty_cache()
    return out


def selector_form(core, torch, w, dm, L, timed):
    """The learned selector on the benchmark sphere: trained on 200k (pair,
    lag) samples of the configuration 1-4 meshes, then the selected assembly
    (FP64, and with the mixed form) against the plain assembly on the maximal
    rule, with the density and displacement errors against the latter."""
    from elastodynamicebem_b200 import selector as S
    t0 = time.perf_counter()
    X, Y = S.training_set(200_000)
    params, losses = S.train(X, Y, epochs=20)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    n3 = 3 * dm.N
    buf = torch.empty((L, n3, n3), dtype=torch.float64, device="cuda")
    p = w.params
    t_max = timed(lambda: core.assemble_sa_rule(dm, p, *S.RULES[-1], 0, L, out=buf), reps=1)
    E = core.assemble_sa_rule(dm, p, *S.RULES[-1], 0, L, out=buf)
    b = core.rhs(dm, p, 7, w.datum)
    phi_max = core.march(E, b)
    u_max = core.pp_sa(dm, p, phi_max, w.points, w.times)
    t_inf = timed(lambda: core.selector_infer(params, dm, p, S.THRESHOLD, 0, L), reps=1)
    cls, counts = core.selector_infer(params, dm, p, S.THRESHOLD, 0, L)
    res = {"rules": [list(r) for r in S.RULES], "train_samples": int(X.shape[0]), "train_s": t_train,
           "final_loss": float(losses[-1]), "lags_per_class": counts, "max_rule_ms": t_max, "inference_ms": t_inf}
    for name, prec in (("fp64", core.PREC_FP64), ("mixed", core.PREC_MIXED)):
        t = timed(lambda: core.assemble_sa_selected(dm, p, cls, S.RULES, 0, L, out=buf, prec=prec), reps=1)
        E, _ = core.assemble_sa_selected(dm, p, cls, S.RULES, 0, L, out=buf, prec=prec)
        phi = core.march(E, b)
        u = core.pp_sa(dm, p, phi, w.points, w.times)
        res[name] = {"assembly_ms": t, "speedup_vs_max_rule": t_max / t,
                     "density_rel_err": float((phi - phi_max).norm() / phi_max.norm()),
                     "displacement_rel_err": float((u - u_max).norm() / u_max.norm())}
    res["scope"] = ("selector classes per (pair, lag) among the rules, lags a wavefront sweeps on the maximal "
                    "rule; the batched launch takes one rule per plan, so selector + mixed is the combination "
                    "measured on this mesh")
    del buf, E, phi_max, cls
    torch.cuda.empty_cache()
    return res


def workload_config(w, L: int, pairs: int, world: int) -> dict:
    """The `config` object of both arms' JSON lines."""
    N, prm = w.mesh.numberTriangles, w.params
    out_gb = 9 * N * N * L * 8 / 1e9          # dense E_0..E_{L-1}, FP64
    rel = "far larger than" if out_gb > 4 * 0.126 else ("larger than" if out_gb > 0.126 else "not larger than")
    return {"workload": f"sphere_icosphere{3 if N == 1280 else 2}_N{N}_L{L}_GH7", "N": N, "L": L, "n_gh": w.n_gh,
            "rho": prm.rho, "mu": prm.mu, "lambda": prm.lam, "dt": prm.dt, "nT": prm.nT,
            "pair_integrals_per_step": pairs, "parallelism": f"source-row panels x{world}, balanced by non-null pair-lags",
            "l2": f"output {out_gb:.2f} GB per step written to HBM, {rel} L2 (126 MB)"}


def reference_arm(args, rank: int):
    """The reference's path on the host cores: the oracle (C++ restatement of
    its MATLAB SA assembly, three instants per lag) on bounded seeded samples
    of the same workload, one sample per step; rank 0 only."""
    from elastodynamicebem_b200 import problem
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    w = problem.sphere_workload(7, subdivisions=3 if args.workload == "sphere1280" else 2)
    L = O.num_blocks(w.mesh, w.params)
    pairs = O.count_nonnull(w.mesh, w.params, L)
    vals, secs, sizes = [], [], []
    info = None
    for _ in range(args.warmup):
        cpu_baseline(w, target_s=min(2.0, args.reference_sample_s))
    for _ in range(args.steps):
        info = cpu_baseline(w, target_s=args.reference_sample_s)
        vals.append(info["value"])
        secs.append(info["seconds"])
        sizes.append(info["pairs"])
    v = statistics.median(vals)
    info["value"] = v
    frac = statistics.median(sizes) / pairs
    cfg = workload_config(w, L, pairs, 1)
    cfg["reference_step"] = (f"each step is a seeded sample of {int(statistics.median(sizes))} of the "
                             f"{pairs} pair-integrals of a full step ({frac:.3f} of it); ms_per_step is the "
                             f"measured time of that sample, value its pair-integrals/s")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": statistics.median(secs) * 1e3,   # the work actually timed per step
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": info,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-peak", action="store_true", help="skip the DGEMM peak measurement")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed-precision and batched measurements")
    ap.add_argument("--reference-sample-s", type=float, default=8.0,
                    help="seconds of host-core work per step of --impl reference")
    ap.add_argument("--workload", default="sphere1280", choices=["sphere1280", "sphere320"],
                    help="sphere1280 is the benchmark; sphere320 (icosphere 2) is the small profiling case")
    args = ap.parse_args()
    if args.warmup < 3:
        log("warning: fewer than 3 warm-up steps")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local_rank))

    from elastodynamicebem_b200 import core, problem, shard

    w = problem.sphere_workload(7, subdivisions=3 if args.workload == "sphere1280" else 2)
    m, prm = w.mesh, w.params
    N = m.numberTriangles
    dm = core.DeviceMesh(m)
    L = core.num_blocks(dm, prm)
    # source-row panels balanced by non-null pair-lags (prefix sum of the row counts)
    src0, nsrc = shard.row_panel(rank, world, N, shard.row_weights(m, prm, L) if world > 1 else None)
    n3 = 3 * N
    out = torch.empty((L, n3, 3 * nsrc), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def step(count=False):
        return core.assemble_sa_panel(dm, prm, w.n_gh, 0, L, src0, nsrc, out=out, stream=stream, count=count)

    _, my_pairs = step(count=True)
    total_pairs = my_pairs
    if world > 1:
        t = torch.tensor([my_pairs], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        total_pairs = int(t.item())
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()

    sampler = ClockSampler(physical_gpu(local_rank))
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    # per-pass device times of the library's own launches (CUDA events on the
    # assembly stream around each launch), from separate steps after the timed
    # ones: reading them synchronises the host at the end of each call, which
    # would leave the GPU idle between the timed steps
    from elastodynamicebem_b200 import lib as _lib
    import ctypes as _C
    L_ = _lib.load()
    prof_ms = (_C.c_double * 2)()
    prof_n = (_C.c_longlong * 2)()
    prof_steps = min(args.steps, 3)
    L_.ebem_profile_read(prof_ms, prof_n, 1)
    L_.ebem_profile_enable(1)
    for _ in range(prof_steps):
        step()
    torch.cuda.synchronize()
    L_.ebem_profile_enable(0)
    L_.ebem_profile_read(prof_ms, prof_n, 1)
    my_s = ev0.elapsed_time(ev1) / 1e3
    t_max = my_s
    if world > 1:
        t = torch.tensor([my_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = total_pairs * args.steps / t_max
    # launches per step of the dominant kernel (the level pass, one per chunk
    # of field columns) and its average launch time; the emission pass is the
    # other launch of each chunk
    launches = max(1, int(prof_n[0]) // prof_steps)
    kernel_s = prof_ms[0] / 1e3 / max(1, int(prof_n[0]))
    emit_ms = prof_ms[1] / prof_steps

    # end to end through the C ABI with host buffers: mesh upload, assembly,
    # copy of E to pinned host memory, every step
    host = torch.empty((L, n3, 3 * nsrc), dtype=torch.float64).pin_memory()
    h2d = m.coordinates.nbytes + m.triangles.astype(np.int32).nbytes
    d2h = host.numel() * 8
    e2e_times = []
    for s in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        dme = core.DeviceMesh(m)
        core.assemble_sa_panel(dme, prm, w.n_gh, 0, L, src0, nsrc, out=host)
        dme.close()
        dt = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([dt], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        if s > 0:
            e2e_times.append(dt)
    e2e_value = total_pairs / statistics.median(e2e_times) if e2e_times else None
    # the host link's device-to-host rate into the same pinned buffer (1 GiB,
    # CUDA events): an end-to-end step takes at least d2h bytes / this rate
    flat = host.view(-1)
    nb = min(flat.numel(), 1 << 27)
    src = torch.zeros(nb, dtype=torch.float64, device="cuda")
    cur = torch.cuda.current_stream()
    flat[:nb].copy_(src, non_blocking=True)
    l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0.record(cur)
    flat[:nb].copy_(src, non_blocking=True)
    l1.record(cur)
    torch.cuda.synchronize()
    link_gbs = nb * 8 / (l0.elapsed_time(l1) / 1e3) / 1e9
    del src

    if rank == 0:
        peak = float("nan") if args.no_peak else fp64_peak_tflops(torch)
        achieved = FLOPS_PER_PAIR_INTEGRAL * (my_pairs / launches) / kernel_s / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(w, L, total_pairs, world),
            "gpu_launches": int(prof_n[0] + prof_n[1]) // prof_steps * args.steps,
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "traffic": NCU_LEVEL_PASS_BYTES_N320 * (my_pairs / launches) / NCU_LEVEL_PASS_UNITS_N320,
                         "peak_source": "measured: cuBLAS DGEMM 8192^3 via torch.matmul float64, best of 5",
                         "flops_per_unit": FLOPS_PER_PAIR_INTEGRAL,
                         "units_per_launch": my_pairs / launches, "launches_per_step": launches,
                         "kernel": KERNEL, "kernel_ms": kernel_s * 1e3,
                         "emission_ms_per_step": emit_ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "path": "ebem_mesh_create + ebem_assemble_sa_panel into pinned host memory + ebem_mesh_destroy",
                    "host_link_d2h_gbs": link_gbs,
                    "copy_bound": total_pairs / (d2h / (link_gbs * 1e9))},
            "clocks": clocks,
        }
        if not args.no_forms and world == 1:
            del out
            torch.cuda.empty_cache()
            line["forms"] = forms(core, problem, torch, w, dm, L, value)
            out = None
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(w)
        print(json.dumps(line), flush=True)
    del out, host
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
