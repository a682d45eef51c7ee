#!/usr/bin/env python
"""Benchmark of PVFMM particle-FMM evaluation on B200 (libpvfmm_b200).

Workload (one "step"): PVFMMEval with setup=1 -- tree build, lists and the
full FMM -- of the Laplace potential+gradient kernel on N = 4,000,000 points
drawn from a mixture of 8 isotropic Gaussians (sigma 0.02, centres uniform in
[0.1,0.9]^3, clipped to [0,1]^3), sources = targets, densities uniform
[-1,1], multipole order 8, at most 256 points per leaf.  Both forms run:
plain FP64 and mixed (FP32 near field and V-list DFTs, split-TF32 tensor-core
V-list products, FP64 check->equivalent chain).  Each form's error is the
relative L2 error of all 4 outputs against an FP64 direct sum over all
sources on 2,000 sampled targets; ``value`` is the targets/s of the fastest
form whose combined and per-component rel-L2 are all <= 1e-6.  `--workload`
selects the other benchmark configurations (100k uniform Laplace m=6, 2M
Stokes m=10, 30M ellipsoid surface m=8); the default is the one above.

Data are synthetic (seeded numpy; no dataset is named by the reference).
`value` is measured with inputs resident in HBM through the device entry
point PVFMMEvalDeviceD; `e2e` through PVFMMEvalD on pinned host buffers
(host<->device copies inside the timed region).

Multi-GPU: the evaluation runs on a single rank (no MPI across GPUs), so
`--gpus N` under torchrun runs N independent replicas (weak scaling) and
reports the summed throughput over the max-over-ranks time.

`--impl reference` times the reference's own CPU FMM (PVFMM's sources built
over a single-rank MPI and SCTL stand-in, oracle/ref_fmm/build.sh ->
oracle/_ref) through its C interface on all host threads, on a bounded sample
of the same workload (`--ref-sample` points, default 500,000).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "targets/s Laplace FMM at rel-L2 ≤1e-6 vs FP64 direct: mixed vs plain, 1 B200"
TOL = 1e-6

# Workloads (the default is the headline one; the others are the remaining
# benchmark configurations, run with --workload NAME).
WORKLOADS = {
    "gaussian4m": dict(kernel=6, m=8, max_pts=256, n=4_000_000, gen="gauss", check_seed=14, n_check=2000,
                       desc="laplace pot+grad FMM (setup=1 per step), {n} gaussian-mixture points "
                            "(8 centres, sigma 0.02), m=8, 256/leaf"),
    "uniform100k": dict(kernel=0, m=6, max_pts=300, n=100_000, gen="uniform", seeds=(1, 2), check_seed=3,
                        n_check=1000, desc="laplace potential FMM (setup=1 per step), {n} uniform points, m=6, 300/leaf"),
    "stokes2m": dict(kernel=3, m=10, max_pts=300, n=2_000_000, gen="stokes", seeds=(21, 22), check_seed=23,
                     n_check=1000, desc="stokes velocity FMM (setup=1 per step), {n} uniform points, N(0,1) forces, "
                                        "m=10, 300/leaf"),
    "ellipsoid30m": dict(kernel=0, m=8, max_pts=128, n=30_000_000, gen="ellipsoid", seeds=(41, 42), check_seed=44,
                         n_check=1000, desc="laplace potential FMM (setup=1 per step), {n} points uniform by area on "
                                            "the (0.45, 0.3, 0.15) ellipsoid, m=8, 128/leaf"),
    # periodic boundaries (box_size 1, the lattice sum over all images),
    # checked against an Ewald sum up to the additive constant of a periodic
    # potential
    "periodic4m": dict(kernel=0, m=8, max_pts=256, n=4_000_000, gen="neutral", seeds=(51, 52), check_seed=53,
                       n_check=200, box=1.0, lattice=True,
                       desc="periodic laplace potential FMM (period 1, lattice sum over all images, setup=1 per "
                            "step), {n} uniform points, charge-neutral densities, m=8, 256/leaf"),
    # the remaining kernels of the C interface (Stokes pressure, velocity
    # gradient, Biot-Savart): 1M uniform points, N(0,1) source vectors, m=6
    "stokespress1m": dict(kernel=2, m=6, max_pts=200, n=1_000_000, gen="stokes", seeds=(61, 62), check_seed=63,
                          n_check=500, desc="stokes pressure FMM (setup=1 per step), {n} uniform points, N(0,1) "
                                            "forces, m=6, 200/leaf"),
    "stokesgrad1m": dict(kernel=4, m=6, max_pts=200, n=1_000_000, gen="stokes", seeds=(64, 65), check_seed=66,
                         n_check=500, desc="stokes velocity gradient FMM (setup=1 per step), {n} uniform points, "
                                           "N(0,1) forces, m=6, 200/leaf"),
    "biotsavart1m": dict(kernel=5, m=6, max_pts=200, n=1_000_000, gen="stokes", seeds=(67, 68), check_seed=69,
                         n_check=500, desc="biot-savart FMM (setup=1 per step), {n} uniform points, N(0,1) "
                                           "currents, m=6, 200/leaf"),
    # the differentiable Laplace potential: one step = forward (pot+grad FMM)
    # + backward (swapped-role FMM on the forward's tree) through
    # pvfmm_b200.autograd.LaplaceFMM, sources = targets
    "autograd1m": dict(kernel=6, m=8, max_pts=256, n=1_000_000, gen="uniform", seeds=(31, 32), check_seed=33,
                       n_check=500, desc="differentiable laplace potential (forward + backward, autograd), {n} "
                                         "uniform points, m=8, 256/leaf"),
}
W = WORKLOADS["gaussian4m"]
KDIM = {0: (1, 1), 2: (3, 1), 3: (3, 3), 4: (3, 9), 5: (3, 3), 6: (1, 4)}   # kernel id -> (k0, k1)
# flops per pair (kernel.txx:1277, 1352, 1367, 1406, 1493; pot+grad 18)
PAIR_FLOPS = {0: 9, 2: 16, 3: 29, 4: 94, 5: 24, 6: 18}


def make_points(w, n):
    """Seeded synthetic inputs of a workload: positions (n,3), densities (n,k0)."""
    if w["gen"] == "gauss":
        return gaussian_mixture(n)
    s0, s1 = w["seeds"]
    if w["gen"] == "uniform":
        return np.random.default_rng(s0).random((n, 3)), np.random.default_rng(s1).uniform(-1, 1, n)
    if w["gen"] == "neutral":  # uniform densities with their mean taken out (a periodic cell without net charge)
        q = np.random.default_rng(s1).uniform(-1, 1, n)
        return np.random.default_rng(s0).random((n, 3)), q - q.mean()
    if w["gen"] == "stokes":
        return np.random.default_rng(s0).random((n, 3)), np.random.default_rng(s1).standard_normal((n, 3))
    if w["gen"] == "ellipsoid":
        rng = np.random.default_rng(s0)
        a = np.array([0.45, 0.3, 0.15])
        out, have = [], 0
        while have < n:
            m = int((n - have) * 2.2) + 1000
            u = rng.standard_normal((m, 3))
            u /= np.linalg.norm(u, axis=1, keepdims=True)
            acc = rng.random(m) < np.linalg.norm(u / a, axis=1) * a.min()
            out.append(0.5 + u[acc] * a)
            have += int(acc.sum())
        return np.concatenate(out)[:n], np.random.default_rng(s1).uniform(-1, 1, n)
    raise ValueError(w["gen"])


def gaussian_mixture(n, seed_c=11, seed_p=12, seed_q=13):
    rng_c = np.random.default_rng(seed_c)
    centres = rng_c.uniform(0.1, 0.9, (8, 3))
    rng = np.random.default_rng(seed_p)
    comp = rng.integers(0, 8, n)
    x = np.clip(centres[comp] + 0.02 * rng.standard_normal((n, 3)), 0.0, 1.0)
    q = np.random.default_rng(seed_q).uniform(-1, 1, n)
    return np.ascontiguousarray(x), q


def direct_gpu(torch, kid, x, q, idx):
    """FP64 direct sum at targets x[idx] over all points (GPU, torch), r == 0
    excluded, r = target - source: Laplace potential (0), Stokes pressure
    (r.f / r^3, 2), Stokes velocity (3), Stokes velocity gradient ((delta_ij
    r.f + r_j f_i - f_j r_i - 3 r.f r_i r_j / r^2) / r^3, 4), Biot-Savart
    (f x r / r^3, 5) or Laplace potential and r q / r^3 (6), with the
    kernels' 1/(8 pi) (3, 4) or 1/(4 pi)."""
    X = torch.as_tensor(x, device="cuda", dtype=torch.float64)
    Q = torch.as_tensor(q, device="cuda", dtype=torch.float64).reshape(X.shape[0], -1)
    T = X[torch.as_tensor(idx, device="cuda")]
    out = torch.zeros((len(idx), KDIM[kid][1]), device="cuda", dtype=torch.float64)
    chunk = 1 << 14
    for a in range(0, X.shape[0], chunk):
        d = T[:, None, :] - X[None, a:a + chunk, :]
        r2 = (d * d).sum(-1)
        rinv = torch.where(r2 > 0, r2.clamp_min(1e-300).rsqrt(), torch.zeros_like(r2))
        qa = Q[a:a + chunk]
        if kid == 3:
            ip = torch.einsum("tsk,sk->ts", d, qa) * rinv * rinv
            out += torch.einsum("ts,sk->tk", rinv, qa) + torch.einsum("ts,tsk->tk", rinv * ip, d)
        elif kid in (2, 4, 5):
            r3 = rinv * rinv * rinv
            rf = torch.einsum("tsk,sk->ts", d, qa)
            if kid == 2:
                out[:, 0] += (rf * r3).sum(1)
            elif kid == 5:
                out += torch.einsum("ts,tsk->tk", r3, torch.cross(qa[None, :, :].expand_as(d), d, dim=-1))
            else:
                c3 = 3 * rf * rinv * rinv
                for i in range(3):
                    for j in range(3):
                        v = d[:, :, j] * qa[None, :, i] - qa[None, :, j] * d[:, :, i] - c3 * d[:, :, i] * d[:, :, j]
                        if i == j:
                            v = v + rf
                        out[:, 3 * i + j] += (v * r3).sum(1)
        else:
            qr = rinv * qa[None, :, 0]
            out[:, 0] += qr.sum(1)
            if kid == 6:
                out[:, 1:] += (d * (qr * rinv * rinv)[:, :, None]).sum(1)
    return (out / (8 * math.pi if kid in (3, 4) else 4 * math.pi)).cpu().numpy()


def ewald_gpu(torch, x, q, idx, alpha=5.5, kmax=10):
    """Periodic potential of the 1/(4 pi r) kernel in the unit cell (Ewald
    sum with a neutralising background) at targets x[idx], which are sources
    (their self term removed); FP64 on the GPU.  alpha = 5.5: the real-space
    sum over the 27 nearest images is complete to erfc(5.5) ~ 7e-15; kmax =
    10: the reciprocal sum to exp(-(2 pi 10)^2 / (4 alpha^2)) ~ 1e-14.  The
    structure factor is separable, S(k) = sum_j q_j ex_j(kx) ey_j(ky) ez_j(kz),
    so it is formed as small matrix products."""
    dev, f64, c128 = "cuda", torch.float64, torch.complex128
    X = torch.as_tensor(x, device=dev, dtype=f64)
    Q = torch.as_tensor(q, device=dev, dtype=f64).reshape(-1)
    T = X[torch.as_tensor(idx, device=dev)]
    phi = torch.zeros(T.shape[0], device=dev, dtype=f64)
    chunk = 1 << 16
    shifts = torch.tensor([[a, b, c] for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)], device=dev,
                          dtype=f64)
    for a in range(0, X.shape[0], chunk):
        d0 = T[:, None, :] - X[None, a:a + chunk, :]
        qa = Q[a:a + chunk]
        for sh in shifts:
            d = d0 + sh
            r = torch.sqrt((d * d).sum(-1))
            v = torch.where(r > 0, torch.special.erfc(alpha * r) / r.clamp_min(1e-300), torch.zeros_like(r))
            phi += (v * qa[None, :]).sum(1) / (4 * math.pi)
    ks = torch.arange(-kmax, kmax + 1, device=dev, dtype=f64) * (2 * math.pi)
    nk = ks.numel()
    S = torch.zeros((nk, nk, nk), device=dev, dtype=c128)
    for a in range(0, X.shape[0], chunk):
        xa = X[a:a + chunk]
        e = [torch.exp(-1j * xa[:, i:i + 1].to(c128) * ks[None, :].to(c128)) for i in range(3)]  # (n, nk)
        w = Q[a:a + chunk].to(c128)[:, None] * e[0]                                                   # (n, kx)
        # S[kx, ky, kz] += sum_j w[j, kx] ey[j, ky] ez[j, kz]
        S += torch.einsum("jx,jy,jz->xyz", w, e[1], e[2])
    kx, ky, kz = torch.meshgrid(ks, ks, ks, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    wk = torch.where(k2 > 0, torch.exp(-k2 / (4 * alpha * alpha)) / k2.clamp_min(1e-300), torch.zeros_like(k2))
    et = [torch.exp(1j * T[:, i:i + 1].to(c128) * ks[None, :].to(c128)) for i in range(3)]        # (t, nk)
    phi += torch.einsum("xyz,tx,ty,tz->t", (wk.to(c128) * S), et[0], et[1], et[2]).real
    phi -= Q[torch.as_tensor(idx, device=dev)] * alpha / (2 * math.pi ** 1.5)
    return phi.cpu().numpy()[:, None]


def rel_err(out, ref, periodic):
    """Relative L2 error; for a periodic potential, defined up to an additive
    constant, after the mean difference is removed."""
    d = out - ref
    if periodic:
        d = d - d.mean(axis=0)
        ref = ref - ref.mean(axis=0)
    return float(np.linalg.norm(d) / np.linalg.norm(ref))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
            return
        # the timed region starts once the sampler is producing samples
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 3.0:
            time.sleep(0.01)
        self.lines.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def rank_tools(world, device):
    """barrier() and max_over_ranks(v) of the replica group (no-ops for one
    rank); the process group is initialised by the caller."""
    import torch
    import torch.distributed as dist

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        if world == 1:
            return v
        t = torch.tensor([v], device=device, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    return barrier, max_over_ranks


def job_throughput(world, n, ms):
    """Whole-job targets/s: every replica evaluates n targets; ms is the
    step time (max over ranks)."""
    return world * n / (ms / 1000)


# The reference has no pot+grad kernel: it evaluates the workload's kernel
# as these C-interface kernels in turn, on the same points (one step = all of
# them).  PVFMMKernel ids: 0 Laplace potential, 1 Laplace gradient, 3 Stokes
# velocity.
REFERENCE_KERNELS = {0: (0,), 2: (2,), 3: (3,), 4: (4,), 5: (5,), 6: (0, 1)}
REF_STAGES = ("InitFMM_Tree", "SetupFMM", "S2U", "U2U", "U-List", "V-List", "W-List", "X-List", "D2D", "D2T")


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_sample(args):
    """A bounded sample of the workload for the CPU reference: `ref_sample`
    points drawn (seed 15) from the workload's points, or all of them."""
    x, q = make_points(W, args.n)
    n = min(args.ref_sample, args.n)
    if n < args.n:
        sel = np.random.default_rng(15).choice(args.n, n, replace=False)
        x, q = x[sel], q[sel]
    return np.ascontiguousarray(x), np.ascontiguousarray(q), n


def reference_contexts(threads):
    """The reference's own FMM (built from its sources, oracle/_ref) through
    its C interface, one context per C-interface kernel of the workload."""
    from oracle.ref_fmm import refpvfmm as R
    t0 = time.perf_counter()
    ctxs = [R.RefContext(k, W["m"], W["max_pts"], threads=threads, box_size=W.get("box", -1.0),
                         lattice=W.get("lattice", False)) for k in REFERENCE_KERNELS[W["kernel"]]]
    return R, ctxs, 1000 * (time.perf_counter() - t0)


def reference_step(ctxs, x, q, setup=True):
    for c in ctxs:
        c.evaluate(x, q, None, setup)


def run_reference(args, world, rank):
    """The reference's own CPU FMM (compiled from its sources, oracle/_ref)
    through its C interface PVFMMCreateContextDWorld / PVFMMEvalD, all host
    threads, FP64, on a bounded sample of the workload; rank 0 only."""
    if rank != 0:
        return
    from oracle.ref_fmm import refpvfmm as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/ref_fmm/build.sh "
                                                              "needs the reference sources)"}), flush=True)
        return
    x, q, n = reference_sample(args)
    cores = os.cpu_count() or 1
    R, ctxs, create_ms = reference_contexts(cores)
    times = []
    stages = {}
    for it in range(args.warmup + args.steps):
        prof = it == args.warmup + args.steps - 1
        if prof:
            R.profile_enable(True)
        t0 = time.perf_counter()
        reference_step(ctxs, x, q, True)
        dt = time.perf_counter() - t0
        if prof:
            R.profile_enable(False)
            for _, tag, sec in R.profile_report():
                if tag in REF_STAGES:
                    stages[tag] = stages.get(tag, 0.0) + 1000 * sec
        if it >= args.warmup:
            times.append(dt)
    t0 = time.perf_counter()
    reference_step(ctxs, x, q, False)          # setup=0: same points, new densities (the tree reused)
    setup0_ms = 1000 * (time.perf_counter() - t0)
    for c in ctxs:
        c.close()
    ms = 1000 * float(np.mean(times))
    value = n / (ms / 1000)
    kernels = "+".join({0: "LaplacePotential", 1: "LaplaceGradient", 2: "StokesPressure", 3: "StokesVelocity",
                        4: "StokesVelocityGrad", 5: "BiotSavartPotential"}[k]
                       for k in REFERENCE_KERNELS[W["kernel"]])
    sample = (f"{n} of the workload's {args.n} points (seed 15), the reference's PVFMMEvalD ({kernels}), FP64, "
              f"setup=1 per step, {cores} threads on {cpu_model()}")
    line = {"metric": METRIC, "value": value, "unit": "targets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": W["desc"].format(n=args.n) + (f" (bounded CPU sample: {n} points)"
                                                                 if n < args.n else "")},
            "impl": "reference",
            "context_create_ms": create_ms,
            "stages_ms": stages,
            "stages_note": "reference profiler tags (pvfmm::Profile) of the last step; V-List runs the reference's "
                           "built-in matrix DFT (FFTW absent)",
            "setup0_ms": setup0_ms,
            "setup0_targets_per_s": n / (setup0_ms / 1000),
            "cpu_baseline": {"value": value, "unit": "targets/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "targets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(args):
    """The reference's own CPU FMM on all host threads, one setup=1 step on a
    bounded sample of the workload (a few seconds to tens of seconds)."""
    from oracle.ref_fmm import refpvfmm as R
    if not R.available():
        return {"value": None, "unit": "targets/s", "cores": 0, "kind": "reference",
                "sample": "reference library not built"}
    x, q, n = reference_sample(args)
    cores = os.cpu_count() or 1
    R, ctxs, _ = reference_contexts(cores)
    reference_step(ctxs, x, q, True)             # first evaluation (allocations)
    t0 = time.perf_counter()
    reference_step(ctxs, x, q, True)
    dt = time.perf_counter() - t0
    for c in ctxs:
        c.close()
    return {"value": n / dt, "unit": "targets/s", "cores": cores, "kind": "reference",
            "sample": f"{n} of the workload's {args.n} points (seed 15), the reference's PVFMMEvalD, FP64, setup=1, "
                      f"{cores} threads on {cpu_model()}, {dt:.2f} s"}


# Per-launch DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of the
# two dominant kernels of each form, measured by ncu on one launch at 1,000,000
# points of the same distribution (m=8, 256/leaf) and scaled here by the units
# a launch processes (traffic grows in proportion).  Units: n_vsrc + n_vtrg for
# the Hadamard kernels, n_trg for the near field.
TRAFFIC_1M = {
    ("hadamard", 4): {"bytes": 844786176 + 671260416, "units": 4768 + 4767},     # hadamard_tc_kernel
    # hadamard_rd_kernel<double> capture; hadamard_dmma1_kernel reads and writes the same spectra
    ("hadamard", 8): {"bytes": 1470638080 + 1367394304, "units": 4768 + 4767},
    ("near_field", 4): {"bytes": 149489664 + 25314816, "units": 1000000},        # near_field_kernel<float>
    ("near_field", 8): {"bytes": 151890688 + 20192256, "units": 1000000},        # near_field_kernel<double>
}
# kernel that computes the V-list Hadamard products: (real bytes, ke) -> name
HADAMARD_KERNEL = {(4, 1): "hadamard_tc_kernel (V-list M2L, TF32 mma.sync x3 split)",
                   (8, 1): "hadamard_dmma1_kernel (V-list M2L, FP64 mma.sync m8n8k4)",
                   (4, 3): "hadamard_tc3_kernel<3> (V-list M2L, TF32 mma.sync x3 split)",
                   (8, 3): "hadamard_dmma3_kernel<3> (V-list M2L, FP64 mma.sync m8n8k4)"}
NEAR_KERNEL = "near_field_kernel (U-list P2P + W + D2T)"


def roofline(B, peaks):
    """Roofline objects of the V-list Hadamard and the fused near field,
    the slower first.

    near field: bound by the SIMT FP32 (mixed) / FP64 (plain) pipes, so its
      object is the FLOP view: `bound` "fp32" / "fp64", achieved = algorithmic
      flops (18 per pair for pot+grad, kernel.txx conventions otherwise, over
      P2P + W + D2T pairs) / kernel time, peak = the nominal SIMT peak (148 SMs
      x 128 FP32 or 64 FP64 lanes x 2 flops x max SM clock; the measured peaks
      have no SIMT figure).  Its HBM view is the `hbm` sub-object.
    Hadamard: the HBM view (the streaming bound it is held to): algorithmic bytes =
      (n_vsrc + n_vtrg) * n3h * 8 children * 2 * rb (input spectra read once,
      output spectra written once) + 26 * n3h * 64 * 2 * rb (operators read
      once) against the measured copy bandwidth; its tensor view (mixed form:
      the split issues 3 TF32 products per product, against a dense TF32 peak
      of half the measured bf16 peak) or FP64 tensor view (plain form, against
      the nominal FP64 peak, the same for the FP64 tensor cores and the FP64
      pipe) is the `compute` sub-object.
    `traffic` is the ncu DRAM traffic of a launch scaled from 1M points."""
    st = B["stats"]
    rb = B["real_bytes"]
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    tf32_peak = peaks.get("bf16_tflops", 1590.0) / 2
    smax = (B["clocks"] or {}).get("sm_max_mhz") or 1965.0
    lanes = 128 if rb == 4 else 64
    simt_peak = 148 * lanes * 2 * smax * 1e6 / 1e12
    m, kid = W["m"], W["kernel"]
    ke = 3 if kid == 3 else 1
    k0, k1 = KDIM[kid]
    n3h = (2 * m) ** 2 * (m + 1)
    ns = 6 * (m - 1) ** 2 + 2

    def traffic(tkey, units):
        tr = TRAFFIC_1M.get((tkey, rb)) if kid == 6 else None
        return tr["bytes"] * units / tr["units"] if tr else None

    had_ms = B["stages_ms"]["V-Hadamard"]
    had_bytes = (st["n_vsrc"] + st["n_vtrg"]) * n3h * 8 * ke * 2 * rb + 26 * n3h * 64 * ke * ke * 2 * rb
    had_flops = 512.0 * ke * ke * n3h * st["v_pairs"]
    had_gbs = had_bytes / (had_ms / 1000) / 1e9 if had_ms > 0 else 0.0
    had_tf = had_flops / (had_ms / 1000) / 1e12 if had_ms > 0 else 0.0
    tensor = rb == 4
    had = {"kernel": HADAMARD_KERNEL[(rb, ke)], "bound": "hbm", "achieved": had_gbs, "peak": hbm_peak, "unit": "GB/s",
           "frac": had_gbs / hbm_peak, "peak_source": peak_src,
           "traffic": traffic("hadamard", st["n_vsrc"] + st["n_vtrg"]), "algorithmic_bytes": had_bytes,
           "kernel_ms": had_ms,
           "compute": ({"pipe": "tensor tf32 x3 (mma.sync)", "achieved_tflops": 3 * had_tf, "peak_tflops": tf32_peak,
                        "peak_source": "half the measured bf16 dense peak", "frac": 3 * had_tf / tf32_peak,
                        "algorithmic_flops": had_flops} if tensor else
                       {"pipe": "fp64 tensor (mma.sync m8n8k4)", "achieved_tflops": had_tf,
                        "peak_tflops": simt_peak, "peak_source": "nominal", "frac": had_tf / simt_peak,
                        "algorithmic_flops": had_flops})}
    near_ms = B["stages_ms"]["near-field kernel"]
    near_bytes = st["n_src"] * (24 + 8 * k0) + st["n_trg"] * (24 + 8 * k1) + st["n_tleaf"] * ns * ke * 8
    near_flops = float(PAIR_FLOPS[kid]) * (st["p2p_pairs"] + st["w_pairs"] + st["d2t_pairs"])
    near_tf = near_flops / (near_ms / 1000) / 1e12 if near_ms > 0 else 0.0
    near_gbs = near_bytes / (near_ms / 1000) / 1e9 if near_ms > 0 else 0.0
    near = {"kernel": NEAR_KERNEL, "bound": "fp32" if rb == 4 else "fp64", "achieved": near_tf, "peak": simt_peak,
            "unit": "TFLOP/s", "frac": near_tf / simt_peak,
            "peak_source": "nominal SIMT peak at the max SM clock (no measured SIMT peak)",
            "traffic": traffic("near_field", st["n_trg"]), "algorithmic_flops": near_flops, "kernel_ms": near_ms,
            "hbm": {"achieved": near_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": near_gbs / hbm_peak,
                    "peak_source": peak_src, "algorithmic_bytes": near_bytes}}
    ranked = sorted([had, near], key=lambda r: -r["kernel_ms"])
    return ranked[0], ranked[1]


def build_line(args, world, N, forms, peaks):
    """The JSON line of the GPU arm from the per-form results: the reported
    form is the fastest whose combined and per-component rel-L2 all meet the
    bar (the first completed form if none does)."""
    k0, k1 = KDIM[W["kernel"]]
    forms_ok = {f: d for f, d in forms.items() if "error" not in d}
    if not forms_ok:
        raise RuntimeError(f"no form completed: {forms}")
    ok = [f for f in forms_ok if max([forms_ok[f]["rel_l2"]] + forms_ok[f]["rel_l2_components"]) <= TOL]
    best = max(ok, key=lambda f: forms_ok[f]["targets_per_s"]) if ok else next(iter(forms_ok))
    B = forms[best]
    worst = max([B["rel_l2"]] + B["rel_l2_components"])
    roof = roofline(B, peaks)
    return {
        "metric": METRIC,
        "value": B["targets_per_s"],
        "unit": "targets/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": B["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if best == "plain" else "f32",
        "data": "synthetic",
        "config": {"workload": W["desc"].format(n=N) + f", form={best}",
                   "l2": "no flush: per-step working set (128 MB inputs + tree + GB-size spectra) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world}"},
        "form": best,
        "meets_bar": bool(ok),
        "rel_l2_worst_component": worst,
        "rel_l2_bar": TOL,
        "forms": forms,
        "mixed_over_plain": (forms_ok["mixed"]["targets_per_s"] / forms_ok["plain"]["targets_per_s"]
                             if "mixed" in forms_ok and "plain" in forms_ok else None),
        "e2e": {"value": B["e2e_targets_per_s"], "unit": "targets/s",
                "h2d_bytes_per_step": N * 3 * 8 + N * k0 * 8, "d2h_bytes_per_step": N * k1 * 8},
        "gpu_launches": B["gpu_launches"],
        "clocks": B["clocks"],
        "roofline": roof[0],
        "roofline_next": roof[1],
    }


def run_autograd(args, world, torch, barrier, max_over_ranks):
    """Forward + backward of the differentiable Laplace potential
    (pvfmm_b200.autograd.LaplaceFMM, mixed form) on one set of points: per
    step phi = FMM(y, q), L = <g, phi>, L.backward() (a swapped-role FMM on the
    forward's octree).  The gradients are checked against an FP64 direct sum
    on a sample of points before the timed steps."""
    from pvfmm_b200.autograd import LaplaceFMM
    N = args.n
    x, q = make_points(W, N)
    y = torch.tensor(x, device="cuda", requires_grad=True)
    d = torch.tensor(np.ascontiguousarray(q.reshape(-1)), device="cuda", requires_grad=True)
    g = torch.tensor(np.random.default_rng(W["check_seed"]).uniform(-1, 1, N), device="cuda")
    fmm = LaplaceFMM(max_points=W["max_pts"], multipole_order=W["m"], precision="mixed")

    def step():
        y.grad = None
        d.grad = None
        phi = fmm(y, d)
        (phi * g).sum().backward()

    try:
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        # dL/dq_j = sum_i G(y_j - y_i) g_i; dL/dy_j adds the source role,
        # q_j sum_i g_i (y_i - y_j) / (4 pi r^3), and the target role,
        # g_j grad phi(y_j) = -g_j sum_i q_i (y_j - y_i) / (4 pi r^3): direct
        # sums with densities g and q, evaluated at a sample of the points
        idx = np.random.default_rng(W["check_seed"] + 1).choice(N, W["n_check"], replace=False)
        ref = direct_gpu(torch, 6, x, g.cpu().numpy(), idx)   # [G g, sum g r / r^3] at the sample
        ref_q = direct_gpu(torch, 6, x, q, idx)                 # [G q, sum q r / r^3]
        got_q = d.grad.cpu().numpy()[idx]
        got_y = y.grad.cpu().numpy()[idx]
        want_y = -q.reshape(-1)[idx, None] * ref[:, 1:] - g.cpu().numpy()[idx, None] * ref_q[:, 1:]
        err_q = float(np.linalg.norm(got_q - ref[:, 0]) / np.linalg.norm(ref[:, 0]))
        err_y = float(np.linalg.norm(got_y - want_y) / np.linalg.norm(want_y))
        clocks = ClockSampler(torch.cuda.current_device())
        barrier()
        torch.cuda.synchronize()
        clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        cl = clocks.stop()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
    finally:
        fmm.close()
    value = job_throughput(world, N, ms)
    return {"metric": "targets/s differentiable Laplace FMM (forward + backward), rel-L2 of the gradients vs FP64 "
                      "direct", "value": value, "unit": "targets/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": W["desc"].format(n=N) + ", form=mixed",
                       "l2": "no flush: per-step working set exceeds the 126 MB L2",
                       "parallelism": f"replicas x{world}"},
            "rel_l2_grad_den": err_q, "rel_l2_grad_pos": err_y, "clocks": cl,
            "e2e": None}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gaussian4m", choices=sorted(WORKLOADS))
    ap.add_argument("--n", type=int, default=None, help="point count (default: the workload's)")
    ap.add_argument("--ref-sample", type=int, default=500_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--forms", default="plain,mixed")
    args = ap.parse_args()
    global W
    W = WORKLOADS[args.workload]
    if args.n is None:
        args.n = W["n"]
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference(args, world, rank)
        return

    import torch
    import torch.distributed as dist
    import pvfmm_b200 as P

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    barrier, max_over_ranks = rank_tools(world, "cuda")
    if args.workload == "autograd1m":
        line = run_autograd(args, world, torch, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    N = args.n
    kid = W["kernel"]
    k0, k1 = KDIM[kid]
    x, q = make_points(W, N)
    q = np.ascontiguousarray(q.reshape(-1))
    idx = np.random.default_rng(W["check_seed"]).choice(N, W["n_check"], replace=False)
    periodic = W.get("box", -1.0) > 0
    ref = ewald_gpu(torch, x, q, idx) if periodic else direct_gpu(torch, kid, x, q, idx)
    torch.cuda.empty_cache()  # the direct sum's temporaries go back to the device
    d_x = torch.as_tensor(x, device="cuda")
    d_q = torch.as_tensor(q, device="cuda")
    d_out = torch.empty((N, k1), device="cuda", dtype=torch.float64)
    stream = torch.cuda.current_stream()

    def run_form(form):
        prec = P.PRECISION_PLAIN if form == "plain" else P.PRECISION_MIXED
        t_ctx = time.perf_counter()
        ctx = P.FMMParticleContext(W.get("box", -1.0), W["max_pts"], W["m"], P.FMMKernel(kid), precision=prec)
        if W.get("lattice"):
            ctx.set_periodic_bc(True)
        context_ms = 1000 * (time.perf_counter() - t_ctx)  # operator precompute + upload, outside the timed steps
        try:
            def step():
                ctx.evaluate_device(d_x.data_ptr(), d_q.data_ptr(), N, d_x.data_ptr(), d_out.data_ptr(), N, True,
                                    stream.cuda_stream)

            for _ in range(args.warmup):
                step()
            torch.cuda.synchronize()
            out = d_out.cpu().numpy()[idx]
            err = rel_err(out, ref, periodic)
            err_comp = [rel_err(out[:, k], ref[:, k], periodic) for k in range(k1)]
            stats = ctx.tree_stats()
            l0 = ctx.launch_count()
            clocks = ClockSampler(local)
            barrier()
            torch.cuda.synchronize()
            clocks.start()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stage_sum = None
            for _ in range(args.steps):
                step()
                st = ctx.stage_times()
                stage_sum = st if stage_sum is None else {k: stage_sum[k] + st[k] for k in st}
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            cl = clocks.stop()
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps)
            launches = (ctx.launch_count() - l0) / args.steps
            stage = {k: v / args.steps for k, v in stage_sum.items()}
            # setup=0: same points, new densities (the tree and lists are
            # reused, as PVFMMEval does with setup=0); reported beside the
            # setup=1 figure
            setup0 = {}
            try:
                def step0():
                    ctx.evaluate_device(d_x.data_ptr(), d_q.data_ptr(), N, d_x.data_ptr(), d_out.data_ptr(), N,
                                        False, stream.cuda_stream)

                step0()
                barrier()
                torch.cuda.synchronize()
                s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                for _ in range(args.steps):
                    step0()
                s1.record(stream)
                torch.cuda.synchronize()
                barrier()
                ms0 = max_over_ranks(s0.elapsed_time(s1) / args.steps)
                setup0 = {"setup0_ms": ms0, "setup0_targets_per_s": job_throughput(world, N, ms0)}
            except RuntimeError as e:
                setup0 = {"setup0_error": str(e)}
            # e2e: public C ABI on pinned host buffers, copies inside the timed region
            lib = P.load_library()
            h_x = torch.from_numpy(x.reshape(-1)).pin_memory()
            h_q = torch.from_numpy(q).pin_memory()
            h_out = torch.empty(N * k1, dtype=torch.float64).pin_memory()
            f = lib.PVFMMEvalD
            for _ in range(2):
                f(ctypes.c_void_p(h_x.data_ptr()), ctypes.c_void_p(h_q.data_ptr()), None, N, ctypes.c_void_p(h_x.data_ptr()),
                  ctypes.c_void_p(h_out.data_ptr()), N, ctypes.c_void_p(ctx._ptr), 1)
            barrier()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                f(ctypes.c_void_p(h_x.data_ptr()), ctypes.c_void_p(h_q.data_ptr()), None, N, ctypes.c_void_p(h_x.data_ptr()),
                  ctypes.c_void_p(h_out.data_ptr()), N, ctypes.c_void_p(ctx._ptr), 1)
            e2e_ms = max_over_ranks(1000 * (time.perf_counter() - t0) / args.steps)
            if P.last_error():
                raise RuntimeError(P.last_error())
            res = {"ms_per_step": ms, "targets_per_s": job_throughput(world, N, ms), "rel_l2": err,
                   "rel_l2_components": err_comp, "stages_ms": stage, "stats": stats, "gpu_launches": launches,
                   "clocks": cl, "e2e_ms": e2e_ms, "e2e_targets_per_s": job_throughput(world, N, e2e_ms),
                   "real_bytes": 8 if form == "plain" else 4, "context_create_ms": context_ms, **setup0}
            return res
        finally:
            ctx.close()

    forms = {}
    for form in args.forms.split(","):
        try:
            forms[form] = run_form(form)
        except RuntimeError as e:  # e.g. a workload too large for one GPU in this form
            forms[form] = {"error": str(e)}
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except OSError:
        pass
    line = build_line(args, world, N, forms, peaks)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
