"""Times the reference's own CPU FMM (built from its sources by
oracle/ref_fmm/build.sh) on the benchmark configurations, on this host's cores.

For each configuration: context creation (operator precompute, read from the
reference's precompute file when present), setup=1 evaluations (tree build +
FMM) and a setup=0 evaluation (same points, new densities), the rel-L2 error
against an FP64 direct sum on 200 sampled targets, and the reference profiler's
per-stage split.  Sizes above --max-n points are run on a seeded subsample of
the configuration's points (stated in the output).  One JSON line per
configuration.

    python oracle/ref_fmm/measure_cpu.py [--max-n 2000000] [--threads 0] [--configs 1,2,3,5]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pvfmm_oracle as O  # noqa: E402
from oracle.ref_fmm import refpvfmm as R  # noqa: E402

STAGES = ("InitFMM_Tree", "SetupFMM", "S2U", "U2U", "U-List", "V-List", "W-List", "X-List", "D2D", "D2T")


def configs():
    import bench
    W = bench.WORKLOADS
    # configuration number: (workload, C-interface kernels evaluated in turn)
    return {1: (W["uniform100k"], (0,)), 2: (W["gaussian4m"], (0, 1)), 3: (W["stokes2m"], (3,)),
            5: (W["ellipsoid30m"], (0,))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--max-n", type=int, default=2_000_000)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--configs", default="1,2,3,5")
    ap.add_argument("--repeats", type=int, default=3)
    args = ap.parse_args()
    import bench
    cfg = configs()
    threads = args.threads or os.cpu_count() or 1
    for c in (int(v) for v in args.configs.split(",")):
        w, kernels = cfg[c]
        x, q = bench.make_points(w, w["n"])
        n = min(args.max_n, w["n"])
        if n < w["n"]:
            sel = np.random.default_rng(15).choice(w["n"], n, replace=False)
            x, q = x[sel], q[sel]
        x = np.ascontiguousarray(x)
        q = np.ascontiguousarray(q)
        t0 = time.perf_counter()
        ctxs = [R.RefContext(k, w["m"], w["max_pts"], threads=threads) for k in kernels]
        create_s = time.perf_counter() - t0
        outs = [c_.evaluate(x, q, None, True) for c_ in ctxs]        # warm-up
        times = []
        for _ in range(args.repeats):
            t0 = time.perf_counter()
            outs = [c_.evaluate(x, q, None, True) for c_ in ctxs]
            times.append(time.perf_counter() - t0)
        R.profile_enable(True)
        t0 = time.perf_counter()
        for c_ in ctxs:
            c_.evaluate(x, q, None, False)
        setup0_s = time.perf_counter() - t0
        R.profile_enable(False)
        stages = {}
        for _, tag, sec in R.profile_report():
            if tag in STAGES:
                stages[tag] = stages.get(tag, 0.0) + sec
        for c_ in ctxs:
            c_.close()
        out = np.concatenate([o.reshape(len(x), -1) for o in outs], axis=1)
        idx = np.random.default_rng(w["check_seed"]).choice(n, min(200, n), replace=False)
        direct = np.concatenate([O.direct_sum(k, x, q, x[idx], chunk=8).reshape(len(idx), -1) for k in kernels],
                                axis=1)
        t = float(np.median(times))
        print(json.dumps({
            "config": c, "workload": w["desc"].format(n=w["n"]), "points_run": n,
            "sample": n < w["n"], "kernels": kernels, "threads": threads,
            "cpu": bench.cpu_model(), "context_create_s": create_s,
            "setup1_s": t, "setup1_targets_per_s": n / t,
            "setup0_s_profiled": setup0_s, "setup0_targets_per_s": n / setup0_s,
            "rel_l2_vs_direct": O.rel_l2(out[idx].reshape(-1), direct.reshape(-1)),
            "stages_setup0_s": stages}), flush=True)


if __name__ == "__main__":
    main()
