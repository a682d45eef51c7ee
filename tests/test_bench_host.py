"""Host-side logic of bench.py, without a GPU: the roofline objects of its
JSON line (bound, achieved / peak, DRAM traffic scaled from the 1M-point ncu
capture by the units a launch processes) and the seeded synthetic workloads.
"""
import numpy as np
import pytest

import bench

# tree statistics of the 1,000,000-point Gaussian-mixture workload (m=8,
# 256/leaf), the size at which the DRAM traffic was captured
STATS_1M = {"n_vsrc": 4768.0, "n_vtrg": 4767.0, "v_pairs": 86308.0, "n_src": 1e6, "n_trg": 1e6,
            "n_tleaf": 31479.0, "p2p_pairs": 1832521088.0, "w_pairs": 24364056.0, "d2t_pairs": 296000000.0}


def _run(rb, had_ms, near_ms, stats=STATS_1M, peaks=None):
    B = {"stats": stats, "real_bytes": rb, "clocks": {"sm_max_mhz": 1965.0},
         "stages_ms": {"V-Hadamard": had_ms, "near-field kernel": near_ms}}
    return bench.roofline(B, {"hbm_gbs": 6449.1} if peaks is None else peaks)


@pytest.mark.parametrize("rb", [4, 8])
def test_roofline_objects_follow_the_contract(rb):
    dom, nxt = _run(rb, 3.26, 3.18)
    assert dom["kernel_ms"] >= nxt["kernel_ms"]
    by = {r["kernel"].split()[0].split("<")[0]: r for r in (dom, nxt)}
    had = by["hadamard_tc_kernel" if rb == 4 else "hadamard_dmma1_kernel"]
    near = by["near_field_kernel"]
    # the Hadamard: HBM view against the measured copy bandwidth
    assert had["bound"] == "hbm" and had["unit"] == "GB/s" and had["peak"] == 6449.1
    assert had["peak_source"] == "measured" and had["frac"] == pytest.approx(had["achieved"] / had["peak"])
    assert had["achieved"] == pytest.approx(had["algorithmic_bytes"] / (had["kernel_ms"] / 1000) / 1e9)
    c = had["compute"]
    assert c["frac"] == pytest.approx(c["achieved_tflops"] / c["peak_tflops"])
    # the near field: FLOP view against the SIMT pipe it is bound by, HBM view beside it
    assert near["bound"] == ("fp32" if rb == 4 else "fp64") and near["unit"] == "TFLOP/s"
    assert near["peak"] == pytest.approx(148 * (128 if rb == 4 else 64) * 2 * 1965e6 / 1e12)
    assert near["achieved"] == pytest.approx(near["algorithmic_flops"] / (near["kernel_ms"] / 1000) / 1e12)
    assert near["frac"] == pytest.approx(near["achieved"] / near["peak"])
    assert near["hbm"]["frac"] == pytest.approx(near["hbm"]["achieved"] / 6449.1)


@pytest.mark.parametrize("rb", [4, 8])
def test_traffic_at_the_capture_size_is_the_capture(rb):
    dom, nxt = _run(rb, 3.26, 3.18)
    by = {r["kernel"].split()[0].split("<")[0]: r for r in (dom, nxt)}
    had = by["hadamard_tc_kernel" if rb == 4 else "hadamard_dmma1_kernel"]
    assert had["traffic"] == bench.TRAFFIC_1M[("hadamard", rb)]["bytes"]
    assert by["near_field_kernel"]["traffic"] == bench.TRAFFIC_1M[("near_field", rb)]["bytes"]


def test_traffic_scales_with_the_units_of_a_launch():
    st = dict(STATS_1M, n_vsrc=2 * 4768.0, n_vtrg=2 * 4767.0, n_trg=4e6)
    dom, nxt = _run(4, 10.0, 12.0, stats=st)
    by = {r["kernel"].split()[0]: r for r in (dom, nxt)}
    assert by["hadamard_tc_kernel"]["traffic"] == pytest.approx(2 * bench.TRAFFIC_1M[("hadamard", 4)]["bytes"])
    assert by["near_field_kernel"]["traffic"] == pytest.approx(4 * bench.TRAFFIC_1M[("near_field", 4)]["bytes"])


def test_hadamard_algorithmic_bytes_at_1m():
    # input spectra read once + output spectra written once + operators once (FP32)
    dom, nxt = _run(4, 3.26, 3.18)
    had = dom if dom["kernel"].startswith("hadamard") else nxt
    assert had["algorithmic_bytes"] == (4768 + 4767) * 2304 * 8 * 2 * 4 + 26 * 2304 * 64 * 2 * 4 == 1436663808


def test_fallback_peak_is_labelled():
    dom, _ = _run(4, 3.26, 3.18, peaks={})
    assert dom["peak"] == 6650.0 and dom["peak_source"] == "fallback"


@pytest.mark.parametrize("name", sorted(bench.WORKLOADS))
def test_workloads_are_seeded(name):
    w = bench.WORKLOADS[name]
    x1, q1 = bench.make_points(w, 2000)
    x2, q2 = bench.make_points(w, 2000)
    assert x1.shape == (2000, 3)
    assert np.array_equal(x1, x2) and np.array_equal(q1, q2)
    assert x1.min() >= 0.0 and x1.max() <= 1.0
    k0 = bench.KDIM[w["kernel"]][0]
    assert q1.reshape(2000, -1).shape[1] == k0


def test_ellipsoid_points_lie_on_the_surface():
    x, _ = bench.make_points(bench.WORKLOADS["ellipsoid30m"], 5000)
    a = np.array([0.45, 0.3, 0.15])
    assert np.allclose((((x - 0.5) / a) ** 2).sum(1), 1.0, atol=1e-12)


def test_reference_arm_line(capsys):
    """The reference arm's JSON line: the reference's own FMM (built from its
    sources) on a bounded sample, with the reference profiler's per-stage
    split, the setup=0 rate and the context-creation time; a line saying it is
    unavailable when the reference library is not built."""
    import json
    from oracle.ref_fmm import refpvfmm as R

    class Args:
        ref_sample, n, warmup, steps, workload = 3000, 20000, 0, 1, "gaussian4m"
    bench.run_reference(Args, 1, 0)
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    if not R.available():
        assert line == {"impl": "reference", "unavailable": line["unavailable"]}
        return
    assert line["impl"] == "reference" and line["value"] > 0
    assert {"S2U", "U2U", "U-List", "V-List", "D2T"} <= set(line["stages_ms"])
    assert line["context_create_ms"] > 0 and line["setup0_targets_per_s"] > 0
    assert line["cpu_baseline"]["kind"] == "reference" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert "3000 of the workload's 20000 points" in line["cpu_baseline"]["sample"]


def test_oracle_setup0_equals_a_fresh_evaluation():
    from oracle import pvfmm_oracle as O
    rng = np.random.default_rng(1)
    x = rng.random((1500, 3))
    q1, q2 = rng.uniform(-1, 1, 1500), rng.uniform(-1, 1, 1500)
    _, fmm = O.pvfmm_eval(6, 4, 60, x, q1, x, return_fmm=True)
    assert np.array_equal(O.pvfmm_eval_setup0(fmm, q2), O.pvfmm_eval(6, 4, 60, x, q2, x))


def _form(tps, err, comps, rb):
    return {"ms_per_step": 4e6 / tps * 1000, "targets_per_s": tps, "rel_l2": err, "rel_l2_components": comps,
            "stages_ms": {"V-Hadamard": 10.0, "near-field kernel": 12.0}, "gpu_launches": 178.0,
            "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 7},
            "e2e_targets_per_s": 0.9 * tps, "real_bytes": rb,
            "stats": dict(STATS_1M, n_vsrc=15240.0, n_vtrg=15237.0, n_trg=4e6, n_src=4e6)}


class _Args:
    steps, warmup = 20, 3


def test_json_line_follows_the_contract():
    forms = {"plain": _form(58e6, 2.1e-7, [6e-8, 2.5e-7, 1.8e-7, 2.0e-7], 8),
             "mixed": _form(109e6, 5.5e-7, [2.3e-7, 6.4e-7, 4.8e-7, 5.6e-7], 4)}
    line = bench.build_line(_Args, 1, 4_000_000, forms, {"hbm_gbs": 6449.1})
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "e2e", "gpu_launches", "clocks", "roofline"):
        assert key in line, key
    assert line["form"] == "mixed" and line["value"] == 109e6 and line["dtype"] == "f32"
    assert line["higher_is_better"] is True and line["scaling"] == "weak" and line["vs_baseline"] is None
    assert line["mixed_over_plain"] == pytest.approx(109 / 58)
    # inputs (positions + densities) in, pot+grad values out, FP64 host buffers
    assert line["e2e"]["h2d_bytes_per_step"] == 4_000_000 * (3 + 1) * 8
    assert line["e2e"]["d2h_bytes_per_step"] == 4_000_000 * 4 * 8
    r = line["roofline"]
    assert set(r) >= {"bound", "achieved", "peak", "unit", "frac", "traffic"}
    assert r["bound"] in ("hbm", "tensor", "fp32", "fp64") and r["traffic"] > 0
    hbm = r if r["bound"] == "hbm" else r["hbm"]
    assert hbm["peak_source"] == "measured"


def test_a_form_over_the_bar_in_one_component_is_not_reported():
    forms = {"plain": _form(58e6, 2.1e-7, [6e-8, 2.5e-7, 1.8e-7, 2.0e-7], 8),
             "mixed": _form(109e6, 5.5e-7, [2.3e-7, 1.2e-6, 4.8e-7, 5.6e-7], 4)}   # one component > 1e-6
    line = bench.build_line(_Args, 1, 4_000_000, forms, {})
    assert line["form"] == "plain" and line["dtype"] == "f64"
    r = line["roofline"]
    assert (r if r["bound"] == "hbm" else r["hbm"])["peak_source"] == "fallback"


def test_a_form_that_failed_is_kept_in_the_line():
    forms = {"plain": {"error": "device allocation failed"},
             "mixed": _form(109e6, 5.5e-7, [2.3e-7, 6.4e-7, 4.8e-7, 5.6e-7], 4)}
    line = bench.build_line(_Args, 2, 4_000_000, forms, {})
    assert line["form"] == "mixed" and line["forms"]["plain"]["error"]
    assert line["mixed_over_plain"] is None and line["n_gpus"] == 2
    with pytest.raises(RuntimeError, match="no form completed"):
        bench.build_line(_Args, 1, 4_000_000, {"plain": {"error": "x"}}, {})


def test_a_line_where_no_form_meets_the_bar_says_so():
    forms = {"plain": _form(58e6, 2.1e-6, [6e-8, 2.5e-6, 1.8e-7, 2.0e-7], 8),
             "mixed": _form(109e6, 5.5e-6, [2.3e-7, 6.4e-6, 4.8e-7, 5.6e-7], 4)}
    line = bench.build_line(_Args, 1, 4_000_000, forms, {})
    assert line["meets_bar"] is False
    assert line["rel_l2_worst_component"] == pytest.approx(2.5e-6) and line["rel_l2_bar"] == 1e-6
    forms["plain"] = _form(58e6, 2.1e-7, [6e-8, 2.5e-7, 1.8e-7, 2.0e-7], 8)
    line = bench.build_line(_Args, 1, 4_000_000, forms, {})
    assert line["meets_bar"] is True and line["form"] == "plain"


def test_periodic_error_ignores_the_additive_constant():
    """A periodic potential is defined up to a constant: the periodic
    workload's error against its Ewald sum removes the mean difference."""
    ref = np.random.default_rng(0).standard_normal((50, 1))
    assert bench.rel_err(ref + 3.0, ref, True) < 1e-15
    assert bench.rel_err(ref + 3.0, ref, False) > 1.0
    assert bench.WORKLOADS["periodic4m"]["box"] > 0
