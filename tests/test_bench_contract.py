"""bench.py's host-side pieces that the JSON line depends on, on the CPU: the roofline
object of each extension kernel (achieved / peak = frac, the bound chosen by the longer
lower-bound time), the clock sampler's reading of nvidia-smi lines, and the CPU baseline
(the oracle on a bounded sample, scaled to the job)."""
import importlib.util
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def sets(bench):
    from phraya_b200 import datagen as D
    return (D.extension_pairs(2000, 100, 300, 0.05, seed=0),
            D.extension_pairs(300, 64, 2048, 0.05, seed=1000, log_uniform=True))


def test_roofline_fields(bench, sets):
    set_a, set_b = sets
    work = {"myers_lane_block_columns": 3.0e6, "myers_lane_redo_pairs": 1,
            "wfa_affine_cells": 7.0e5, "wfa_affine_lcp_words": 6.0e5,
            "wfa_linear_cells": 2.4e5, "wfa_linear_lcp_words": 2.6e5}
    int_peak, hbm_peak = 37.2e12, 6.65e12
    for name in ("myers_lane", "wfa_affine", "wfa_linear"):
        r = bench.roofline(name, 0.5, 1.0, work, set_a, set_b, int_peak, hbm_peak, "fallback")
        for key in ("bound", "achieved", "peak", "unit", "frac", "traffic", "kernel", "work", "int_frac", "hbm_frac"):
            assert key in r, (name, key)
        assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
        # the bound is the resource with the longer lower-bound time
        assert r["bound"] == ("hbm" if r["hbm_frac"] >= r["int_frac"] else "int")
        assert r["unit"] == ("GB/s" if r["bound"] == "hbm" else "Tops/s")
    for ckpt in (0, 1):
        r = bench.roofline("myers_lane", 0.5, 1.0, work, set_a, set_b, int_peak, hbm_peak, "fallback", ckpt=ckpt)
        assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    # traffic: from the capture record only when it was taken of the current kernel source
    # (the checkpointed and the record-mode kernels have records of their own)
    for ckpt, key in ((1, "myers_lane_ck"), (0, "myers_lane")):
        per, why = bench.traffic_record(key)
        r = bench.roofline("myers_lane", 0.5, 1.0, work, set_a, set_b, int_peak, hbm_peak, "fallback", ckpt=ckpt)
        if per is None:
            assert r["traffic"] is None and r["traffic_source"] == why
        else:
            assert r["traffic"] == pytest.approx(per * set_b.n)
    assert bench.roofline("myers_lane", 0.5, 1.0, work, set_a, set_b, int_peak, hbm_peak, "fallback",
                          traffic_gb=2.0)["traffic"] == pytest.approx(2.0e9)
    assert bench.roofline("pack", 0.5, 1.0, work, set_a, set_b, int_peak, hbm_peak, "fallback")["bound"] is None


def test_clock_sampler_reasons(bench):
    s = bench.ClockSampler(0)  # parsing only: a stand-in for the nvidia-smi process
    s.lines = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
               "0, 1900, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
               "garbage line"]

    class _P:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

    s.proc = _P()
    c = s.stop()
    assert c["samples"] == 2 and c["sm_max_mhz"] == 1965.0 and c["sm_mhz"] == pytest.approx(1932.5)
    assert c["reasons"] == ["sw_power_cap"]


def test_cpu_baseline_scales_sample(bench, sets):
    set_a, set_b = sets
    b = bench.cpu_baseline(set_a, set_b, 1_000_000, 1_000_000, 2, sample_a=500, sample_b=50)
    assert b["kind"] == "port" and b["cores"] == 2 and b["unit"] == "pairs/s" and b["value"] > 0
    assert "500 set-A pairs" in b["sample"]


def test_read_parity_reports_first_mismatch(bench):
    """Per-read parity counts mismatches over the checked reads and describes the first
    one: outcome, has_result, reverse, then (ed, qs, qe, ts, te, CIGAR length) per
    alignment, for the GPU and the oracle."""
    row = (0, 1, 0, [("10M", 0, 0, 10, 5, 15)])
    other = (4, 0, 0, [])
    gpu = [row, other, row]
    par = bench._read_parity(gpu, [row, row, row])
    assert par["reads"] == 3 and par["mismatches"] == 1 and par["first_mismatch"] == 1
    assert par["first_mismatch_detail"] == {"gpu": [4, 0, 0, []], "oracle": [0, 1, 0, [[0, 0, 10, 5, 15, 3]]]}
    # a subset of the reads, by index
    par = bench._read_parity(gpu, [row, row], [0, 2])
    assert par == {"reads": 2, "mismatches": 0}


def test_reference_arm_keeps_the_job_mix(bench, monkeypatch):
    """The reference arm's JSON line on small sizes, with the engine arm's generator run
    on the CPU: the sample keeps the job's set-A : set-B proportion, and value,
    ms_per_step and the projection agree."""
    import contextlib
    import io
    import json
    import types

    from phraya_b200 import datagen as D

    def arm_pairs_cpu(n_a, n_b, rank, dev):
        return (D.extension_pairs_device(n_a, 100, 300, 0.05, seed=2 * rank, device="cpu"),
                D.extension_pairs_device(n_b, 64, 2048, 0.05, seed=2 * rank + 1, log_uniform=True, device="cpu"))

    monkeypatch.setattr(bench, "arm_pairs", arm_pairs_cpu)
    monkeypatch.setattr(bench, "REF_SAMPLE_A", 200)
    args = types.SimpleNamespace(n_a=2000, n_b=1000, steps=2, warmup=1, gpus=1)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, 0, 1)
    line = json.loads(buf.getvalue())
    assert line["impl"] == "reference"
    assert line["config"]["n_pairs_wfa"] == 200 and line["config"]["n_pairs_myers"] == 100
    per_step = 2 * 200 + 100
    assert line["value"] == pytest.approx(per_step / (line["ms_per_step"] / 1000.0))
    assert line["projected_full_job_ms"] == pytest.approx((2 * 2000 + 1000) / line["value"] * 1000.0)
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"
