"""Benchmark: phraya-align's batched extension microbench on B200.

Workload (one step = the whole job, all pairs resident in HBM):
  set A: N_A query/target pairs, query lengths uniform in [100, 300] bp, targets =
         query mutated at per-pair divergence U[0, 5 %] (70 % substitutions, 30 % 1-5 bp
         indels); aligned with WFA affine (mismatch 4, gap open 6, gap extend 2) AND WFA
         linear;
  set B: N_B pairs with lengths log-uniform in [64, 2048] bp, same mutation model;
         aligned with Myers bit-parallel edit distance + CIGAR (myers_edit_distance).
Metric: aligned pairs per second over the whole job (2 N_A + N_B alignments per step);
DP-equivalent GCUPS (sum q*t / s) is reported beside it. Synthetic seeded data.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "reads/s & GCUPS on 1 B200, served vs per-call GPU; p50/p99 latency; bit-exact"
N_A_DEFAULT = 1_000_000
N_B_DEFAULT = 1_000_000
COSTS_A = (4, 6, 2)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sms, maxs, reasons = [], [], set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxs) if maxs else None,
                "reasons": sorted(reasons), "samples": len(sms)}


def make_workload(n_a, n_b, seed):
    from phraya_b200 import datagen as D
    set_a = D.extension_pairs(n_a, 100, 300, 0.05, seed=seed)
    set_b = D.extension_pairs(n_b, 64, 2048, 0.05, seed=seed + 1000, log_uniform=True)
    return set_a, set_b


def dp_cells(p):
    return float(np.dot(p.q_len.astype(np.float64), p.t_len.astype(np.float64)))


def input_bytes(p):
    return int(p.seq.nbytes + p.q_off.nbytes + p.q_len.nbytes + p.t_off.nbytes + p.t_len.nbytes + 8 * p.n)


def packed_bytes(p):
    """2-bit packed bytes of every query and target (16 bases per 32-bit word)."""
    return 4.0 * float(((p.q_len.astype(np.int64) + 15) // 16).sum() + ((p.t_len.astype(np.int64) + 15) // 16).sum())


def roofline(name, step_ms, launches, work, set_a, set_b, int_peak, hbm_peak, peak_src, traffic_gb=None):
    """Roofline of one kernel over a step: algorithmic work from the kernel's own counters,
    bound = the resource (integer issue or HBM) whose lower-bound time is longer."""
    sec = step_ms / 1000.0
    if name == "myers_lane":
        cols = work["myers_lane_block_columns"]      # 64-row block x column steps evaluated
        ops = cols * 64 * 22.0 / 32.0                # 22 word operations per 32 rows per column
        # {VP, HP} records written (16 B per block-column), read back along the path
        # (>= one 16 B record per target column), packed inputs
        nbytes = cols * 16.0 + float(set_b.t_len.astype(np.float64).sum()) * 16.0 + packed_bytes(set_b)
        t_int, t_hbm = ops / int_peak, nbytes / hbm_peak
        work_txt = ("band cells = 64 x block-columns evaluated (kernel counter); int ops = cells x 22/32; "
                    "bytes = 16 B {VP,HP} record per block-column + 16 B read back per target column + 2-bit inputs")
    elif name in ("wfa_affine", "wfa_linear"):
        cells, words = work[name + "_cells"], work[name + "_lcp_words"]
        per = 30.0 if name == "wfa_affine" else 10.0   # ops per wavefront diagonal (3 layers / 1)
        ops = per * cells + 4.0 * words                # + 4 ops per word compare of match extension
        nbytes = packed_bytes(set_a) + 40.0 * set_a.n  # 2-bit inputs + one alignment record per pair
        t_int, t_hbm = ops / int_peak, nbytes / hbm_peak
        work_txt = (f"wavefront diagonals x {per:.0f} ops + LCP word compares x 4 ops (kernel counters); "
                    "bytes = 2-bit inputs + result records")
        cols = None
    else:
        return {"kernel": name, "kernel_ms_per_step": step_ms, "bound": None,
                "note": "no work counter for this kernel"}
    if t_hbm >= t_int:
        bound, achieved, peak, unit = "hbm", nbytes / sec / 1e9, hbm_peak / 1e9, "GB/s"
        psrc = f"measured copy bandwidth ({peak_src})"
    else:
        bound, achieved, peak, unit = "int", ops / sec / 1e12, int_peak / 1e12, "Tops/s"
        psrc = "nominal integer issue rate 148 SMs x 4 x 32 lanes x max SM clock"
    traffic, traffic_src = None, None
    if traffic_gb is not None:
        traffic, traffic_src = traffic_gb * 1e9, "--traffic-gb-per-step"
    elif name == "myers_lane":
        # ncu dram__bytes_read.sum + write.sum of one launch on 100,000 pairs of the same
        # distribution (3.01 + 4.58 GB, profiles/myers_lane_kernel_set_b_100k.md), scaled by
        # the pair count
        traffic = 7.59e9 * set_b.n / 100000
        traffic_src = "ncu capture of 100,000 pairs (7.59 GB), scaled by pairs"
    out = {"bound": bound, "achieved": achieved, "peak": peak, "unit": unit, "frac": achieved / peak,
           "traffic": traffic, "traffic_source": traffic_src, "kernel": name, "kernel_ms_per_step": step_ms,
           "launches_per_step": launches, "work": work_txt, "peak_source": psrc,
           "int_frac": ops / sec / int_peak, "hbm_frac": nbytes / sec / hbm_peak}
    if name == "myers_lane":
        out.update(band_cells_per_step=cols * 64, redo_pairs_per_step=work["myers_lane_redo_pairs"])
    else:
        out.update(wavefront_diagonals_per_step=work[name + "_cells"], lcp_words_per_step=work[name + "_lcp_words"])
    return out


def cpu_baseline(set_a, set_b, n_a, n_b, nthreads, sample_a=60000, sample_b=6000):
    """Times the oracle (CPU restatement) on a bounded sample and scales to the job."""
    import oracle as O
    from phraya_b200 import _abi as A
    from phraya_b200.batch import PackedPairs

    def sub(p, k):
        k = min(k, p.n)
        return PackedPairs.from_arrays(p.seq, p.q_off[:k].copy(), p.q_len[:k].copy(), p.t_off[:k].copy(),
                                       p.t_len[:k].copy())

    sa, sb = sub(set_a, sample_a), sub(set_b, sample_b)
    L = O.lib()
    t = {}
    for name, eng, p, costs in (("affine", A.ENGINE_WFA_AFFINE, sa, COSTS_A), ("linear", A.ENGINE_WFA_LINEAR, sa, (2, 4, 1)),
                                ("myers", A.ENGINE_MYERS_GLOBAL, sb, (2, 4, 1))):
        b = p.batch()
        t0 = time.perf_counter()
        L.orc_extend_batch_time(eng, b, A.AffineCosts(*costs), nthreads)
        t[name] = time.perf_counter() - t0
    job_s = (t["affine"] + t["linear"]) * (n_a / sa.n) + t["myers"] * (n_b / sb.n)
    return {"value": (2 * n_a + n_b) / job_s, "unit": "pairs/s", "cores": nthreads, "kind": "port",
            "sample": f"{sa.n} set-A pairs (WFA affine 4/6/2 + WFA linear) and {sb.n} set-B pairs (Myers), "
                      f"scaled to {n_a}+{n_a}+{n_b} alignments; {t['affine']:.2f}+{t['linear']:.2f}+{t['myers']:.2f} s"}


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU algorithm (the oracle restatement; the Rust
    reference cannot be built without a Rust toolchain) on the host cores."""
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    n_a, n_b = args.n_a, args.n_b
    set_a, set_b = make_workload(min(n_a, 60000), min(n_b, 6000), seed=0)
    vals = []
    base = None
    for s in range(args.warmup + args.steps):
        base = cpu_baseline(set_a, set_b, n_a, n_b, nthreads, sample_a=set_a.n, sample_b=set_b.n)
        if s >= args.warmup:
            vals.append(base["value"])
    v = statistics.median(vals)
    ms = (2 * n_a + n_b) / v * 1000.0
    line = {"metric": METRIC, "value": v, "unit": "pairs/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
            "config": {"workload": "batched extension microbench", "n_pairs_wfa": n_a, "n_pairs_myers": n_b,
                       "note": "CPU restatement of phraya-align (Rust toolchain absent); bounded sample per step"},
            "cpu_baseline": {**base, "value": v},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_engine(args, rank, world):
    import ctypes as C

    import torch

    from phraya_b200 import _abi as A
    from phraya_b200 import api as P
    from phraya_b200 import dist as R

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    n_a, n_b = args.n_a, args.n_b
    from phraya_b200 import datagen as D
    t_gen = time.perf_counter()
    dev_a = D.extension_pairs_device(n_a, 100, 300, 0.05, seed=2 * rank, device=f"cuda:{dev}")
    dev_b = D.extension_pairs_device(n_b, 64, 2048, 0.05, seed=2 * rank + 1, log_uniform=True, device=f"cuda:{dev}")
    set_a, set_b = D.to_packed(dev_a), D.to_packed(dev_b)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    eng = P.Engine(dev)
    L = eng._lib
    stream = torch.cuda.ExternalStream(L.phr_ctx_stream(eng.handle), device=dev)

    # ---- device-resident batches (value) -------------------------------------
    def to_dev(p):
        d = {k: torch.from_numpy(np.ascontiguousarray(getattr(p, k))).to(f"cuda:{dev}")
             for k in ("seq", "q_off", "q_len", "t_off", "t_len")}
        b = A.PairBatch()
        b.n_pairs = p.n
        b.seq = d["seq"].data_ptr()
        b.seq_bytes = p.seq.nbytes
        b.q_off, b.q_len = d["q_off"].data_ptr(), d["q_len"].data_ptr()
        b.t_off, b.t_len = d["t_off"].data_ptr(), d["t_len"].data_ptr()
        b.q_seed = b.t_seed = None
        cap = int(0.75 * (p.q_len.sum() + p.t_len.sum())) + 64 * p.n
        aln = torch.empty(p.n * C.sizeof(A.Alignment), dtype=torch.uint8, device=f"cuda:{dev}")
        cig = torch.empty(cap, dtype=torch.uint8, device=f"cuda:{dev}")
        arena = A.ResultArena(aln.data_ptr(), cig.data_ptr(), cap, 0)
        return d, b, aln, cig, arena

    jobs = [(A.ENGINE_WFA_AFFINE, COSTS_A, *to_dev(set_a)), (A.ENGINE_WFA_LINEAR, (2, 4, 1), *to_dev(set_a)),
            (A.ENGINE_MYERS_GLOBAL, (2, 4, 1), *to_dev(set_b))]
    torch.cuda.synchronize()

    def step():
        for eng_id, costs, _d, b, _aln, _cig, arena in jobs:
            eng.check(L.phr_extend_batch_device(eng.handle, eng_id, C.byref(b), A.AffineCosts(*costs),
                                                C.byref(arena)))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    R.barrier()
    L.phr_ctx_reset_timing(eng.handle)
    L.phr_ctx_set_timing(eng.handle, 1)
    launches0 = eng.kernel_launches
    clocks = ClockSampler(dev)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    L.phr_ctx_set_timing(eng.handle, 0)
    launches = eng.kernel_launches - launches0
    elapsed_ms = R.max_over_ranks(e0.elapsed_time(e1), device=f"cuda:{dev}")
    ms_per_step = elapsed_ms / args.steps
    per_step_pairs = 2 * n_a + n_b
    value = per_step_pairs * world / (ms_per_step / 1000.0)
    cells = 2 * dp_cells(set_a) + dp_cells(set_b)
    gcups = cells * world / (ms_per_step / 1000.0) / 1e9

    # per-kernel device times (CUDA events on the launching stream)
    recs = (A.KernelTiming * 64)()
    nrec = L.phr_ctx_get_timing(eng.handle, recs, 64)
    ktimes = {recs[i].name.decode(): (recs[i].launches, recs[i].total_ms) for i in range(min(nrec, 64))
              if not recs[i].name.startswith(b"host:")}
    # work counters of the timed steps (reset with the timings)
    work = {k: eng.counter(k) / args.steps for k in ("myers_lane_block_columns", "myers_lane_redo_pairs",
                                                      "wfa_affine_cells", "wfa_affine_lcp_words",
                                                      "wfa_linear_cells", "wfa_linear_lcp_words")}

    # ---- end to end through the host API, pinned host buffers ----------------
    def pinned_pairs(p):
        from phraya_b200.batch import PackedPairs
        arrs = {}
        for k in ("seq", "q_off", "q_len", "t_off", "t_len"):
            src = np.ascontiguousarray(getattr(p, k))
            t = torch.empty(src.shape, dtype=torch.from_numpy(src[:1]).dtype, pin_memory=True)
            t.numpy()[...] = src
            arrs[k] = t
        for k in ("q_seed", "t_seed"):  # zero seeds, pinned like the rest (pageable copies would block)
            arrs[k] = torch.zeros(p.n, dtype=torch.int32, pin_memory=True)
        pp = PackedPairs.from_arrays(*(arrs[k].numpy() for k in ("seq", "q_off", "q_len", "t_off", "t_len")),
                                     q_seed=arrs["q_seed"].numpy().view(np.uint32),
                                     t_seed=arrs["t_seed"].numpy().view(np.uint32))
        pp._pins = arrs
        return pp

    pa, pb = pinned_pairs(set_a), pinned_pairs(set_b)

    def host_outputs(p):
        aln = torch.empty(p.n * C.sizeof(A.Alignment), dtype=torch.uint8, pin_memory=True)
        cap = int(0.75 * (p.q_len.sum() + p.t_len.sum())) + 64 * p.n
        cig = torch.empty(cap, dtype=torch.uint8, pin_memory=True)
        return aln, cig, cap

    outs = [host_outputs(pa), host_outputs(pa), host_outputs(pb)]
    e2e_jobs = [(A.ENGINE_WFA_AFFINE, COSTS_A, pa, outs[0]), (A.ENGINE_WFA_LINEAR, (2, 4, 1), pa, outs[1]),
                (A.ENGINE_MYERS_GLOBAL, (2, 4, 1), pb, outs[2])]
    d2h = 0

    def e2e_step():
        nonlocal d2h
        d2h = 0
        for eng_id, costs, p, (aln, cig, cap) in e2e_jobs:
            arena = A.ResultArena(aln.data_ptr(), cig.data_ptr(), cap, 0)
            b = p.batch()
            eng.check(L.phr_extend_batch(eng.handle, eng_id, C.byref(b), A.AffineCosts(*costs), C.byref(arena)))
            d2h += p.n * C.sizeof(A.Alignment) + arena.cigar_used

    for _ in range(max(1, args.warmup)):
        e2e_step()
    torch.cuda.synchronize()
    R.barrier()
    # CUDA events on the context stream: the host copies of phr_extend_batch run on it
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_s = R.max_over_ranks(f0.elapsed_time(f1) / 1000.0 / args.steps, device=f"cuda:{dev}")
    h2d = 2 * input_bytes(set_a) + input_bytes(set_b)

    if rank != 0:
        return
    # ---- roofline of the dominant kernel (its device time per step, CUDA events) ----
    peaks, peak_src = load_peaks()
    kms = {k: tot / args.steps for k, (_nl, tot) in ktimes.items()}
    name = max(kms, key=kms.get)
    step_ms = kms[name]
    int_peak = 148 * 4 * 32 * peaks.get("sm_max_mhz", 1965.0) * 1e6   # ops/s, nominal issue
    hbm_peak = peaks.get("hbm_gbs", 6650.0) * 1e9                      # bytes/s, measured copy
    roof = roofline(name, step_ms, ktimes[name][0] / args.steps, work, set_a, set_b, int_peak, hbm_peak,
                    peak_src, args.traffic_gb_per_step)
    # the other extension kernels, each against its own bound
    roofs = {k: roofline(k, kms[k], ktimes[k][0] / args.steps, work, set_a, set_b, int_peak, hbm_peak, peak_src)
             for k in ("myers_lane", "wfa_affine", "wfa_linear") if k in kms}
    pipe = None
    if not args.no_pipeline:
        # the read pipeline and the server start from a fresh context and an empty torch
        # cache: the extension bench's arenas and buffers would otherwise hold device
        # memory that the server's admission control waits for
        del jobs
        eng.close()
        torch.cuda.empty_cache()
        eng = P.Engine(dev)
        pipe = run_pipeline(eng, dev, args)
    cpu = cpu_baseline(set_a, set_b, n_a, n_b, os.cpu_count() or 1) if not args.no_cpu else None
    line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
            "config": {"workload": "batched extension microbench", "n_pairs_wfa": n_a, "n_pairs_myers": n_b,
                       "wfa_affine_costs": list(COSTS_A), "lengths_wfa": [100, 300],
                       "lengths_myers": [64, 2048, "log-uniform"], "divergence": [0.0, 0.05],
                       "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"},
            "gcups_dp_equivalent": gcups,
            "e2e": {"value": per_step_pairs * world / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1000.0},
            "gpu_launches": launches,
            "roofline": roof,
            "rooflines": roofs,
            "kernel_ms": {k: round(v[1] / args.steps, 3) for k, v in ktimes.items()},
            "clocks": clk,
            "cpu_baseline": cpu,
            "pipeline": pipe,
            "datagen_s": round(t_gen, 1)}
    print(json.dumps(line))


def run_pipeline(eng, dev, args):
    """Read-pipeline figures: align_read over a 1 Mbp reference (20,000 x 150 bp reads, 1 %
    substitutions + 0.05 % 1-3 bp indels, both strands): batched vs one read per call,
    and a served mixed Poisson stream (90 % 150 bp at 1 % error, 10 % long reads with
    lognormal lengths, median 8 kb, 5 % error) with p50/p99 latency of the short reads."""
    import ctypes as C
    import numpy as np
    from phraya_b200 import _abi as A
    from phraya_b200 import datagen as D
    from phraya_b200.batch import PackedReads

    out = {}
    ref = D.random_reference(1_000_000, seed=100)
    idx = eng.index(ref)
    packed, _, _ = D.reads_on_reference(ref, args.reads, 150, 0.0105, seed=101, sub_frac=0.952, max_indel=3)
    reads = [bytes(packed.seq[o:o + l]) for o, l in zip(packed.off, packed.len)]
    for strat, name in ((A.BALANCED, "balanced"), (A.SENSITIVE, "sensitive_affine")):
        eng.align_packed(idx, packed, strat, A.GAP_AFFINE)  # warm-up
        t0 = time.perf_counter()
        rr, aln, cig, st = eng.align_packed(idx, packed, strat, A.GAP_AFFINE)
        dt = time.perf_counter() - t0
        out[f"batched_{name}_reads_per_s"] = len(reads) / dt
        out[f"batched_{name}_placed_frac"] = st[0] / len(reads)
    # variant observations of every read with a result (extract_variants_from_cigar with
    # local coverage, executor.rs:735-775, 814-1096) on the device, in the same call
    eng.align_packed_variants(idx, packed, A.BALANCED, A.GAP_AFFINE)  # warm-up
    t0 = time.perf_counter()
    vres = eng.align_packed_variants(idx, packed, A.BALANCED, A.GAP_AFFINE)
    dt = time.perf_counter() - t0
    n_var = len(vres[5])
    out["batched_balanced_with_variants_reads_per_s"] = len(reads) / dt
    out["variant_observations"] = n_var
    out["coverage_cells"] = len(vres[6])
    eng._lib.phr_ctx_reset_timing(eng.handle)
    eng.set_timing(True)
    eng.align_packed_variants(idx, packed, A.BALANCED, A.GAP_AFFINE)
    kt = eng.kernel_times()
    eng.set_timing(False)
    vk_ms = sum(kt.get(k, (0, 0.0))[1] for k in ("variant_count", "variant_write"))
    out["variant_kernels_ms"] = vk_ms
    out["variant_observations_per_s_device"] = n_var / (vk_ms / 1000.0) if vk_ms > 0 else None
    if not args.no_cpu:
        import oracle as O
        otg = O.Target(ref)
        t0 = time.perf_counter()
        O_res = otg.variants_packed(packed, vres[0], vres[1], vres[2], A.BALANCED)
        cdt = time.perf_counter() - t0
        out["variants_cpu_baseline"] = {"value": len(O_res[1]) / cdt, "unit": "observations/s", "cores": 1,
                                        "kind": "port", "sample": f"{len(reads)} reads, balanced, 1 Mbp"}
    # one read per call (the reference API's shape), on a sample
    k = min(300, len(reads))
    one = [PackedReads([r]) for r in reads[:k]]
    eng.align_packed(idx, one[0], A.BALANCED, A.GAP_AFFINE)
    t0 = time.perf_counter()
    for pr in one:
        eng.align_packed(idx, pr, A.BALANCED, A.GAP_AFFINE)
    out["percall_balanced_reads_per_s"] = k / (time.perf_counter() - t0)
    out["batched_over_percall"] = out["batched_balanced_reads_per_s"] / out["percall_balanced_reads_per_s"]
    # served mixed stream
    rng = np.random.default_rng(102)
    n_req = args.reads
    n_long = n_req // 10
    longp, _, _ = D.reads_on_reference(
        ref, n_long, error=0.05, seed=103, sub_frac=0.4, max_indel=3,
        length_sampler=lambda g, n: np.clip(np.exp(g.normal(np.log(8000), 0.5, n)), 1000, 50000).astype(np.int64))
    longs = [bytes(longp.seq[o:o + l]) for o, l in zip(longp.off, longp.len)]
    stream = reads[:n_req - n_long] + longs
    order = rng.permutation(len(stream))
    stream = [stream[i] for i in order]
    is_short = [len(r) <= 500 for r in stream]

    def serve(rate):
        gaps = np.random.default_rng(104).exponential(1.0 / rate, len(stream))
        arrive = np.cumsum(gaps)
        srv = eng.server(idx, strategy=A.BALANCED, max_batch_reads=2048, max_wait_us=1000, n_streams=3)
        # warm the workers with a slice of the same mix (long reads included), so every
        # worker's first long batch is behind it
        warm = stream[:512]
        srv.submit_many(warm)
        got = 0
        while got < len(warm):
            got += len(srv.poll(4096, wait_us=20000))
        lat = {}
        ids = {}
        t_start = time.perf_counter()
        i = 0
        done = 0
        while done < len(stream):
            now = time.perf_counter() - t_start
            j = int(np.searchsorted(arrive, now, side="right"))
            if j > i:  # every read whose arrival time has passed, in one call
                for k, rid in enumerate(srv.submit_many(stream[i:j])):
                    ids[rid] = i + k
                i = j
            for rid, res, l in srv.poll(4096, wait_us=200 if i >= len(stream) else 0):
                lat[ids[rid]] = l
                done += 1
        t_total = time.perf_counter() - t_start
        srv.close()
        sl = sorted(lat[j] for j in range(len(stream)) if is_short[j])
        al = sorted(lat.values())
        return {"rate_offered_reads_per_s": rate, "reads": len(stream), "long_reads": n_long,
                "throughput_reads_per_s": len(stream) / t_total,
                "p50_ms_150bp": sl[len(sl) // 2] / 1000.0, "p99_ms_150bp": sl[int(len(sl) * 0.99)] / 1000.0,
                "p99_ms_all": al[int(len(al) * 0.99)] / 1000.0}

    sweep = [serve(r) for r in args.served_rates]
    ok = [x for x in sweep if x["p99_ms_150bp"] <= 50.0]
    best = max(ok, key=lambda x: x["throughput_reads_per_s"]) if ok else max(sweep, key=lambda x: x["rate_offered_reads_per_s"])
    out["served"] = dict(best, p99_target_ms=50.0, meets_p99_target=bool(ok))
    out["served_sweep"] = sweep
    out["served_over_percall"] = out["served"]["throughput_reads_per_s"] / out["percall_balanced_reads_per_s"]
    out["workload"] = ("align_read, 1 Mbp i.i.d. reference, 150 bp reads both strands, 1 % subs + 0.05 % "
                       "1-3 bp indels; served: Poisson arrivals, 90 % 150 bp + 10 % lognormal long reads")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20,
                    help="timed steps (20 keep the timed region near 0.7 s, several clock samples)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n-a", type=int, default=N_A_DEFAULT)
    ap.add_argument("--n-b", type=int, default=N_B_DEFAULT)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-pipeline", action="store_true", help="skip the read-pipeline / serving section")
    ap.add_argument("--reads", type=int, default=20000, help="reads of the read-pipeline section")
    ap.add_argument("--served-rates", type=float, nargs="+", default=[25000.0, 50000.0, 100000.0],
                    help="Poisson arrival rates (reads/s) of the served sweep")
    ap.add_argument("--traffic-gb-per-step", type=float, default=None,
                    help="DRAM bytes per step of the dominant kernel from an ncu capture (reported as is)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and args.impl == "engine":
        import datetime

        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_engine(args, rank, world)
    finally:
        if world > 1 and args.impl == "engine":
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
