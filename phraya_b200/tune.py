"""Autotuner for the extension kernels' launch parameters.

The kernels' results never depend on these settings (lanes per WFA pair, the length
bucket edge between short and long WFA pairs, threads per block, resident blocks per
SM, the Myers stored-band base and checkpointing, the threshold of the one-CTA-per-pair
WFA kernels and the gap-affine one's threads per CTA);
only their speed does. The tuner runs a coordinate descent over a small candidate grid
per key: for each key in turn it times every candidate on the given workloads with the
other keys at their current best, keeps the fastest, and repeats the sweep. Time is the
device time of the engine's kernels (CUDA events, phr_ctx timing), summed over the
workloads, best of `repeats` runs. Every candidate's results are compared with the
first run's, so a setting that changed a result would stop the tuner.

The chosen values are written as "key value" lines, the tune-file format that
phr_ctx_create reads when phr_config.tune_file_enable is set
(api.Engine(tune_file=...)).

    python -m phraya_b200.tune --out phraya_b200_tune.txt
"""
import argparse
import ctypes as C

from . import _abi as A
from . import api as P

SPACE = {
    "wfa_group_short": [4, 8, 16, 32],
    "wfa_affine_group_short": [8, 16, 32],
    "wfa_group_long": [16, 32],
    "wfa_long_min": [512, 1024, 2048],
    "block_threads": [128, 256],
    "max_blocks_per_sm": [2, 3, 4],
    "myers_band_base": [32, 48, 64, 128],
    "myers_lane_ckpt": [0, 1],
    "wfa_big_min": [0, 2048, 4096, 8192],
    "wfa_affine_big_threads": [256, 512, 1024],
}

KEYS_FOR = {
    A.ENGINE_WFA_LINEAR: ["wfa_group_short", "wfa_group_long", "wfa_long_min", "block_threads",
                          "max_blocks_per_sm", "wfa_big_min"],
    A.ENGINE_WFA_AFFINE: ["wfa_affine_group_short", "wfa_group_long", "wfa_long_min", "block_threads",
                          "max_blocks_per_sm", "wfa_big_min", "wfa_affine_big_threads"],
    A.ENGINE_MYERS_FIT: ["myers_band_base", "block_threads", "max_blocks_per_sm"],
    A.ENGINE_MYERS_GLOBAL: ["myers_band_base", "myers_lane_ckpt", "block_threads", "max_blocks_per_sm"],
}


def _device_ms(eng):
    recs = (A.KernelTiming * 64)()
    n = eng._lib.phr_ctx_get_timing(eng.handle, recs, 64)
    return sum(recs[i].total_ms for i in range(n) if not recs[i].name.startswith(b"host:"))


def measure(eng, workloads, repeats=3):
    """Best-of-`repeats` device milliseconds of all workloads, and their results."""
    L = eng._lib
    best, results = None, []
    for rep in range(repeats + 1):
        L.phr_ctx_reset_timing(eng.handle)
        L.phr_ctx_set_timing(eng.handle, 1 if rep else 0)
        out = []
        for engine, packed, costs in workloads:
            aln, cig = eng.extend_packed(engine, packed, P.AffineCosts(*costs))
            out.append(P.unpack(aln, cig))
        L.phr_ctx_set_timing(eng.handle, 0)
        if rep == 0:
            results = out  # warm-up run: arenas grow, modules load
            continue
        ms = _device_ms(eng)
        best = ms if best is None else min(best, ms)
    return best, results


def tune(eng, workloads, rounds=2, repeats=3, space=None, log=None, min_gain=0.02):
    """Coordinate descent over `space` (default SPACE restricted to the workloads'
    engines). A candidate replaces the current value only when it is faster by more
    than `min_gain` (relative), so timing noise does not move settings the workloads
    do not exercise. Returns ({key: value}, best_ms). Leaves the engine at the best
    values."""
    space = dict(space or SPACE)
    keys = []
    for engine, _, _ in workloads:
        for k in KEYS_FOR[engine]:
            if k in space and k not in keys:
                keys.append(k)
    current = {k: eng.get_tune(k) for k in keys}
    best_ms, reference = measure(eng, workloads, repeats)
    for _ in range(rounds):
        changed = False
        for k in keys:
            for v in space[k]:
                if v == current[k]:
                    continue
                eng.set_tune(k, v)
                ms, res = measure(eng, workloads, repeats)
                if res != reference:
                    raise AssertionError(f"tune key {k}={v} changed a result")
                if log:
                    log(f"{k}={v}: {ms:.3f} ms (best {best_ms:.3f})")
                if ms < best_ms * (1.0 - min_gain):
                    best_ms, current[k], changed = ms, v, True
                eng.set_tune(k, current[k])
        if not changed:
            break
    return current, best_ms


def write_tune_file(path, values):
    with open(path, "w") as f:
        for k, v in values.items():
            f.write(f"{k} {int(v)}\n")


def read_tune_file(path):
    out = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) == 2:
                out[parts[0]] = int(parts[1])
    return out


def default_workloads(n_wfa=100_000, n_myers=20_000, seed=7):
    """Config-2-shaped workloads: WFA pairs of 100-300 bp at 0-5 % divergence (affine
    (4, 6, 2) and linear) and Myers pairs log-uniform 64-2048 bp."""
    from . import datagen as D
    a = D.extension_pairs(n_wfa, 100, 300, 0.05, seed=seed)
    b = D.extension_pairs(n_myers, 64, 2048, 0.05, seed=seed + 1, log_uniform=True)
    return [(A.ENGINE_WFA_AFFINE, a, (4, 6, 2)), (A.ENGINE_WFA_LINEAR, a, (2, 4, 1)),
            (A.ENGINE_MYERS_GLOBAL, b, (2, 4, 1))]


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default="phraya_b200_tune.txt")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--n-wfa", type=int, default=100_000)
    ap.add_argument("--n-myers", type=int, default=20_000)
    ap.add_argument("--rounds", type=int, default=2)
    args = ap.parse_args()
    eng = P.Engine(args.device)
    values, ms = tune(eng, default_workloads(args.n_wfa, args.n_myers), rounds=args.rounds, log=print)
    write_tune_file(args.out, values)
    print(f"best {ms:.3f} ms: {values} -> {args.out}")


if __name__ == "__main__":
    main()
