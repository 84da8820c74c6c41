"""Serving loop: every read's result is identical alone, in a mixed continuous stream,
and through the batched align_reads call."""
import time

import pytest

from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import datagen as D

pytestmark = pytest.mark.gpu


def drain(srv, want, timeout_s=120):
    got = {}
    t0 = time.time()
    while len(got) < want and time.time() - t0 < timeout_s:
        for rid, res, lat in srv.poll(4096, wait_us=20000):
            got[rid] = (res, lat)
    assert len(got) == want
    return got


@pytest.mark.parametrize("strat", [A.BALANCED, A.SENSITIVE])
def test_alone_equals_mixed_equals_batched(strat):
    eng = P.Engine(0)
    ref = D.random_reference(400_000, seed=41)
    idx = eng.index(ref)
    short, _, _ = D.reads_on_reference(ref, 240, 150, 0.01, seed=42)
    longr, _, _ = D.reads_on_reference(ref, 24, 1500, 0.05, seed=43)
    reads = [bytes(short.seq[o:o + l]) for o, l in zip(short.off, short.len)]
    reads += [bytes(longr.seq[o:o + l]) for o, l in zip(longr.off, longr.len)]
    reads = [reads[i] for i in sorted(range(len(reads)), key=lambda i: (i * 7919) % len(reads))]  # interleave
    batched, _ = eng.align_reads(idx, reads, strat)
    srv = eng.server(idx, strategy=strat, max_batch_reads=64, max_wait_us=500, n_streams=3)
    # alone: one request in flight at a time
    alone = []
    for r in reads[:40]:
        rid = srv.submit(r)
        got = drain(srv, 1)
        alone.append(got[rid][0])
    # mixed: everything in flight together, batches formed continuously
    ids = [srv.submit(r) for r in reads]
    got = drain(srv, len(reads))
    mixed = [got[i][0] for i in ids]
    srv.close()
    assert alone == batched[:40]
    assert mixed == batched
    lat = [got[i][1] for i in ids]
    assert min(lat) > 0


@pytest.mark.parametrize("short_lane", [1, -1])
def test_submit_many_and_lanes(short_lane):
    """Batched submission and both lane layouts return the batched call's results; long
    reads (one-CTA-per-pair WFA path) and short reads share the stream."""
    eng = P.Engine(0)
    ref = D.random_reference(400_000, seed=44)
    idx = eng.index(ref)
    short, _, _ = D.reads_on_reference(ref, 300, 150, 0.01, seed=45)
    longr, _, _ = D.reads_on_reference(ref, 12, 5000, 0.05, seed=46)
    reads = [bytes(short.seq[o:o + l]) for o, l in zip(short.off, short.len)]
    reads += [bytes(longr.seq[o:o + l]) for o, l in zip(longr.off, longr.len)]
    reads = [reads[i] for i in sorted(range(len(reads)), key=lambda i: (i * 7919) % len(reads))]
    batched, _ = eng.align_reads(idx, reads, A.BALANCED)
    srv = eng.server(idx, strategy=A.BALANCED, max_batch_reads=128, max_wait_us=300, n_streams=3,
                     short_lane=short_lane, long_blocks_per_sm=1)
    ids = []
    for k in range(0, len(reads), 50):
        ids += srv.submit_many(reads[k:k + 50])
    assert len(set(ids)) == len(reads)
    got = drain(srv, len(reads))
    srv.close()
    assert [got[i][0] for i in ids] == batched
