"""A plan file feeding align_read on the device: the short-read case's target and read
sketches written to a `.phrayaplan` v7 file, read back, and used as the index's sketch
and the reads' stored sketches (executor.rs:615-624) give the same results as sketching
on the device, and as the oracle given the same stored sketches; the placements go to a
`.phraya.queries` sidecar and read back."""
import numpy as np
import pytest

import oracle as O
from phraya_b200 import _abi as A
from phraya_b200 import api as P
from phraya_b200 import casegen as G
from phraya_b200 import planio as IO
from phraya_b200.batch import PackedReads

pytestmark = pytest.mark.gpu


def test_plan_round_trip_drives_align_reads(tmp_path):
    c = G.case2_short(genome_size=200_000, num_reads=1500, read_len=150, divergence=0.01, indel_rate=0.0005,
                      indel_max_len=3, seed=3)
    with P.Engine(0) as eng:
        tv, tp = eng.sketch([c.genome])[0]
        plan = IO.Plan(input_files=["ref.fa", "reads.fq"], timestamp="t", total_read_count=len(c.reads),
                       kmer_index={"synthetic_ref": IO.Sketch(list(zip(tv.tolist(), tp.tolist())))},
                       batch_num_chunks=2)
        for r, (v, p) in zip(c.reads, eng.sketch(c.reads)):
            h = IO.read_content_hash(r)
            plan.read_sketches[h] = IO.Sketch(list(zip(v.tolist(), p.tolist())))
            plan.read_hash_order.append(h)
        f = tmp_path / "case.phrayaplan"
        IO.write_plan(f, plan)
        got = IO.read_plan(f)
        sk = got.kmer_index["synthetic_ref"]
        stored = [got.stored_sketch(r) for r in c.reads]
        assert all(s is not None for s in stored)
        idx = eng.index(c.genome, sketch=(np.array([v for v, _ in sk.minimizers], np.uint64),
                                          np.array([p for _, p in sk.minimizers], np.uint32)))
        plain_idx = eng.index(c.genome)
        for strat in (A.BALANCED, A.SENSITIVE):
            with_plan, st1 = eng.align_reads(idx, c.reads, strat, stored=stored)
            plain, st2 = eng.align_reads(plain_idx, c.reads, strat)
            assert with_plan == plain and st1 == st2
            otg = O.Target(c.genome)
            ores, ost = otg.align_reads(c.reads, strat, stored=stored)
            assert with_plan == ores and tuple(st1) == tuple(ost)
        ids = [f"read_{i}" for i in range(len(c.reads))]
        qf = tmp_path / "case.phraya.queries"
        qi = IO.query_index(ids, with_plan)
        IO.write_queries(qf, qi)
        back = IO.read_queries(qf)
        assert back == {k: [(p, sc) for p, sc in v] for k, v in IO.queries_wire(qi).items()}
        assert len(back) == sum(1 for r in with_plan if r[1] and 1 - r[3][0][1] / max(r[3][0][3], 1) >= 0.95)
        idx.close()
        plain_idx.close()
