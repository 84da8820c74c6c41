"""phraya-io's formats on the host (phraya_b200.planio): the reference's own round-trip
and filtering cases for `.phraya.queries` (phraya-io/src/queries.rs test module), plan
v7 layout and round trip (plan.rs:561-873), `.phraya` round trip (phraya.rs:67-97),
CoverageTrack quantization (types.rs:618-660) and the FNV-1a content hash (plan.rs:29-41)."""
import os

import pytest

from phraya_b200 import planio as IO


def test_zstd_round_trip_and_concatenated_frames():
    a, b = b"ACGT" * 5000, bytes(range(256)) * 40
    assert IO.zstd_decompress(IO.zstd_compress(a)) == a
    assert IO.zstd_decompress(IO.zstd_compress(a) + IO.zstd_compress(b)) == a + b
    with pytest.raises(IO.FormatError):
        IO.zstd_decompress(IO.zstd_compress(a)[:-5])


def test_fnv1a_content_hash_known_values():
    # FNV-1a 64 published test vectors
    assert IO.read_content_hash(b"") == 0xCBF29CE484222325
    assert IO.read_content_hash(b"a") == 0xAF63DC4C8601EC8C
    assert IO.read_content_hash(b"foobar") == 0x85944171F73967E8


def test_queries_round_trip(tmp_path):
    # queries.rs: round trip of five positions at or above the threshold
    pos = [(100, 0.99), (200, 0.98), (300, 0.97), (400, 0.96), (500, 0.95)]
    f = tmp_path / "q.phraya.queries"
    IO.write_queries(f, {"test_query": pos})
    assert IO.read_queries(f)["test_query"] == pos


def test_queries_empty_and_subthreshold_dropped(tmp_path):
    f = tmp_path / "q"
    IO.write_queries(f, {"query_no_hits": [], "query_subthreshold": [(10, 0.40)]})
    assert IO.read_queries(f) == {}
    IO.write_queries(f, {"mixed": [(100, 0.98), (200, 0.40)]})
    assert IO.read_queries(f) == {"mixed": [(100, 0.98)]}


def test_queries_bytes_do_not_depend_on_insertion_order(tmp_path):
    keys = [f"read_{i}" for i in range(64)]
    a = {k: [(300 - i, 0.97), (i, 0.99), (i, 0.96)] for i, k in enumerate(keys)}
    b = {k: a[k][::-1] for k in reversed(keys)}
    IO.write_queries(tmp_path / "a", a)
    IO.write_queries(tmp_path / "b", b)
    assert (tmp_path / "a").read_bytes() == (tmp_path / "b").read_bytes()
    # positions sorted by (position, score descending)
    assert IO.read_queries(tmp_path / "a")["read_0"] == [(0, 0.99), (0, 0.96), (300, 0.97)]


def sample_plan(chunks=3):
    sk = lambda n, base: IO.Sketch([(base + i * 7, i * 3) for i in range(n)])  # noqa: E731
    reads = [b"ACGT" * (i + 5) for i in range(10)]
    p = IO.Plan(use_case="ReadsWithRef", input_files=["ref.fa", "reads.fq"], timestamp="2026-01-01T00:00:00Z",
                reference_space=[IO.ReferenceSpace("ab" * 32, "E. coli", {"chr": sk(5, 100)})],
                kmer_index={"chr": sk(8, 1000), "plasmid": sk(3, 50)}, kmer_uniqueness={5: 0.5, 1: 1.0},
                task_list=[(0, 0), (1, 0)], hotspot_intervals=[(10, 20), (40, 45)], reads_per_file=[10],
                total_read_count=10, batch_num_chunks=chunks, batch_reads_per_chunk=4,
                read_byte_offsets=[[i * 100 for i in range(10)]], batch_output_paths=["o1", "o2", "o3"])
    for i, r in enumerate(reads):
        h = IO.read_content_hash(r)
        p.read_sketches[h] = sk(i + 1, i * 1000)
        p.read_hash_order.append(h)
    return p, reads


def test_plan_v7_round_trip_and_layout(tmp_path):
    p, reads = sample_plan(3)
    f = tmp_path / "x.phrayaplan"
    IO.write_plan(f, p)
    data = f.read_bytes()
    assert data[:4] == b"PHR7"
    toc = IO.read_plan_toc(f)
    assert toc["num_chunks"] == 3 and toc["shared_frame_offset"] == 12
    # frames are back to back and the table of contents follows the last one
    ends = [toc["shared_frame_offset"] + toc["shared_frame_len"]] + [o + n for o, n in toc["chunk_frame_offsets"]]
    assert [o for o, _ in toc["chunk_frame_offsets"]] == ends[:-1]
    assert int.from_bytes(data[4:12], "little") == ends[-1]
    q = IO.read_plan(f)
    for name in ("use_case", "input_files", "timestamp", "kmer_index", "kmer_uniqueness", "task_list",
                 "hotspot_intervals", "reads_per_file", "total_read_count", "batch_num_chunks",
                 "batch_reads_per_chunk", "batch_output_paths", "alphabet", "read_sketches"):
        assert getattr(q, name) == getattr(p, name), name
    assert q.reference_space == p.reference_space
    assert q.read_byte_offsets == p.read_byte_offsets
    # chunk c holds reads [4c, 4c + 4) of the plan's order (chunk size ceil(10 / 3))
    w1 = IO.read_plan(f, worker=(1, 3))
    assert set(w1.read_sketches) == set(p.read_hash_order[4:8])
    assert w1.read_byte_offsets == [[400, 500, 600, 700]]
    # stored sketch lookup by content hash
    v, pos = q.stored_sketch(reads[2])
    assert v == [2000, 2007, 2014] and pos == [0, 3, 6]
    assert q.stored_sketch(b"NOTINPLAN") is None


def test_plan_without_read_order_puts_everything_in_chunk_zero(tmp_path):
    p, _ = sample_plan(2)
    p.read_hash_order = []
    f = tmp_path / "y"
    IO.write_plan(f, p)
    assert set(IO.read_plan(f, worker=(0, 2)).read_sketches) == set(p.read_sketches)
    assert IO.read_plan(f, worker=(1, 2)).read_sketches == {}


def test_plan_trailing_optional_fields(tmp_path):
    p, _ = sample_plan(1)
    p.insert_size_distribution = [350, 40, "FR", 1000]
    p.dense_kmer_index = {"chr": IO.Sketch([(1, 2)], 21, 5)}
    f = tmp_path / "z"
    IO.write_plan(f, p)
    q = IO.read_plan(f)
    assert q.insert_size_distribution == p.insert_size_distribution and q.dense_kmer_index == p.dense_kmer_index
    assert q.w11_membership == {} and q.sparse_mode is False


def test_bad_plan_files_are_refused(tmp_path):
    f = tmp_path / "bad"
    f.write_bytes(b"PHR6" + bytes(20))
    with pytest.raises(IO.FormatError):
        IO.read_plan(f)
    f.write_bytes(b"PHR7" + (1 << 40).to_bytes(8, "little"))
    with pytest.raises(IO.FormatError):
        IO.read_plan(f)


def test_coverage_track_quantization_and_runs():
    # quantize: 0-2 -> 0, 3-7 -> 5, 8-12 -> 10, capped at 255 (types.rs:650-656)
    runs, n = IO.coverage_track([0, 1, 2, 3, 7, 8, 12, 13, 1000, 1000])
    assert n == 10 and runs == [(0, 3), (5, 2), (10, 2), (15, 1), (255, 2)]
    assert IO.coverage_track([]) == ([], 0)
    assert IO.coverage_track([1, 1, 1]) == ([(0, 3)], 3)


def test_phraya_round_trip(tmp_path):
    obs = [IO.Observation(10, ord("A"), {ord("C"): 1, ord("A"): 3}, 0.97, "148M1X1M", 60, 1, [1, 1, 2], 40.0,
                          "s:read1", variant_type="snp", strand="-", coverage_window_variant_offset=1),
           IO.Observation(20, ord("."), {ord("G"): 1}, 0.5, "10M1D10M", 60, 1, [1], 40.0, "s:read2",
                          variant_type="insertion")]
    track = IO.coverage_track([0, 5, 5, 9])
    f = tmp_path / "s.phraya"
    IO.write_phraya(f, 4, "s", "2026", obs, track)
    h, o, t = IO.read_phraya(f)
    assert h == {"version": 1, "reference_length": 4, "sample_id": "s", "timestamp": "2026", "observation_count": 2}
    assert o == obs and t == track
