"""ctypes mirror of include/phraya_gpu.h (structs, enums and function prototypes).

Kept in one place so the product wrapper (phraya_b200.api) and any test harness bind
the same layouts. Field order and types must match the header exactly.
"""
import ctypes as C

PHR_OK = 0
PHR_INVALID_INPUT = 1
PHR_ALIGNMENT_FAILED = 2
PHR_ERR_OOM = 3
PHR_ERR_CUDA = 5
PHR_ERR_ARG = 6
PHR_ERR_CAPACITY = 7
PHR_ERR_STATE = 8

ENGINE_WFA_LINEAR = 0
ENGINE_WFA_AFFINE = 1
ENGINE_MYERS_FIT = 2
ENGINE_MYERS_GLOBAL = 3

ALPHABET_DNA = 0
ALPHABET_PROTEIN = 1

COVERAGE_QUANTIZED = 0
COVERAGE_DEPTH = 1

FAST = 0
BALANCED = 1
SENSITIVE = 2
GAP_LINEAR = 0
GAP_AFFINE = 1

OUT_PLACED = 0
OUT_NO_SEED = 1
OUT_BELOW_THRESHOLD = 2
OUT_FAST_CUTOFF = 3
OUT_NO_ALIGNMENT = 4

u8p = C.POINTER(C.c_uint8)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


class AffineCosts(C.Structure):
    _fields_ = [("mismatch", C.c_int32), ("gap_open", C.c_int32), ("gap_extend", C.c_int32)]


class PairBatch(C.Structure):
    _fields_ = [
        ("n_pairs", C.c_uint64),
        ("seq", C.c_void_p),
        ("seq_bytes", C.c_uint64),
        ("q_off", C.c_void_p),
        ("q_len", C.c_void_p),
        ("t_off", C.c_void_p),
        ("t_len", C.c_void_p),
        ("q_seed", C.c_void_p),
        ("t_seed", C.c_void_p),
    ]


class Alignment(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("edit_distance", C.c_uint32),
        ("query_start", C.c_uint32),
        ("query_end", C.c_uint32),
        ("target_start", C.c_uint32),
        ("target_end", C.c_uint32),
        ("cigar_off", C.c_uint64),
        ("cigar_len", C.c_uint32),
        ("affine_score", C.c_uint32),
    ]


class ResultArena(C.Structure):
    _fields_ = [
        ("aln", C.c_void_p),
        ("cigar", C.c_void_p),
        ("cigar_capacity", C.c_uint64),
        ("cigar_used", C.c_uint64),
    ]


class Config(C.Structure):
    _fields_ = [
        ("workspace_bytes", C.c_uint64),
        ("tune_file_enable", C.c_int32),
        ("tune_file", C.c_char_p),
    ]


class Sketch(C.Structure):
    _fields_ = [
        ("values", C.c_void_p),
        ("positions", C.c_void_p),
        ("n", C.c_uint64),
        ("k", C.c_int32),
        ("w", C.c_int32),
    ]


class IndexInfo(C.Structure):
    _fields_ = [
        ("n_minimizers", C.c_uint64),
        ("n_distinct", C.c_uint64),
        ("occurrence_cap", C.c_uint64),
        ("target_len", C.c_uint64),
        ("device_bytes", C.c_uint64),
    ]


class SeqBatch(C.Structure):
    _fields_ = [
        ("n", C.c_uint64),
        ("seq", C.c_void_p),
        ("seq_bytes", C.c_uint64),
        ("off", C.c_void_p),
        ("len", C.c_void_p),
    ]


class Seed(C.Structure):
    _fields_ = [("query_pos", C.c_uint32), ("target_pos", C.c_uint32), ("minimizer", C.c_uint64)]


class Chain(C.Structure):
    _fields_ = [
        ("score", C.c_int64),
        ("seed_off", C.c_uint32),
        ("n_seeds", C.c_uint32),
        ("target_start", C.c_uint32),
        ("_pad", C.c_uint32),
    ]


class ChainArena(C.Structure):
    _fields_ = [
        ("n_seeds_found", C.c_void_p),
        ("n_chains", C.c_void_p),
        ("chain_off", C.c_void_p),
        ("chains", C.c_void_p),
        ("chain_capacity", C.c_uint64),
        ("seeds", C.c_void_p),
        ("seed_capacity", C.c_uint64),
    ]


class AlignConfig(C.Structure):
    _fields_ = [("strategy", C.c_int32), ("gap_model", C.c_int32)]


class ReadBatch(C.Structure):
    _fields_ = [
        ("n_reads", C.c_uint64),
        ("seq", C.c_void_p),
        ("seq_bytes", C.c_uint64),
        ("off", C.c_void_p),
        ("len", C.c_void_p),
        ("has_stored", C.c_void_p),
        ("s_off", C.c_void_p),
        ("s_n", C.c_void_p),
        ("s_values", C.c_void_p),
        ("s_positions", C.c_void_p),
    ]


class ReadResult(C.Structure):
    _fields_ = [
        ("outcome", C.c_int32),
        ("has_result", C.c_uint8),
        ("reverse", C.c_uint8),
        ("_pad", C.c_uint16),
        ("n_aln", C.c_uint32),
        ("_pad2", C.c_uint32),
        ("aln_off", C.c_uint64),
    ]


class ReadResultArena(C.Structure):
    _fields_ = [
        ("reads", C.c_void_p),
        ("aln", C.c_void_p),
        ("aln_capacity", C.c_uint64),
        ("aln_used", C.c_uint64),
        ("cigar", C.c_void_p),
        ("cigar_capacity", C.c_uint64),
        ("cigar_used", C.c_uint64),
    ]


class AlignStats(C.Structure):
    _fields_ = [
        ("placed", C.c_uint64),
        ("no_seed", C.c_uint64),
        ("below_threshold", C.c_uint64),
        ("fast_cutoff", C.c_uint64),
        ("no_alignment", C.c_uint64),
    ]


class VariantConfig(C.Structure):
    _fields_ = [
        ("coverage_radius", C.c_uint32),
        ("_pad", C.c_uint32),
        ("hotspot_start", C.c_void_p),
        ("hotspot_end", C.c_void_p),
        ("n_hotspots", C.c_uint64),
    ]


class VariantArena(C.Structure):
    _fields_ = [
        ("read_variant_off", C.c_void_p),
        ("variants", C.c_void_p),
        ("variant_capacity", C.c_uint64),
        ("variant_used", C.c_uint64),
        ("coverage", C.c_void_p),
        ("coverage_capacity", C.c_uint64),
        ("coverage_used", C.c_uint64),
        ("alleles", C.c_void_p),
        ("allele_capacity", C.c_uint64),
        ("allele_used", C.c_uint64),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("align", AlignConfig),
        ("max_batch_reads", C.c_uint32),
        ("max_batch_bases", C.c_uint64),
        ("hbm_reserve_bytes", C.c_uint64),
        ("max_wait_us", C.c_uint32),
        ("n_streams", C.c_uint32),
        ("short_lane", C.c_int32),
        ("long_blocks_per_sm", C.c_uint32),
    ]


class ServerResult(C.Structure):
    _fields_ = [
        ("request_id", C.c_uint64),
        ("outcome", C.c_int32),
        ("has_result", C.c_uint8),
        ("reverse", C.c_uint8),
        ("_pad", C.c_uint16),
        ("n_aln", C.c_uint32),
        ("_pad2", C.c_uint32),
        ("latency_us", C.c_double),
    ]


class KernelTiming(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_uint64), ("total_ms", C.c_double)]


# Every exported symbol of libphraya_b200.so, with its ctypes prototype.
PROTOTYPES = {
    "phr_abi_version": (C.c_int32, []),
    "phr_status_string": (C.c_char_p, [C.c_int32]),
    "phr_ctx_create": (C.c_int32, [C.c_int32, C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "phr_ctx_destroy": (None, [C.c_void_p]),
    "phr_ctx_last_error": (C.c_char_p, [C.c_void_p]),
    "phr_ctx_kernel_launches": (C.c_uint64, [C.c_void_p]),
    "phr_ctx_set_timing": (C.c_int32, [C.c_void_p, C.c_int32]),
    "phr_ctx_set_tune": (C.c_int32, [C.c_void_p, C.c_char_p, C.c_int64]),
    "phr_ctx_get_tune": (C.c_int32, [C.c_void_p, C.c_char_p, C.POINTER(C.c_int64)]),
    "phr_ctx_get_timing": (C.c_uint32, [C.c_void_p, C.c_void_p, C.c_uint32]),
    "phr_ctx_reset_timing": (None, [C.c_void_p]),
    "phr_ctx_counter": (C.c_uint64, [C.c_void_p, C.c_char_p]),
    "phr_ctx_stream": (C.c_void_p, [C.c_void_p]),
    "phr_extend_batch": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(PairBatch), AffineCosts,
                                     C.POINTER(ResultArena)]),
    "phr_extend_batch_device": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(PairBatch), AffineCosts,
                                            C.POINTER(ResultArena)]),
    "phr_extend_percall": (C.c_int32, [C.c_void_p, C.c_int32, C.POINTER(PairBatch), AffineCosts,
                                       C.POINTER(ResultArena)]),
    "phr_index_create": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64, C.POINTER(Sketch), C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "phr_index_destroy": (None, [C.c_void_p]),
    "phr_index_get_info": (C.c_int32, [C.c_void_p, C.POINTER(IndexInfo)]),
    "phr_sketch_batch": (C.c_int32, [C.c_void_p, C.POINTER(SeqBatch), C.c_int32, C.c_int32, C.c_int32,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "phr_seed_chain_batch": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(Sketch), C.c_uint64,
                                         C.POINTER(ChainArena)]),
    "phr_align_reads": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(ReadBatch), C.POINTER(AlignConfig),
                                    C.POINTER(ReadResultArena), C.POINTER(AlignStats)]),
    "phr_align_reads_variants": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(ReadBatch),
                                             C.POINTER(AlignConfig), C.POINTER(ReadResultArena),
                                             C.POINTER(VariantConfig), C.POINTER(VariantArena),
                                             C.POINTER(AlignStats)]),
    "phr_index_repeat_regions": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                             C.POINTER(C.c_uint64)]),
    "phr_coverage_create": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "phr_coverage_add": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "phr_coverage_read": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint64]),
    "phr_coverage_destroy": (None, [C.c_void_p]),
    "phr_server_create": (C.c_int32, [C.c_void_p, C.c_void_p, C.POINTER(ServerConfig),
                                      C.POINTER(C.c_void_p)]),
    "phr_server_submit": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64)]),
    "phr_server_submit_many": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                           C.c_void_p]),
    "phr_server_poll": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p,
                                    C.c_uint64, C.c_uint32, C.POINTER(C.c_uint32)]),
    "phr_server_destroy": (C.c_int32, [C.c_void_p]),
    "phr_myers_extend_noalloc": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                             C.c_void_p, C.c_void_p]),
}


def bind(lib):
    """Attach restype/argtypes for every prototype to a loaded CDLL."""
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib
