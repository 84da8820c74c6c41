/*
 * phraya_gpu.h -- C ABI of the B200 (sm_100a) seed -> chain -> extend engine.
 *
 * Every entry point is a plain C function over caller-owned buffers: pointers, sizes
 * and POD structs only. Host-buffer entry points copy inputs to HBM, run the CUDA
 * kernels and copy results back; "_device" entry points take device pointers and keep
 * results resident. There is no CPU fallback: if the CUDA library cannot run, every
 * compute call returns PHR_ERR_CUDA.
 *
 * Conventions shared with phraya-align (the Rust crate this replaces):
 *   - CIGAR text uses the reference's letters: M (match), X (mismatch),
 *     D = query-extra base, I = target-extra base  (phraya-align/src/wfa_simd.rs:1101-1105).
 *   - Status codes map 1:1 onto WfaError (phraya-align/src/lib.rs:44-49):
 *     PHR_INVALID_INPUT == WfaError::InvalidInput, PHR_ALIGNMENT_FAILED ==
 *     WfaError::AlignmentFailed; the rest are engine errors with no Rust counterpart.
 *   - A phr_ctx is bound to one device and one stream; it is not thread-safe. Use one
 *     context per host thread (or wrap it in a mutex).
 */
#ifndef PHRAYA_GPU_H
#define PHRAYA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHR_ABI_VERSION 1

typedef enum {
    PHR_OK = 0,
    PHR_INVALID_INPUT = 1,     /* WfaError::InvalidInput (seed beyond sequence end)   */
    PHR_ALIGNMENT_FAILED = 2,  /* WfaError::AlignmentFailed (search exhausted)         */
    PHR_ERR_OOM = 3,           /* device allocation failed / not enough free HBM      */
    /* 4 is unused: no entry point waits on the device with a time limit (no kernel spins
     * on a flag; the persistent kernels take work from an atomic queue head). */
    PHR_ERR_CUDA = 5,          /* CUDA runtime error or no usable device               */
    PHR_ERR_ARG = 6,           /* bad argument: NULL pointer, size over a stated limit */
    PHR_ERR_CAPACITY = 7,      /* caller-supplied output arena too small               */
    PHR_ERR_STATE = 8          /* call out of order (e.g. server not started)          */
} phr_status;

/* Extension engines, one per phraya-align entry point. */
typedef enum {
    PHR_ENGINE_WFA_LINEAR = 0,   /* wfa_extend            phraya-align/src/lib.rs:74      */
    PHR_ENGINE_WFA_AFFINE = 1,   /* wfa_extend_affine     phraya-align/src/lib.rs:139-167 */
    PHR_ENGINE_MYERS_FIT = 2,    /* myers_extend          phraya-align/src/lib.rs:106-127 */
    PHR_ENGINE_MYERS_GLOBAL = 3  /* myers_edit_distance   phraya-align/src/lib.rs:94-96   */
} phr_engine;

/* AffineCosts (phraya-align/src/wfa_simd.rs:521-540); default {2,4,1}. */
typedef struct {
    int32_t mismatch;
    int32_t gap_open;
    int32_t gap_extend;
} phr_affine_costs;

/*
 * A batch of query/target pairs (structure of arrays over one byte arena).
 * Pair i aligns seq[q_off[i] .. q_off[i]+q_len[i]) [q_seed[i]..] against
 * seq[t_off[i] .. t_off[i]+t_len[i]) [t_seed[i]..]  -- the SeedAnchor of lib.rs:25-28.
 * q_seed / t_seed may be NULL (anchor (0,0)). Bytes are compared exactly as given
 * (case-sensitive, N == N), as the reference does.
 */
typedef struct {
    uint64_t n_pairs;
    const uint8_t* seq;
    uint64_t seq_bytes;
    const uint64_t* q_off;
    const uint32_t* q_len;
    const uint64_t* t_off;
    const uint32_t* t_len;
    const uint32_t* q_seed;
    const uint32_t* t_seed;
} phr_pair_batch;

/*
 * One Alignment (phraya-align/src/lib.rs:31-39). The CIGAR is
 * arena.cigar[cigar_off .. cigar_off + cigar_len), not NUL-terminated.
 * For PHR_ENGINE_MYERS_GLOBAL the coordinates are (0, |q|, 0, |t|).
 */
typedef struct {
    int32_t status;          /* phr_status of this pair (PHR_OK, PHR_INVALID_INPUT, ...) */
    uint32_t edit_distance;
    uint32_t query_start;
    uint32_t query_end;
    uint32_t target_start;
    uint32_t target_end;
    uint64_t cigar_off;
    uint32_t cigar_len;
    uint32_t affine_score;   /* WFA affine search score (0 for other engines) */
} phr_alignment;

/* Caller-owned result arena. cigar_used is written by the call. */
typedef struct {
    phr_alignment* aln;      /* n_pairs entries */
    char* cigar;
    uint64_t cigar_capacity;
    uint64_t cigar_used;
} phr_result_arena;

/* Upper bound of the CIGAR bytes one pair can produce: 2 * (|q| + |t|). */
#define PHR_CIGAR_BOUND(qlen, tlen) (2ull * ((uint64_t)(qlen) + (uint64_t)(tlen)))

/* ------------------------------------------------------------------------- */
/* Context                                                                    */
/* ------------------------------------------------------------------------- */

typedef struct phr_ctx phr_ctx;

typedef struct {
    uint64_t workspace_bytes;  /* cap on extension scratch; 0 = default (a fifth of the
                                  device memory, within 8 GiB .. 48 GiB)                */
    int32_t tune_file_enable;  /* 1 = read/write autotuner cache file                   */
    const char* tune_file;     /* NULL = "phraya_b200_tune.txt" in the working dir      */
} phr_config;

/* Reports the ABI version compiled into the library. */
int32_t phr_abi_version(void);
const char* phr_status_string(phr_status s);

phr_status phr_ctx_create(int32_t device, const phr_config* cfg, phr_ctx** out);
void phr_ctx_destroy(phr_ctx* ctx);
/* Launch parameters of the extension kernels. No counterpart in the reference (its
 * kernels are CPU code with nothing to tune); results never depend on them. Keys:
 *   "wfa_group_short", "wfa_group_long"  lanes per WFA pair below / from qlen+tlen
 *                                        wfa_long_min (power of two, 1..32)
 *   "wfa_affine_group_short"             lanes per gap-affine WFA pair below that edge
 *                                        (power of two, 1..32; "wfa_group_short" is then
 *                                        the linear engine's)
 *   "wfa_long_min"                       that length-bucket edge (default 1024)
 *   "myers_band_base"                    Myers stored-band half-width base (>= 0)
 *   "block_threads"                      threads per block of the warp-per-pair kernels
 *                                        (32..256, multiple of 32)
 *   "wfa_big_min"                        WFA pairs (linear and gap-affine) with qlen+tlen
 *                                        >= this run one per CTA (0 = never)
 *   "wfa_big_smem"                       shared memory of those kernels, bytes (16 KiB..200
 *                                        KiB; longer pairs are read from global memory)
 *   "wfa_affine_big_threads"             threads per CTA of the gap-affine one-CTA-per-pair
 *                                        kernel: 1024 (default, one CTA per SM), 512 or 256
 *   "max_blocks_per_sm"                  resident blocks per SM of the persistent extension
 *                                        kernels (1..4)
 *   "host_chunks"                        chunks a host batch of more than 128 MiB of sequence
 *                                        is copied and aligned in, overlapped (2..32, default 4)
 *   "myers_lane_ckpt"                    banded Myers (global 2-bit pairs): 1 = keep the band's
 *                                        state every 8th column and recompute 8 columns at a
 *                                        time for the traceback (default), 0 = store every
 *                                        column's records
 * With phr_config.tune_file_enable, phr_ctx_create applies "key value" lines of the tune
 * file (written by the autotuner); unknown keys and bad values there are ignored. */
phr_status phr_ctx_set_tune(phr_ctx* ctx, const char* key, int64_t value);
phr_status phr_ctx_get_tune(const phr_ctx* ctx, const char* key, int64_t* value);
/* Message describing the last non-PHR_OK status returned on this context. */
const char* phr_ctx_last_error(const phr_ctx* ctx);
/* Number of the library's own kernel launches issued on this context so far. */
uint64_t phr_ctx_kernel_launches(const phr_ctx* ctx);

/*
 * Instrumentation (no counterpart in the reference). With timing enabled, every
 * kernel the library launches is bracketed by CUDA events on the context's stream and
 * its device time accumulated per kernel name.
 */
typedef struct {
    char name[32];
    uint64_t launches;
    double total_ms;
} phr_kernel_timing;

phr_status phr_ctx_set_timing(phr_ctx* ctx, int32_t enable);
/* Copies up to `max` per-kernel records; returns how many kernels have records. */
uint32_t phr_ctx_get_timing(const phr_ctx* ctx, phr_kernel_timing* out, uint32_t max);
/* Clears the kernel times and the work counters below. */
void phr_ctx_reset_timing(phr_ctx* ctx);
/*
 * Work counters accumulated over the context's extension calls (no counterpart in the
 * reference): "myers_lane_block_columns" counts the 64-row block x column steps the
 * banded Myers kernel evaluated (64 DP cells each); "myers_lane_redo_pairs" the pairs
 * it handed to the every-block redo pass; "wfa_affine_cells" / "wfa_linear_cells" count
 * wavefront diagonals computed (the M band of each score) and "wfa_affine_lcp_words" /
 * "wfa_linear_lcp_words" the word compares of match extension. Unknown names read 0.
 * With the environment variable PHRAYA_EXTEND_TRACE=<file> set, each redo round of an
 * extension call appends one line to that file: engine, round, pairs, scratch budget
 * and the eight largest scratch needs as qlen:tlen:bytes; and each call appends one line
 * per pair of qlen + tlen >= 65536 with its final status and distance.
 */
uint64_t phr_ctx_counter(const phr_ctx* ctx, const char* name);
/* The cudaStream_t the context launches on (for callers that order their own work). */
void* phr_ctx_stream(const phr_ctx* ctx);

/* ------------------------------------------------------------------------- */
/* Pairs API -- replaces per-call wfa_extend / wfa_extend_affine /            */
/* myers_extend / myers_edit_distance (phraya-align/src/lib.rs:63-167).       */
/* ------------------------------------------------------------------------- */

/*
 * Aligns every pair of `batch` (host memory) with `engine` and writes one
 * phr_alignment per pair plus packed CIGAR text into `out` (host memory).
 * `costs` is read only by PHR_ENGINE_WFA_AFFINE. Pairs are independent; per-pair
 * failures are reported in phr_alignment.status, the call itself returns PHR_OK. A pair
 * whose extension needs more scratch than the context's workspace budget (a very
 * divergent pair of very long sequences: the reference's own full-width history would
 * need more memory still) reports PHR_ERR_OOM in its status and no alignment; align_read
 * skips such an anchor as it skips a failed extension (executor.rs:558). The context
 * counter "scratch_oom_pairs" counts them.
 */
phr_status phr_extend_batch(phr_ctx* ctx, phr_engine engine, const phr_pair_batch* batch,
                            phr_affine_costs costs, phr_result_arena* out);

/*
 * Same as phr_extend_batch, but every pointer in `batch` and `out` is DEVICE memory
 * (out->aln, out->cigar). Work is queued on the context's stream; the call returns
 * after the results are complete in device memory. Used by callers that keep data
 * resident in HBM.
 */
phr_status phr_extend_batch_device(phr_ctx* ctx, phr_engine engine, const phr_pair_batch* batch,
                                   phr_affine_costs costs, phr_result_arena* out);

/*
 * Per-call variant: one launch sequence per pair, the shape of the reference's
 * one-call-per-pair API. Exists as the baseline the batched path is measured against.
 */
phr_status phr_extend_percall(phr_ctx* ctx, phr_engine engine, const phr_pair_batch* batch,
                              phr_affine_costs costs, phr_result_arena* out);

/*
 * Allocation-free Myers fitting extension. No counterpart in the reference.
 *
 * For callers that must not allocate device memory: code running next to a caching
 * allocator that already holds the device's memory (where a cudaMalloc of its own can
 * fail or fragment that pool), and latency-critical loops that cannot afford the
 * implicit device-wide synchronisation cudaMalloc/cudaFree may bring. It computes
 * exactly what phr_extend_batch(PHR_ENGINE_MYERS_FIT) computes (myers_extend with the
 * anchor at (0, 0), phraya-align/src/lib.rs:106-127), but every byte of scratch it
 * needs lives in one fixed array inside the library (PHR_NOALLOC_SCRATCH_BYTES of
 * device memory, held by each GPU that loads the library until the process exits).
 *
 * All pointers are DEVICE memory owned by the caller: pair i aligns
 * seq[q_off[i] .. +q_len[i]) against seq[t_off[i] .. +t_len[i]); results go to
 * status[i], edit_distance[i], target_consumed[i], cigar_len[i] and the CIGAR text at
 * cigar + i * cigar_stride. `stream` is a cudaStream_t (NULL = default stream); every
 * call copies its error flags device -> host on `stream` and synchronises the stream, so
 * it returns after the work on it has finished.
 * Limits: |q| <= PHR_NOALLOC_MAX_QUERY, |t| <= PHR_NOALLOC_MAX_TARGET (the reference's
 * Myers regime: queries of at most 500 bases against windows of twice that); longer
 * pairs get status PHR_ERR_ARG and the call returns PHR_ERR_ARG. cigar_stride must be at
 * least PHR_NOALLOC_CIGAR_STRIDE.
 * The first call on a device looks up the scratch array's device address (once per
 * device, with that device current); make that first call before any stream capture.
 * Every call shares the one scratch array, so calls that overlap on the GPU (other
 * streams, other host threads) race: serialise them.
 */
#define PHR_NOALLOC_MAX_QUERY 512u
#define PHR_NOALLOC_MAX_TARGET 1024u
#define PHR_NOALLOC_CIGAR_STRIDE 3072u
#define PHR_NOALLOC_SCRATCH_BYTES (64ull << 20)
phr_status phr_myers_extend_noalloc(const uint8_t* seq, const uint64_t* q_off, const uint32_t* q_len,
                                    const uint64_t* t_off, const uint32_t* t_len, uint64_t n_pairs,
                                    int32_t* status, uint32_t* edit_distance, uint32_t* target_consumed,
                                    char* cigar, uint32_t cigar_stride, uint32_t* cigar_len, void* stream);

/* ------------------------------------------------------------------------- */
/* Sketches, target index, seeding and chaining                               */
/* ------------------------------------------------------------------------- */

typedef enum { PHR_ALPHABET_DNA = 0, PHR_ALPHABET_PROTEIN = 1 } phr_alphabet;

/* MinimizerSketch (phraya-core/src/types.rs:1803-1810) as two parallel arrays. */
typedef struct {
    const uint64_t* values;
    const uint32_t* positions;
    uint64_t n;
    int32_t k;
    int32_t w;
} phr_sketch;

typedef struct phr_index phr_index;

typedef struct {
    uint64_t n_minimizers;     /* target sketch length                          */
    uint64_t n_distinct;       /* distinct minimizer values                     */
    uint64_t occurrence_cap;   /* seed_occurrence_cap(index, 256)               */
    uint64_t target_len;
    uint64_t device_bytes;     /* HBM held by the index                         */
} phr_index_info;

/*
 * TargetContext::build (phraya-align/src/executor.rs:431-449): uploads the target
 * bytes, builds the minimizer index (build_minimizer_index, seeding.rs:31-37) and the
 * occurrence cap (seed_occurrence_cap(index, 256), seeding.rs:94-102) on the device, and
 * finds the target's tandem-repeat regions (detect_tandem_repeats, phraya-core/src/
 * lib.rs:79-135). `sketch` may be NULL: the target is then sketched with the library's
 * sketcher at the alphabet's default k/w (DNA 21/11 canonical, protein 6/5 plain).
 * Sketches of up to 2^31 - 16 minimizers.
 */
phr_status phr_index_create(phr_ctx* ctx, const uint8_t* target, uint64_t target_len,
                            const phr_sketch* sketch, phr_alphabet alphabet, phr_index** out);
void phr_index_destroy(phr_index* idx);
phr_status phr_index_get_info(const phr_index* idx, phr_index_info* info);

/*
 * The library's minimizer sketcher: canonical (DNA) or plain (protein) (k, w)
 * minimizers of every sequence in the batch, k in 1..32. Restates simd-minimizers
 * 2.3.1 as phraya-core/src/types.rs:1848-1869 calls it (over packed-seq's AsciiSeq):
 * characters as 2-bit codes (b >> 1) & 3; 32-bit ntHash order hashes (canonical: the
 * smaller of the forward and reverse-complement hashes); per window of w k-mers the
 * leftmost minimum, or, for canonical minimizers, the rightmost one in windows whose
 * w + k - 1 characters hold no more T/G than A/C; each selected k-mer once per run of
 * windows; value = the 2-bit k-mer, first character lowest (DNA: the smaller of the
 * k-mer and its reverse complement). The crate itself is not available to check
 * against, so sketches are not guaranteed identical to its.
 * Sequence i is seq[off[i] .. off[i]+len[i]). Output: sequence i's minimizers at
 * values/positions[out_off[i] .. out_off[i] + out_n[i]); capacity per sequence is
 * max(len[i] - k + 1, 0) entries, so out_off must leave that much room.
 */
typedef struct {
    uint64_t n;
    const uint8_t* seq;
    uint64_t seq_bytes;
    const uint64_t* off;
    const uint32_t* len;
} phr_seq_batch;

phr_status phr_sketch_batch(phr_ctx* ctx, const phr_seq_batch* seqs, int32_t k, int32_t w,
                            phr_alphabet alphabet, const uint64_t* out_off, uint64_t* values,
                            uint32_t* positions, uint32_t* out_n);

/* Chain (phraya-align/src/chaining.rs:24-35): seeds and score. */
typedef struct {
    uint32_t query_pos;
    uint32_t target_pos;
    uint64_t minimizer;
} phr_seed;

typedef struct {
    int64_t score;
    uint32_t seed_off;         /* into phr_chain_arena.seeds */
    uint32_t n_seeds;
    uint32_t target_start;     /* Chain::target_start()      */
    uint32_t _pad;
} phr_chain;

typedef struct {
    /* per query: chains[chain_off[i] .. chain_off[i] + n_chains[i]) */
    uint32_t* n_seeds_found;   /* raw seed count (find_seeds_indexed_capped length) */
    uint32_t* n_chains;
    uint64_t* chain_off;       /* written by the call */
    phr_chain* chains;
    uint64_t chain_capacity;
    phr_seed* seeds;
    uint64_t seed_capacity;
} phr_chain_arena;

/*
 * seed_and_chain (phraya-align/src/executor.rs:511-519) for every query sketch:
 * find_seeds_indexed_capped (seeding.rs:58-80) against the index with its occurrence
 * cap, then chain_seeds with ChainParams::default() (chaining.rs:134-226).
 * sketches[i] are host arrays.
 */
phr_status phr_seed_chain_batch(phr_ctx* ctx, const phr_index* idx, const phr_sketch* sketches,
                                uint64_t n_queries, phr_chain_arena* out);

/* ------------------------------------------------------------------------- */
/* align_read -- the whole per-read pipeline up to `scored`                   */
/* (phraya-align/src/executor.rs:573-733, 777-787)                            */
/* ------------------------------------------------------------------------- */

typedef enum { PHR_FAST = 0, PHR_BALANCED = 1, PHR_SENSITIVE = 2 } phr_strategy;
typedef enum { PHR_GAP_LINEAR = 0, PHR_GAP_AFFINE = 1 } phr_gap_model;

/* AlignConfig (executor.rs:107-166) minus the coverage radius, which only feeds
 * host-side variant extraction. */
typedef struct {
    phr_strategy strategy;
    phr_gap_model gap_model;   /* consulted only for PHR_SENSITIVE */
} phr_align_config;

/*
 * Reads: seq[off[i] .. off[i]+len[i]). Optional stored forward sketches
 * (plan.get_read_sketch, executor.rs:615-624): when has_stored[i] != 0, read i uses
 * sketch values/positions[s_off[i] .. s_off[i]+s_n[i]) as its forward sketch
 * (an empty stored sketch with no seeds means NoSeed, executor.rs:671-674).
 * All four stored-sketch pointers may be NULL.
 */
typedef struct {
    uint64_t n_reads;
    const uint8_t* seq;
    uint64_t seq_bytes;
    const uint64_t* off;
    const uint32_t* len;
    const uint8_t* has_stored;
    const uint64_t* s_off;
    const uint32_t* s_n;
    const uint64_t* s_values;
    const uint32_t* s_positions;
} phr_read_batch;

/* AlignStats outcome buckets (executor.rs:269-322). */
typedef enum {
    PHR_OUT_PLACED = 0,
    PHR_OUT_NO_SEED = 1,
    PHR_OUT_BELOW_THRESHOLD = 2,
    PHR_OUT_FAST_CUTOFF = 3,
    PHR_OUT_NO_ALIGNMENT = 4
} phr_outcome;

/*
 * Per read: the winning orientation's ScoredAlignments (primary first, then the
 * alternatives with score ratio >= 0.95, lib.rs:170-199) as alignments
 * aln[aln_off .. aln_off + n_aln); `reverse` = 1 when the reverse complement won
 * (0 whenever has_result = 0).
 * has_result = 0 when align_read would return None (NoAlignment, FastCutoff, stored
 * empty sketch); `outcome` is always set. query_positions of the reference
 * (executor.rs:777-781) are (aln.target_start, 1 - aln.edit_distance / max(|q|,1)).
 */
typedef struct {
    int32_t outcome;
    uint8_t has_result;
    uint8_t reverse;
    uint16_t _pad;
    uint32_t n_aln;
    uint32_t _pad2;
    uint64_t aln_off;
} phr_read_result;

typedef struct {
    phr_read_result* reads;    /* n_reads entries */
    phr_alignment* aln;
    uint64_t aln_capacity;
    uint64_t aln_used;
    char* cigar;
    uint64_t cigar_capacity;
    uint64_t cigar_used;
} phr_read_result_arena;

typedef struct {
    uint64_t placed;
    uint64_t no_seed;
    uint64_t below_threshold;
    uint64_t fast_cutoff;
    uint64_t no_alignment;
} phr_align_stats;

/*
 * align_read for every read of the batch against `idx`, bit-exact with
 * phraya-align's executor. `stats` may be NULL; when given, outcomes are ADDED to it.
 */
phr_status phr_align_reads(phr_ctx* ctx, const phr_index* idx, const phr_read_batch* reads,
                           const phr_align_config* cfg, phr_read_result_arena* out,
                           phr_align_stats* stats);

/* ------------------------------------------------------------------------- */
/* Variant observations and coverage of the aligned reads                    */
/* (phraya-align/src/executor.rs:735-775, 814-1096)                           */
/* ------------------------------------------------------------------------- */

/*
 * One VariantObservation (phraya-core/src/types.rs:217-283) as extract_variants_from_cigar
 * (executor.rs:814-1046) builds it from a read's primary alignment. The per-read fields
 * the device does not know -- mapq, avg_base_quality, provenance, the CIGAR string
 * (the read's primary CIGAR) and mate information -- are the host's, shared by every
 * variant of read `read`.
 */
typedef struct {
    uint32_t position;               /* 0-based reference position                     */
    uint8_t ref_base;                /* '.' for an insertion                           */
    uint8_t variant_type;            /* VariantType: 0 SNP, 1 insertion, 2 deletion    */
    uint8_t in_tandem_repeat;        /* is_in_repeat_region (executor.rs:806-809)       */
    uint8_t strand;                  /* 0 forward, 1 reverse complement                */
    uint32_t read;                   /* index of the read in its batch                 */
    uint32_t edit_distance;          /* the primary alignment's                        */
    double confidence;               /* kmer_uniqueness * (1 - ed / max(|q|, 1))        */
    double kmer_uniqueness;          /* 0 inside a hotspot interval (is_in_hotspot), 1  */
    uint64_t coverage_off;           /* local_coverage = coverage[off .. off + len)     */
    uint32_t coverage_len;
    uint32_t coverage_variant_offset;/* index of `position` within local_coverage       */
    uint64_t allele_off;             /* all_alleles = alleles[off .. off + n), ascending */
    uint32_t n_alleles;
    uint32_t _pad;
} phr_variant;

typedef struct {
    uint8_t base;                    /* allele byte ('.' = deleted)                    */
    uint8_t _pad[3];
    uint32_t count;
} phr_allele;

typedef struct {
    uint32_t coverage_radius;        /* 0: the strategy's (AlignConfig, executor.rs:124-128:
                                        Fast 150, Balanced 50, Sensitive 25)             */
    uint32_t _pad;
    const uint32_t* hotspot_start;   /* plan.hotspot_intervals: sorted, non-overlapping */
    const uint32_t* hotspot_end;     /* [start, end) intervals, host arrays; may be NULL */
    uint64_t n_hotspots;
} phr_variant_config;

typedef struct {
    uint64_t* read_variant_off;      /* n_reads + 1 entries: read i's variants are
                                        variants[off[i] .. off[i + 1])                 */
    phr_variant* variants;
    uint64_t variant_capacity;
    uint64_t variant_used;
    uint32_t* coverage;
    uint64_t coverage_capacity;
    uint64_t coverage_used;
    phr_allele* alleles;
    uint64_t allele_capacity;
    uint64_t allele_used;
} phr_variant_arena;

/*
 * phr_align_reads plus, for every read with a result, the variant observations of its
 * primary alignment on the device: local coverage is the read's raw windowed coverage
 * (compute_windowed_coverage, executor.rs:1071-1090: one window per alignment, primary
 * then alternatives, count 1 over [target_start, target_end)), in_tandem_repeat comes
 * from the index's tandem-repeat regions (detect_tandem_repeats with
 * min_repeat_count 3, phraya-core/src/lib.rs:79-135). The coverage track the reference
 * stores per read is each alignment's span with quantize_coverage(1) = 0
 * (executor.rs:1092-1096), i.e. derived from the alignments alone.
 * `vcfg` may be NULL (the strategy's radius, no hotspots). If the variant arena is too
 * small the call returns PHR_ERR_CAPACITY with variant_used / coverage_used /
 * allele_used set to the sizes needed (the read results in `out` are complete); call
 * again with a larger arena.
 */
phr_status phr_align_reads_variants(phr_ctx* ctx, const phr_index* idx, const phr_read_batch* reads,
                                    const phr_align_config* cfg, phr_read_result_arena* out,
                                    const phr_variant_config* vcfg, phr_variant_arena* vout,
                                    phr_align_stats* stats);

/* The index's tandem-repeat regions (TargetContext::build, executor.rs:440): region r
 * covers [start[r], end[r]] (end inclusive, RepeatRegion, phraya-core/src/lib.rs:10-18).
 * Writes min(n, cap) regions and the total count in *n. */
phr_status phr_index_repeat_regions(const phr_index* idx, uint32_t* start, uint32_t* end, uint64_t cap,
                                    uint64_t* n);

/*
 * Genome coverage track, resident on the device, merged batch by batch as the CLI's
 * merge_result does (phraya-cli/src/main.rs:556-572): every alignment of a read with a
 * result contributes its window [min(target_start, len), min(target_end, len)) with
 * per-position count 1, quantized per window by quantize_coverage
 * (executor.rs:1092-1096, ((c + 2) / 5) * 5) before it is added.
 * PHR_COVERAGE_QUANTIZED reproduces that track exactly (quantize(1) = 0, so it stays
 * all zero, as the reference's does); PHR_COVERAGE_DEPTH adds the raw count instead
 * (read depth). Tracks are target_len uint32 entries.
 */
typedef struct phr_coverage phr_coverage;
typedef enum { PHR_COVERAGE_QUANTIZED = 0, PHR_COVERAGE_DEPTH = 1 } phr_coverage_mode;

phr_status phr_coverage_create(phr_ctx* ctx, const phr_index* idx, phr_coverage_mode mode, phr_coverage** out);
/* Adds the windows of aln[0 .. n_aln) (host array; e.g. a phr_read_result_arena's
 * aln[0 .. aln_used), which holds only alignments of reads with a result). */
phr_status phr_coverage_add(phr_coverage* cov, const phr_alignment* aln, uint64_t n_aln);
/* Copies the track out (len must equal the index's target_len). */
phr_status phr_coverage_read(phr_coverage* cov, uint32_t* track, uint64_t len);
void phr_coverage_destroy(phr_coverage* cov);

/* ------------------------------------------------------------------------- */
/* Serving loop: device-resident index, admission by free HBM, continuous    */
/* batching. No counterpart in the reference (its CLI is batch-only).         */
/* ------------------------------------------------------------------------- */

typedef struct phr_server phr_server;

typedef struct {
    phr_align_config align;
    uint32_t max_batch_reads;      /* reads per device batch (0 = 4096)            */
    uint64_t max_batch_bases;      /* bases per device batch (0 = 16 Mbp)          */
    uint64_t hbm_reserve_bytes;    /* free HBM kept back when admitting (0 = 2 GiB) */
    uint32_t max_wait_us;          /* batch-forming window after first arrival     */
    uint32_t n_streams;            /* concurrent batches in flight (0 = 2)         */
    int32_t short_lane;            /* worker 0 takes only reads <= 500 bases, on a
                                      high-priority stream, and the other workers
                                      only longer reads: 0 = on when n_streams >= 2,
                                      1 = on, -1 = off                               */
    uint32_t long_blocks_per_sm;   /* resident blocks per SM of the extension kernels
                                      of the other workers while a short lane runs
                                      (0 = 2; the short lane keeps the rest)        */
} phr_server_config;

typedef struct {
    uint64_t request_id;
    int32_t outcome;
    uint8_t has_result;
    uint8_t reverse;
    uint16_t _pad;
    uint32_t n_aln;
    uint32_t _pad2;
    double latency_us;             /* submit -> result ready */
} phr_server_result;

/* While a server exists, the device's default CUDA memory pool keeps memory freed to it
 * (release threshold raised to the maximum), so the workers' arenas can grow again
 * without the driver mapping memory while other workers' kernels run. Servers on one
 * device share that setting: the threshold in force before the first of them was
 * created is restored when the last of them is destroyed. Create and destroy leave the
 * caller's current device unchanged. */
phr_status phr_server_create(phr_ctx* ctx, const phr_index* idx, const phr_server_config* cfg,
                             phr_server** out);
/* Enqueues one read (bytes copied); returns its request id in *request_id. */
phr_status phr_server_submit(phr_server* srv, const uint8_t* read, uint32_t len,
                             uint64_t* request_id);
/* Enqueues n reads (read i = seq[off[i] .. off[i] + len[i]), bytes copied) with one
 * lock round trip; their request ids are written to ids[0..n). Each read's latency
 * starts at this call. */
phr_status phr_server_submit_many(phr_server* srv, const uint8_t* seq, const uint64_t* off,
                                  const uint32_t* len, uint64_t n, uint64_t* ids);
/*
 * Copies up to `max_results` finished requests into `res` (and their alignments and
 * CIGARs, packed, into the given arrays), returns how many in *n_out.
 * `wait_us` > 0 blocks up to that long for at least one result.
 */
phr_status phr_server_poll(phr_server* srv, phr_server_result* res, uint32_t max_results,
                           phr_alignment* aln, uint64_t aln_capacity, char* cigar,
                           uint64_t cigar_capacity, uint32_t wait_us, uint32_t* n_out);
/* Stops after draining every submitted request. */
phr_status phr_server_destroy(phr_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* PHRAYA_GPU_H */
