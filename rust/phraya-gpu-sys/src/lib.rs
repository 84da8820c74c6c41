//! Raw bindings of `include/phraya_gpu.h`, the C ABI of the phraya B200 (sm_100a)
//! seed -> chain -> extend engine, plus a small safe layer (`gpu`) with the shapes of
//! phraya-align's extension API (phraya-align/src/lib.rs:63-199) and of the CLI's
//! per-batch `align_read` loop (phraya-cli/src/main.rs:583-590).
//!
//! Every `#[repr(C)]` struct below is a field-for-field copy of the header's; the
//! repository's test-suite checks each size and field offset against the header with a
//! C++ compiler. C enums are passed as `i32`.
#![allow(non_camel_case_types)]

use std::os::raw::{c_char, c_void};

pub const PHR_ABI_VERSION: i32 = 1;

// phr_status
pub const PHR_OK: i32 = 0;
pub const PHR_INVALID_INPUT: i32 = 1;
pub const PHR_ALIGNMENT_FAILED: i32 = 2;
pub const PHR_ERR_OOM: i32 = 3;
pub const PHR_ERR_CUDA: i32 = 5;
pub const PHR_ERR_ARG: i32 = 6;
pub const PHR_ERR_CAPACITY: i32 = 7;
pub const PHR_ERR_STATE: i32 = 8;

// phr_engine
pub const PHR_ENGINE_WFA_LINEAR: i32 = 0;
pub const PHR_ENGINE_WFA_AFFINE: i32 = 1;
pub const PHR_ENGINE_MYERS_FIT: i32 = 2;
pub const PHR_ENGINE_MYERS_GLOBAL: i32 = 3;

// phr_alphabet, phr_strategy, phr_gap_model, phr_outcome, phr_coverage_mode
pub const PHR_ALPHABET_DNA: i32 = 0;
pub const PHR_ALPHABET_PROTEIN: i32 = 1;
pub const PHR_FAST: i32 = 0;
pub const PHR_BALANCED: i32 = 1;
pub const PHR_SENSITIVE: i32 = 2;
pub const PHR_GAP_LINEAR: i32 = 0;
pub const PHR_GAP_AFFINE: i32 = 1;
pub const PHR_OUT_PLACED: i32 = 0;
pub const PHR_OUT_NO_SEED: i32 = 1;
pub const PHR_OUT_BELOW_THRESHOLD: i32 = 2;
pub const PHR_OUT_FAST_CUTOFF: i32 = 3;
pub const PHR_OUT_NO_ALIGNMENT: i32 = 4;
pub const PHR_COVERAGE_QUANTIZED: i32 = 0;
pub const PHR_COVERAGE_DEPTH: i32 = 1;

pub const PHR_NOALLOC_MAX_QUERY: u32 = 512;
pub const PHR_NOALLOC_MAX_TARGET: u32 = 1024;
pub const PHR_NOALLOC_CIGAR_STRIDE: u32 = 3072;
pub const PHR_NOALLOC_SCRATCH_BYTES: u64 = 64 << 20;

/// Upper bound of the CIGAR bytes one pair can produce (PHR_CIGAR_BOUND).
pub const fn phr_cigar_bound(qlen: u64, tlen: u64) -> u64 {
    2 * (qlen + tlen)
}

#[repr(C)]
pub struct phr_ctx {
    _p: [u8; 0],
}
#[repr(C)]
pub struct phr_index {
    _p: [u8; 0],
}
#[repr(C)]
pub struct phr_coverage {
    _p: [u8; 0],
}
#[repr(C)]
pub struct phr_server {
    _p: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct phr_affine_costs {
    pub mismatch: i32,
    pub gap_open: i32,
    pub gap_extend: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_pair_batch {
    pub n_pairs: u64,
    pub seq: *const u8,
    pub seq_bytes: u64,
    pub q_off: *const u64,
    pub q_len: *const u32,
    pub t_off: *const u64,
    pub t_len: *const u32,
    pub q_seed: *const u32,
    pub t_seed: *const u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_alignment {
    pub status: i32,
    pub edit_distance: u32,
    pub query_start: u32,
    pub query_end: u32,
    pub target_start: u32,
    pub target_end: u32,
    pub cigar_off: u64,
    pub cigar_len: u32,
    pub affine_score: u32,
}

#[repr(C)]
pub struct phr_result_arena {
    pub aln: *mut phr_alignment,
    pub cigar: *mut c_char,
    pub cigar_capacity: u64,
    pub cigar_used: u64,
}

#[repr(C)]
pub struct phr_config {
    pub workspace_bytes: u64,
    pub tune_file_enable: i32,
    pub tune_file: *const c_char,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_kernel_timing {
    pub name: [c_char; 32],
    pub launches: u64,
    pub total_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_sketch {
    pub values: *const u64,
    pub positions: *const u32,
    pub n: u64,
    pub k: i32,
    pub w: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_index_info {
    pub n_minimizers: u64,
    pub n_distinct: u64,
    pub occurrence_cap: u64,
    pub target_len: u64,
    pub device_bytes: u64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_seq_batch {
    pub n: u64,
    pub seq: *const u8,
    pub seq_bytes: u64,
    pub off: *const u64,
    pub len: *const u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_seed {
    pub query_pos: u32,
    pub target_pos: u32,
    pub minimizer: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_chain {
    pub score: i64,
    pub seed_off: u32,
    pub n_seeds: u32,
    pub target_start: u32,
    pub _pad: u32,
}

#[repr(C)]
pub struct phr_chain_arena {
    pub n_seeds_found: *mut u32,
    pub n_chains: *mut u32,
    pub chain_off: *mut u64,
    pub chains: *mut phr_chain,
    pub chain_capacity: u64,
    pub seeds: *mut phr_seed,
    pub seed_capacity: u64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_align_config {
    pub strategy: i32,
    pub gap_model: i32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_read_batch {
    pub n_reads: u64,
    pub seq: *const u8,
    pub seq_bytes: u64,
    pub off: *const u64,
    pub len: *const u32,
    pub has_stored: *const u8,
    pub s_off: *const u64,
    pub s_n: *const u32,
    pub s_values: *const u64,
    pub s_positions: *const u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_read_result {
    pub outcome: i32,
    pub has_result: u8,
    pub reverse: u8,
    pub _pad: u16,
    pub n_aln: u32,
    pub _pad2: u32,
    pub aln_off: u64,
}

#[repr(C)]
pub struct phr_read_result_arena {
    pub reads: *mut phr_read_result,
    pub aln: *mut phr_alignment,
    pub aln_capacity: u64,
    pub aln_used: u64,
    pub cigar: *mut c_char,
    pub cigar_capacity: u64,
    pub cigar_used: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_align_stats {
    pub placed: u64,
    pub no_seed: u64,
    pub below_threshold: u64,
    pub fast_cutoff: u64,
    pub no_alignment: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_variant {
    pub position: u32,
    pub ref_base: u8,
    pub variant_type: u8,
    pub in_tandem_repeat: u8,
    pub strand: u8,
    pub read: u32,
    pub edit_distance: u32,
    pub confidence: f64,
    pub kmer_uniqueness: f64,
    pub coverage_off: u64,
    pub coverage_len: u32,
    pub coverage_variant_offset: u32,
    pub allele_off: u64,
    pub n_alleles: u32,
    pub _pad: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_allele {
    pub base: u8,
    pub _pad: [u8; 3],
    pub count: u32,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_variant_config {
    pub coverage_radius: u32,
    pub _pad: u32,
    pub hotspot_start: *const u32,
    pub hotspot_end: *const u32,
    pub n_hotspots: u64,
}

#[repr(C)]
pub struct phr_variant_arena {
    pub read_variant_off: *mut u64,
    pub variants: *mut phr_variant,
    pub variant_capacity: u64,
    pub variant_used: u64,
    pub coverage: *mut u32,
    pub coverage_capacity: u64,
    pub coverage_used: u64,
    pub alleles: *mut phr_allele,
    pub allele_capacity: u64,
    pub allele_used: u64,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct phr_server_config {
    pub align: phr_align_config,
    pub max_batch_reads: u32,
    pub max_batch_bases: u64,
    pub hbm_reserve_bytes: u64,
    pub max_wait_us: u32,
    pub n_streams: u32,
    pub short_lane: i32,
    pub long_blocks_per_sm: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct phr_server_result {
    pub request_id: u64,
    pub outcome: i32,
    pub has_result: u8,
    pub reverse: u8,
    pub _pad: u16,
    pub n_aln: u32,
    pub _pad2: u32,
    pub latency_us: f64,
}

extern "C" {
    pub fn phr_abi_version() -> i32;
    pub fn phr_status_string(s: i32) -> *const c_char;

    pub fn phr_ctx_create(device: i32, cfg: *const phr_config, out: *mut *mut phr_ctx) -> i32;
    pub fn phr_ctx_destroy(ctx: *mut phr_ctx);
    pub fn phr_ctx_set_tune(ctx: *mut phr_ctx, key: *const c_char, value: i64) -> i32;
    pub fn phr_ctx_get_tune(ctx: *const phr_ctx, key: *const c_char, value: *mut i64) -> i32;
    pub fn phr_ctx_last_error(ctx: *const phr_ctx) -> *const c_char;
    pub fn phr_ctx_kernel_launches(ctx: *const phr_ctx) -> u64;
    pub fn phr_ctx_set_timing(ctx: *mut phr_ctx, enable: i32) -> i32;
    pub fn phr_ctx_get_timing(ctx: *const phr_ctx, out: *mut phr_kernel_timing, max: u32) -> u32;
    pub fn phr_ctx_reset_timing(ctx: *mut phr_ctx);
    pub fn phr_ctx_counter(ctx: *const phr_ctx, name: *const c_char) -> u64;
    pub fn phr_ctx_stream(ctx: *const phr_ctx) -> *mut c_void;

    pub fn phr_extend_batch(ctx: *mut phr_ctx, engine: i32, batch: *const phr_pair_batch,
                            costs: phr_affine_costs, out: *mut phr_result_arena) -> i32;
    pub fn phr_extend_batch_device(ctx: *mut phr_ctx, engine: i32, batch: *const phr_pair_batch,
                                   costs: phr_affine_costs, out: *mut phr_result_arena) -> i32;
    pub fn phr_extend_percall(ctx: *mut phr_ctx, engine: i32, batch: *const phr_pair_batch,
                              costs: phr_affine_costs, out: *mut phr_result_arena) -> i32;
    pub fn phr_myers_extend_noalloc(seq: *const u8, q_off: *const u64, q_len: *const u32, t_off: *const u64,
                                    t_len: *const u32, n_pairs: u64, status: *mut i32, edit_distance: *mut u32,
                                    target_consumed: *mut u32, cigar: *mut c_char, cigar_stride: u32,
                                    cigar_len: *mut u32, stream: *mut c_void) -> i32;

    pub fn phr_index_create(ctx: *mut phr_ctx, target: *const u8, target_len: u64, sketch: *const phr_sketch,
                            alphabet: i32, out: *mut *mut phr_index) -> i32;
    pub fn phr_index_destroy(idx: *mut phr_index);
    pub fn phr_index_get_info(idx: *const phr_index, info: *mut phr_index_info) -> i32;
    pub fn phr_sketch_batch(ctx: *mut phr_ctx, seqs: *const phr_seq_batch, k: i32, w: i32, alphabet: i32,
                            out_off: *const u64, values: *mut u64, positions: *mut u32, out_n: *mut u32) -> i32;
    pub fn phr_seed_chain_batch(ctx: *mut phr_ctx, idx: *const phr_index, sketches: *const phr_sketch,
                                n_queries: u64, out: *mut phr_chain_arena) -> i32;

    pub fn phr_align_reads(ctx: *mut phr_ctx, idx: *const phr_index, reads: *const phr_read_batch,
                           cfg: *const phr_align_config, out: *mut phr_read_result_arena,
                           stats: *mut phr_align_stats) -> i32;
    pub fn phr_align_reads_variants(ctx: *mut phr_ctx, idx: *const phr_index, reads: *const phr_read_batch,
                                    cfg: *const phr_align_config, out: *mut phr_read_result_arena,
                                    vcfg: *const phr_variant_config, vout: *mut phr_variant_arena,
                                    stats: *mut phr_align_stats) -> i32;
    pub fn phr_index_repeat_regions(idx: *const phr_index, start: *mut u32, end: *mut u32, cap: u64,
                                    n: *mut u64) -> i32;

    pub fn phr_coverage_create(ctx: *mut phr_ctx, idx: *const phr_index, mode: i32,
                               out: *mut *mut phr_coverage) -> i32;
    pub fn phr_coverage_add(cov: *mut phr_coverage, aln: *const phr_alignment, n_aln: u64) -> i32;
    pub fn phr_coverage_read(cov: *mut phr_coverage, track: *mut u32, len: u64) -> i32;
    pub fn phr_coverage_destroy(cov: *mut phr_coverage);

    pub fn phr_server_create(ctx: *mut phr_ctx, idx: *const phr_index, cfg: *const phr_server_config,
                             out: *mut *mut phr_server) -> i32;
    pub fn phr_server_submit(srv: *mut phr_server, read: *const u8, len: u32, request_id: *mut u64) -> i32;
    pub fn phr_server_submit_many(srv: *mut phr_server, seq: *const u8, off: *const u64, len: *const u32, n: u64,
                                  ids: *mut u64) -> i32;
    pub fn phr_server_poll(srv: *mut phr_server, res: *mut phr_server_result, max_results: u32,
                           aln: *mut phr_alignment, aln_capacity: u64, cigar: *mut c_char, cigar_capacity: u64,
                           wait_us: u32, n_out: *mut u32) -> i32;
    pub fn phr_server_destroy(srv: *mut phr_server) -> i32;
}

/// Safe shapes of phraya-align's API over the raw bindings.
pub mod gpu {
    use super::*;

    /// `WfaError` (phraya-align/src/lib.rs:44-49) plus the engine's own failures.
    #[derive(Debug, Clone, PartialEq, Eq)]
    pub enum Error {
        InvalidInput,
        AlignmentFailed,
        Engine(i32, String),
    }

    /// `SeedAnchor` (phraya-align/src/lib.rs:25-28).
    #[derive(Debug, Clone, Copy, Default)]
    pub struct SeedAnchor {
        pub query_pos: usize,
        pub target_pos: usize,
    }

    /// `Alignment` (phraya-align/src/lib.rs:31-39).
    #[derive(Debug, Clone, PartialEq, Eq)]
    pub struct Alignment {
        pub cigar: String,
        pub edit_distance: usize,
        pub query_start: usize,
        pub query_end: usize,
        pub target_start: usize,
        pub target_end: usize,
    }

    /// One device context (one device, one stream; not thread-safe: one per worker).
    pub struct Context {
        raw: *mut phr_ctx,
    }

    unsafe impl Send for Context {}

    fn status(ctx: *const phr_ctx, st: i32) -> Result<(), Error> {
        if st == PHR_OK {
            return Ok(());
        }
        let msg = unsafe {
            let p = if ctx.is_null() { phr_status_string(st) } else { phr_ctx_last_error(ctx) };
            if p.is_null() { String::new() } else { std::ffi::CStr::from_ptr(p).to_string_lossy().into_owned() }
        };
        Err(Error::Engine(st, msg))
    }

    impl Context {
        pub fn new(device: i32) -> Result<Self, Error> {
            let mut raw = std::ptr::null_mut();
            status(std::ptr::null(), unsafe { phr_ctx_create(device, std::ptr::null(), &mut raw) })?;
            Ok(Context { raw })
        }

        /// One batched call for every pair: the per-pair results of `wfa_extend`,
        /// `wfa_extend_affine`, `myers_extend` or `myers_edit_distance` (by `engine`).
        pub fn extend_batch(&mut self, engine: i32, pairs: &[(&[u8], &[u8], SeedAnchor)],
                            costs: phr_affine_costs) -> Result<Vec<Result<Alignment, Error>>, Error> {
            let n = pairs.len();
            let mut seq = Vec::new();
            let (mut q_off, mut q_len, mut t_off, mut t_len) = (Vec::new(), Vec::new(), Vec::new(), Vec::new());
            let (mut q_seed, mut t_seed) = (Vec::new(), Vec::new());
            let mut bound = 16u64;
            for (q, t, a) in pairs {
                q_off.push(seq.len() as u64);
                q_len.push(q.len() as u32);
                seq.extend_from_slice(q);
                t_off.push(seq.len() as u64);
                t_len.push(t.len() as u32);
                seq.extend_from_slice(t);
                q_seed.push(a.query_pos as u32);
                t_seed.push(a.target_pos as u32);
                bound += phr_cigar_bound(q.len() as u64, t.len() as u64);
            }
            let batch = phr_pair_batch {
                n_pairs: n as u64, seq: seq.as_ptr(), seq_bytes: seq.len() as u64, q_off: q_off.as_ptr(),
                q_len: q_len.as_ptr(), t_off: t_off.as_ptr(), t_len: t_len.as_ptr(), q_seed: q_seed.as_ptr(),
                t_seed: t_seed.as_ptr(),
            };
            let mut aln = vec![phr_alignment::default(); n];
            let mut cigar = vec![0u8; bound as usize];
            let mut arena = phr_result_arena {
                aln: aln.as_mut_ptr(), cigar: cigar.as_mut_ptr() as *mut c_char, cigar_capacity: bound, cigar_used: 0,
            };
            status(self.raw, unsafe { phr_extend_batch(self.raw, engine, &batch, costs, &mut arena) })?;
            Ok(aln.iter().map(|a| match a.status {
                PHR_OK => Ok(Alignment {
                    cigar: String::from_utf8_lossy(&cigar[a.cigar_off as usize..(a.cigar_off + a.cigar_len as u64) as usize])
                        .into_owned(),
                    edit_distance: a.edit_distance as usize,
                    query_start: a.query_start as usize,
                    query_end: a.query_end as usize,
                    target_start: a.target_start as usize,
                    target_end: a.target_end as usize,
                }),
                PHR_INVALID_INPUT => Err(Error::InvalidInput),
                PHR_ALIGNMENT_FAILED => Err(Error::AlignmentFailed),
                s => Err(Error::Engine(s, String::new())),
            }).collect())
        }

        pub fn raw(&mut self) -> *mut phr_ctx {
            self.raw
        }
    }

    impl Drop for Context {
        fn drop(&mut self) {
            unsafe { phr_ctx_destroy(self.raw) };
        }
    }
}
