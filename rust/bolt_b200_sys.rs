// bolt_b200_sys.rs — Rust FFI declarations of libboltb200 (include/bolt_b200.h).
//
// Drop-in file for the reference crate: `src/cuda/bolt_b200_sys.rs`, declared
// from `src/cuda/mod.rs` with `pub mod bolt_b200_sys;`. Link with
// `println!("cargo:rustc-link-search=native=<dir of libboltb200.so>");` and
// `println!("cargo:rustc-link-lib=dylib=boltb200");` in build.rs.
//
// Every struct is #[repr(C)] and mirrors the header field for field; the C
// layouts themselves are checked against the header by gcc in
// tests/test_abi.py. This file is not compiled in this repository (its build
// image has no Rust toolchain); it is kept as source for the reference's
// maintainers, next to the wrappers in bolt_b200_exec.rs.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_int, c_void};

// ---------------------------------------------------------------------------
// Status codes (the reference's BoltResult taxonomy, src/error.rs:21-100,
// plus the executors' Option "decline", src/exec/groupby_shmem_exec.rs:53).
// ---------------------------------------------------------------------------
pub type bolt_status = c_int;
pub const BOLT_OK: bolt_status = 0;
pub const BOLT_DECLINE: bolt_status = 1;
pub const BOLT_ERR_SPILL: bolt_status = 2;
pub const BOLT_ERR_OVERFLOW: bolt_status = 3;
pub const BOLT_ERR_CAPACITY: bolt_status = 4;
pub const BOLT_ERR_TIMEOUT: bolt_status = 5;
pub const BOLT_ERR_CUDA: bolt_status = 6;
pub const BOLT_ERR_INVALID: bolt_status = 7;

// Column dtypes (bolt_dtype).
pub const BOLT_I32: i32 = 0;
pub const BOLT_I64: i32 = 1;
pub const BOLT_F32: i32 = 2;
pub const BOLT_F64: i32 = 3;
pub const BOLT_DEC128: i32 = 4;
pub const BOLT_U32: i32 = 5;

// Aggregate operators (bolt_agg_op).
pub const BOLT_AGG_SUM: i32 = 0;
pub const BOLT_AGG_COUNT_STAR: i32 = 1;
pub const BOLT_AGG_COUNT: i32 = 2;
pub const BOLT_AGG_MIN: i32 = 3;
pub const BOLT_AGG_MAX: i32 = 4;
pub const BOLT_AGG_AVG: i32 = 5;

// Comparisons of a WHERE conjunct (bolt_cmp).
pub const BOLT_CMP_LT: i32 = 0;
pub const BOLT_CMP_LE: i32 = 1;
pub const BOLT_CMP_GT: i32 = 2;
pub const BOLT_CMP_GE: i32 = 3;
pub const BOLT_CMP_EQ: i32 = 4;
pub const BOLT_CMP_NE: i32 = 5;

// Call flags.
pub const BOLT_FLAG_ASYNC: u32 = 0x1;
pub const BOLT_FLAG_PROFILE: u32 = 0x2;
pub const BOLT_FLAG_FORCE_GLOBAL: u32 = 0x4;
pub const BOLT_FLAG_FORCE_SHMEM: u32 = 0x8;
pub const BOLT_FLAG_NO_TUNE: u32 = 0x10;
pub const BOLT_FLAG_KERNEL_REGS: u32 = 0x20;
pub const BOLT_FLAG_KERNEL_STAGED: u32 = 0x40;
pub const BOLT_FLAG_NO_PART: u32 = 0x80;
pub const BOLT_FLAG_FORCE_PART: u32 = 0x100;
pub const BOLT_FLAG_KERNEL_TIMES: u32 = 0x200;

// ---------------------------------------------------------------------------
// Column borrows (== GpuView / GpuViewMut, src/cuda/smart_ptrs.rs:268,367).
// ---------------------------------------------------------------------------
#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_col_view {
    pub data: *const c_void,
    pub validity: *const u8, // Arrow LSB bitmap or null
    pub len: u64,
    pub dtype: i32,
    pub scale: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_col_mut {
    pub data: *mut c_void,
    pub validity: *mut u8,
    pub cap: u64,
    pub dtype: i32,
    pub scale: i32,
}

pub type bolt_stream = *mut c_void; // CUstream / cudaStream_t

#[repr(C)]
pub struct bolt_ctx {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct bolt_join_table {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct bolt_graph {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct bolt_server {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_agg_spec {
    pub op: i32,
    pub input_col: i32, // -1 for COUNT(*)
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_pred {
    pub col: i32,
    pub cmp: i32,
    pub lit_i: i64,
    pub lit_f: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_groupby_desc {
    pub cols: *const bolt_col_view,
    pub n_cols: i32,
    pub key_cols: *const i32,
    pub n_keys: i32,
    pub preds: *const bolt_pred,
    pub n_preds: i32,
    pub aggs: *const bolt_agg_spec,
    pub n_aggs: i32,
    pub groups_hint: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_groupby_out {
    pub keys: *mut bolt_col_mut,
    pub aggs: *mut bolt_col_mut,
    pub n_groups: u64,
    pub n_groups_dev: *mut u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_query {
    pub desc: bolt_groupby_desc,
    pub out: bolt_groupby_out,
    pub row_begin: u64,
    pub row_end: u64,
    pub status: bolt_status,
}

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct bolt_server_config {
    pub device: i32,
    pub scratch_bytes: u64,
    pub max_batch: i32,
    pub n_lanes: i32,
}

extern "C" {
    // Context.
    pub fn bolt_ctx_create(device: c_int, scratch_bytes: u64, out: *mut *mut bolt_ctx) -> bolt_status;
    pub fn bolt_ctx_destroy(ctx: *mut bolt_ctx);
    pub fn bolt_ctx_last_error(ctx: *const bolt_ctx) -> *const c_char;
    pub fn bolt_status_str(s: bolt_status) -> *const c_char;
    pub fn bolt_ctx_last_device_ms(ctx: *const bolt_ctx) -> f64;
    pub fn bolt_ctx_last_launches(ctx: *const bolt_ctx) -> u32;
    pub fn bolt_ctx_last_groupby_tier(ctx: *const bolt_ctx) -> i32;
    pub fn bolt_ctx_kernel_times(ctx: *mut bolt_ctx, ms: *mut f64, max: u32) -> u32;
    pub fn bolt_ctx_sync_status(ctx: *mut bolt_ctx, stream: bolt_stream) -> bolt_status;
    pub fn bolt_ctx_scratch_bytes(ctx: *const bolt_ctx) -> u64;
    pub fn bolt_version() -> *const c_char;

    // GROUP BY.
    pub fn bolt_groupby(ctx: *mut bolt_ctx, desc: *const bolt_groupby_desc, out: *mut bolt_groupby_out,
                        flags: u32, stream: bolt_stream) -> bolt_status;
    pub fn bolt_groupby_host(ctx: *mut bolt_ctx, desc: *const bolt_groupby_desc, out: *mut bolt_groupby_out,
                             flags: u32, stream: bolt_stream) -> bolt_status;
    pub fn bolt_groupby_noalloc(desc: *const bolt_groupby_desc, out: *mut bolt_groupby_out, stream: bolt_stream,
                                err: *mut c_char, err_cap: i32) -> bolt_status;
    pub fn bolt_groupby_autotune(ctx: *mut bolt_ctx, desc: *const bolt_groupby_desc, out: *mut bolt_groupby_out,
                                 stream: bolt_stream, best_ms: *mut f64) -> bolt_status;
    pub fn bolt_ctx_tuning_save(ctx: *const bolt_ctx, path: *const c_char) -> bolt_status;
    pub fn bolt_ctx_tuning_load(ctx: *mut bolt_ctx, path: *const c_char) -> bolt_status;

    // Hash join.
    pub fn bolt_hash_join_build(ctx: *mut bolt_ctx, build_key: *const bolt_col_view, payload: *const bolt_col_view,
                                flags: u32, stream: bolt_stream, table_out: *mut *mut bolt_join_table) -> bolt_status;
    pub fn bolt_hash_join_probe(ctx: *mut bolt_ctx, table: *const bolt_join_table, probe_key: *const bolt_col_view,
                                probe_idx: *mut bolt_col_mut, build_idx: *mut bolt_col_mut, n_out: *mut u64,
                                flags: u32, stream: bolt_stream) -> bolt_status;
    pub fn bolt_hash_join_release(ctx: *mut bolt_ctx, table: *mut bolt_join_table);
    pub fn bolt_join_groupby(ctx: *mut bolt_ctx, table: *const bolt_join_table, probe_key: *const bolt_col_view,
                             value: *const bolt_col_view, out_group: *mut bolt_col_mut, out_sum: *mut bolt_col_mut,
                             out_count: *mut bolt_col_mut, n_groups: *mut u64, flags: u32,
                             stream: bolt_stream) -> bolt_status;

    // ORDER BY.
    pub fn bolt_radix_sort_perm(ctx: *mut bolt_ctx, key: *const bolt_col_view, descending: i32, nulls_first: i32,
                                perm: *mut bolt_col_mut, flags: u32, stream: bolt_stream) -> bolt_status;
    pub fn bolt_radix_sort_perm_multi(ctx: *mut bolt_ctx, keys: *const bolt_col_view, n_keys: i32,
                                      descending: *const i32, nulls_first: *const i32, perm: *mut bolt_col_mut,
                                      flags: u32, stream: bolt_stream) -> bolt_status;

    // WHERE compaction.
    pub fn bolt_compact(ctx: *mut bolt_ctx, cols: *const bolt_col_view, n_cols: i32, preds: *const bolt_pred,
                        n_preds: i32, out: *mut bolt_col_mut, row_ids: *mut bolt_col_mut, n_out: *mut u64,
                        flags: u32, stream: bolt_stream) -> bolt_status;
    pub fn bolt_compact_mask(ctx: *mut bolt_ctx, cols: *const bolt_col_view, n_cols: i32, mask: *const u8,
                             out: *mut bolt_col_mut, row_ids: *mut bolt_col_mut, n_out: *mut u64, flags: u32,
                             stream: bolt_stream) -> bolt_status;

    // Batched and served forms (no counterpart in the reference).
    pub fn bolt_batch_groupby(ctx: *mut bolt_ctx, qs: *mut bolt_query, n: i32, flags: u32,
                              stream: bolt_stream) -> bolt_status;
    pub fn bolt_groupby_footprint(desc: *const bolt_groupby_desc, n_rows: u64) -> u64;
    pub fn bolt_batch_graph_create(device: c_int, qs: *mut bolt_query, n: i32, out: *mut *mut bolt_graph) -> bolt_status;
    pub fn bolt_graph_launch(g: *mut bolt_graph, stream: bolt_stream) -> bolt_status;
    pub fn bolt_graph_sync_status(g: *mut bolt_graph, stream: bolt_stream, statuses: *mut i32,
                                  n_groups: *mut u64) -> bolt_status;
    pub fn bolt_graph_destroy(g: *mut bolt_graph);
    pub fn bolt_server_create(cfg: *const bolt_server_config, out: *mut *mut bolt_server) -> bolt_status;
    pub fn bolt_server_submit(srv: *mut bolt_server, q: *mut bolt_query, ticket: *mut u64) -> bolt_status;
    pub fn bolt_server_submit_batch(srv: *mut bolt_server, qs: *mut bolt_query, n: i32,
                                    tickets: *mut u64) -> bolt_status;
    pub fn bolt_server_wait(srv: *mut bolt_server, ticket: u64, latency_us: *mut f64) -> bolt_status;
    pub fn bolt_server_destroy(srv: *mut bolt_server);
}
