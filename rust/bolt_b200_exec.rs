// bolt_b200_exec.rs — the reference-side executors over libboltb200.
//
// Drop-in file for the reference crate: `src/exec/bolt_b200_exec.rs`, declared
// from `src/exec/mod.rs` with `pub mod bolt_b200_exec;`, beside the FFI block
// in bolt_b200_sys.rs. It cannot be compiled in this repository (no Rust
// toolchain in its build image); it is written against the reference's own
// types and call sites, listed per function below.
//
// Wiring in the reference (one line each):
//   * src/exec/groupby.rs:355 — first in the fast-path chain:
//       try_fast_path!(crate::exec::bolt_b200_exec::try_execute_bolt_b200(plan, table_batch));
//     The status mapping below makes BOLT_ERR_SPILL a `partition_reduce
//     spill:` error, which `try_fast_path!` (groupby.rs:329-354) treats as a
//     soft miss and falls through, exactly like the reference's Tier-2
//     reduce; BOLT_DECLINE is `None` (next strategy); every other error
//     propagates. Two integer keys wider than 64 bits (an Int64 among them,
//     no WHERE) take the library's sort-based wide form through the same
//     call, ahead of the host reducer at groupby.rs:513-522; other wide
//     shapes decline to it.
//   * src/exec/groupby_with_pre.rs:248-252 — the multi-column reject becomes
//       if let Some(r) = crate::exec::bolt_b200_exec::try_execute_bolt_b200(plan, table_batch) { return r; }
//     ahead of it, so WHERE + two-key GROUP BY runs here instead of erroring.
//   * src/exec/join.rs:1336 — `try_gpu_inner_join` calls
//       try_join_indices_bolt_b200(build_key, probe_key)
//     for single Int32/Int64 keys before its Stage-1 and Stage-2 kernels
//     (duplicate build keys included: every matching build row, ascending);
//     `None` keeps the existing path (multi-column keys, other dtypes).
//   * src/exec/sort.rs:191-196 — the `BOLT_GPU_SORT` gate routes through
//       try_sort_perm_bolt_b200(&batch, sort_exprs)
//     instead of `try_gpu_sort_radix`; the permutation feeds the same `take`.
//   * src/exec/gpu_compact.rs:1005 — `compact_columns_on_gpu` becomes a
//     call to `bolt_compact_mask` over the same device columns.
//
// One `BoltB200` per Engine (like the reference's Engine, it is !Sync: the
// raw context pointer makes it so).

use std::ffi::CStr;
use std::sync::Arc;

use arrow_array::{
    Array, ArrayRef, Decimal128Array, Float32Array, Float64Array, Int32Array, Int64Array, RecordBatch, UInt32Array,
};
use arrow_buffer::{BooleanBuffer, NullBuffer};
use arrow_schema::{DataType as ArrowType, Schema as ArrowSchema};

use crate::cuda::bolt_b200_sys::*;
use crate::cuda::GpuVec;
use crate::error::{BoltError, BoltResult};
use crate::exec::groupby_tier2_orchestrator::PARTITION_REDUCE_SPILL_PREFIX;
use crate::plan::logical_plan::{AggregateExpr, BinaryOp, Expr, Literal};
use crate::plan::physical_plan::{KernelSpec, Op, PhysicalPlan};

/// The library's context: scratch arena, stream-ordered status word, tuning
/// cache (bolt_ctx_create / bolt_ctx_destroy).
pub struct BoltB200 {
    ctx: *mut bolt_ctx,
}

impl BoltB200 {
    /// `scratch_bytes == 0` takes a quarter of the device's free memory.
    pub fn new(device: i32, scratch_bytes: u64) -> BoltResult<Self> {
        let mut ctx = std::ptr::null_mut();
        let st = unsafe { bolt_ctx_create(device, scratch_bytes, &mut ctx) };
        if st != BOLT_OK {
            return Err(BoltError::Cuda(format!("bolt_ctx_create failed: status {st}")));
        }
        Ok(Self { ctx })
    }

    fn last_error(&self) -> String {
        unsafe { CStr::from_ptr(bolt_ctx_last_error(self.ctx)) }.to_string_lossy().into_owned()
    }

    /// The reference's result shape for one call: `None` = decline (the caller
    /// takes its next path), `Some(Ok)` = served, `Some(Err)` = the matching
    /// BoltError variant (src/error.rs:21-100). BOLT_ERR_SPILL carries the
    /// Tier-2 soft-miss prefix so `try_fast_path!` falls through on it.
    fn status(&self, st: bolt_status) -> Option<BoltResult<()>> {
        let msg = || self.last_error();
        match st {
            BOLT_OK => Some(Ok(())),
            BOLT_DECLINE => None,
            BOLT_ERR_SPILL => Some(Err(BoltError::Other(format!("{PARTITION_REDUCE_SPILL_PREFIX} {}", msg())))),
            BOLT_ERR_OVERFLOW => Some(Err(BoltError::Type(msg()))),
            BOLT_ERR_CAPACITY => Some(Err(BoltError::GpuCapacity(msg()))),
            BOLT_ERR_TIMEOUT | BOLT_ERR_CUDA => Some(Err(BoltError::Cuda(msg()))),
            BOLT_ERR_INVALID => Some(Err(BoltError::Plan(msg()))),
            other => Some(Err(BoltError::Other(format!("libboltb200 status {other}: {}", msg())))),
        }
    }
}

impl Drop for BoltB200 {
    fn drop(&mut self) {
        unsafe { bolt_ctx_destroy(self.ctx) }
    }
}

thread_local! {
    // One context per host thread (the reference's Engine is !Sync).
    static BOLT: std::cell::RefCell<Option<BoltB200>> = std::cell::RefCell::new(None);
}

fn with_bolt<R>(f: impl FnOnce(&BoltB200) -> Option<R>) -> Option<R> {
    BOLT.with(|b| {
        let mut b = b.borrow_mut();
        if b.is_none() {
            *b = BoltB200::new(0, 0).ok();
        }
        b.as_ref().and_then(f)
    })
}

// ---------------------------------------------------------------------------
// Host Arrow arrays as column views (the library reads host columns through
// bolt_groupby_host, streaming them to the device in chunks).
// ---------------------------------------------------------------------------
fn bolt_dtype(t: &ArrowType) -> Option<(i32, i32, usize)> {
    Some(match t {
        ArrowType::Int32 => (BOLT_I32, 0, 4),
        ArrowType::Int64 => (BOLT_I64, 0, 8),
        ArrowType::Float32 => (BOLT_F32, 0, 4),
        ArrowType::Float64 => (BOLT_F64, 0, 8),
        ArrowType::Decimal128(_, s) => (BOLT_DEC128, *s as i32, 16),
        _ => return None,
    })
}

/// A view of a host Arrow array. Declines (None) on sliced arrays whose
/// validity bitmap does not start on bit 0.
fn host_view(a: &ArrayRef) -> Option<bolt_col_view> {
    let (dtype, scale, width) = bolt_dtype(a.data_type())?;
    let data = a.to_data();
    let values = data.buffers().first()?;
    let validity = match data.nulls() {
        Some(n) if n.null_count() > 0 => {
            if n.offset() != 0 {
                return None;
            }
            n.buffer().as_ptr()
        }
        _ => std::ptr::null(),
    };
    let base = unsafe { values.as_ptr().add(data.offset() * width) };
    Some(bolt_col_view { data: base as *const _, validity, len: a.len() as u64, dtype, scale })
}

// ---------------------------------------------------------------------------
// Lowering the pre-aggregation kernel: pass-through loads, literals, widening
// casts and comparisons of a column with a literal, joined by AND. Anything
// else (arithmetic, OR, NULL tests) declines.
// ---------------------------------------------------------------------------
#[derive(Clone)]
enum Val {
    Col(usize),
    Lit(Literal),
    Preds(Vec<(usize, i32, Literal)>),
}

fn cmp_code(op: &BinaryOp, swapped: bool) -> Option<i32> {
    let c = match op {
        BinaryOp::Lt => BOLT_CMP_LT,
        BinaryOp::LtEq => BOLT_CMP_LE,
        BinaryOp::Gt => BOLT_CMP_GT,
        BinaryOp::GtEq => BOLT_CMP_GE,
        BinaryOp::Eq => return Some(BOLT_CMP_EQ),
        BinaryOp::NotEq => return Some(BOLT_CMP_NE),
        _ => return None,
    };
    Some(if !swapped {
        c
    } else {
        match c {
            BOLT_CMP_LT => BOLT_CMP_GT,
            BOLT_CMP_LE => BOLT_CMP_GE,
            BOLT_CMP_GT => BOLT_CMP_LT,
            _ => BOLT_CMP_LE,
        }
    })
}

/// (pre output ordinal -> pre input ordinal, WHERE conjuncts over pre inputs).
fn lower_pre(k: &KernelSpec) -> Option<(Vec<usize>, Vec<(usize, i32, Literal)>)> {
    let mut regs: std::collections::HashMap<u32, Val> = Default::default();
    let mut outs = vec![usize::MAX; k.outputs.len()];
    for op in &k.ops {
        match op {
            Op::LoadColumn { dst, col_idx, .. } => {
                regs.insert(dst.0, Val::Col(*col_idx));
            }
            Op::Const { dst, lit } => {
                regs.insert(dst.0, Val::Lit(lit.clone()));
            }
            Op::Cast { dst, src, .. } => {
                let v = regs.get(&src.0)?.clone();
                regs.insert(dst.0, v);
            }
            Op::Binary { dst, op, lhs, rhs, .. } => {
                let (l, r) = (regs.get(&lhs.0)?.clone(), regs.get(&rhs.0)?.clone());
                let v = match (op, l, r) {
                    (BinaryOp::And, Val::Preds(mut a), Val::Preds(b)) => {
                        a.extend(b);
                        Val::Preds(a)
                    }
                    (op, Val::Col(c), Val::Lit(x)) => Val::Preds(vec![(c, cmp_code(op, false)?, x)]),
                    (op, Val::Lit(x), Val::Col(c)) => Val::Preds(vec![(c, cmp_code(op, true)?, x)]),
                    _ => return None,
                };
                regs.insert(dst.0, v);
            }
            Op::Store { src, col_idx, .. } => match regs.get(&src.0)? {
                Val::Col(c) => outs[*col_idx] = *c,
                _ => return None,
            },
            _ => return None,
        }
    }
    let preds = match &k.predicate {
        None => Vec::new(),
        Some(r) => match regs.get(&r.0)? {
            Val::Preds(p) => p.clone(),
            _ => return None,
        },
    };
    if outs.iter().any(|&c| c == usize::MAX) {
        return None;
    }
    Some((outs, preds))
}

fn bolt_literal(l: &Literal) -> Option<(i64, f64)> {
    Some(match l {
        Literal::Int32(v) => (*v as i64, *v as f64),
        Literal::Int64(v) => (*v, *v as f64),
        Literal::Float32(v) => (0, *v as f64),
        Literal::Float64(v) => (0, *v),
        _ => return None,
    })
}

// ---------------------------------------------------------------------------
// GROUP BY (replaces the fast-path chain of src/exec/groupby.rs:355-457 and
// the WHERE + GROUP BY executor of src/exec/groupby_with_pre.rs:222).
// ---------------------------------------------------------------------------

/// Output column of the GROUP BY, allocated on the device by the reference's
/// allocator and read back after the call.
struct OutCol {
    data: GpuVec<u8>,
    validity: GpuVec<u8>,
    dtype: i32,
    scale: i32,
    width: usize,
}

impl OutCol {
    fn new(dtype: i32, scale: i32, cap: usize) -> BoltResult<Self> {
        let width = match dtype {
            BOLT_I32 | BOLT_F32 | BOLT_U32 => 4,
            BOLT_DEC128 => 16,
            _ => 8,
        };
        Ok(Self {
            data: GpuVec::<u8>::zeros(cap * width)?,
            validity: GpuVec::<u8>::zeros((cap + 7) / 8)?,
            dtype,
            scale,
            width,
        })
    }

    fn as_mut(&mut self, cap: usize) -> bolt_col_mut {
        bolt_col_mut {
            data: self.data.device_ptr() as *mut _,
            validity: self.validity.device_ptr() as *mut _,
            cap: cap as u64,
            dtype: self.dtype,
            scale: self.scale,
        }
    }

    fn to_arrow(&self, n: usize) -> BoltResult<ArrayRef> {
        let bytes = self.data.to_vec()?;
        let bits = self.validity.to_vec()?;
        let nulls = NullBuffer::new(BooleanBuffer::new(bits.into(), 0, n));
        let nulls = if nulls.null_count() > 0 { Some(nulls) } else { None };
        let b = &bytes[..n * self.width];
        Ok(match self.dtype {
            BOLT_I32 => Arc::new(Int32Array::new(b.chunks_exact(4).map(|c| i32::from_le_bytes(c.try_into().unwrap())).collect(), nulls)),
            BOLT_I64 => Arc::new(Int64Array::new(b.chunks_exact(8).map(|c| i64::from_le_bytes(c.try_into().unwrap())).collect(), nulls)),
            BOLT_F32 => Arc::new(Float32Array::new(b.chunks_exact(4).map(|c| f32::from_le_bytes(c.try_into().unwrap())).collect(), nulls)),
            BOLT_F64 => Arc::new(Float64Array::new(b.chunks_exact(8).map(|c| f64::from_le_bytes(c.try_into().unwrap())).collect(), nulls)),
            _ => Arc::new(
                Decimal128Array::new(b.chunks_exact(16).map(|c| i128::from_le_bytes(c.try_into().unwrap())).collect(), nulls)
                    .with_precision_and_scale(38, self.scale as i8)
                    .map_err(|e| BoltError::Other(e.to_string()))?,
            ),
        })
    }
}

/// Output dtype of an aggregate over an input of dtype `t` (the reference's
/// result types: COUNT -> Int64, AVG -> Float64, SUM of integers -> Int64,
/// SUM / MIN / MAX otherwise keep the input type).
fn agg_out(op: i32, t: Option<(i32, i32)>) -> (i32, i32) {
    match (op, t) {
        (BOLT_AGG_COUNT_STAR, _) | (BOLT_AGG_COUNT, _) => (BOLT_I64, 0),
        (BOLT_AGG_AVG, _) => (BOLT_F64, 0),
        (BOLT_AGG_SUM, Some((BOLT_I32, _))) => (BOLT_I64, 0),
        (_, Some(t)) => t,
        (_, None) => (BOLT_I64, 0),
    }
}

pub fn try_execute_bolt_b200(plan: &PhysicalPlan, batch: &RecordBatch) -> Option<BoltResult<RecordBatch>> {
    let (pre, agg) = match plan {
        PhysicalPlan::Aggregate { pre, aggregate, .. } => (pre, aggregate),
        _ => return None,
    };
    if agg.group_by.is_empty() || agg.group_by.len() > 2 {
        return None;
    }
    // Aggregate inputs -> table column names, through the pre kernel if any.
    let (name_of, preds): (Vec<String>, Vec<(String, i32, Literal)>) = match pre {
        None => (agg.inputs.iter().map(|c| c.name.clone()).collect(), Vec::new()),
        Some(k) => {
            let (outs, preds) = lower_pre(k)?;
            (
                outs.iter().map(|&c| k.inputs[c].name.clone()).collect(),
                preds.into_iter().map(|(c, cmp, l)| (k.inputs[c].name.clone(), cmp, l)).collect(),
            )
        }
    };
    // The table's columns the query reads, each once.
    let mut names: Vec<String> = Vec::new();
    let mut col_of = |n: &str, names: &mut Vec<String>| -> i32 {
        match names.iter().position(|x| x == n) {
            Some(i) => i as i32,
            None => {
                names.push(n.to_string());
                (names.len() - 1) as i32
            }
        }
    };
    let key_cols: Vec<i32> = agg.group_by.iter().map(|&g| col_of(&name_of[g], &mut names)).collect();
    let mut aggs: Vec<bolt_agg_spec> = Vec::new();
    for a in &agg.aggregates {
        let (op, e) = match a {
            AggregateExpr::Sum(e) => (BOLT_AGG_SUM, Some(e)),
            AggregateExpr::Min(e) => (BOLT_AGG_MIN, Some(e)),
            AggregateExpr::Max(e) => (BOLT_AGG_MAX, Some(e)),
            AggregateExpr::Avg(e) => (BOLT_AGG_AVG, Some(e)),
            // COUNT(*) is lowered as COUNT(<literal 1>) (sql_frontend.rs:2851).
            AggregateExpr::Count(Expr::Literal(_)) => (BOLT_AGG_COUNT_STAR, None),
            AggregateExpr::Count(e) => (BOLT_AGG_COUNT, Some(e)),
            _ => return None,
        };
        let input_col = match e {
            None => -1,
            Some(Expr::Column(c)) => {
                let i = agg.inputs.iter().position(|x| &x.name == c)?;
                col_of(&name_of[i], &mut names)
            }
            Some(_) => return None,
        };
        aggs.push(bolt_agg_spec { op, input_col });
    }
    let mut bpreds: Vec<bolt_pred> = Vec::new();
    for (n, cmp, lit) in &preds {
        let (lit_i, lit_f) = bolt_literal(lit)?;
        bpreds.push(bolt_pred { col: col_of(n, &mut names), cmp: *cmp, lit_i, lit_f });
    }
    let mut arrays: Vec<ArrayRef> = Vec::new();
    for n in &names {
        arrays.push(batch.column(batch.schema().index_of(n).ok()?).clone());
    }
    let cols: Vec<bolt_col_view> = arrays.iter().map(host_view).collect::<Option<_>>()?;

    with_bolt(|b| {
        let run = || -> Option<BoltResult<RecordBatch>> {
            // Output capacity: the rows bound the groups; a smaller first guess
            // with a capacity retry would save device memory for huge inputs.
            let cap = batch.num_rows().max(1) + 1;
            let mut key_out: Vec<OutCol> = Vec::new();
            for &k in &key_cols {
                let c = &cols[k as usize];
                match OutCol::new(c.dtype, c.scale, cap) {
                    Ok(o) => key_out.push(o),
                    Err(e) => return Some(Err(e)),
                }
            }
            let mut agg_out_cols: Vec<OutCol> = Vec::new();
            for a in &aggs {
                let t = (a.input_col >= 0).then(|| (cols[a.input_col as usize].dtype, cols[a.input_col as usize].scale));
                let (dt, sc) = agg_out(a.op, t);
                match OutCol::new(dt, sc, cap) {
                    Ok(o) => agg_out_cols.push(o),
                    Err(e) => return Some(Err(e)),
                }
            }
            let mut kmut: Vec<bolt_col_mut> = key_out.iter_mut().map(|o| o.as_mut(cap)).collect();
            let mut amut: Vec<bolt_col_mut> = agg_out_cols.iter_mut().map(|o| o.as_mut(cap)).collect();
            let desc = bolt_groupby_desc {
                cols: cols.as_ptr(),
                n_cols: cols.len() as i32,
                key_cols: key_cols.as_ptr(),
                n_keys: key_cols.len() as i32,
                preds: if bpreds.is_empty() { std::ptr::null() } else { bpreds.as_ptr() },
                n_preds: bpreds.len() as i32,
                aggs: aggs.as_ptr(),
                n_aggs: aggs.len() as i32,
                groups_hint: 0,
            };
            let mut out = bolt_groupby_out {
                keys: kmut.as_mut_ptr(),
                aggs: amut.as_mut_ptr(),
                n_groups: 0,
                n_groups_dev: std::ptr::null_mut(),
            };
            let st = unsafe { bolt_groupby_host(b.ctx, &desc, &mut out, 0, std::ptr::null_mut()) };
            if let Err(e) = b.status(st)? {
                return Some(Err(e));
            }
            let n = out.n_groups as usize;
            let mut arrays: Vec<ArrayRef> = Vec::new();
            for o in key_out.iter().chain(agg_out_cols.iter()) {
                match o.to_arrow(n) {
                    Ok(a) => arrays.push(a),
                    Err(e) => return Some(Err(e)),
                }
            }
            // The reference's own conversion (groupby.rs:830,3244).
            let schema: Arc<ArrowSchema> =
                match crate::exec::schema_convert::plan_schema_to_arrow_schema_minmax_temporal(&agg.output_schema) {
                    Ok(s) => s,
                    Err(e) => return Some(Err(e)),
                };
            Some(RecordBatch::try_new(schema, arrays).map_err(|e| BoltError::Other(e.to_string())))
        };
        run()
    })
}

// ---------------------------------------------------------------------------
// Hash join indices (replaces Stage 1 of try_gpu_inner_join, join.rs:1336,
// and gpu_join::hash_join_indices_on_gpu, gpu_join.rs:1403). Pairs come back
// in probe order; a duplicated build key pairs with each of its build rows in
// ascending order.
// ---------------------------------------------------------------------------
pub fn try_join_indices_bolt_b200(build_key: &ArrayRef, probe_key: &ArrayRef)
    -> Option<BoltResult<(UInt32Array, UInt32Array)>> {
    if !matches!(build_key.data_type(), ArrowType::Int32 | ArrowType::Int64) || build_key.data_type() != probe_key.data_type() {
        return None;
    }
    with_bolt(|b| {
        let run = || -> BoltResult<Option<(UInt32Array, UInt32Array)>> {
            let width = if build_key.data_type() == &ArrowType::Int32 { 4 } else { 8 };
            let up = |a: &ArrayRef| -> BoltResult<(GpuVec<u8>, bolt_col_view)> {
                let v = host_view(a).ok_or_else(|| BoltError::Other("sliced join key".into()))?;
                if !v.validity.is_null() {
                    return Err(BoltError::Other("NULL join keys take the reference path".into()));
                }
                let bytes = unsafe { std::slice::from_raw_parts(v.data as *const u8, a.len() * width) };
                let d = GpuVec::<u8>::from_slice(bytes)?;
                let view = bolt_col_view { data: d.device_ptr() as *const _, validity: std::ptr::null(), len: a.len() as u64,
                                           dtype: v.dtype, scale: 0 };
                Ok((d, view))
            };
            let (_bk, bview) = match up(build_key) { Ok(x) => x, Err(_) => return Ok(None) };
            let (_pk, pview) = match up(probe_key) { Ok(x) => x, Err(_) => return Ok(None) };
            let mut table = std::ptr::null_mut();
            match b.status(unsafe { bolt_hash_join_build(b.ctx, &bview, std::ptr::null(), 0, std::ptr::null_mut(), &mut table) }) {
                None => return Ok(None),
                Some(r) => r?,
            }
            let n = probe_key.len();
            let mut pi = GpuVec::<u32>::zeros(n.max(1))?;
            let mut bi = GpuVec::<u32>::zeros(n.max(1))?;
            let mut pm = bolt_col_mut { data: pi.device_ptr() as *mut _, validity: std::ptr::null_mut(), cap: n as u64, dtype: BOLT_U32, scale: 0 };
            let mut bm = bolt_col_mut { data: bi.device_ptr() as *mut _, validity: std::ptr::null_mut(), cap: n as u64, dtype: BOLT_U32, scale: 0 };
            let mut n_out = 0u64;
            let st = unsafe { bolt_hash_join_probe(b.ctx, table, &pview, &mut pm, &mut bm, &mut n_out, 0, std::ptr::null_mut()) };
            unsafe { bolt_hash_join_release(b.ctx, table) };
            match b.status(st) {
                None => return Ok(None),
                Some(r) => r?,
            }
            let k = n_out as usize;
            let (mut p, mut q) = (pi.to_vec()?, bi.to_vec()?);
            p.truncate(k);
            q.truncate(k);
            let _ = (&mut pi, &mut bi);
            Ok(Some((UInt32Array::from(q), UInt32Array::from(p)))) // (build rows, probe rows)
        };
        run().transpose()
    })
}

// ---------------------------------------------------------------------------
// ORDER BY permutation (replaces try_gpu_sort_radix behind the BOLT_GPU_SORT
// gate, sort.rs:191-196, and gpu_sort::sort_indices_on_gpu_radix_multi,
// gpu_sort.rs:995-1058). Stable; NULLs first or last per key.
// ---------------------------------------------------------------------------
pub fn try_sort_perm_bolt_b200(keys: &[(ArrayRef, bool /* descending */, bool /* nulls_first */)])
    -> Option<BoltResult<UInt32Array>> {
    if keys.is_empty() {
        return None;
    }
    let n = keys[0].0.len();
    let mut views = Vec::new();
    let mut keep = Vec::new(); // device copies of the keys and bitmaps
    for (a, _, _) in keys {
        if !matches!(a.data_type(), ArrowType::Int32 | ArrowType::Int64 | ArrowType::Float32 | ArrowType::Float64) {
            return None;
        }
        let v = host_view(a)?;
        let width = if matches!(a.data_type(), ArrowType::Int32 | ArrowType::Float32) { 4 } else { 8 };
        let d = GpuVec::<u8>::from_slice(unsafe { std::slice::from_raw_parts(v.data as *const u8, n * width) }).ok()?;
        let vb = if v.validity.is_null() {
            None
        } else {
            Some(GpuVec::<u8>::from_slice(unsafe { std::slice::from_raw_parts(v.validity, (n + 7) / 8) }).ok()?)
        };
        views.push(bolt_col_view {
            data: d.device_ptr() as *const _,
            validity: vb.as_ref().map_or(std::ptr::null(), |x| x.device_ptr() as *const u8),
            len: n as u64,
            dtype: v.dtype,
            scale: 0,
        });
        keep.push((d, vb));
    }
    let desc: Vec<i32> = keys.iter().map(|k| k.1 as i32).collect();
    let nf: Vec<i32> = keys.iter().map(|k| k.2 as i32).collect();
    with_bolt(|b| {
        let perm = match GpuVec::<u32>::zeros(n.max(1)) {
            Ok(p) => p,
            Err(e) => return Some(Err(e)),
        };
        let mut pm = bolt_col_mut { data: perm.device_ptr() as *mut _, validity: std::ptr::null_mut(), cap: n as u64, dtype: BOLT_U32, scale: 0 };
        let st = unsafe {
            bolt_radix_sort_perm_multi(b.ctx, views.as_ptr(), views.len() as i32, desc.as_ptr(), nf.as_ptr(), &mut pm, 0,
                                       std::ptr::null_mut())
        };
        if let Err(e) = b.status(st)? {
            return Some(Err(e));
        }
        Some(perm.to_vec().map(|mut v| {
            v.truncate(n);
            UInt32Array::from(v)
        }))
    })
}
