"""CPU: the C-ABI library loads, exports every entry point the header
declares, its struct layouts match the ctypes binding, and calls without a
GPU fail with a typed status (no crash) — the reference's cuda-stub contract
(tests/cuda_stub_contract_test.rs:1-20)."""

from __future__ import annotations

import ctypes as C
import re
import subprocess
import tempfile
from pathlib import Path

import pytest

from conftest import REPO, gpu_available, load_bolt

HEADER = REPO / "include" / "bolt_b200.h"


def header_functions() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bolt_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    bolt = load_bolt()
    from importlib import import_module
    build = import_module("craton_bolt_b200.build")
    build.build()
    return bolt.lib()


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_binding_covers_every_declared_function():
    from importlib import import_module
    load_bolt()
    abi = import_module("craton_bolt_b200._abi")
    assert sorted(abi.SIGNATURES) == header_functions()


def test_struct_layouts_match_header(tmp_path):
    from importlib import import_module
    load_bolt()
    abi = import_module("craton_bolt_b200._abi")
    structs = {"bolt_col_view": abi.ColView, "bolt_col_mut": abi.ColMut, "bolt_agg_spec": abi.AggSpec,
               "bolt_pred": abi.Pred, "bolt_groupby_desc": abi.GroupbyDesc, "bolt_groupby_out": abi.GroupbyOut,
               "bolt_query": abi.Query, "bolt_server_config": abi.ServerConfig}
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        src.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            src.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    src.append("return 0;}")
    c_file = tmp_path / "layout.c"
    c_file.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-o", str(exe), str(c_file)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = dict(line.rsplit(" ", 1) for line in out if line)
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, f"{cname}.{fname}"


def test_status_strings(lib):
    lib.bolt_status_str.restype = C.c_char_p
    assert lib.bolt_status_str(0) == b"ok"
    assert lib.bolt_status_str(3) == b"overflow"
    assert lib.bolt_version().startswith(b"bolt-b200")


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU contract")
def test_no_gpu_gives_typed_error(lib):
    h = C.c_void_p()
    st = lib.bolt_ctx_create(0, 0, C.byref(h))
    assert st == 6 and not h.value  # BOLT_ERR_CUDA, no context


def test_null_context_is_rejected(lib):
    assert lib.bolt_groupby(None, None, None, 0, None) == 7
    assert lib.bolt_radix_sort_perm(None, None, 0, 0, None, 0, None) == 7


def test_footprint_tracks_rows_not_only_the_hint(lib):
    """The admission footprint (host arithmetic, no GPU) sizes the table from
    min(groups hint, rows): a small query hinted at many groups stays small,
    and the footprint never shrinks as rows grow."""
    from importlib import import_module
    load_bolt()
    abi = import_module("craton_bolt_b200._abi")
    aggs = (abi.AggSpec * 2)(abi.AggSpec(0, 1), abi.AggSpec(1, -1))
    d = abi.GroupbyDesc(None, 2, None, 1, None, 0, aggs, 2, 1_000_000)
    small = lib.bolt_groupby_footprint(C.byref(d), 10_000)
    big = lib.bolt_groupby_footprint(C.byref(d), 50_000_000)
    assert small < big / 50
    sizes = [lib.bolt_groupby_footprint(C.byref(d), n) for n in (1, 100, 10_000, 1_000_000, 10_000_000)]
    assert sizes == sorted(sizes)


RUST_SYS = REPO / "rust" / "bolt_b200_sys.rs"


def header_constants() -> dict[str, int]:
    """Enum values and #define flags of the header, by name."""
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    vals = {m[0]: int(m[1], 0) for m in re.findall(r"#define\s+(BOLT_FLAG_[A-Z_]+)\s+(0x[0-9a-fA-F]+)u", text)}
    for body in re.findall(r"typedef enum\s*\{(.*?)\}", text, flags=re.S):
        for name, val in re.findall(r"(BOLT_[A-Z0-9_]+)\s*=\s*(\d+)", body):
            vals[name] = int(val)
    return vals


def test_rust_ffi_declares_every_function_and_constant():
    """The Rust FFI file a maintainer drops into the reference declares every
    entry point of the header and carries the header's constant values (it
    is not compiled here: there is no Rust toolchain)."""
    rs = RUST_SYS.read_text()
    declared = set(re.findall(r"pub fn (bolt_[a-z0-9_]+)\s*\(", rs))
    missing = [n for n in header_functions() if n not in declared]
    assert not missing, f"rust/bolt_b200_sys.rs lacks {missing}"
    consts = {m[0]: int(m[1], 0) for m in re.findall(r"pub const (BOLT_[A-Z0-9_]+): [a-z0-9_]+ = (0x[0-9a-fA-F]+|\d+);", rs)}
    want = header_constants()
    assert len(want) >= 30
    wrong = {k: (consts.get(k), v) for k, v in want.items() if consts.get(k) != v}
    assert not wrong, f"rust constants differ from the header (rust, header): {wrong}"
