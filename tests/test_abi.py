"""CPU-side checks of the C ABI: the library builds, loads and exports every
entry point declared in include/*.h; host-side validation behaves like the
reference's error enums without touching a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

import lzx_b200
from lzx_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    declared = _lib.declared_functions()
    assert "lc_ntt_forward" in declared and "lc_ntt_plan_create_u32" in declared
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (lc_\w+)", out))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    L = _lib.lib()
    for f in declared:
        assert hasattr(L, f)


def test_build_targets_sm100a_only():
    from lzx_b200 import build
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS
    assert build.up_to_date(), "in-tree library is older than its sources"


def test_status_strings_and_version():
    L = _lib.lib()
    assert L.lc_version() == lzx_b200.__version__.encode()
    assert L.lc_status_string(0) == b"ok"
    assert L.lc_status_string(_lib.LC_ERR_ADICITY_TOO_SMALL) == b"adicity too small"
    assert L.lc_status_string(12345) == b"unknown status"


def test_host_validation_precedes_device():
    """NttTables::new rejects log_n + 1 > adicity (ntt.rs:47-50) before any device work."""
    with pytest.raises(lzx_b200.NttError) as e:
        lzx_b200.NttTables(lzx_b200.Modulus32.Q_12289, 12)
    assert e.value.kind == "AdicityTooSmall"
    with pytest.raises(lzx_b200.NttError):
        lzx_b200.NttTables(lzx_b200.CRT_SET_30BIT, 10)  # adicity 9 and 10 primes
    L = _lib.lib()
    h = C.c_void_p()
    arr = lambda *xs: (C.c_uint32 * len(xs))(*xs)
    assert L.lc_ntt_plan_create_u32(8, arr(4), arr(30), arr(3), 1, C.byref(h)) == \
        _lib.LC_ERR_INVALID_ARGUMENT  # even modulus
    assert L.lc_ntt_plan_create_u32(8, arr(12289), arr(12), arr(11), 0, C.byref(h)) == \
        _lib.LC_ERR_INVALID_ARGUMENT  # no moduli
    assert L.lc_ntt_plan_create_goldilocks(32, C.byref(h)) == _lib.LC_ERR_ADICITY_TOO_SMALL
    assert L.lc_ntt_forward(None, None, None, 1, None) == _lib.LC_ERR_INVALID_ARGUMENT


def test_no_cpu_fallback_without_gpu():
    L = _lib.lib()
    if L.lc_device_available():
        pytest.skip("a GPU is present")
    with pytest.raises(lzx_b200.LatticeCudaError) as e:
        lzx_b200.NttTables(lzx_b200.Modulus32.Q_32, 8)
    assert e.value.status == _lib.LC_ERR_NO_DEVICE


def test_header_cites_reference_interfaces():
    src = open(os.path.join(ROOT, "include", "lattice_cuda.h")).read()
    for cite in ("ntt.rs:46-106", "ntt.rs:118-146", "ntt.rs:187-216", "ntt.rs:38-42"):
        assert cite in src


def test_integration_binding_declares_every_entry_point():
    """The Rust FFI module given in INTEGRATION.md declares every entry point
    of the header, so a maintainer who copies it reaches the whole ABI."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```rust\n(.*?)\n```", doc, re.S)
    declared_rust = {f for b in blocks if 'extern "C"' in b for f in re.findall(r"pub fn (lc_\w+)\(", b)}
    missing = [f for f in _lib.declared_functions() if f not in declared_rust]
    assert not missing, missing


def test_rust_hooks_call_only_header_entry_points():
    """The hook code for the two hot-path crates (NttTables dispatch,
    AjtaiPublicKey::commit / commit_batch) calls only functions the header
    declares, and the hooks cover the reference methods they replace."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```rust\n(.*?)\n```", doc, re.S)
    called = {f for b in blocks for f in re.findall(r"ffi::(lc_\w+)\(", b)}
    declared = set(_lib.declared_functions())
    assert called and not (called - declared), sorted(called - declared)
    code = "\n".join(blocks)
    for hook in ("fn with_gpu", "fn forward_fast", "fn inverse_fast", "fn forward_batch", "fn inverse_batch",
                 "fn from_seed_gpu", "fn commit(", "fn commit_batch", "AjtaiError::DimensionMismatch"):
        assert hook in code, hook


def test_null_handles_are_rejected():
    """Every entry point that takes a plan, key, batch, pipeline or output
    pointer rejects null with LC_ERR_INVALID_ARGUMENT (the getters with -1)
    before touching a device, like the reference's Result errors."""
    L = _lib.lib()
    bad = _lib.LC_ERR_INVALID_ARGUMENT
    calls = {
        "lc_ajtai_key_set_fused": (L.lc_ajtai_key_set_fused, (None, 1)),
        "lc_ajtai_key_set_slot_products": (L.lc_ajtai_key_set_slot_products, (None, 0)),
        "lc_ajtai_key_set_engine": (L.lc_ajtai_key_set_engine, (None, 0)),
        "lc_ajtai_key_info": (L.lc_ajtai_key_info, (None, None, None, None)),
        "lc_ajtai_commit": (L.lc_ajtai_commit, (None, None, 1, None, None)),
        "lc_ajtai_commit_i8": (L.lc_ajtai_commit_i8, (None, None, 1, None, None)),
        "lc_ajtai_commit_u8": (L.lc_ajtai_commit_u8, (None, None, 1, None, None)),
        "lc_ajtai_commit_host": (L.lc_ajtai_commit_host, (None, None, 1, None)),
        "lc_ajtai_commit_noalloc": (L.lc_ajtai_commit_noalloc, (None, None, 1, None, None)),
        "lc_ajtai_key_check": (L.lc_ajtai_key_check, (None, None)),
        "lc_ajtai_key_view": (L.lc_ajtai_key_view, (None, 1, 1, None)),
        "lc_ntt_inverse": (L.lc_ntt_inverse, (None, None, None, 1, None)),
        "lc_ntt_forward_host": (L.lc_ntt_forward_host, (None, None, None, 1)),
        "lc_ntt_plan_info": (L.lc_ntt_plan_info, (None, None, None, None)),
        "lc_ntt_plan_set_variant": (L.lc_ntt_plan_set_variant, (None, 0)),
        "lc_ntt_plan_check": (L.lc_ntt_plan_check, (None, None)),
        "lc_batch_run": (L.lc_batch_run, (None, None)),
        "lc_batch_info": (L.lc_batch_info, (None, None, None, None, None)),
        "lc_batch_set_config": (L.lc_batch_set_config, (None, 1, 1, 1)),
        "lc_fold_pipeline_run": (L.lc_fold_pipeline_run, (None, None)),
        "lc_fold_pipeline_buffers": (L.lc_fold_pipeline_buffers, (None, None, None, None, None)),
        "lc_quad50_mul_host": (L.lc_quad50_mul_host, (None, None, None, None, 1)),
        "lc_quad50_plan_info": (L.lc_quad50_plan_info, (None, None, None)),
        "lc_lb_commit_host": (L.lc_lb_commit_host, (None, None, 1, None, None, None)),
        "lc_lb_key_info": (L.lc_lb_key_info, (None, None, None, None, None)),
        "lc_tc_i8_rate": (L.lc_tc_i8_rate, (1, 1, None, None)),
    }
    for name, (fn, args) in calls.items():
        assert fn(*args) == bad, name
    for getter in (L.lc_ajtai_key_get_fused, L.lc_ajtai_key_get_slot_products, L.lc_ajtai_key_get_engine):
        assert getter(None) == -1


def test_every_status_has_a_message_and_maps_to_an_error():
    """Each lc_status of the header has its own message; the Python layer
    turns LC_ERR_DIMENSION_MISMATCH into AjtaiError::DimensionMismatch
    (ajtai.rs:44-49) and every other failure into LatticeCudaError."""
    from lzx_b200.commitment import AjtaiError, _map_status
    src = open(os.path.join(ROOT, "include", "lattice_cuda.h")).read()
    codes = {name: int(v) for name, v in re.findall(r"\b(LC_(?:OK|ERR_\w+))\s*=\s*(\d+)", src)}
    assert codes["LC_OK"] == 0 and len(codes) >= 10
    L = _lib.lib()
    msgs = {c: L.lc_status_string(v) for c, v in codes.items()}
    assert all(m and m != b"unknown status" for m in msgs.values()), msgs
    assert len(set(msgs.values())) == len(msgs)
    _map_status(0, "ok")
    for name, v in codes.items():
        if v == 0:
            continue
        if name == "LC_ERR_DIMENSION_MISMATCH":
            with pytest.raises(AjtaiError) as e:
                _map_status(v, "commit")
            assert e.value.kind == "DimensionMismatch"
        else:
            with pytest.raises(_lib.LatticeCudaError) as e:
                _map_status(v, "commit")
            assert e.value.status == v and "commit" in str(e.value)
