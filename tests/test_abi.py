"""The C ABI: the libraries load without a GPU and export every declared entry point."""
import ctypes
import os
import re

import numpy as np
import pytest

import bohrium_b200 as bh
from bohrium_b200 import ir

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "bohrium_b200", "lib")


def declared_functions():
    src = open(os.path.join(ROOT, "include", "bh_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bh[a-z_0-9]+)\s*\(", src)))


def test_header_declares_the_bridge():
    names = declared_functions()
    for required in ["bhb_runtime_create", "bhb_ir_create", "bhb_ir_execute", "bhb_data_get", "bhb_data_set",
                     "bhb_message", "bhb_extmethod", "bh_ve_cuda_dry_run"]:
        assert required in names


def test_every_declared_symbol_is_exported():
    core = ctypes.CDLL(os.path.join(LIB, "libbh_core.so"), mode=ctypes.RTLD_GLOBAL)
    ve = ctypes.CDLL(os.path.join(LIB, "libbh_ve_cuda.so"))
    for name in declared_functions():
        lib = ve if name.startswith("bh_ve_cuda") else core
        assert hasattr(lib, name), f"{name} missing"


def test_components_export_create_and_destroy():
    for so in ["libbh_ve_cuda.so", "libbh_vem_node.so"]:
        lib = ctypes.CDLL(os.path.join(LIB, so))
        assert hasattr(lib, "create") and hasattr(lib, "destroy"), so


def test_base_handles():
    lib = bh.load_library()
    b = lib.bhb_base_create(ir.FLOAT32, 123)
    assert b and lib.bhb_base_dtype(b) == ir.FLOAT32 and lib.bhb_base_nelem(b) == 123
    assert lib.bhb_base_data(b) is None
    lib.bhb_base_destroy(b)
    assert not lib.bhb_base_create(99, 1)
    assert b"bad dtype" in lib.bhb_last_error()


def test_decode_rejects_malformed_bytecode():
    lib = bh.load_library()
    base = lib.bhb_base_create(ir.FLOAT64, 4)
    good = np.array([ir.OPCODES["ADD"], 3, -1, 0, 0, base, 0, 1, 4, 1, base, 0, 1, 4, 1, base, 0, 1, 4, 1],
                    dtype=np.int64)
    h = lib.bhb_ir_create(good.ctypes.data, len(good), None, 0, 1, None, None, 0)
    assert h
    lib.bhb_ir_destroy(h)
    truncated = good[:-3].copy()
    assert not lib.bhb_ir_create(truncated.ctypes.data, len(truncated), None, 0, 1, None, None, 0)
    assert b"truncated" in lib.bhb_last_error()
    wrong_nop = good.copy()
    wrong_nop[0] = ir.OPCODES["SQRT"]
    assert not lib.bhb_ir_create(wrong_nop.ctypes.data, len(wrong_nop), None, 0, 1, None, None, 0)
    assert b"expects 2 operands" in lib.bhb_last_error()
    unknown = good.copy()
    unknown[0] = 70
    assert not lib.bhb_ir_create(unknown.ctypes.data, len(unknown), None, 0, 1, None, None, 0)
    lib.bhb_base_destroy(base)


def test_stack_selection_and_env_override(tmp_path, monkeypatch):
    """config.ini stack selection and BH_<SECTION>_<OPTION> overrides (core/bh_config_parser.cpp)."""
    lib = bh.load_library()
    cfg = tmp_path / "config.ini"
    cfg.write_text(f"[stacks]\ndefault = node\nbroken = missing\n[node]\nimpl = {LIB}/libbh_vem_node.so\n"
                   f"[missing]\nimpl = {tmp_path}/nothing.so\n")
    rt = lib.bhb_runtime_create(str(cfg).encode(), b"default")
    assert rt, lib.bhb_last_error()
    assert lib.bhb_message(rt, b"info") == b""
    lib.bhb_runtime_destroy(rt)
    assert not lib.bhb_runtime_create(str(cfg).encode(), b"broken")
    assert b"cannot load library" in lib.bhb_last_error()
    # An environment override of `impl` takes precedence over the file.
    monkeypatch.setenv("BH_MISSING_IMPL", f"{LIB}/libbh_vem_node.so")
    rt = lib.bhb_runtime_create(str(cfg).encode(), b"broken")
    assert rt, lib.bhb_last_error()
    lib.bhb_runtime_destroy(rt)
    monkeypatch.delenv("BH_MISSING_IMPL")
    monkeypatch.setenv("BH_STACK", "default")


def test_cuda_stack_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA|device"):
        bh.NativeExecutor(stack="cuda")
