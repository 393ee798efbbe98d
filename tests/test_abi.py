"""The C-ABI library loads without a GPU and exports every function include/vgpu.h declares."""
import ctypes as C

import numpy as np

from vectisdb_b200 import abi
from vectisdb_b200.engine import sha256_hex


def test_library_exports_every_declared_symbol():
    lib = abi.lib()
    declared = abi.declared_functions()
    assert len(declared) >= 30
    missing = [name for name in declared if not hasattr(lib, name)]
    assert not missing, missing
    bound = {name for name, _, _ in abi.SIGNATURES}
    assert set(declared) == bound, set(declared) ^ bound


def test_abi_version_and_status_strings():
    lib = abi.lib()
    assert lib.vgpu_abi_version() == abi.ABI_VERSION
    assert lib.vgpu_status_string(abi.ERR_UNSUPPORTED) == b"UNSUPPORTED"


def test_sha256_known_vectors():
    # KernelCache::HashSource known answers (cuda_engine/tests/test_kernel_cache.cpp:68-75)
    assert sha256_hex(b"") == "e3b0c44298fc1c149afbf4c8996fb92427ae41e4649b934ca495991b7852b855"
    assert sha256_hex(b"abc") == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"
    assert len(sha256_hex(b"x")) == 64
    assert sha256_hex(b"out[idx] = a + b;") != sha256_hex(b"out[idx] = a - b;")
    long = bytes(range(256)) * 17
    import hashlib
    assert sha256_hex(long) == hashlib.sha256(long).hexdigest()


def test_malformed_plans_fail_cleanly_without_a_device():
    lib = abi.lib()
    res = C.c_void_p()
    # empty plan
    plan = abi.vgpu_plan()
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"empty plan" in lib.vgpu_last_error()
    # child index out of range
    nodes = (abi.vgpu_plan_node * 1)()
    kids = (C.c_uint32 * 1)(5)
    nodes[0].op = 1
    nodes[0].n_children = 1
    nodes[0].children = C.cast(kids, C.POINTER(C.c_uint32))
    plan = abi.vgpu_plan(C.cast(nodes, C.POINTER(abi.vgpu_plan_node)), 1, 0)
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    # a cycle
    kids[0] = 0
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert b"cycle" in lib.vgpu_last_error()
    # unknown op
    nodes[0].op = 99
    nodes[0].n_children = 0
    assert lib.vgpu_execute_plan(C.byref(plan), None, 0, None, C.byref(res)) == abi.ERR_INVALID_ARGUMENT
    assert not res.value


def test_row_independence_and_working_set():
    from vectisdb_b200 import workloads as W
    from vectisdb_b200.engine import estimate_working_set, is_row_independent, make_expr, make_projection, make_scan
    from vectisdb_b200.engine import GpuValueType as T
    assert not is_row_independent(W.c0_plan())
    p = make_projection([make_expr("((int*)out)[idx] = ((const int*)inputs[0])[row];", ["k"], T.INT32)],
                        make_scan(["k"]))
    assert is_row_independent(p)
    plan = W.c1_plan(0)
    plan.children[0].children[0].estimated_rows = 1 << 27
    plan.children[0].children[0].estimated_row_width_bytes = 32
    ws = estimate_working_set(plan)
    assert ws.total_bytes >= (1 << 27) * 32
    assert ws.largest_operator in (b"GROUP_BY_AGGREGATE", b"SCAN")
