"""CPU-only checks of the C ABI boundary: the library loads, exports every entry point the
header declares, and reports a missing device as an error instead of falling back."""
import ctypes as C
import os
import re
import subprocess

import pytest

from fluxion_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    return sorted(L.parse_header().keys())


def test_header_declares_the_backend_surface():
    names = set(_declared())
    # one entry point per Backend trait op (crates/core/src/backend.rs:43-406)
    trait = ["fx_alloc", "fx_upload_f64", "fx_upload_f32", "fx_apply_stencil", "fx_copy", "fx_fill", "fx_axpy",
             "fx_scale", "fx_apply_stencil_var", "fx_stencil_axpy", "fx_norm_l2", "fx_reduce_sum",
             "fx_reduce_max", "fx_reduce_min", "fx_dot", "fx_dot2", "fx_restrict", "fx_prolong",
             "fx_weighted_jacobi", "fx_pointwise_mult", "fx_pointwise_div", "fx_waxpy", "fx_aypx",
             "fx_reciprocal", "fx_abs_val", "fx_pointwise_max", "fx_pointwise_min", "fx_apply_conv_diff",
             "fx_conv_diff_axpy", "fx_copy_to_host_f64", "fx_copy_to_host_f32", "fx_backend_name"]
    solvers = ["fx_cg_solve", "fx_cg_solve_preconditioned", "fx_pipelined_cg_solve", "fx_bicgstab_solve",
               "fx_bicgstab_solve_preconditioned", "fx_gmres_solve", "fx_gmres_solve_preconditioned",
               "fx_mg_create", "fx_mg_v_cycle", "fx_mg_depth", "fx_precond_identity"]
    missing = [n for n in trait + solvers if n not in names]
    assert not missing, missing


def test_library_exports_every_declared_symbol():
    assert os.path.exists(L.LIB_PATH), "libfluxion_cuda.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (fx_\w+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing


def test_library_loads_and_binds_all_prototypes():
    lib = L.lib()
    for name in _declared():
        assert getattr(lib, name).argtypes is not None
    assert lib.fx_backend_name() == b"cuda"
    assert lib.fx_version() >= 10000


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.lib()
    h = C.c_void_p()
    st = lib.fx_ctx_create(0, C.byref(h))
    assert st == L.FX_ERR_NO_DEVICE
    assert "CUDA" in L.last_error() or "device" in L.last_error()
    from fluxion_b200 import Device, BackendUnavailable
    with pytest.raises(BackendUnavailable):
        Device.best()


def test_null_handles_are_rejected():
    lib = L.lib()
    assert lib.fx_fill(None, None, 1.0) == L.FX_ERR_INVALID_ARGUMENT
    assert lib.fx_ctx_synchronize(None) == L.FX_ERR_INVALID_ARGUMENT
    out = C.c_double()
    assert lib.fx_dot(None, None, None, C.byref(out)) == L.FX_ERR_INVALID_ARGUMENT


def test_device_lanes_are_distinct_values():
    from fluxion_b200 import Device
    assert Device.Cuda(0) == Device(0, 0) and str(Device.Cuda(0)) == "cuda:0"
    d = Device.Cuda(0, lane=3)
    assert d.lane == 3 and d != Device.Cuda(0) and str(d) == "cuda:0/lane3"
    assert len({Device.Cuda(0, k) for k in range(4)}) == 4


def test_checked_library_exports_the_same_symbols_and_says_so():
    checked = os.path.join(ROOT, "fluxion_b200", "libfluxion_cuda_checked.so")
    assert os.path.exists(checked), "libfluxion_cuda_checked.so not built"
    out = subprocess.run(["nm", "-D", "--defined-only", checked], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (fx_\w+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing
    # fx_checked_build touches no device: 1 in the checked library, 0 in the default one
    assert C.CDLL(checked).fx_checked_build() == 1
    assert L.lib().fx_checked_build() == (1 if os.environ.get("FLUXION_CHECKED") == "1" else 0)
