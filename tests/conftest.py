import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


# Under the checked build (FLUXION_CHECKED=1, libfluxion_cuda_checked.so) every GPU test ends by
# reading the kernels' index-check status words: an out-of-range index anywhere fails the test.
if os.environ.get("FLUXION_CHECKED") == "1":
    @pytest.fixture(autouse=True)
    def _checked_status(request):
        yield
        if "gpu" not in request.keywords or not cuda_available():
            return
        import ctypes as C

        from fluxion_b200 import CudaBackend
        from fluxion_b200 import _lib as L
        be = CudaBackend.get(0)
        cnt, line, idx, ext = C.c_size_t(), C.c_int(), C.c_longlong(), C.c_longlong()
        name = C.create_string_buffer(256)
        rc = L.lib().fx_checked_status(be.ctx, C.byref(cnt), name, 256, C.byref(line), C.byref(idx), C.byref(ext))
        assert rc == 0, L.lib().fx_last_error()
        assert cnt.value == 0, (f"{cnt.value} unit(s) saw an out-of-range index; first: {name.value.decode()}:"
                                f"{line.value} index {idx.value} of {ext.value}")
