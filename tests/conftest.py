import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def dev():
    import torch
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def stab_dirs(dev):
    """stab_dirs(n, i0=0) -> float32 [n, 32, 3]: the raystab directions of
    queries i0 .. i0+n-1 as the reference's CUDA build computes them (its
    fibonacci_dir<32> with the device sincosf, from oracle/_ref/libref_bvh.so),
    for the raystab oracle (oracle.sdf_raystab64(..., dirs=...)).  Where that
    library is not built, the library's own directions, which
    tests/test_gpu_ref_bvh.py compares with the reference's bit for bit."""
    import ctypes

    import torch
    from oracle import oracle as O

    def get(n, i0=0):
        out = torch.empty(n, 32, 3, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if O.ref_bvh_available():
            O.ref_stab_dirs_gpu_ptr(i0, n, out.data_ptr(), stream)
        else:
            from cubvh_b200._lib import lib
            assert lib().cubvh_stab_directions(i0, n, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)) == 0
        torch.cuda.synchronize(dev)
        return out.cpu().numpy()
    return get
