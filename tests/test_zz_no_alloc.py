"""ds2d_dot_f64_noalloc (static device scratch, no context) against ds2d_dot_f64, through the C ABI.

Collected last on purpose (file name): it must pass both alone in a fresh process and after
every other test has loaded and used the library in the same process."""
import ctypes

import pytest

from ds2d_b200 import Elastic2D
from ds2d_b200._lib import load

pytestmark = pytest.mark.gpu

DS2D_E_ARG = -1
MAX_ELEMS = 536_870_912  # 32768 partial sums x 16384 elements


def _noalloc(lib, a, b, n, stream):
    out = ctypes.c_double(float("nan"))
    rc = lib.ds2d_dot_f64_noalloc(ctypes.c_void_p(a), ctypes.c_void_p(b), int(n),
                                  ctypes.c_void_p(stream), ctypes.byref(out))
    return rc, out.value


def test_noalloc_matches_dot_f64_on_consecutive_calls(cuda_device):
    import torch
    lib = load()
    g = torch.Generator().manual_seed(11)
    n1, n2 = 3_000_001, 1000
    a = torch.randn(n1, generator=g, dtype=torch.float32).cuda()
    b = torch.randn(n1, generator=g, dtype=torch.float32).cuda()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    with Elastic2D(16, 16, 16, 8, 4, 10.0, 10.0, 0.001) as e:
        want1 = e.dot_f64(a.data_ptr(), b.data_ptr(), n1)
        want2 = e.dot_f64(a.data_ptr(), b.data_ptr(), n2)
    scale1 = float((a.double().abs() * b.double().abs()).sum())
    scale2 = float((a[:n2].double().abs() * b[:n2].double().abs()).sum())
    # two calls in a row, the second much shorter than the first: partial sums left in the static
    # scratch by the first call must not leak into the second
    rc1, got1 = _noalloc(lib, a.data_ptr(), b.data_ptr(), n1, stream)
    rc2, got2 = _noalloc(lib, a.data_ptr(), b.data_ptr(), n2, stream)
    assert rc1 == 0 and rc2 == 0, lib.ds2d_last_error(None)
    assert abs(got1 - want1) <= 1e-12 * scale1, (got1, want1)
    assert abs(got2 - want2) <= 1e-12 * scale2, (got2, want2)
    # repeat: deterministic, and no device memory taken by the calls.  This process's own
    # allocator must not move at all; the device-wide free memory (which other processes on the
    # same GPU also change) is allowed a small slack and one retry.
    reserved0 = torch.cuda.memory_reserved()
    for attempt in range(2):
        free0 = torch.cuda.mem_get_info()[0]
        rc3, got3 = _noalloc(lib, a.data_ptr(), b.data_ptr(), n1, stream)
        rc4, got4 = _noalloc(lib, a.data_ptr(), b.data_ptr(), n2, stream)
        assert rc3 == 0 and rc4 == 0
        assert got3 == got1 and got4 == got2
        if abs(torch.cuda.mem_get_info()[0] - free0) < (2 << 20):
            break
    else:
        pytest.fail("device free memory moved by 2 MiB or more across two no-allocation calls")
    assert torch.cuda.memory_reserved() == reserved0


def test_noalloc_rejects_oversize_and_bad_arguments(cuda_device):
    import torch
    lib = load()
    a = torch.ones(8, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    # rejected on the host before any launch: the pointers are never dereferenced
    rc, _ = _noalloc(lib, a.data_ptr(), a.data_ptr(), MAX_ELEMS + 1, 0)
    assert rc == DS2D_E_ARG
    assert b"static scratch limit" in lib.ds2d_last_error(None)
    rc, _ = _noalloc(lib, a.data_ptr(), a.data_ptr(), -1, 0)
    assert rc == DS2D_E_ARG
    rc, _ = _noalloc(lib, 0, a.data_ptr(), 8, 0)
    assert rc == DS2D_E_ARG
    rc, got = _noalloc(lib, a.data_ptr(), a.data_ptr(), 0, 0)
    assert rc == 0 and got == 0.0
    rc, got = _noalloc(lib, a.data_ptr(), a.data_ptr(), 8, 0)
    assert rc == 0 and got == 8.0
