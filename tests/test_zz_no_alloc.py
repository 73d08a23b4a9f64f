"""prima_dot_no_alloc against prima_dot.

prima_dot_no_alloc serves callers that own their device memory and cannot
let a library allocate (a host with its own device pool or a fixed memory
budget: cudaFree synchronises the whole device).  It takes caller-owned
device arrays, keeps its block partials in a fixed device array inside the
library, and must give the same dot product as the context entry point
prima_dot on the same data, call after call, whatever the previous call
left in that array.  The inputs here are torch device tensors: the test owns
the memory, as such a caller would.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from noaidi_b200.prima import cuda

MAX_ELEMENTS = 16_777_216


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _no_alloc_dot(lib, x, y, bits, stream):
    import torch
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=x.device)
    rc = lib.prima_dot_no_alloc(_ptr(x), _ptr(y), x.numel(), bits, _ptr(out), C.c_void_p(stream.cuda_stream))
    assert rc == cuda.OK, lib.prima_last_error()
    stream.synchronize()
    return float(out.item())


@pytest.mark.gpu
@pytest.mark.parametrize("bits", [64, 32])
def test_matches_prima_dot_on_consecutive_calls(bits):
    import torch
    lib = cuda.library()
    kernels = cuda.CudaKernels(0, bits)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    dtype = torch.float64 if bits == 64 else torch.float32
    rng = np.random.default_rng(17)
    # a large call leaves many partials behind; the smaller calls after it
    # must read only their own
    for n in (3_000_001, 70_001, 8_192, 1):
        x = rng.standard_normal(n)
        y = rng.standard_normal(n)
        want = kernels.dot(kernels.upload(x), kernels.upload(y))
        xd = torch.from_numpy(x).to(device="cuda:0", dtype=dtype)
        yd = torch.from_numpy(y).to(device="cuda:0", dtype=dtype)
        got = _no_alloc_dot(lib, xd, yd, bits, stream)
        xr, yr = xd.double().cpu().numpy(), yd.double().cpu().numpy()  # the inputs as the device holds them
        scale = float(np.abs(xr * yr).sum())
        assert abs(got - want) <= 1e-9 * scale, (n, got, want)
        # and, independently of the library, a float64 sum on the host of the
        # same (rounded) inputs
        host = float(np.dot(xr, yr))
        assert abs(got - host) <= 1e-9 * scale, (n, got, host)


@pytest.mark.gpu
def test_empty_and_oversized_inputs():
    import torch
    lib = cuda.library()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    x = torch.ones(4, dtype=torch.float64, device="cuda:0")
    out = torch.full((1,), 7.0, dtype=torch.float64, device="cuda:0")
    assert lib.prima_dot_no_alloc(_ptr(x), _ptr(x), 0, 64, _ptr(out), C.c_void_p(stream.cuda_stream)) == cuda.OK
    stream.synchronize()
    assert out.item() == 0.0
    # rejected before anything is launched: nothing reads past x
    rc = lib.prima_dot_no_alloc(_ptr(x), _ptr(x), MAX_ELEMENTS + 1, 64, _ptr(out), C.c_void_p(stream.cuda_stream))
    assert rc == cuda.ERR_INVALID_ARGUMENT
    assert b"16777216" in lib.prima_last_error()
    rc = lib.prima_dot_no_alloc(_ptr(x), _ptr(x), 4, 16, _ptr(out), C.c_void_p(stream.cuda_stream))
    assert rc == cuda.ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_host_memory_is_refused_before_any_launch():
    """The arrays come from the caller; a host buffer handed over by mistake
    is refused (nothing is queued that would read it), and a device call on
    the same stream works afterwards."""
    import torch
    lib = cuda.library()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    host = np.ones(1024, dtype=np.float64)
    xd = torch.ones(1024, dtype=torch.float64, device="cuda:0")
    out = torch.full((1,), 7.0, dtype=torch.float64, device="cuda:0")
    host_out = np.zeros(1)
    hp = C.c_void_p(host.ctypes.data)
    for x, y, o in ((hp, _ptr(xd), _ptr(out)), (_ptr(xd), hp, _ptr(out)),
                    (_ptr(xd), _ptr(xd), C.c_void_p(host_out.ctypes.data))):
        rc = lib.prima_dot_no_alloc(x, y, 1024, 64, o, C.c_void_p(stream.cuda_stream))
        assert rc == cuda.ERR_INVALID_ARGUMENT
        assert b"current device" in lib.prima_last_error()
    stream.synchronize()
    assert out.item() == 7.0
    assert _no_alloc_dot(lib, xd, xd, 64, stream) == 1024.0
