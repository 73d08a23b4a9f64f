"""The C ABI: libprima_cuda.so builds for sm_100a, loads, and exports every
symbol include/*.h declares, with the binding's signatures.  No
compute calls (these run without a GPU)."""
import ctypes
import os
import re

import pytest

from noaidi_b200 import build as B
from noaidi_b200.prima import cuda

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_functions():
    names = set()
    for header in sorted(os.listdir(INCLUDE)):
        if header.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(INCLUDE, header)).read(), flags=re.S)
            names |= set(re.findall(r"\b(prima_[a-z_0-9]+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    path = B.build()
    return ctypes.CDLL(path)


def test_library_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 20
    for name in sorted(names):
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_binding_covers_the_header():
    assert declared_functions() == set(cuda.SIGNATURES)


def test_library_is_sm_100a_native():
    # the build line targets sm_100a only; no other architecture, no PTX for JIT
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_open_without_a_device_fails_loudly(lib):
    if os.environ.get("CUDA_VISIBLE_DEVICES") is None:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    h = ctypes.c_int64()
    rc = lib.prima_open(0, 64, ctypes.byref(h))
    assert rc == cuda.ERR_NO_DEVICE


def test_defaults_match_the_reference(lib):
    p = cuda.CParams()
    lib.prima_params_default(ctypes.byref(p))
    assert (p.eps_abs, p.eps_rel, p.max_iterations, p.evaluation_frequency) == (1e-8, 1e-8, 100000, 64)
    assert (p.ruiz_iterations, p.apply_pock_chambolle, p.pock_chambolle_alpha) == (10, 1, 1.0)
    assert (p.restart_sufficient_reduction, p.restart_necessary_reduction, p.restart_artificial_fraction,
            p.primal_weight_smoothing, p.infeasibility_tolerance) == (0.2, 0.8, 0.36, 0.5, 1e-8)
    assert p.time_limit_ms < 0
    m = cuda.CMixedParams()
    lib.prima_mixed_params_default(ctypes.byref(m))
    assert (m.reduced_tolerance, m.reduced_max_iterations, m.always_refine, m.reduced_time_share) == \
        (1e-5, 20000, 0, 0.5)
