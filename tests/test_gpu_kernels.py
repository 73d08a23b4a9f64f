"""KernelContractSuite (core/src/test/.../KernelsSuite.scala:19-245) held
against the B200 backend through the C ABI, in both precisions, plus
randomized parity of every seam op against the oracle's ScalaKernels /
Float32Kernels on the same inputs."""
import json
import math
import os

import numpy as np
import pytest

from noaidi_b200.prima import SparseMatrix
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))["kernel_contract"]


def _f(v):
    return [float(t) for t in v]


@pytest.fixture(params=[64, 32], ids=["fp64", "fp32"])
def kernels(request):
    from noaidi_b200.prima.cuda import CudaKernels
    k = CudaKernels(0, request.param)
    yield k
    k.close()


def tol(k):
    return PINS["tolerance"]["fp64" if k.capabilities.supports_float64 else "fp32"]


def down(k, v):
    out = np.zeros(k.length(v))
    k.download(v, out)
    return out


def assert_vec(k, actual, expected):
    assert len(actual) == len(expected)
    for a, e in zip(actual, expected):
        assert abs(a - e) <= tol(k) * max(1.0, abs(e))


def test_round_trip_and_copy_semantics(kernels):
    data = np.array(PINS["round_trip"])
    assert list(down(kernels, kernels.upload(data))) == list(data)
    src = np.array([1.0, 2.0])
    v = kernels.upload(src)
    src[0] = 99.0
    assert down(kernels, v)[0] == 1.0
    assert list(down(kernels, kernels.allocate(5))) == [0.0] * 5


def test_spmv(kernels):
    g = PINS["spmv"]
    m = kernels.upload_matrix(SparseMatrix.from_dense(g["dense"], 3))
    out = kernels.allocate(2)
    kernels.spmv(m, kernels.upload(g["x"]), out)
    assert_vec(kernels, down(kernels, out), g["out"])


def test_axpby_aliased(kernels):
    g = PINS["axpby"]
    x, y, out = kernels.upload(g["x"]), kernels.upload(g["y"]), kernels.allocate(3)
    kernels.axpby(g["alpha"], x, g["beta"], y, out)
    assert_vec(kernels, down(kernels, out), g["out"])
    kernels.axpby(g["alpha"], x, g["beta"], y, y)
    assert_vec(kernels, down(kernels, y), g["out"])


def test_dot_and_norm(kernels):
    g = PINS["dot"]
    x, y = kernels.upload(g["x"]), kernels.upload(g["y"])
    assert abs(kernels.dot(x, y) - g["dot"]) <= tol(kernels)
    assert abs(kernels.squared_norm(x) - g["squared_norm_x"]) <= tol(kernels)
    assert kernels.squared_norm(kernels.allocate(3)) == 0.0


def test_primal_step_box_and_infinite_bounds(kernels):
    for key in ("primal_step_box", "primal_step_inf"):
        g = PINS[key]
        args = [kernels.upload(_f(g[n])) for n in ("x", "kty", "c", "l", "u")]
        out = kernels.allocate(len(g["x"]))
        kernels.primal_step(*args, g["tau"], out)
        assert_vec(kernels, down(kernels, out), g["out"])


def test_dual_step(kernels):
    g = PINS["dual_step"]
    out = kernels.allocate(4)
    kernels.dual_step(kernels.upload(_f(g["y"])), kernels.upload(_f(g["kxbar"])), kernels.upload(g["q"]), g["sigma"],
                      g["neq"], out)
    assert_vec(kernels, down(kernels, out), g["out"])


def test_capabilities(kernels):
    caps = kernels.capabilities
    assert caps.name
    assert caps.requires_double_precision_refinement == (not caps.supports_float64)


def test_fp32_narrowing_and_infinities():
    from noaidi_b200.prima.cuda import CudaKernels
    with CudaKernels(0, 32) as k:
        assert down(k, k.upload([1.0 + 2.0 ** -30]))[0] == 1.0
        v = down(k, k.upload([-math.inf, math.inf, 1e300]))
        assert v[0] == -math.inf and v[1] == math.inf and v[2] == math.inf
    with CudaKernels(0, 64) as k:
        assert down(k, k.upload([1.0 + 2.0 ** -30]))[0] != 1.0


def test_closed_context_is_rejected_and_close_is_idempotent():
    from noaidi_b200.prima.cuda import CudaKernels, PrimaError
    k = CudaKernels(0, 64)
    v = k.upload([1.0])
    k.close()
    k.close()
    with pytest.raises(PrimaError):
        k.length(v)


@pytest.mark.parametrize("precision,mode", [(64, O.FP64), (32, O.FP32)], ids=["fp64", "fp32"])
def test_random_parity_with_the_oracle_ops(precision, mode):
    """Every seam op on seeded random data.  SpMV and the elementwise ops are
    bit-identical to the reference kernels (same per-row order, no FMA);
    reductions agree to reduction-order tolerance."""
    from noaidi_b200.prima.cuda import CudaKernels
    rng = np.random.default_rng(7)
    rows, cols = 3000, 2000
    r = rng.integers(0, rows, 20000)
    c = rng.integers(0, cols, 20000)
    A = SparseMatrix.from_triplets(rows, cols, r, c, rng.standard_normal(20000))
    ops = O.Ops(mode)
    x, y = rng.standard_normal(cols), rng.standard_normal(rows)
    l, u = -rng.uniform(0, 1, cols), rng.uniform(0, 1, cols)
    l[::7], u[::5] = -np.inf, np.inf
    cc, kt = rng.standard_normal(cols), rng.standard_normal(cols)
    with CudaKernels(0, precision) as k:
        ux, uy = ops.upload(x), ops.upload(y)
        dA = k.upload_matrix(A)
        out = k.allocate(rows)
        k.spmv(dA, k.upload(x), out)
        # every row summed in index order: bit-exact in both precisions
        got, want = down(k, out), ops.spmv(A, ux)
        assert np.array_equal(got, want)
        o = k.allocate(cols)
        k.axpby(0.37, k.upload(x), -1.25, k.upload(kt), o)
        assert np.array_equal(down(k, o), ops.axpby(0.37, ux, -1.25, ops.upload(kt)))
        k.scale(0.3, k.upload(x), o)
        assert np.array_equal(down(k, o), ops.scale(0.3, ux))
        k.primal_step(k.upload(x), k.upload(kt), k.upload(cc), k.upload(l), k.upload(u), 0.7, o)
        assert np.array_equal(down(k, o), ops.primal_step(ux, ops.upload(kt), ops.upload(cc), ops.upload(l),
                                                          ops.upload(u), 0.7))
        od = k.allocate(rows)
        q = rng.standard_normal(rows)
        k.dual_step(k.upload(y), k.upload(q), k.upload(y), 0.9, 1000, od)
        assert np.array_equal(down(k, od), ops.dual_step(uy, ops.upload(q), uy, 0.9, 1000))
        d = k.dot(k.upload(x), k.upload(kt))
        assert abs(d - float(np.dot(ux, ops.upload(kt)))) <= 1e-9 * np.abs(ux * ops.upload(kt)).sum()
        assert abs(k.squared_norm(k.upload(x)) - float(ux @ ux)) <= 1e-9 * float(ux @ ux)


@pytest.mark.parametrize("mode,precision", [(O.FP64, 64), (O.FP32, 32)], ids=["fp64", "fp32"])
def test_spmv_bit_exact_on_long_and_short_rows(mode, precision):
    """A matrix whose rows range from empty to 12,000 nonzeros, large enough
    that the seam's autotuner times both of its kernels: every row is the
    reference's index-order sum, whichever kernel the tuner kept and whether
    or not a row's tile fits the kernel's staging area."""
    from noaidi_b200.prima.cuda import CudaKernels
    rng = np.random.default_rng(11)
    rows, cols = 20000, 15000
    lengths = rng.integers(0, 9, rows)
    lengths[[3, 777, 19999]] = [12000, 5000, 4097]
    r = np.repeat(np.arange(rows), lengths)
    c = np.concatenate([rng.choice(cols, size=k, replace=False) for k in lengths])
    A = SparseMatrix.from_triplets(rows, cols, r, c, rng.standard_normal(len(r)))
    ops = O.Ops(mode)
    x = rng.standard_normal(cols)
    with CudaKernels(0, precision) as k:
        dA = k.upload_matrix(A)
        out = k.allocate(rows)
        for _ in range(2):  # twice: the second call reuses the same kernel choice
            k.spmv(dA, k.upload(x), out)
            assert np.array_equal(down(k, out), ops.spmv(A, ops.upload(x)))
