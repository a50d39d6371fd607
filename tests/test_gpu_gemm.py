"""The GEMM utility API (compas/utils/gemm.h:7-70): compute_gemm, compute_complex_gemm and the planar
converters, through the C ABI, against numpy in FP64.

result = alpha·lhs·rhsᵀ + beta·result. Tolerances (relative L2 against FP64): Regular and Pedantic
(FP32 on the CUDA cores) 1e-5; Fast (split-BF16 on the tensor cores) 1e-4, also at K = 50176 where
the chunked accumulation matters; bfloat16 inputs 1e-5 against FP64 of the rounded inputs.
Shapes are ragged (no multiple of the 128 x 128 tiles or of the 64-wide K stages)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {"Regular": 1e-5, "Pedantic": 1e-5, "Fast": 1e-4}
SHAPES = [(1, 1, 1), (37, 53, 29), (130, 257, 70), (256, 128, 1100)]


@pytest.fixture(scope="module")
def cb():
    import compas_b200

    compas_b200.library()
    return compas_b200


@pytest.fixture(scope="module")
def ctx(cb):
    return cb.Context(0)


def _rel(a, b):
    a, b = np.asarray(a, np.complex128), np.asarray(b, np.complex128)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("method", ["Regular", "Pedantic", "Fast"])
@pytest.mark.parametrize("shape", SHAPES)
def test_real_gemm(cb, ctx, method, shape):
    m, n, k = shape
    rng = np.random.default_rng(m * 7 + n + k)
    a, b = rng.standard_normal((m, k)).astype(np.float32), rng.standard_normal((n, k)).astype(np.float32)
    c0 = rng.standard_normal((m, n)).astype(np.float32)
    for alpha, beta in ((1.0, 0.0), (1.5, -0.5)):
        out = cb.CompasArray.from_numpy(ctx, c0)
        cb.compute_gemm(ctx, out, cb.CompasArray.from_numpy(ctx, a), cb.CompasArray.from_numpy(ctx, b), alpha, beta,
                        method)
        ref = alpha * (a.astype(np.float64) @ b.astype(np.float64).T) + beta * c0
        assert _rel(out.to_numpy(), ref) < TOL[method], (alpha, beta)


@pytest.mark.parametrize("method", ["Regular", "Fast"])
@pytest.mark.parametrize("shape", SHAPES)
def test_complex_gemm(cb, ctx, method, shape):
    m, n, k = shape
    rng = np.random.default_rng(m + 3 * n + k)
    a = rng.standard_normal((2, m, k)).astype(np.float32)
    b = rng.standard_normal((2, n, k)).astype(np.float32)
    c0 = rng.standard_normal((2, m, n)).astype(np.float32)
    A, B, C0 = (x[0].astype(np.float64) + 1j * x[1] for x in (a, b, c0))
    for alpha, beta in ((1.0, 0.0), (0.75, 2.0)):
        out = cb.CompasArray.from_numpy(ctx, c0)
        cb.compute_complex_gemm(ctx, out, cb.CompasArray.from_numpy(ctx, a), cb.CompasArray.from_numpy(ctx, b), alpha,
                                beta, method)
        got = out.to_numpy()
        ref = alpha * (A @ B.T) + beta * C0
        assert _rel(got[0] + 1j * got[1], ref) < TOL[method], (alpha, beta)


def test_complex_gemm_long_k_fast(cb, ctx):
    # K = 50176 (the voxel contraction of the MR-STAT slice): the two alternating TMEM accumulators
    # keep the split-BF16 result within 1e-4 of FP64
    m, n, k = 64, 48, 50176
    rng = np.random.default_rng(5)
    a = rng.standard_normal((2, m, k)).astype(np.float32)
    b = rng.standard_normal((2, n, k)).astype(np.float32)
    out = cb.CompasArray.from_numpy(ctx, np.zeros((2, m, n), np.float32))
    cb.compute_complex_gemm(ctx, out, cb.CompasArray.from_numpy(ctx, a), cb.CompasArray.from_numpy(ctx, b), 1.0, 0.0,
                            "Fast")
    got = out.to_numpy()
    A, B = (x[0].astype(np.float64) + 1j * x[1] for x in (a, b))
    assert _rel(got[0] + 1j * got[1], A @ B.T) < 1e-4


@pytest.mark.parametrize("cplx", [False, True])
def test_bfloat16_inputs(cb, ctx, cplx):
    m, n, k = 70, 45, 333
    rng = np.random.default_rng(9)
    shape_a, shape_b, shape_c = ((2, m, k), (2, n, k), (2, m, n)) if cplx else ((m, k), (n, k), (m, n))
    a, b = rng.standard_normal(shape_a).astype(np.float32), rng.standard_normal(shape_b).astype(np.float32)
    ab, bb = cb.CompasArray.from_bfloat16(ctx, a), cb.CompasArray.from_bfloat16(ctx, b)
    ar, br = cb.bfloat16_values(ab.to_numpy()).astype(np.float64), cb.bfloat16_values(bb.to_numpy()).astype(np.float64)
    assert np.array_equal(ab.to_numpy(), cb.bfloat16_bits(a))
    out = cb.CompasArray.from_numpy(ctx, np.zeros(shape_c, np.float32))
    if cplx:
        cb.compute_complex_gemm(ctx, out, ab, bb, 1.0, 0.0, "Regular")
        got = out.to_numpy()
        ref = (ar[0] + 1j * ar[1]) @ (br[0] + 1j * br[1]).T
        assert _rel(got[0] + 1j * got[1], ref) < 1e-5
    else:
        cb.compute_gemm(ctx, out, ab, bb, 1.0, 0.0, "Fast")
        assert _rel(out.to_numpy(), ar @ br.T) < 1e-5


def test_planar_converters(cb, ctx):
    rng = np.random.default_rng(3)
    x = (rng.standard_normal((17, 23)) + 1j * rng.standard_normal((17, 23))).astype(np.complex64)
    planar = cb.convert_complex_to_planar(ctx, x)
    p = planar.to_numpy()
    assert p.shape == (2, 17, 23) and np.array_equal(p[0], x.real) and np.array_equal(p[1], x.imag)
    assert np.array_equal(cb.convert_planar_to_complex(ctx, planar).to_numpy(), x)
    pb = cb.convert_complex_to_planar(ctx, x, bfloat16=True).to_numpy()
    assert np.array_equal(pb[0], cb.bfloat16_bits(x.real)) and np.array_equal(pb[1], cb.bfloat16_bits(x.imag))


def test_empty_k_and_shape_errors(cb, ctx):
    c0 = np.arange(12, dtype=np.float32).reshape(3, 4)
    out = cb.CompasArray.from_numpy(ctx, c0)
    z = lambda *s: cb.CompasArray.from_numpy(ctx, np.zeros(s, np.float32))  # noqa: E731
    # k = 0: result = beta·result, and 0 when beta = 0 (result not read)
    for method in ("Regular", "Fast"):
        out = cb.CompasArray.from_numpy(ctx, c0)
        cb.compute_gemm(ctx, out, z(3, 0), z(4, 0), 1.0, 2.0, method)
        assert np.array_equal(out.to_numpy(), 2.0 * c0)
        cb.compute_gemm(ctx, out, z(3, 0), z(4, 0), 1.0, 0.0, method)
        assert not out.to_numpy().any()
    with pytest.raises(cb.CompasError):
        cb.compute_gemm(ctx, out, z(3, 5), z(4, 6), 1.0, 0.0, "Fast")
    with pytest.raises(cb.CompasError):
        cb.compute_complex_gemm(ctx, z(2, 3, 4), z(2, 3, 5), z(2, 5, 5), 1.0, 0.0, "Regular")
