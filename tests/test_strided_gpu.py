"""The HERK branch of quda::stridedBatchGEMMCutlass (lib/cutlass_interface.cu:316-381)
through ftdx_strided_batch_gemm: FP32 interleaved complex input, packed lower
triangle complex64 output, the reference's flop count; other patterns -1.
Default arithmetic: the reference's FP32 -> FP16 -> E4M3 narrowing with FP16
results; opt-in: per-channel-scaled FP8 with FP32 results."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import FtdxError  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
OP_N, OP_T, OP_C = 0, 1, 2
DT_S, DT_C = 0, 2


def _fp16_voltages(seed, batch, n, k):
    # FP16-representable components of magnitude 0.25..4 with full FP16
    # mantissas (so FP16 -> E4M3 rounds), some zeros: every E4M3 product is a
    # multiple of 2^-10 below 16, so FP32 partial sums over k <= 64 are exact
    # and the only roundings are the narrowing and the FP16 results
    rng = np.random.default_rng(seed)
    mag = np.exp2(rng.uniform(-2, 2, size=(batch, n, k, 2)))
    x = (mag * rng.choice([-1.0, 1.0], size=mag.shape)).astype(np.float16)
    x[rng.random(size=x.shape) < 0.05] = 0
    x = x.astype(np.float32)
    return x[..., 0] + 1j * x[..., 1]


@pytest.mark.parametrize("shape", [(300, 64, 3), (129, 17, 2), (1, 1, 1)])
def test_default_is_the_reference_fp16_narrowing_bit_exact(shape):
    n, k, batch = shape
    v = _fp16_voltages(41 + n, batch, n, k).astype(np.complex64)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(batch, n, k, 2)).to(DEV)
    C = torch.full((batch, tri_size(n), 2), float("nan"), device=DEV)
    with Correlator() as c:
        for _ in range(2):  # the second call reuses the staging buffers
            assert c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_C) == \
                8 * n * n * k * batch
            assert np.array_equal(C.cpu().numpy(), oracle.herk_fp16_narrowed(v))


def test_narrowing_rounds_fp32_to_fp16_first():
    # components that FP16 rounds to an E4M3 tie, so the double rounding
    # FP32 -> FP16 -> E4M3 differs from a direct FP32 -> E4M3 rounding
    n, k, batch = 8, 16, 1
    rng = np.random.default_rng(9)
    base = np.float32(1.0625)  # halfway between the E4M3 values 1.0 and 1.125
    x = (base + np.float32(2.0 ** -13)) * rng.choice([-1, 1], size=(batch, n, k, 2))
    x = x.astype(np.float32)  # FP16 rounds the offset away: an exact tie, to even (1.0)
    v = (x[..., 0] + 1j * x[..., 1]).astype(np.complex64)
    A = torch.from_numpy(np.ascontiguousarray(x)).to(DEV)
    C = torch.empty(batch, tri_size(n), 2, device=DEV)
    with Correlator() as c:
        c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_C)
    got = C.cpu().numpy()
    assert np.array_equal(got, oracle.herk_fp16_narrowed(v))
    assert got[0, 0, 0] == 2 * k * 1.0  # |1.0|^2 + |1.0|^2 per sample, not 1.125^2


def test_scaled_fp8_mode_and_other_patterns():
    n, k, batch = 300, 256, 3
    v = oracle.workload4_voltages(21, batch, n, k, rfi_time_frac=0.0)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(batch, n, k, 2)).to(DEV)
    C = torch.full((batch, tri_size(n), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.set_strided_mode(1)
        flops = c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_C)
        assert flops == 8 * n * n * k * batch
        # not a HERK: different B, wrong ops, real data, m != n
        B = A.clone()
        assert c.strided_batch_gemm(A, B, C, n, n, k, OP_C, OP_N, batch, DT_C) == -1
        assert c.strided_batch_gemm(A, A, C, n, n, k, OP_T, OP_N, batch, DT_C) == -1
        assert c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_S) == -1
        assert c.strided_batch_gemm(A, A, C, n, n - 1, k, OP_C, OP_N, batch, DT_C) == -1
        with pytest.raises(FtdxError):
            c.set_strided_mode(7)
    ref = oracle.herk_c128(v.astype(np.complex128), n, k, batch)
    err = oracle.correlation_errors(C.cpu().numpy(), ref, n)
    # FP8 E4M3 with a per-channel scale, FP32 results
    assert err["max_norm"] < 3e-2 and err["rms_norm"] < 3e-3
