"""The HERK branch of quda::stridedBatchGEMMCutlass (lib/cutlass_interface.cu:316-381)
through ftdx_strided_batch_gemm: FP32 interleaved complex input, packed lower
triangle complex64 output, the reference's flop count; other patterns -1."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
OP_N, OP_T, OP_C = 0, 1, 2
DT_S, DT_C = 0, 2


def test_herk_pattern():
    n, k, batch = 300, 256, 3
    v = oracle.workload4_voltages(21, batch, n, k, rfi_time_frac=0.0)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(batch, n, k, 2)).to(DEV)
    C = torch.full((batch, tri_size(n), 2), float("nan"), device=DEV)
    with Correlator() as c:
        flops = c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_C)
        assert flops == 8 * n * n * k * batch
        # not a HERK: different B, wrong ops, real data, m != n
        B = A.clone()
        assert c.strided_batch_gemm(A, B, C, n, n, k, OP_C, OP_N, batch, DT_C) == -1
        assert c.strided_batch_gemm(A, A, C, n, n, k, OP_T, OP_N, batch, DT_C) == -1
        assert c.strided_batch_gemm(A, A, C, n, n, k, OP_C, OP_N, batch, DT_S) == -1
        assert c.strided_batch_gemm(A, A, C, n, n - 1, k, OP_C, OP_N, batch, DT_C) == -1
    ref = oracle.herk_c128(v.astype(np.complex128), n, k, batch)
    err = oracle.correlation_errors(C.cpu().numpy(), ref, n)
    # FP8 E4M3 with a per-channel scale (the reference narrows to unscaled FP16 -> FP8)
    assert err["max_norm"] < 3e-2 and err["rms_norm"] < 3e-3
