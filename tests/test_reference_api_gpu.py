"""The reference's own GPU HERK API (cutlass_gemm_api::CutlassComplexGemm::herk,
built unmodified from the reference's sources by baseline/build_cutlass_ref.sh)
and this library give identical packed triangles on the same QC input, in each
of the reference's dispatch modes: its default (K-adaptive), its direct kernel
and its CUTLASS tcgen05 sub-GEMM baseline.  All of them sum exact integer
products in FP32, so the comparison is bit-exact; the oracle pins both.
The reference's CUTLASS GEMMs need K a multiple of 16 (for K = 200 its
can_implement fails with status 11, and its default dispatch takes that
path), so the ragged case uses K = 208."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import bench  # noqa: E402
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import IN_INT4, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("N,K,B", [(256, 256, 3), (300, 208, 2), (1024, 1024, 2)])
@pytest.mark.parametrize("mode", [0, 1, 2])  # Auto, ForceDirect, ForceBaseline
def test_reference_api_equals_library(N, K, B, mode):
    L = bench.load_reference_api()
    if L is None:
        pytest.skip("the reference's API library is not built")
    qc_np = oracle.gaussian_qc(4400 + N + K, B, N, K)
    qc = torch.from_numpy(qc_np.reshape(B, N, K)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
    torch.cuda.synchronize()
    R = torch.full_like(C, float("nan"))
    with bench._StdoutToStderr():
        h = L.ref_api_create()
        assert h
        try:
            rc = L.ref_api_herk_qc_fp32(h, ctypes.c_void_p(qc.data_ptr()),
                                        ctypes.c_void_p(R.data_ptr()), N, K, B, mode, None)
            torch.cuda.synchronize()
        finally:
            L.ref_api_destroy(h)
    assert rc == 0
    assert torch.equal(R, C)
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc_np, N, K, B).astype(np.float32))
