"""The reference's own Blackwell direct HERK kernel (herk_direct_fp8_precast_kernel
with its INT4 -> FP8 cast, built from the reference's sources by
baseline/build_direct_ref.sh) and this library give identical triangles on
the same QC input: both sum exact integer products in FP32."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
import bench  # noqa: E402
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import IN_INT4, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.mark.parametrize("N,K,B", [(96, 64, 2), (300, 256, 3)])
def test_reference_direct_kernel_equals_library(N, K, B):
    if bench.load_reference_direct() is None:
        pytest.skip("reference direct kernel not built")
    qc_np = oracle.gaussian_qc(77 + N, B, N, K)
    qc = torch.from_numpy(qc_np.reshape(B, N, K)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator() as c:
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
    torch.cuda.synchronize()
    out = bench.run_reference_direct_leg(torch, torch.device(DEV), qc, C, N, K, B, steps=3)
    assert out is not None and out["bit_exact_vs_library"]
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc_np, N, K, B).astype(np.float32))
