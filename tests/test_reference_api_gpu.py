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
from ftd_b200._lib import IN_FP16, IN_INT4, OUT_FP16, OUT_FP32  # noqa: E402

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


def _ref_call(L, A, R, N, K, B, inp, out, mode, alpha=1.0, beta=0.0):
    with bench._StdoutToStderr():
        h = L.ref_api_create()
        assert h
        try:
            rc = L.ref_api_herk(h, ctypes.c_void_p(A.data_ptr()), ctypes.c_void_p(R.data_ptr()),
                                N, K, B, inp, out, alpha, beta, mode, None)
            torch.cuda.synchronize()
        finally:
            L.ref_api_destroy(h)
    return rc


def _need_api():
    L = bench.load_reference_api()
    if L is None:
        pytest.skip("the reference's API library is not built")
    return L


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reference_api_fp16_output_equals_library(mode):
    # QC input, FP16 packed output (herkBatchedCutlassQC_FP16's form): the
    # exact FP32 sums rounded to FP16 the same way
    L = _need_api()
    N, K, B = 256, 256, 2
    qc = torch.from_numpy(oracle.gaussian_qc(4500, B, N, K).reshape(B, N, K)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), dtype=torch.float16, device=DEV)
    with Correlator() as c:
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP16, tune=False)
    R = torch.full_like(C, float("nan"))
    assert _ref_call(L, qc, R, N, K, B, 1, 0, mode) == 0
    assert torch.equal(R, C)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_reference_api_fp16_input_matches_library(mode):
    # interleaved FP16 input (herkBatchedCutlassFP16's form), unscaled E4M3
    # operands on both sides; the sums of the same exact products differ only
    # by FP32 summation order (measured <= 3.6e-7 of the largest element)
    L = _need_api()
    N, K, B = 256, 256, 2
    rng = np.random.default_rng(4600)
    a = (rng.standard_normal((B, N, K, 2)) * 3.0).astype(np.float16)
    A = torch.from_numpy(a).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk(A, C, N, K, B, input=IN_FP16, output=OUT_FP32, tune=False)
    R = torch.full_like(C, float("nan"))
    assert _ref_call(L, A, R, N, K, B, 0, 1, mode) == 0
    assert float((R - C).abs().max()) <= 2e-6 * float(C.abs().max())


@pytest.mark.parametrize("alpha,beta", [(0.5, -2.0), (1.0, 1.0), (2.0, 0.0)])
def test_reference_api_alpha_beta(alpha, beta):
    # The reference's direct kernel applies alpha and beta exactly as this
    # library (Im(C_ii) zeroed before beta).  Its CUTLASS baseline instead
    # leaves Im(C_ii) = 0 after beta: for a non-Hermitian old C the two
    # reference paths differ there, and only there.
    L = _need_api()
    N, K, B = 256, 256, 2
    qc = torch.from_numpy(oracle.gaussian_qc(4700, B, N, K).reshape(B, N, K)).to(DEV)
    old = torch.randn(B, tri_size(N), 2, device=DEV)
    C = old.clone()
    with Correlator() as c:
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, alpha=alpha, beta=beta, tune=False)
    Rd = old.clone()
    assert _ref_call(L, qc, Rd, N, K, B, 1, 1, 1, alpha, beta) == 0
    assert torch.equal(Rd, C)
    Rb = old.clone()
    assert _ref_call(L, qc, Rb, N, K, B, 1, 1, 2, alpha, beta) == 0
    i = torch.arange(N, device=DEV)
    diag = i * (i + 1) // 2 + i
    want = C.clone()
    want[:, diag, 1] = 0.0
    assert torch.equal(Rb, want)


@pytest.mark.parametrize("cfg", [2, 3, 6])  # GemmOptimal, WideN, SmallTile
def test_reference_baseline_tile_configs_equal_library(cfg):
    # the reference's CUTLASS baseline under each single-CTA-cluster tile
    # configuration its autotuner can choose gives this library's triangles
    L = _need_api()
    N, K, B = 256, 256, 2
    qc = torch.from_numpy(oracle.gaussian_qc(4800, B, N, K).reshape(B, N, K)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
    R = torch.full_like(C, float("nan"))
    with bench._StdoutToStderr():
        h = L.ref_api_create()
        try:
            assert L.ref_api_set_tile_config(h, cfg) == 0
            assert L.ref_api_set_tile_config(h, 4) == -2  # cluster configurations are refused
            assert L.ref_api_set_tile_config(h, cfg) == 0
            rc = L.ref_api_herk(h, ctypes.c_void_p(qc.data_ptr()), ctypes.c_void_p(R.data_ptr()),
                                N, K, B, 1, 1, 1.0, 0.0, 2, None)
            torch.cuda.synchronize()
        finally:
            L.ref_api_destroy(h)
    assert rc == 0 and torch.equal(R, C)
