"""Split-K (K cut into ranges, partial triangles reduced afterwards): bit-exact
for QC input at every split count, with alpha/beta, FP16 output, the CTA-pair
kernel, graph replay and float inputs; and the autotuner picks a split for a
call whose tiles do not fill the GPU."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import COMPUTE_FP8, COMPUTE_FP8_SPLIT, IN_FP32, IN_INT4, OUT_FP16, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def run(qc, N, K, B, splits, mode=0, out=OUT_FP32, alpha=1.0, beta=0.0, C=None):
    dt = torch.float32 if out == OUT_FP32 else torch.float16
    if C is None:
        C = torch.full((B, tri_size(N), 2), float("nan"), dtype=dt, device=DEV)
    with Correlator() as c:
        c.set_strategy(mode, 0, splits=splits)
        c.herk(torch.from_numpy(qc.reshape(-1)).to(DEV), C, N, K, B, input=IN_INT4, output=out,
               alpha=alpha, beta=beta, tune=False)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    return C


@pytest.mark.parametrize("splits", [2, 3, 7, 32])
@pytest.mark.parametrize("N,K,B", [(256, 4096, 1), (130, 1000, 2), (64, 300, 3)])
def test_bit_exact(splits, N, K, B):
    qc = oracle.gaussian_qc(N + K + splits, B, N, K)
    C = run(qc, N, K, B, splits).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_pair_kernel_fp16_alpha_beta():
    N, K, B = 300, 2048, 2
    qc = oracle.gaussian_qc(77, B, N, K)
    R = oracle.herk_qc(qc, N, K, B)
    C = run(qc, N, K, B, 4, mode=2, out=OUT_FP16).cpu().numpy()
    assert np.array_equal(C, R.astype(np.float32).astype(np.float16))
    old = torch.randn(B, tri_size(N), 2, device=DEV)
    C = run(qc, N, K, B, 5, alpha=0.5, beta=2.0, C=old.clone())
    np.testing.assert_allclose(C.double().cpu().numpy(),
                               0.5 * R + 2.0 * old.double().cpu().numpy(), rtol=1e-6, atol=1e-3)


def test_float_inputs_close_to_unsplit():
    B, N, K = 2, 200, 2048
    v = oracle.workload4_voltages(3, B, N, K)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    for compute in (COMPUTE_FP8, COMPUTE_FP8_SPLIT):
        outs = []
        for splits in (1, 4):
            C = torch.empty(B, tri_size(N), 2, device=DEV)
            with Correlator() as c:
                c.set_strategy(0, 0, splits=splits)
                c.herk(A, C, N, K, B, input=IN_FP32, compute=compute, output=OUT_FP32, tune=False)
                assert c.device_status() == 0
            outs.append(C.cpu().numpy())
        # FP32 accumulation in another order: K = 2048 products per element,
        # rounding of order K * 2^-24 relative at worst
        np.testing.assert_allclose(outs[1], outs[0], rtol=2e-4, atol=1e-6 * np.abs(outs[0]).max())


def test_graph_replay_and_tuner_pick():
    N, K, B = 256, 8192, 1          # 3 tiles on 148 SMs: split-K should win
    qc = oracle.gaussian_qc(5, B, N, K)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.tune(d, C, N, K, B)
        assert c.tuned_split_k(N, K, B) > 1
        c.set_graph_mode(True)
        for _ in range(3):
            C.fill_(float("nan"))
            c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=True)
        assert c.graph_count() >= 1
        assert c.device_status() == 0
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
