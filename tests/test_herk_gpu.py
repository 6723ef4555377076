"""Parity of the tcgen05 correlator (through the C ABI) with the oracle.

QC int4 input with alpha = 1, beta = 0 must be bit-exact: every product of
two E4M3-encoded integers in [-7, 7] is exact, and every partial sum is an
integer below 2^24, so FP32 accumulation loses nothing.
"""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, herk_batched_cutlass_qc, tri_size  # noqa: E402
from ftd_b200._lib import IN_FP16, IN_INT4, OUT_FP16, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module")
def corr():
    c = Correlator()
    yield c
    assert c.device_status() == 0
    c.close()


def run_qc(corr, qc_np, N, K, B, out=OUT_FP32, alpha=1.0, beta=0.0, C=None):
    qc = torch.from_numpy(np.ascontiguousarray(qc_np).reshape(-1)).to(DEV)
    dt = torch.float32 if out == OUT_FP32 else torch.float16
    if C is None:
        C = torch.full((B, tri_size(N), 2), float("nan"), dtype=dt, device=DEV)
    corr.herk(qc, C, N, K, B, input=IN_INT4, output=out, alpha=alpha, beta=beta)
    torch.cuda.synchronize()
    return C


def test_golden_fixtures_bit_exact(corr, golden_dir):
    files = sorted(glob.glob(os.path.join(golden_dir, "*.npz")))
    assert files
    for f in files:
        z = np.load(f)
        N, K, B = int(z["N"]), int(z["K"]), int(z["batch"])
        C = run_qc(corr, z["qc"], N, K, B).cpu().numpy()
        ref = z["tri"].astype(np.float32)
        assert np.array_equal(C, ref), os.path.basename(f)


def test_small_config_bit_exact(corr):
    # 64 antennas x 2 pol = 128 inputs, 32 channels, K = 256, Gaussian sigma 2.5
    N, K, B = 128, 256, 32
    qc = oracle.gaussian_qc(1, B, N, K)
    C = run_qc(corr, qc, N, K, B).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


@pytest.mark.parametrize("N,K,B", [(256, 1024, 2), (300, 100, 2), (129, 64, 3), (2, 1, 5), (257, 96, 3),
                                   (384, 63, 1), (513, 200, 1)])
def test_ragged_shapes_bit_exact(corr, N, K, B):
    qc = oracle.gaussian_qc(N * 1000 + K, B, N, K)
    C = run_qc(corr, qc, N, K, B).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_adversarial_pm7_long_k_bit_exact(corr):
    # all samples +-7: |R| up to 98 K = 200704 at K = 2048, still < 2^24
    N, K, B = 256, 2048, 1
    rng = np.random.default_rng(7)
    s = rng.integers(0, 2, size=(2, B, N, K)) * 2 - 1
    qc = oracle.encode_qc(7 * s[0], 7 * s[1])
    C = run_qc(corr, qc, N, K, B).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))
    # all +7: every element equals 98 K exactly
    qc = oracle.encode_qc(np.full((B, N, K), 7), np.full((B, N, K), 7))
    C = run_qc(corr, qc, N, K, B).cpu().numpy()
    assert np.all(C[..., 0] == 98.0 * K) and np.all(C[..., 1] == 0.0)


def test_fp16_output(corr):
    N, K, B = 200, 128, 2
    qc = oracle.gaussian_qc(11, B, N, K)
    C = run_qc(corr, qc, N, K, B, out=OUT_FP16).cpu().numpy()
    ref = oracle.herk_qc(qc, N, K, B).astype(np.float32).astype(np.float16)
    assert np.array_equal(C, ref)


def test_alpha_beta(corr):
    N, K, B = 160, 96, 2
    qc = oracle.gaussian_qc(12, B, N, K)
    old = torch.randn(B, tri_size(N), 2, device=DEV)
    C = old.clone()
    run_qc(corr, qc, N, K, B, alpha=0.5, beta=-2.0, C=C)
    R = oracle.herk_qc(qc, N, K, B).astype(np.float64)
    ref = 0.5 * R + (-2.0) * old.double().cpu().numpy()
    # Im of the diagonal is zeroed before beta is applied (reference store rule)
    got = C.double().cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-4)


def test_fp16_input(corr):
    # interleaved FP16 complex input, E4M3 conversion with saturation at 448
    N, K, B = 130, 80, 2
    rng = np.random.default_rng(13)
    a = (rng.uniform(-0.5, 0.5, (B, N, K)) + 1j * rng.uniform(-0.5, 0.5, (B, N, K)))
    a16 = np.stack([a.real, a.imag], -1).astype(np.float16)
    A = torch.from_numpy(a16).to(DEV)
    C = torch.empty(B, tri_size(N), 2, dtype=torch.float16, device=DEV)
    corr.herk(A, C, N, K, B, input=IN_FP16, output=OUT_FP16)
    torch.cuda.synchronize()
    # oracle on the E4M3-quantised input (torch's float8_e4m3fn rounds to nearest-even)
    q = torch.from_numpy(a16.astype(np.float32)).to(torch.float8_e4m3fn).to(torch.float64).numpy()
    ref = oracle.herk_c128(q[..., 0] + 1j * q[..., 1], N, K, B)
    np.testing.assert_allclose(C.double().cpu().numpy(), ref, rtol=2e-3, atol=2e-2)


# None: the autotuner's choice on this GPU; then every strategy it can pick
# for QC input: 1 single CTA + bulk stores, 2 CTA pair, 3 pair + bulk stores,
# 10 / 11 the pair on int8 operands, 16 promotion fused into the single CTA
@pytest.mark.parametrize("strategy", [None, 1, 2, 3, 10, 11, 16])
def test_dsa2000_scale_spot_rows(strategy):
    # 4096 inputs x 64 channels x K = 1024 (the DSA-2000 configuration): full
    # output on the GPU, exact check of two whole channels, of row blocks in
    # three more and of the whole diagonal (sum |v|^2) of every channel.
    N, K, B = 4096, 1024, 64
    g = torch.Generator(device=DEV).manual_seed(3)
    re = torch.clamp(torch.round(torch.randn(B, N, K, device=DEV, generator=g) * 2.5), -7, 7)
    im = torch.clamp(torch.round(torch.randn(B, N, K, device=DEV, generator=g) * 2.5), -7, 7)
    def nib(v):
        v = v.to(torch.int32)
        return torch.where(v < 0, 8 | (-v), v)
    qc = ((nib(re) << 4) | nib(im)).to(torch.uint8)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    C.fill_(float("nan"))
    with Correlator() as c:
        if strategy is not None:
            c.set_strategy(strategy, 0)
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=strategy is None)
        assert c.device_status() == 0
    assert not torch.isnan(C).any()
    diag_idx = torch.arange(N, device=DEV, dtype=torch.int64)
    diag_idx = diag_idx * (diag_idx + 1) // 2 + diag_idx
    power = (re * re + im * im).sum(-1)
    assert torch.equal(C[:, diag_idx, 0], power)
    assert torch.all(C[:, diag_idx, 1] == 0)
    qc_h = qc.cpu().numpy()
    for b, (i0, i1) in [(0, (0, 130)), (63, (3968, 4096)), (17, (2000, 2060))]:
        ref = oracle.herk_qc_rows(qc_h, N, K, b, i0, i1).astype(np.float32)
        got = C[b, tri_size(i0):tri_size(i1)].cpu().numpy()
        assert np.array_equal(got, ref), (b, i0, i1)
    # two whole channels, all 8,390,656 elements of each, against the int64 oracle
    for b in (5, 40):
        ref = oracle.herk_qc(np.ascontiguousarray(qc_h[b:b + 1]), N, K, 1)[0].astype(np.float32)
        assert np.array_equal(C[b].cpu().numpy(), ref), b


def test_ggp_entry_point(corr):
    N, K, B = 96, 64, 3
    qc_np = oracle.gaussian_qc(21, B, N, K)
    qc = torch.from_numpy(qc_np.reshape(-1)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    assert herk_batched_cutlass_qc(qc, C, N, K, B) == 0
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc_np, N, K, B).astype(np.float32))


# Promotion fused into the correlator (strategy 16): raw QC tiles by TMA,
# converted to E4M3 in shared memory.  Bit-exact against the oracle, over
# ragged N (partial tiles, channel rows running into the next channel's),
# K tails that are multiples of 16 but not of 128 (zeros from the TMA past K),
# K = 16, alpha / beta, FP16 output, split-K; and calls it cannot take (K not
# a multiple of 16, A not 16-byte aligned) run the two-pass path and stay exact.
@pytest.mark.parametrize("N,K,B", [(200, 208, 3), (128, 1024, 2), (300, 16, 2), (64, 48, 5),
                                   (260, 100, 2), (1, 16, 3), (129, 2048, 1)])
def test_fused_promotion_exact(N, K, B):
    qc = oracle.gaussian_qc(4000 + N + K, B, N, K)
    ref = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    with Correlator() as c:
        c.set_strategy(16, 0)
        got = run_qc(c, qc, N, K, B).cpu().numpy()
        assert c.device_status() == 0
    assert np.array_equal(got, ref)


def test_fused_promotion_options():
    N, K, B = 192, 320, 3
    qc = oracle.gaussian_qc(4100, B, N, K)
    ref = oracle.herk_qc(qc, N, K, B)
    with Correlator() as c:
        c.set_strategy(16, 0)
        # FP16 output: the FP32 result rounded to nearest
        h = run_qc(c, qc, N, K, B, out=OUT_FP16).cpu().numpy()
        assert np.array_equal(h, ref.astype(np.float32).astype(np.float16))
        # alpha and beta
        old = torch.randn(B, tri_size(N), 2, device=DEV)
        C = old.clone()
        run_qc(c, qc, N, K, B, alpha=0.5, beta=-2.0, C=C)
        want = 0.5 * ref.astype(np.float64) + (-2.0) * old.double().cpu().numpy()
        np.testing.assert_allclose(C.double().cpu().numpy(), want, rtol=1e-6, atol=1e-4)
        # split-K into 3 ranges, exact
        c.set_strategy(16, 0, splits=3)
        got = run_qc(c, qc, N, K, B).cpu().numpy()
        assert np.array_equal(got, ref.astype(np.float32))
        assert c.device_status() == 0


def test_fused_promotion_falls_back_when_misaligned():
    N, K, B = 96, 64, 2
    qc = oracle.gaussian_qc(4200, B, N, K)
    buf = torch.zeros(qc.size + 16, dtype=torch.uint8, device=DEV)
    A = buf[1:1 + qc.size]  # 1 byte past a 16-byte boundary
    A.copy_(torch.from_numpy(qc.reshape(-1)).to(DEV))
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.set_strategy(16, 0)
        c.herk(A, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        torch.cuda.synchronize()
        assert c.device_status() == 0
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_fused_promotion_kahan_and_graph_replay():
    # Kahan accumulation over three dumps, and graph replay with new voltages
    # in the same buffers: the fused kernel reads the QC bytes at every replay.
    N, K, B = 256, 192, 2
    dumps = [oracle.gaussian_qc(4300 + i, B, N, K) for i in range(3)]
    want = sum(oracle.herk_qc(q, N, K, B) for q in dumps).astype(np.float32)
    with Correlator() as c:
        c.set_strategy(16, 0)
        S = torch.zeros(B, tri_size(N), 2, device=DEV)
        comp = torch.zeros_like(S)
        for q in dumps:
            c.herk_kahan(torch.from_numpy(q.reshape(-1)).to(DEV), S, comp, N, K, B,
                         input=IN_INT4)
        torch.cuda.synchronize()
        assert np.array_equal(S.cpu().numpy(), want)
        c.set_graph_mode(True)
        A = torch.empty(B * N * K, dtype=torch.uint8, device=DEV)
        C = torch.empty(B, tri_size(N), 2, device=DEV)
        for q in dumps:
            A.copy_(torch.from_numpy(q.reshape(-1)).to(DEV))
            C.fill_(float("nan"))
            c.herk(A, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
            torch.cuda.synchronize()
            assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(q, N, K, B).astype(np.float32))
        assert c.graph_count() >= 1 and c.device_status() == 0
