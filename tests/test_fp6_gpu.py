"""FP6 operand form of the correlator (store modes + 4): QC voltages promoted
to packed E3M2 planes (16 codes per 12 bytes, unpacked by the TMA), the
MMAs reading E3M2 operands.  E3M2 holds every QC value exactly, so the
results must equal the FP8 form and the int64 oracle bit for bit."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError, tri_size  # noqa: E402
from ftd_b200._lib import COMPUTE_FP6, IN_FP32, IN_INT4, OUT_FP16, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
FP6 = 4


def run(qc, N, K, B, store_mode, output=OUT_FP32, alpha=1.0, beta=0.0, C0=None):
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    dt = torch.float32 if output == OUT_FP32 else torch.float16
    C = (torch.full((B, tri_size(N), 2), float("nan"), device=DEV, dtype=dt) if C0 is None
         else torch.from_numpy(C0).to(DEV))
    with Correlator() as c:
        c.set_strategy(store_mode, 0)
        c.herk(d, C, N, K, B, input=IN_INT4, output=output, alpha=alpha, beta=beta, tune=False)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    return C.cpu().numpy()


@pytest.mark.parametrize("store_mode", [0, 1, 2, 3])
@pytest.mark.parametrize("N,K,B", [(160, 256, 3), (130, 100, 2), (300, 1000, 2), (640, 96, 2)])
def test_fp6_bit_exact(store_mode, N, K, B):
    qc = oracle.gaussian_qc(600 + N + K + store_mode, B, N, K, sigma=3.0)
    want = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    got = run(qc, N, K, B, store_mode + FP6)
    assert np.array_equal(got, want)


def test_fp6_full_scale_values():
    # every QC code, including -0 and the extremes +-7, in both components
    N, K, B = 256, 512, 2
    rng = np.random.default_rng(61)
    qc = rng.integers(0, 256, size=(B, N, K), dtype=np.uint8)
    want = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    for mode in (0 + FP6, 2 + FP6):
        assert np.array_equal(run(qc, N, K, B, mode), want)


def test_fp6_alpha_beta_fp16_equal_fp8_form():
    N, K, B = 200, 320, 2
    qc = oracle.gaussian_qc(62, B, N, K)
    rng = np.random.default_rng(63)
    C0 = rng.normal(size=(B, tri_size(N), 2)).astype(np.float32)
    for mode in (0, 2):
        a = run(qc, N, K, B, mode, alpha=0.5, beta=2.0, C0=C0)
        b = run(qc, N, K, B, mode + FP6, alpha=0.5, beta=2.0, C0=C0)
        assert np.array_equal(a, b)
        h8 = run(qc, N, K, B, mode, output=OUT_FP16)
        h6 = run(qc, N, K, B, mode + FP6, output=OUT_FP16)
        assert np.array_equal(h8, h6)


def test_fp6_ignored_for_float_input():
    # FP32 input cannot take the E3M2 form; the strategy falls back to E4M3
    N, K, B = 130, 128, 2
    rng = np.random.default_rng(64)
    v = (rng.normal(size=(B, N, K, 2))).astype(np.float32)
    A = torch.from_numpy(v).to(DEV)
    outs = []
    for mode in (2, 2 + FP6):
        C = torch.empty(B, tri_size(N), 2, device=DEV)
        with Correlator() as c:
            c.set_strategy(mode, 0)
            c.herk(A, C, N, K, B, input=IN_FP32, output=OUT_FP32, tune=False)
            assert c.device_status() == 0
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_compute_fp6_int4_exact_and_float_refused():
    # ComputePrecision::FP6 on INT4 input runs the E3M2 operand form (exact)
    N, K, B = 192, 256, 2
    qc = oracle.gaussian_qc(65, B, N, K)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk(d, C, N, K, B, input=IN_INT4, compute=COMPUTE_FP6, output=OUT_FP32)
        assert c.device_status() == 0
        torch.cuda.synchronize()
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
        A = torch.zeros(B, N, K, 2, device=DEV)
        with pytest.raises(FtdxError):
            c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP6, output=OUT_FP32)


# ------------------------------------------------ signed 8-bit operands
S8_PAIR = 2 + 8  # CTA-pair kernel with kind::i8 MMAs and S32 accumulators


@pytest.mark.parametrize("N,K,B", [(160, 256, 3), (130, 100, 2), (300, 1000, 2)])
def test_s8_pair_bit_exact(N, K, B):
    qc = oracle.gaussian_qc(700 + N + K, B, N, K, sigma=3.0)
    want = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    assert np.array_equal(run(qc, N, K, B, S8_PAIR), want)


def test_s8_pair_all_codes_alpha_beta_fp16():
    N, K, B = 256, 512, 2
    rng = np.random.default_rng(71)
    qc = rng.integers(0, 256, size=(B, N, K), dtype=np.uint8)
    assert np.array_equal(run(qc, N, K, B, S8_PAIR),
                          oracle.herk_qc(qc, N, K, B).astype(np.float32))
    C0 = rng.normal(size=(B, tri_size(N), 2)).astype(np.float32)
    assert np.array_equal(run(qc, N, K, B, 2, alpha=0.5, beta=2.0, C0=C0),
                          run(qc, N, K, B, S8_PAIR, alpha=0.5, beta=2.0, C0=C0))
    assert np.array_equal(run(qc, N, K, B, 2, output=OUT_FP16),
                          run(qc, N, K, B, S8_PAIR, output=OUT_FP16))


@pytest.mark.parametrize("N,K,B", [(1, 1, 1), (7, 3, 2), (129, 17, 1), (257, 129, 2)])
@pytest.mark.parametrize("store_mode", [0 + FP6, 2 + FP6, S8_PAIR])
def test_operand_forms_edge_sizes(N, K, B, store_mode):
    qc = oracle.gaussian_qc(800 + N + K, B, N, K, sigma=3.0)
    assert np.array_equal(run(qc, N, K, B, store_mode), oracle.herk_qc(qc, N, K, B).astype(np.float32))


# ------------------------------------------------ CTA pair with bulk-copy stores
@pytest.mark.parametrize("mode", [3, 3 + 8])
@pytest.mark.parametrize("N,K,B", [(640, 192, 2), (1000, 130, 1), (300, 64, 3)])
def test_pair_bulk_stores_bit_exact(mode, N, K, B):
    # store mode 3: interior tiles (all 128 columns of a CTA below every row,
    # rows inside n) leave through shared memory and one bulk copy per row;
    # the others through the direct / sector path; 3 + 8 on int8 operands
    qc = oracle.gaussian_qc(1000 + N + K + mode, B, N, K, sigma=3.0)
    want = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    assert np.array_equal(run(qc, N, K, B, mode), want)


def test_pair_bulk_stores_fall_back_for_alpha_fp16():
    N, K, B = 640, 128, 2
    qc = oracle.gaussian_qc(1100, B, N, K)
    assert np.array_equal(run(qc, N, K, B, 2, alpha=0.5), run(qc, N, K, B, 3, alpha=0.5))
    assert np.array_equal(run(qc, N, K, B, 2, output=OUT_FP16), run(qc, N, K, B, 3, output=OUT_FP16))


@pytest.mark.parametrize("mode", [1, 3, 10, 11])
def test_strategies_under_graph_replay(mode):
    # the bench replays the tuned strategy as a captured CUDA graph: every
    # store mode / operand form stays bit-exact across replays
    N, K, B = 640, 256, 3
    qc = oracle.gaussian_qc(1200 + mode, B, N, K)
    want = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator() as c:
        c.set_strategy(mode, 0)
        c.init_herk(N, K, B)
        c.set_graph_mode(True)
        for _ in range(3):
            C.fill_(float("nan"))
            c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
            torch.cuda.synchronize()
            assert np.array_equal(C.cpu().numpy(), want)
        assert c.graph_count() >= 1 and c.device_status() == 0


@pytest.mark.parametrize("bad", [-1, 9, 12, 13, 14, 15, 17, 18, 20, 24, 32, 2 + 8 + 4])
def test_invalid_store_modes_refused(bad):
    # 8 (int8 operands) only with the pair modes 2 / 3, never with 4 (FP6);
    # 16 (fused promotion) only alone; no bits above 16
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.set_strategy(bad, 0)


def test_fp6_compute_with_kahan_refused():
    N, K, B = 64, 32, 1
    qc = oracle.gaussian_qc(1300, B, N, K)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    S = torch.zeros(B, tri_size(N), 2, device=DEV)
    comp = torch.zeros_like(S)
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.herk_kahan(d, S, comp, N, K, B, input=IN_INT4, compute=COMPUTE_FP6)
