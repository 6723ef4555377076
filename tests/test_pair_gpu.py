"""Parity of the CTA-pair correlator kernel (store_mode 2: one tcgen05
cta_group::2 MMA over two SMs per 256 x 128 tile) with the oracle, through
the C ABI.  QC int4 input is bit-exact as for the single-CTA kernel (every
partial sum is an integer below 2^24); float modes must match the
single-CTA kernel's result."""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import (COMPUTE_FP8, COMPUTE_FP8_SPLIT, IN_FP32, IN_INT4,  # noqa: E402
                           OUT_FP16, OUT_FP32)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


@pytest.fixture(scope="module")
def pair():
    c = Correlator()
    c.set_strategy(2, 0)
    yield c
    assert c.device_status() == 0
    c.close()


def run_qc(corr, qc_np, N, K, B, out=OUT_FP32, alpha=1.0, beta=0.0, C=None):
    qc = torch.from_numpy(np.ascontiguousarray(qc_np).reshape(-1)).to(DEV)
    dt = torch.float32 if out == OUT_FP32 else torch.float16
    if C is None:
        C = torch.full((B, tri_size(N), 2), float("nan"), dtype=dt, device=DEV)
    corr.herk(qc, C, N, K, B, input=IN_INT4, output=out, alpha=alpha, beta=beta, tune=False)
    torch.cuda.synchronize()
    return C


def test_golden_fixtures_bit_exact(pair, golden_dir):
    files = sorted(glob.glob(os.path.join(golden_dir, "*.npz")))
    assert files
    for f in files:
        z = np.load(f)
        N, K, B = int(z["N"]), int(z["K"]), int(z["batch"])
        C = run_qc(pair, z["qc"], N, K, B).cpu().numpy()
        assert np.array_equal(C, z["tri"].astype(np.float32)), os.path.basename(f)


@pytest.mark.parametrize("N,K,B", [(256, 1024, 2), (300, 100, 2), (129, 64, 3), (2, 1, 5),
                                   (257, 96, 3), (384, 63, 1), (513, 200, 1), (640, 384, 2),
                                   (1000, 128, 1)])
def test_ragged_shapes_bit_exact(pair, N, K, B):
    qc = oracle.gaussian_qc(N * 1000 + K + 7, B, N, K)
    C = run_qc(pair, qc, N, K, B).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_adversarial_pm7_bit_exact(pair):
    N, K, B = 512, 2048, 1
    rng = np.random.default_rng(8)
    s = rng.integers(0, 2, size=(2, B, N, K)) * 2 - 1
    qc = oracle.encode_qc(7 * s[0], 7 * s[1])
    C = run_qc(pair, qc, N, K, B).cpu().numpy()
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


@pytest.mark.parametrize("grid", [-1, 2, 7, 1000])
def test_grid_shapes(grid):
    # one pair per tile, a single pair, an odd request (rounded down to 6
    # CTAs) and more than fit (capped at the co-resident pairs)
    N, K, B = 700, 128, 3
    qc = oracle.gaussian_qc(50 + grid, B, N, K)
    with Correlator() as c:
        c.set_strategy(2, grid)
        C = run_qc(c, qc, N, K, B).cpu().numpy()
        assert c.device_status() == 0
    assert np.array_equal(C, oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_fp16_output_and_alpha_beta(pair):
    N, K, B = 520, 128, 2
    qc = oracle.gaussian_qc(11, B, N, K)
    C = run_qc(pair, qc, N, K, B, out=OUT_FP16).cpu().numpy()
    R = oracle.herk_qc(qc, N, K, B)
    assert np.array_equal(C, R.astype(np.float32).astype(np.float16))
    old = torch.randn(B, tri_size(N), 2, device=DEV)
    C = old.clone()
    run_qc(pair, qc, N, K, B, alpha=0.5, beta=-2.0, C=C)
    ref = 0.5 * R.astype(np.float64) - 2.0 * old.double().cpu().numpy()
    np.testing.assert_allclose(C.double().cpu().numpy(), ref, rtol=1e-6, atol=1e-4)


def test_float_modes_match_single_cta():
    B, N, K = 3, 384, 512
    v = oracle.workload4_voltages(77, B, N, K)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    for compute in (COMPUTE_FP8, COMPUTE_FP8_SPLIT):
        outs = []
        for mode in (0, 2):
            C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
            with Correlator() as c:
                c.set_strategy(mode, 0)
                c.herk(A, C, N, K, B, input=IN_FP32, compute=compute, output=OUT_FP32, tune=False)
                assert c.device_status() == 0
            torch.cuda.synchronize()
            outs.append(C.cpu().numpy())
        assert np.isfinite(outs[1]).all()
        np.testing.assert_allclose(outs[1], outs[0], rtol=1e-6, atol=1e-6 * np.abs(outs[0]).max())


def test_kahan_matches_single_cta():
    N, K, B, dumps = 300, 256, 2, 5
    res = []
    for mode in (0, 2):
        S = torch.zeros(B, tri_size(N), 2, device=DEV)
        comp = torch.zeros_like(S)
        with Correlator() as c:
            c.set_strategy(mode, 0)
            for d in range(dumps):
                qc = oracle.gaussian_qc(1000 + d, B, N, K, sigma=5.0)
                c.herk_kahan(torch.from_numpy(qc.reshape(-1)).to(DEV), S, comp, N, K, B,
                             input=IN_INT4, compute=COMPUTE_FP8)
            assert c.device_status() == 0
        torch.cuda.synchronize()
        res.append((S.cpu().numpy(), comp.cpu().numpy()))
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])
    exact = sum(oracle.herk_qc(oracle.gaussian_qc(1000 + d, B, N, K, sigma=5.0), N, K, B)
                for d in range(dumps))
    assert np.array_equal(res[1][0].astype(np.int64), exact)


def test_graph_replay(pair):
    N, K, B = 400, 256, 2
    qc = oracle.gaussian_qc(61, B, N, K)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    pair.set_graph_mode(True)
    try:
        for _ in range(3):
            C.fill_(float("nan"))
            pair.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        assert pair.graph_count() >= 1
    finally:
        pair.set_graph_mode(False)
    torch.cuda.synchronize()
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_dsa2000_scale_spot_rows():
    # 4096 inputs x 64 channels x K = 1024: diagonal of every channel and
    # row blocks of three channels exact
    N, K, B = 4096, 1024, 64
    g = torch.Generator(device=DEV).manual_seed(4)
    re = torch.clamp(torch.round(torch.randn(B, N, K, device=DEV, generator=g) * 2.5), -7, 7)
    im = torch.clamp(torch.round(torch.randn(B, N, K, device=DEV, generator=g) * 2.5), -7, 7)

    def nib(v):
        v = v.to(torch.int32)
        return torch.where(v < 0, 8 | (-v), v)
    qc = ((nib(re) << 4) | nib(im)).to(torch.uint8)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator() as c:
        c.set_strategy(2, 0)
        c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        assert c.device_status() == 0
    idx = torch.arange(N, device=DEV, dtype=torch.int64)
    idx = idx * (idx + 1) // 2 + idx
    assert torch.equal(C[:, idx, 0], (re * re + im * im).sum(-1))
    assert torch.all(C[:, idx, 1] == 0)
    qc_h = qc.cpu().numpy()
    for b, (i0, i1) in [(0, (0, 130)), (63, (3968, 4096)), (17, (2000, 2060)), (30, (255, 260))]:
        ref = oracle.herk_qc_rows(qc_h, N, K, b, i0, i1).astype(np.float32)
        got = C[b, tri_size(i0):tri_size(i1)].cpu().numpy()
        assert np.array_equal(got, ref), (b, i0, i1)


def test_tuner_considers_pair(tmp_path):
    N, K, B = 1024, 512, 4
    qc = oracle.gaussian_qc(90, B, N, K)
    d = torch.from_numpy(qc.reshape(-1)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator(verbosity=2) as c:
        win = c.tune(d, C, N, K, B)
        # 0 direct, 1 bulk, 2 pair, 3 pair + bulk; + 8: the pair on int8
        # operands; 16 the single CTA with the promotion fused in
        assert win["store_mode"] in (0, 1, 2, 3, 10, 11, 16)
        torch.cuda.synchronize()
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
