"""Correlation straight from raw packet-ordered QC voltages (ftdx_herk_ftd:
corner turn fused into the promotion pass) against the oracle's corner turn +
int64 HERK and the reference's cpu_herk_ftd fixtures.  Bit-exact."""
import glob
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError, tri_size  # noqa: E402
from ftd_b200._lib import (LAYOUT_CHAN_POL_ANT_TIME, LAYOUT_TIME_ANT_CHAN_POL,  # noqa: E402
                           OUT_FP16, OUT_FP32)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
LAYOUTS = (LAYOUT_TIME_ANT_CHAN_POL, LAYOUT_CHAN_POL_ANT_TIME)


@pytest.fixture(scope="module")
def corr():
    c = Correlator()
    yield c
    assert c.device_status() == 0
    c.close()


def expected(raw, a, c, p, t, ti, layout, pol_sum):
    bf = oracle.ftd_to_batch_first(raw, a, c, p, t, ti, layout, pol_sum)
    return oracle.herk_qc(bf, a, bf.shape[2], bf.shape[0]).astype(np.float32)


def run(corr, raw, a, c, p, t, ti, layout, pol_sum=False, out=OUT_FP32, **kw):
    nb = c * ti * (1 if pol_sum else p)
    dt = torch.float32 if out == OUT_FP32 else torch.float16
    C = torch.full((nb, tri_size(a), 2), float("nan"), dtype=dt, device=DEV)
    d = torch.from_numpy(np.ascontiguousarray(raw)).to(DEV)
    corr.herk_ftd(d, C, a, c, p, t, ti, layout=layout, pol_sum=pol_sum, output=out, **kw)
    torch.cuda.synchronize()
    return C


def test_reference_fixtures_bit_exact(corr, golden_dir):
    files = sorted(glob.glob(os.path.join(golden_dir, "ftd", "*.npz")))
    assert files
    for f in files:
        z = np.load(f)
        a, c, p = int(z["n_ant"]), int(z["n_chan"]), int(z["n_pol"])
        ti, t = int(z["n_time_inner"]), int(z["n_time"])
        C = run(corr, z["raw"], a, c, p, t, ti, LAYOUT_TIME_ANT_CHAN_POL).cpu().numpy()
        assert np.array_equal(C, z["tri"].astype(np.float32)), os.path.basename(f)


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("pol_sum", [False, True])
@pytest.mark.parametrize("a,c,p,ti,K", [(130, 3, 2, 2, 96), (64, 2, 2, 1, 256), (257, 1, 2, 3, 61),
                                         (7, 5, 1, 4, 17), (200, 2, 3, 1, 130)])
def test_layouts_bit_exact(corr, layout, pol_sum, a, c, p, ti, K):
    t = ti * K
    rng = np.random.default_rng(a * 1000 + K + layout)
    re, im = oracle.gaussian_int4(rng, (t * a * c * p,))
    raw = oracle.encode_qc(re, im)
    C = run(corr, raw, a, c, p, t, ti, layout, pol_sum).cpu().numpy()
    assert np.array_equal(C, expected(raw, a, c, p, t, ti, layout, pol_sum))


@pytest.mark.parametrize("layout", LAYOUTS)
def test_pair_kernel_and_unaligned_rows(layout):
    # CTA-pair strategy (third operand plane written by the corner turn) and a
    # time-slice length that is not a multiple of 4 bytes
    a, c, p, ti, K = 301, 3, 1, 2, 77
    t = ti * K
    raw = np.random.default_rng(9).integers(0, 256, size=t * a * c * p, dtype=np.uint8)
    with Correlator() as cp:
        cp.set_strategy(2, 0)
        C = run(cp, raw, a, c, p, t, ti, layout, True).cpu().numpy()
        assert cp.device_status() == 0
    assert np.array_equal(C, expected(raw, a, c, p, t, ti, layout, True))


def test_fp16_output_alpha_beta(corr):
    a, c, p, ti, K = 96, 2, 2, 2, 64
    t = ti * K
    raw = oracle.encode_qc(*oracle.gaussian_int4(np.random.default_rng(12), (t * a * c * p,)))
    R = expected(raw, a, c, p, t, ti, LAYOUT_TIME_ANT_CHAN_POL, False)
    C = run(corr, raw, a, c, p, t, ti, LAYOUT_TIME_ANT_CHAN_POL, out=OUT_FP16).cpu().numpy()
    assert np.array_equal(C, R.astype(np.float16))
    old = torch.randn(c * p * ti, tri_size(a), 2, device=DEV)
    C = old.clone()
    corr.herk_ftd(torch.from_numpy(raw).to(DEV), C, a, c, p, t, ti, alpha=2.0, beta=0.5)
    torch.cuda.synchronize()
    np.testing.assert_allclose(C.double().cpu().numpy(),
                               2.0 * R.astype(np.float64) + 0.5 * old.double().cpu().numpy(),
                               rtol=1e-6, atol=1e-4)


def test_bad_geometry_rejected(corr):
    d = torch.zeros(1000, dtype=torch.uint8, device=DEV)
    C = torch.empty(10, 2, device=DEV)
    with pytest.raises(FtdxError):
        corr.herk_ftd(d, C, 4, 1, 1, 10, 3)          # n_time not a multiple of n_time_inner
    with pytest.raises(FtdxError):
        corr.herk_ftd(d, C, 0, 1, 1, 10, 1)
    with pytest.raises(FtdxError):
        corr.herk_ftd(d, C, 4, 1, 1, 10, 1, layout=7)
    assert corr.device_status() == 0
