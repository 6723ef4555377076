"""Uneven-K, antenna-flagged channels in one launch (ftdx_herk_batched_v):
every channel bit-exact against the oracle on its gathered active rows."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import OUT_FP16, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def make_channels(rng, specs):
    """specs: (rows, n_active or None, K, lda_pad) -> host and device descriptors."""
    chans, host = [], []
    for rows, n_act, K, pad in specs:
        lda = K + pad
        re, im = oracle.gaussian_int4(rng, (rows, lda))
        block = oracle.encode_qc(re, im)
        if n_act is None:
            active = None
            rows_used = np.arange(min(rows, rows))
            n = rows
        else:
            active = np.sort(rng.choice(rows, size=n_act, replace=False)).astype(np.int32)
            rows_used = active
            n = n_act
        dA = torch.from_numpy(block.reshape(-1)).to(DEV)
        dC = torch.full((tri_size(n), 2), float("nan"), device=DEV)
        dact = torch.from_numpy(active).to(DEV) if active is not None else None
        chans.append({"A": dA, "C": dC, "n_inputs": n, "K": K, "lda": lda, "active": dact})
        host.append((block, rows_used, n, K))
    return chans, host


def expected(block, rows_used, n, K):
    qc = np.ascontiguousarray(block[rows_used][:, :K]).reshape(1, n, K)
    return oracle.herk_qc(qc, n, K, 1)[0].astype(np.float32)


def check(chans, host):
    torch.cuda.synchronize()
    for ch, hb in zip(chans, host):
        assert np.array_equal(ch["C"].cpu().numpy(), expected(*hb)), (ch["n_inputs"], ch["K"])


def test_uneven_flagged_small():
    rng = np.random.default_rng(70)
    specs = [(1, None, 1, 0), (200, 130, 64, 16), (300, 257, 200, 3), (64, None, 1000, 0),
             (310, 300, 2048, 0), (129, 129, 65, 7), (500, 17, 130, 0)]
    chans, host = make_channels(rng, specs)
    with Correlator() as c:
        c.herk_batched_v(chans, output=OUT_FP32)
        assert c.device_status() == 0
    check(chans, host)


def test_uneven_flagged_medium_tuned_and_graph():
    rng = np.random.default_rng(71)
    specs = []
    for _ in range(12):
        K = int(rng.integers(2, 33)) * 64
        n = int(rng.integers(300, 700))
        specs.append((768, n, K, 0))
    chans, host = make_channels(rng, specs)
    with Correlator() as c:
        c.herk_batched_v(chans, tune=True)          # autotunes on the first call
        check(chans, host)
        c.set_graph_mode(True)
        for ch in chans:
            ch["C"].fill_(float("nan"))
        for _ in range(2):
            c.herk_batched_v(chans, tune=True)      # captured once, then replayed
        assert c.graph_count() == 1
        check(chans, host)
        # new flag lists written into the same device arrays are honoured
        for ch, hb in zip(chans, host):
            block, rows_used, n, K = hb
            new = np.sort(rng.choice(768, size=n, replace=False)).astype(np.int32)
            ch["active"].copy_(torch.from_numpy(new))
            host[host.index(hb)] = (block, new, n, K)
        c.herk_batched_v(chans, tune=True)
        check(chans, host)
        assert c.device_status() == 0


def test_batched_fp16_out_and_beta():
    rng = np.random.default_rng(72)
    specs = [(150, 140, 96, 0), (90, None, 160, 0)]
    chans, host = make_channels(rng, specs)
    olds = []
    for ch in chans:
        ch["C"] = torch.randn(tri_size(ch["n_inputs"]), 2, device=DEV)
        olds.append(ch["C"].clone())
    with Correlator() as c:
        c.herk_batched_v(chans, output=OUT_FP32, alpha=2.0, beta=0.5)
    torch.cuda.synchronize()
    for ch, hb, old in zip(chans, host, olds):
        ref = 2.0 * expected(*hb).astype(np.float64) + 0.5 * old.double().cpu().numpy()
        np.testing.assert_allclose(ch["C"].double().cpu().numpy(), ref, rtol=1e-6, atol=1e-3)
    chans16, host16 = make_channels(rng, specs)
    for ch in chans16:
        ch["C"] = torch.empty(tri_size(ch["n_inputs"]), 2, dtype=torch.float16, device=DEV)
    with Correlator() as c:
        c.herk_batched_v(chans16, output=OUT_FP16)
    torch.cuda.synchronize()
    for ch, hb in zip(chans16, host16):
        assert np.array_equal(ch["C"].cpu().numpy(), expected(*hb).astype(np.float16))


def test_batched_bad_descriptor_rejected():
    from ftd_b200 import FtdxError
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.herk_batched_v([{"A": 0, "C": 0, "n_inputs": 4, "K": 4}])
        A = torch.zeros(64, dtype=torch.uint8, device=DEV)
        C = torch.zeros(20, 2, device=DEV)
        with pytest.raises(FtdxError):  # lda < K
            c.herk_batched_v([{"A": A, "C": C, "n_inputs": 4, "K": 16, "lda": 8}])
