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
        for k, ch in enumerate(chans):
            block, rows_used, n, K = host[k]
            new = np.sort(rng.choice(768, size=n, replace=False)).astype(np.int32)
            ch["active"].copy_(torch.from_numpy(new))
            host[k] = (block, new, n, K)
        c.herk_batched_v(chans, tune=True)
        check(chans, host)
        assert c.device_status() == 0


@pytest.mark.parametrize("mode", [1, 2, 3])
def test_uneven_flagged_store_modes(mode):
    """Bulk stores and the CTA-pair kernel (with and without bulk stores) on
    the gathered channels: bit-exact, including channels narrower than one
    256-input pair tile and ones ending mid-tile."""
    rng = np.random.default_rng(80 + mode)
    specs = [(1, None, 1, 0), (200, 130, 64, 16), (300, 257, 200, 3), (64, None, 1000, 0),
             (700, 600, 2048, 0), (129, 129, 65, 7), (500, 17, 130, 0), (1100, 1023, 384, 0)]
    chans, host = make_channels(rng, specs)
    with Correlator() as c:
        c.set_strategy(mode, 0)
        c.herk_batched_v(chans, output=OUT_FP32)
        assert c.device_status() == 0
        check(chans, host)
        # a second call on the same plan after a single-CTA call
        c.set_strategy(0, 0)
        c.herk_batched_v(chans, output=OUT_FP32)
        c.set_strategy(mode, 0)
        for ch in chans:
            ch["C"].fill_(float("nan"))
        c.herk_batched_v(chans, output=OUT_FP32)
        assert c.device_status() == 0
    check(chans, host)


@pytest.mark.parametrize("mode", [0, 2])
def test_batched_fp16_out_and_beta(mode):
    """alpha / beta and FP16 output on the single-CTA kernel and the CTA pair."""
    rng = np.random.default_rng(72)
    specs = [(150, 140, 96, 0), (90, None, 160, 0), (600, 530, 256, 0)]
    chans, host = make_channels(rng, specs)
    olds = []
    for ch in chans:
        ch["C"] = torch.randn(tri_size(ch["n_inputs"]), 2, device=DEV)
        olds.append(ch["C"].clone())
    with Correlator() as c:
        c.set_strategy(mode, 0)
        c.herk_batched_v(chans, output=OUT_FP32, alpha=2.0, beta=0.5)
    torch.cuda.synchronize()
    for ch, hb, old in zip(chans, host, olds):
        ref = 2.0 * expected(*hb).astype(np.float64) + 0.5 * old.double().cpu().numpy()
        np.testing.assert_allclose(ch["C"].double().cpu().numpy(), ref, rtol=1e-6, atol=1e-3)
    chans16, host16 = make_channels(rng, specs)
    for ch in chans16:
        ch["C"] = torch.empty(tri_size(ch["n_inputs"]), 2, dtype=torch.float16, device=DEV)
    with Correlator() as c:
        c.set_strategy(mode, 0)
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


def make_workload3(seed, n_chans=96, inputs=4096):
    """96 channels; K ~ U{128, 192, ..., 2048}; active inputs ~ U[1536, 4096]
    after seeded random flagging of a 4096-input array; Gaussian int4 (sigma 2.5)."""
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=DEV).manual_seed(seed)
    chans = []
    for _ in range(n_chans):
        K = int(rng.integers(2, 33)) * 64
        n = int(rng.integers(1536, inputs + 1))
        active = np.sort(rng.choice(inputs, size=n, replace=False)).astype(np.int32)
        re = torch.clamp(torch.round(torch.randn(inputs, K, device=DEV, generator=g) * 2.5), -7, 7).to(torch.int32)
        im = torch.clamp(torch.round(torch.randn(inputs, K, device=DEV, generator=g) * 2.5), -7, 7).to(torch.int32)
        qc = ((torch.where(re < 0, 8 | (-re), re) << 4) | torch.where(im < 0, 8 | (-im), im)).to(torch.uint8)
        chans.append({"A": qc, "C": torch.empty(tri_size(n), 2, device=DEV), "n_inputs": n, "K": K,
                      "active": torch.from_numpy(active).to(DEV), "re": re, "im": im})
    return chans


def test_workload3_full_size_properties():
    chans = make_workload3(2027)
    with Correlator() as c:
        c.herk_batched_v(chans, tune=True)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    for k, ch in enumerate(chans):
        n = ch["n_inputs"]
        act = ch["active"].long()
        # diagonal: sum |v|^2 of each active input, exactly
        power = (ch["re"][act] ** 2 + ch["im"][act] ** 2).sum(-1).float()
        idx = torch.arange(n, device=DEV, dtype=torch.int64)
        assert torch.equal(ch["C"][idx * (idx + 1) // 2 + idx, 0], power), k
        if k % 24 == 0:  # exact rows against the oracle for a few channels
            qc = ch["A"][act].cpu().numpy()[None]
            i0 = n - 40
            ref = oracle.herk_qc_rows(qc, n, ch["K"], 0, i0, n).astype(np.float32)
            got = ch["C"][tri_size(i0):tri_size(n)].cpu().numpy()
            assert np.array_equal(got, ref), k


def test_workload3_pair_modes_match_single():
    """The full-size uneven workload through the CTA-pair kernel (store modes
    2 and 3) equals the single-CTA result bit for bit."""
    chans = make_workload3(2028, n_chans=24)
    with Correlator() as c:
        c.set_strategy(0, 0)
        c.herk_batched_v(chans)
        ref = [ch["C"].clone() for ch in chans]
        for mode in (2, 3):
            for ch in chans:
                ch["C"].fill_(float("nan"))
            c.set_strategy(mode, 0)
            c.herk_batched_v(chans)
            assert c.device_status() == 0
            torch.cuda.synchronize()
            for k, ch in enumerate(chans):
                assert torch.equal(ch["C"], ref[k]), (mode, k)
