"""Host-to-host correlation pipeline (ftdx_pipeline_*, the VisibilityPipeline
correlate / correlate_pipelined replacement) against the oracle: pageable and
pinned host buffers, batch-first and raw packet-ordered payloads, several
payloads in flight.  Bit-exact."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError, Pipeline, tri_size  # noqa: E402
from ftd_b200._lib import LAYOUT_CHAN_POL_ANT_TIME, LAYOUT_TIME_ANT_CHAN_POL, OUT_FP16  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_payloads", [1, 2, 5])
@pytest.mark.parametrize("pinned", [False, True])
def test_batch_first_payloads(n_payloads, pinned):
    N, K, B = 200, 160, 3
    qcs = [oracle.gaussian_qc(100 + p, B, N, K) for p in range(n_payloads)]
    if pinned:
        ins = [torch.from_numpy(q.reshape(-1)).pin_memory() for q in qcs]
        outs = [torch.full((B, tri_size(N), 2), float("nan")).pin_memory() for _ in qcs]
    else:
        ins = [np.ascontiguousarray(q.reshape(-1)) for q in qcs]
        outs = [np.full((B, tri_size(N), 2), np.nan, dtype=np.float32) for _ in qcs]
    with Correlator() as c, Pipeline(c, N, K, B) as p:
        assert p.sizes == (B * N * K, B * tri_size(N) * 8)
        p.correlate(outs, ins)
        p.correlate(outs, ins[::-1])   # reuse: outs[j] now holds payload n-1-j
    for q, o in zip(qcs[::-1], outs):
        got = o.numpy() if hasattr(o, "numpy") else o
        assert np.array_equal(got, oracle.herk_qc(q, N, K, B).astype(np.float32))


@pytest.mark.parametrize("layout", [LAYOUT_TIME_ANT_CHAN_POL, LAYOUT_CHAN_POL_ANT_TIME])
def test_raw_layout_payloads(layout):
    a, ch, pol, ti, K = 96, 2, 2, 2, 64
    t = ti * K
    ftd = {"n_ant": a, "n_chan": ch, "n_pol": pol, "n_time": t, "n_time_inner": ti,
           "layout": layout, "pol_sum": True}
    rng = np.random.default_rng(layout + 5)
    raws = [oracle.encode_qc(*oracle.gaussian_int4(rng, (t * a * ch * pol,))) for _ in range(3)]
    outs = [np.empty((ch * ti, tri_size(a), 2), dtype=np.float32) for _ in raws]
    with Correlator() as c, Pipeline(c, ftd=ftd) as p:
        p.correlate(outs, raws)
    for r, o in zip(raws, outs):
        bf = oracle.ftd_to_batch_first(r, a, ch, pol, t, ti, layout, True)
        assert np.array_equal(o, oracle.herk_qc(bf, a, pol * K, bf.shape[0]).astype(np.float32))


def test_fp16_output_and_errors():
    N, K, B = 64, 96, 2
    q = oracle.gaussian_qc(7, B, N, K)
    out = np.empty((B, tri_size(N), 2), dtype=np.float16)
    with Correlator() as c:
        with Pipeline(c, N, K, B, output=OUT_FP16) as p:
            p.correlate([out], [q.reshape(-1)])
            assert np.array_equal(out, oracle.herk_qc(q, N, K, B).astype(np.float32)
                                  .astype(np.float16))
            with pytest.raises(FtdxError):
                p.correlate([out], [q.reshape(-1), q.reshape(-1)])
        with pytest.raises(FtdxError):
            Pipeline(c, 0, K, B)
