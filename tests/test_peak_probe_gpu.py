"""ftdx_peak_probe: every kind runs to completion with the device status clear
and reports a throughput between 10% and 150% of the datasheet's dense
figure for its format (FP8 4.5 PFLOPS, NVFP4 9 PFLOPS); an unknown kind is
rejected before any launch."""
import pytest

pytest.importorskip("torch")
from ftd_b200 import Correlator, FtdxError  # noqa: E402

pytestmark = pytest.mark.gpu

NOMINAL = {0: 4500.0, 1: 9000.0, 2: 4500.0, 3: 4500.0}


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_probe_kinds(kind):
    with Correlator() as c:
        tf = c.peak_probe(kind, iters=2001, reps=1)  # 2001: rounded up to whole steps
        assert c.device_status() == 0
    assert 0.1 * NOMINAL[kind] < tf < 1.5 * NOMINAL[kind], tf


@pytest.mark.parametrize("kind", [-1, 4])
def test_probe_rejects_unknown_kind(kind):
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.peak_probe(kind, iters=100, reps=1)
