"""XEngine-compatible correlation (ftdx_xengine): two's-complement (4,4)b
payload blocks [K][n_ant], C = M^H M as the packed upper triangle or the
full matrix, against the oracle restating tests/xengine_test.cpp.  Exact."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError  # noqa: E402
from ftd_b200._lib import OUT_FP16, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def run(n, K, B, fmt, out=OUT_FP32, seed=0, mode=0):
    """mode: the strategy (0 single-CTA kernel, 2 CTA pair)."""
    p = np.random.default_rng(seed).integers(0, 256, size=B * K * n, dtype=np.uint8)
    size = n * n if fmt == 0 else n * (n + 1) // 2
    dt = torch.float32 if out == OUT_FP32 else torch.float16
    C = torch.full((B, size, 2), float("nan"), dtype=dt, device=DEV)
    with Correlator() as c:
        c.set_strategy(mode, 0)
        c.xengine(torch.from_numpy(p).to(DEV), C, n, K, B, mat_format=fmt, output=out)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    got = C.double().cpu().numpy()
    ref = oracle.xengine(p, n, K, B, fmt).reshape(B, size)
    return got[..., 0] + 1j * got[..., 1], ref


@pytest.mark.parametrize("mode", [0, 2])
@pytest.mark.parametrize("fmt", [0, 1])
# 640 and 1000: interior tiles (the unmasked store paths); 257, 1000: a last
# 256-input block of the pair kernel that is partly or mostly empty
@pytest.mark.parametrize("n,K,B", [(64, 128, 3), (130, 100, 2), (257, 64, 1), (5, 3, 4),
                                   (640, 96, 2), (1000, 160, 1)])
def test_formats_exact(mode, fmt, n, K, B):
    got, ref = run(n, K, B, fmt, seed=n + K + fmt, mode=mode)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("mode", [0, 2])
def test_fp16_output(mode):
    got, ref = run(96, 64, 2, 1, out=OUT_FP16, seed=9, mode=mode)
    assert np.array_equal(got, ref.real.astype(np.float16) + 1j * ref.imag.astype(np.float16))


def test_bad_format_rejected():
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.xengine(torch.zeros(64, dtype=torch.uint8, device=DEV),
                      torch.zeros(16, 2, device=DEV), 4, 4, 1, mat_format=2)
