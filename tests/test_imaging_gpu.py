"""Imaging from the packed triangles (ftdx_image_beams: pillbox gridding with
fused pol sum and taper, cuFFT inverse FFT, beam extraction) against the
numpy oracle that restates the reference's kernels.  Cell indices are exact;
sums of FP32 atomics agree with the exact oracle sums to FP32 rounding."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def case(seed, n_ant, n_chan, n_pol, ng, outside=0.1):
    rng = np.random.default_rng(seed)
    n_bl = n_ant * (n_ant + 1) // 2
    freq = 1.0e9 + 1.0e6 * np.arange(n_chan)
    lam = oracle.C_LIGHT / freq[0]
    # cell 1 rad: u in wavelengths = cell index offset; some baselines off the grid
    span = 0.5 * ng * (1 + outside)
    uv = (rng.uniform(-span, span, size=(n_bl, 2)) * lam).astype(np.float32)
    vis = rng.standard_normal((n_chan, n_pol, n_bl, 2)).astype(np.float32)
    taper = rng.uniform(0.2, 1.0, size=(ng, ng)).astype(np.float32)
    return vis, uv, freq, taper


def run(c, vis, uv, freq, n_ant, ng, stage, taper=None, chan_tile=0, pix=None):
    n_chan, n_pol = vis.shape[0], vis.shape[1]
    out = torch.empty(n_chan, ng, ng, 2, device=DEV)
    beams = torch.empty(n_chan, 0 if pix is None else len(pix), device=DEV)
    c.image_beams(dev(vis), beams, n_ant, n_chan, n_pol, ng, 1.0, dev(uv), dev(freq),
                  taper=None if taper is None else dev(taper),
                  beam_pixels=None if pix is None else dev(np.asarray(pix, dtype=np.int32)),
                  n_beam=0 if pix is None else len(pix), chan_tile=chan_tile,
                  output_stage=stage, grid_out=None if stage == 0 else out)
    torch.cuda.synchronize()
    if stage == 0:
        return beams.cpu().numpy()
    o = out.cpu().numpy()
    return o[..., 0] + 1j * o[..., 1]


def test_reference_point_and_mirror():
    # baseline (1, 0) at (2, 3) wavelengths, cell 1: (1, 0.5) at (Ng/2+2, Ng/2+3),
    # conjugate at (Ng/2-2, Ng/2-3) (lib/test_imaging.cu:109-160)
    n, ng, f = 4, 32, 1.0e9
    lam = oracle.C_LIGHT / f
    uv = np.zeros((10, 2), dtype=np.float32)
    uv[1] = [2.0 * lam, 3.0 * lam]
    vis = np.zeros((1, 1, 10, 2), dtype=np.float32)
    vis[0, 0, 1] = [1.0, 0.5]
    with Correlator() as c:
        g = run(c, vis, uv, np.array([f]), n, ng, 1)
    h = ng // 2
    assert g[0, h + 3, h + 2] == 1 + 0.5j and g[0, h - 3, h - 2] == 1 - 0.5j
    assert np.count_nonzero(g) == 2


@pytest.mark.parametrize("n_pol,use_taper", [(1, False), (2, True), (3, True)])
def test_grid_image_beams_random(n_pol, use_taper):
    n_ant, n_chan, ng = 40, 5, 64
    vis, uv, freq, taper = case(n_pol * 10 + 1, n_ant, n_chan, n_pol, ng)
    taper = taper if use_taper else None
    ref_grid = oracle.image_grid(vis, uv, freq, n_ant, ng, 1.0, taper)
    ref_img = oracle.image_from_grid(ref_grid)
    pix = [(0, 0), (ng // 2, ng // 2), (3, 60), (63, 63), (ng, 1), (-1, 4)]
    ref_beams = oracle.beam_intensity(ref_img, pix)
    with Correlator() as c:
        g = run(c, vis, uv, freq, n_ant, ng, 1, taper)
        img = run(c, vis, uv, freq, n_ant, ng, 2, taper, chan_tile=2)
        beams = run(c, vis, uv, freq, n_ant, ng, 0, taper, chan_tile=3, pix=pix)
        assert c.device_status() == 0
    # same cells, same sums to FP32 rounding
    assert np.array_equal(g != 0, ref_grid != 0)
    np.testing.assert_allclose(g, ref_grid, rtol=1e-5, atol=1e-5 * np.abs(ref_grid).max())
    np.testing.assert_allclose(img, ref_img, rtol=1e-4, atol=1e-5 * np.abs(ref_img).max())
    np.testing.assert_allclose(beams, ref_beams, rtol=1e-3, atol=1e-6 * np.abs(ref_beams).max())
    assert np.all(beams[:, 4:] == 0)


def test_long_beam_list_sorted_gather():
    # 70,000 beams (past the length from which the pixels are sorted once per
    # call and gathered in image order), repeats and off-image pixels
    # included: every beam is the direct gather's value for its own pixel
    n_ant, n_chan, ng = 40, 3, 64
    vis, uv, freq, taper = case(77, n_ant, n_chan, 2, ng)
    rng = np.random.default_rng(78)
    pix = rng.integers(-2, ng + 2, size=(70000, 2))
    ref_img = oracle.image_from_grid(oracle.image_grid(vis, uv, freq, n_ant, ng, 1.0, taper))
    with Correlator() as c:
        long_b = run(c, vis, uv, freq, n_ant, ng, 0, taper, pix=pix)
        short_b = run(c, vis, uv, freq, n_ant, ng, 0, taper, pix=pix[:1000])
        assert c.device_status() == 0
    # two calls grid with FP32 atomics in different orders: equal to rounding
    np.testing.assert_allclose(long_b[:, :1000], short_b, rtol=1e-4,
                               atol=1e-6 * np.abs(short_b).max())
    ref = oracle.beam_intensity(ref_img, [tuple(p) for p in pix[:2000]])
    np.testing.assert_allclose(long_b[:, :2000], ref, rtol=1e-3, atol=1e-6 * np.abs(ref).max())
    off = (pix[:, 0] < 0) | (pix[:, 0] >= ng) | (pix[:, 1] < 0) | (pix[:, 1] >= ng)
    assert np.all(long_b[:, off] == 0)


def test_large_triangle_auto_cross_split():
    # 3000 antennas: packed indices past 2^22, where a float square-root decode
    # of the row misclassifies baselines; every baseline at u = v = 0 with
    # vis 1: the centre cell counts n_bl + (n_bl - N) exactly
    n = 3000
    n_bl = n * (n + 1) // 2
    vis = np.zeros((1, 1, n_bl, 2), dtype=np.float32)
    vis[..., 0] = 1.0
    uv = np.zeros((n_bl, 2), dtype=np.float32)
    with Correlator() as c:
        g = run(c, vis, uv, np.array([1.0e9]), n, 16, 1)
    assert g[0, 8, 8] == 2 * n_bl - n and np.count_nonzero(g) == 1


def test_bad_config_rejected():
    with Correlator() as c:
        with pytest.raises(FtdxError):
            c.image_beams(torch.zeros(4, device=DEV), None, 1, 1, 1, 1, 1.0,
                          torch.zeros(2, device=DEV), torch.zeros(1, dtype=torch.float64,
                                                                  device=DEV))
