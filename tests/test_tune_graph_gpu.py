"""Autotuner, its disk cache, and CUDA-graph replay (through the C ABI)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError, tri_size  # noqa: E402
from ftd_b200._lib import IN_INT4, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def inputs(N, K, B, seed):
    qc = oracle.gaussian_qc(seed, B, N, K)
    return qc, torch.from_numpy(qc.reshape(-1)).to(DEV)


def test_tune_writes_and_reloads_cache(tmp_path):
    N, K, B = 384, 256, 2
    qc, d = inputs(N, K, B, 31)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    path = str(tmp_path / "tune.txt")
    with Correlator(tune_cache=path) as c:
        assert c.lookup_tuned(N, K, B) is None
        win = c.tune(d, C, N, K, B)
        assert win["store_mode"] in (0, 1, 2, 3, 10, 11, 16) and win["ms"] > 0
        assert c.lookup_tuned(N, K, B)["store_mode"] == win["store_mode"]
        torch.cuda.synchronize()
        # the sweep leaves a correct result behind
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
    lines = open(path).read().splitlines()
    assert len(lines) == 1 and lines[0].startswith("ftdx-tune 2 ")
    with Correlator(tune_cache=path) as c2:  # a new handle reads it back
        got = c2.lookup_tuned(N, K, B)
        assert got is not None and got["store_mode"] == win["store_mode"]
        # tune=True on a cached shape runs without another sweep
        C.fill_(float("nan"))
        c2.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=True)
        torch.cuda.synchronize()
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
    assert len(open(path).read().splitlines()) == 1


def test_corrupt_cache_lines_skipped(tmp_path):
    path = tmp_path / "tune.txt"
    path.write_text("garbage line\nftdx-tune 1 NVIDIA_B200 256 128 1 1 1 1 148 0.01\n"
                    "ftdx-tune 1 NVIDIA_B200 -5 x\n")
    with Correlator() as c:
        with pytest.raises(FtdxError) as ei:
            c.set_tune_cache(str(path))
        assert "2 malformed" in str(ei.value)
        # the valid entry was still loaded (device name as this build records it)
        name = torch.cuda.get_device_name(0).replace(" ", "_")
        if name == "NVIDIA_B200":
            assert c.lookup_tuned(256, 100, 1)["grid"] == 148


def test_tune_then_herk_autotunes_on_miss(tmp_path):
    N, K, B = 256, 128, 3
    qc, d = inputs(N, K, B, 32)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=True)
        assert c.lookup_tuned(N, K, B) is not None
        torch.cuda.synchronize()
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
        assert c.device_status() == 0


@pytest.mark.parametrize("store_mode", [0, 1, 2])
def test_both_store_modes_bit_exact(tmp_path, store_mode):
    # force each epilogue through a cache entry and compare with the oracle
    N, K, B = 640, 192, 2
    qc, d = inputs(N, K, B, 40 + store_mode)
    name = torch.cuda.get_device_name(0).replace(" ", "_")
    path = tmp_path / "t.txt"
    path.write_text(f"ftdx-tune 1 {name} {N} 256 {B} 1 1 {store_mode} 0 1.0\n")
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator(tune_cache=str(path)) as c:
        assert c.lookup_tuned(N, K, B)["store_mode"] == store_mode
        c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=True)
        assert c.device_status() == 0
    assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))


def test_graph_replay_and_lru():
    N, K, B = 200, 96, 2
    qc, d = inputs(N, K, B, 50)
    ref = oracle.herk_qc(qc, N, K, B).astype(np.float32)
    with Correlator() as c:
        c.set_graph_mode(True)
        outs = [torch.full((B, tri_size(N), 2), float("nan"), device=DEV) for _ in range(6)]
        for _ in range(3):
            c.herk(d, outs[0], N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        assert c.graph_count() == 1
        for o in outs[1:]:
            c.herk(d, o, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        assert c.graph_count() == 4  # least-recently-used entries evicted
        torch.cuda.synchronize()
        for o in outs:
            assert np.array_equal(o.cpu().numpy(), ref)
        # replay sees new input data written into the same buffer
        qc2 = oracle.gaussian_qc(51, B, N, K)
        d.copy_(torch.from_numpy(qc2.reshape(-1)))
        c.herk(d, outs[5], N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
        torch.cuda.synchronize()
        assert np.array_equal(outs[5].cpu().numpy(), oracle.herk_qc(qc2, N, K, B).astype(np.float32))
        c.set_graph_mode(False)
        assert c.graph_count() == 0


def test_capture_into_user_graph():
    # ftdx_herk inside the caller's own stream capture, after init_herk
    N, K, B = 160, 64, 2
    qc, d = inputs(N, K, B, 60)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    s = torch.cuda.Stream()
    with Correlator() as c:
        c.init_herk(N, K, B)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False, stream=s)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
        del g


def test_capture_without_workspace_fails_cleanly():
    N, K, B = 160, 64, 2
    _, d = inputs(N, K, B, 61)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    s = torch.cuda.Stream()
    with Correlator() as c:
        g = torch.cuda.CUDAGraph()
        with pytest.raises(FtdxError) as ei:
            with torch.cuda.graph(g, stream=s):
                c.herk(d, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False, stream=s)
        assert "CAPACITY" in str(ei.value)


def test_tuned_entries_kept_per_compute_mode():
    # FP32 input tuned under NVFP4 leaves an NVFP4 entry only; the FP8 lookup
    # of the same shape stays empty until an FP8 call tunes it
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP8, IN_FP32
    N, K, B = 256, 256, 2
    rng = np.random.default_rng(60)
    A = torch.from_numpy(rng.standard_normal((B, N, K, 2)).astype(np.float32)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator() as c:
        c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP4, output=OUT_FP32, tune=True)
        fp4 = c.lookup_tuned(N, K, B, input=IN_FP32, output=OUT_FP32, compute=COMPUTE_FP4)
        assert fp4 is not None and fp4["ms"] > 0
        assert c.lookup_tuned(N, K, B, input=IN_FP32, output=OUT_FP32,
                              compute=COMPUTE_FP8) is None
        c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP32, tune=True)
        assert c.lookup_tuned(N, K, B, input=IN_FP32, output=OUT_FP32,
                              compute=COMPUTE_FP8) is not None
        assert c.device_status() == 0
