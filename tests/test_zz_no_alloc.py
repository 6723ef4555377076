"""ftdx_herk_static: the entry point for callers that cannot let the library
allocate GPU memory (real-time pipelines with buffers fixed at start-up,
frameworks that own all device memory through their own pool).  It must give
exactly what ftdx_herk gives on the same input (QC int4 correlations are
bit-exact), call after call, with its scratch in the library's static device
array.  This file is collected last so that a failure here comes after every
other test has run; it also passes on its own in a fresh process."""
import ctypes

import numpy as np
import pytest

from ftd_b200 import _lib

STATIC_BYTES = 32 << 20


def _sizes(N, K, batch):
    Kp = (K + 127) // 128 * 128
    nb = (N + 127) // 128
    tiles = batch * nb * (nb + 1) // 2
    plan = batch * 40 + tiles * 8  # ChanDesc (40 B) per channel, TileDesc (8 B) per tile
    z_off = (256 + plan + 1023) // 1024 * 1024
    return z_off + 2 * N * batch * Kp


def test_static_rejects_oversize_without_gpu_work():
    # a problem beyond the static scratch is refused before touching the device
    L = _lib.load()
    used = ctypes.c_size_t(0)
    N, K, B = 4096, 1024, 64
    st = L.ftdx_herk_static(ctypes.c_void_p(16), ctypes.c_void_p(16), N, K, B, None, None,
                            ctypes.byref(used))
    assert st == 6  # FTDX_ERR_CAPACITY
    assert used.value == _sizes(N, K, B) > STATIC_BYTES
    # the sizes are reported through the calling thread's error text, not stderr
    msg = L.ftdx_last_error(None).decode()
    assert f"needs {used.value} bytes" in msg and str(STATIC_BYTES) in msg
    assert L.ftdx_herk_static(None, None, 1, 1, 1, None, None, None) == 1
    # a tile count that overflows 32-bit arithmetic is refused as too large
    st = L.ftdx_herk_static(ctypes.c_void_p(16), ctypes.c_void_p(16), 6_000_000, 1, 1, None,
                            None, ctypes.byref(used))
    assert st == 6 and used.value == _sizes(6_000_000, 1, 1)


@pytest.mark.gpu
def test_static_matches_ftdx_herk_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    from oracle import oracle
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP32

    L = _lib.load()
    dev = "cuda:0"
    torch.cuda.set_device(0)
    # two different problems back to back: the second call reuses (and must
    # fully rewrite) the scratch the first one left behind
    for (N, K, B, seed) in [(1024, 1024, 15, 101), (300, 77, 3, 102)]:
        qc_np = oracle.gaussian_qc(seed, B, N, K)
        qc = torch.from_numpy(qc_np.reshape(-1)).to(dev)
        ref = torch.full((B, tri_size(N), 2), float("nan"), device=dev)
        with Correlator(device=0) as c:
            c.herk(qc, ref, N, K, B, input=IN_INT4, output=OUT_FP32, tune=False)
            assert c.device_status() == 0
        got = torch.full((B, tri_size(N), 2), float("nan"), device=dev)
        bits = ctypes.c_uint32(123)
        used = ctypes.c_size_t(0)
        st = L.ftdx_herk_static(ctypes.c_void_p(qc.data_ptr()), ctypes.c_void_p(got.data_ptr()),
                                N, K, B, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream),
                                ctypes.byref(bits), ctypes.byref(used))
        assert st == 0 and bits.value == 0
        assert used.value == _sizes(N, K, B) <= STATIC_BYTES
        torch.cuda.synchronize()
        assert torch.equal(got, ref), (N, K, B)
        # and against the oracle on a few rows (the full oracle is slow at N=1024)
        rows = oracle.herk_qc_rows(qc_np, N, K, B - 1, N - 8, N).astype(np.float32)
        assert np.array_equal(got[B - 1, tri_size(N - 8):tri_size(N)].cpu().numpy(), rows)
