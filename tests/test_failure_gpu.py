"""Failure detection on the GPU without faulting it: bounded device waits
are made to run out (an mbarrier nothing arrives on, then a global flag
nothing sets), the timeout shows up in the status word, and the same handle
then correlates bit-exactly."""
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, FtdxError, tri_size  # noqa: E402
from ftd_b200._lib import IN_INT4, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def test_bounded_wait_times_out_and_handle_recovers():
    with Correlator() as c:
        assert c.device_status() == 0
        t0 = time.perf_counter()
        c.wait_selftest(100)
        bits = c.device_status()
        dt = time.perf_counter() - t0
        assert bits != 0                 # the timeout bit
        assert 0.19 < dt < 5.0           # it waited about the limit twice, then gave up
        assert c.device_status() == 0    # reading clears it
        # the handle and the context are still good
        N, K, B = 200, 96, 2
        qc = oracle.gaussian_qc(5, B, N, K)
        C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
        c.herk(torch.from_numpy(qc.reshape(-1)).to(DEV), C, N, K, B, input=IN_INT4,
               output=OUT_FP32, tune=False)
        assert c.device_status() == 0
        assert np.array_equal(C.cpu().numpy(), oracle.herk_qc(qc, N, K, B).astype(np.float32))
        with pytest.raises(FtdxError):
            c.wait_selftest(0)
