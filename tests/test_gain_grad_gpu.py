"""Gain-calibration loss and gradient (ftdx_gain_gradient) against the FP64
oracle and against central finite differences (eps = 1e-3) of the device
loss.  R_obs and R_mod come from the correlator on two seeded voltage sets."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import IN_INT4, OUT_FP32  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def setup(N, K, B, seed):
    rng = np.random.default_rng(seed)
    qo = oracle.gaussian_qc(seed + 1, B, N, K)
    qm = oracle.gaussian_qc(seed + 2, B, N, K)
    Ro = torch.empty(B, tri_size(N), 2, device=DEV)
    Rm = torch.empty_like(Ro)
    with Correlator() as c:
        c.herk(torch.from_numpy(qo.reshape(-1)).to(DEV), Ro, N, K, B, input=IN_INT4, output=OUT_FP32)
        c.herk(torch.from_numpy(qm.reshape(-1)).to(DEV), Rm, N, K, B, input=IN_INT4, output=OUT_FP32)
    W = torch.from_numpy(rng.uniform(0, 1, size=(B, tri_size(N))).astype(np.float32)).to(DEV)
    g = (1.0 + rng.uniform(-0.1, 0.1, N)) * np.exp(1j * rng.uniform(-np.pi, np.pi, N))
    return Ro, Rm, W, g


def gpu_loss_grad(c, Ro, Rm, W, g, N, B):
    gd = torch.from_numpy(np.stack([g.real, g.imag], -1).astype(np.float32)).to(DEV)
    grad = torch.empty(N, 2, dtype=torch.float64, device=DEV)
    loss = torch.empty(1, dtype=torch.float64, device=DEV)
    c.gain_gradient(Ro, Rm, W, gd, N, B, grad, loss)
    torch.cuda.synchronize()
    return float(loss.item()), grad[:, 0].cpu().numpy() + 1j * grad[:, 1].cpu().numpy()


def test_gain_gradient_matches_fp64_and_fd():
    N, K, B = 320, 128, 3
    Ro, Rm, W, g = setup(N, K, B, 500)
    g32 = g.astype(np.complex64).astype(np.complex128)  # the device sees FP32 gains
    L_ref, grad_ref = oracle.gain_loss_grad(Ro.cpu().numpy(), Rm.cpu().numpy(),
                                            W.cpu().numpy(), g32, N)
    with Correlator() as c:
        L, grad = gpu_loss_grad(c, Ro, Rm, W, g32, N, B)
        assert abs(L - L_ref) / L_ref < 1e-6
        rel = np.abs(grad - grad_ref) / np.max(np.abs(grad_ref))
        assert rel.max() < 1e-5, rel.max()
        # central finite differences of the device loss, eps = 1e-3
        eps = 1e-3
        for k in [0, 7, N // 2, N - 1]:
            fd = 0j
            for unit, part in [(1.0, 1.0), (1j, 1j)]:
                gp, gm = g32.copy(), g32.copy()
                gp[k] += eps * unit
                gm[k] -= eps * unit
                Lp, _ = gpu_loss_grad(c, Ro, Rm, W, gp.astype(np.complex64).astype(np.complex128), N, B)
                Lm, _ = gpu_loss_grad(c, Ro, Rm, W, gm.astype(np.complex64).astype(np.complex128), N, B)
                fd += part * (Lp - Lm) / (2 * eps)
            assert abs(fd - grad[k]) / np.max(np.abs(grad_ref)) < 2e-3, (k, fd, grad[k])


def test_gain_gradient_dsa_half_scale():
    # 1024 antennas x 2 pol = 2048 inputs, 32 channels, K = 512
    N, K, B = 2048, 512, 32
    Ro, Rm, W, g = setup(N, K, B, 600)
    g32 = g.astype(np.complex64).astype(np.complex128)
    with Correlator() as c:
        L, grad = gpu_loss_grad(c, Ro, Rm, W, g32, N, B)
        assert c.device_status() == 0
    # FP64 reference on 4 of the 32 channels (the sum is linear in channels)
    sub = [0, 9, 20, 31]
    Ls, gs = 0.0, np.zeros(N, dtype=np.complex128)
    for f in sub:
        l, gr = oracle.gain_loss_grad(Ro[f:f + 1].cpu().numpy(), Rm[f:f + 1].cpu().numpy(),
                                      W[f:f + 1].cpu().numpy(), g32, N)
        Ls += l
        gs += gr
    with Correlator() as c:
        Lsub, gsub = gpu_loss_grad(c, Ro[sub].contiguous(), Rm[sub].contiguous(),
                                   W[sub].contiguous(), g32, N, len(sub))
    assert abs(Lsub - Ls) / Ls < 1e-6
    assert np.max(np.abs(gsub - gs)) / np.max(np.abs(gs)) < 1e-5
    assert np.isfinite(L) and np.all(np.isfinite(grad))
