"""Adjoint of the correlator, dV = (G + G^H) V (ftdx_herk_adjoint), against
FP64 numpy, plus the defining identity: for L = Re <G, V V^H>,
dL/dRe(V) + i dL/dIm(V) = (G + G^H) V, checked with central finite
differences (eps = 1e-3) on a few voltages."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator  # noqa: E402

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def run(G, qc, N, K, B):
    dG = torch.from_numpy(np.ascontiguousarray(G.astype(np.complex64)).view(np.float32)).to(DEV)
    dV = torch.from_numpy(qc.reshape(-1)).to(DEV)
    out = torch.full((B, N, K, 2), float("nan"), device=DEV)
    with Correlator() as c:
        c.herk_adjoint(dG, dV, out, N, K, B)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return o[..., 0].astype(np.float64) + 1j * o[..., 1]


def voltages(qc):
    re, im = oracle.decode_qc(qc)
    return re.astype(np.float64) + 1j * im.astype(np.float64)


def test_adjoint_general_g_ragged():
    rng = np.random.default_rng(80)
    N, K, B = 264, 200, 3
    G = (rng.normal(size=(B, N, N)) + 1j * rng.normal(size=(B, N, N))).astype(np.complex64)
    qc = oracle.gaussian_qc(81, B, N, K)
    got = run(G, qc, N, K, B)
    G64 = G.astype(np.complex128)
    ref = (G64 + np.conj(np.transpose(G64, (0, 2, 1)))) @ voltages(qc)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("adjoint rel err", err)
    assert err < 1e-4


def test_adjoint_g_only_8_byte_aligned():
    # G one complex64 into an allocation (8- but not 16-byte aligned): the
    # symmetrisation pass reads it element-wise, same result as aligned
    rng = np.random.default_rng(83)
    N, K, B = 136, 72, 2
    G = (rng.normal(size=(B, N, N)) + 1j * rng.normal(size=(B, N, N))).astype(np.complex64)
    qc = oracle.gaussian_qc(84, B, N, K)
    flat = np.concatenate([np.zeros(1, np.complex64), G.reshape(-1)])
    buf = torch.from_numpy(flat.view(np.float32)).to(DEV)
    dG = buf[2:]  # offset by one complex64
    assert dG.data_ptr() % 16 == 8
    dV = torch.from_numpy(qc.reshape(-1)).to(DEV)
    out = torch.empty(B, N, K, 2, device=DEV)
    with Correlator() as c:
        c.herk_adjoint(dG, dV, out, N, K, B)
        assert c.device_status() == 0
    o = out.cpu().numpy()
    got = o[..., 0].astype(np.float64) + 1j * o[..., 1]
    assert np.array_equal(got, run(G, qc, N, K, B))


def test_adjoint_matches_finite_differences():
    rng = np.random.default_rng(82)
    N, K, B = 64, 40, 1
    A = rng.normal(size=(N, N)) + 1j * rng.normal(size=(N, N))
    G = ((A + A.conj().T) / 2).astype(np.complex64)[None]  # Hermitian upstream gradient
    qc = oracle.gaussian_qc(83, B, N, K)
    got = run(G, qc, N, K, B)[0]
    V = voltages(qc)[0]
    G64 = G[0].astype(np.complex128)

    def loss(Vx):
        return float(np.real(np.sum(np.conj(G64) * (Vx @ Vx.conj().T))))
    eps = 1e-3
    for (a, t) in [(0, 0), (5, 17), (63, 39)]:
        fd = 0j
        for unit in (1.0, 1j):
            Vp, Vm = V.copy(), V.copy()
            Vp[a, t] += eps * unit
            Vm[a, t] -= eps * unit
            fd += unit * (loss(Vp) - loss(Vm)) / (2 * eps)
        assert abs(fd - got[a, t]) / np.abs(got).max() < 1e-4, (a, t, fd, got[a, t])


def test_adjoint_half_dsa_scale():
    # 1024 antennas x 2 pol = 2048 inputs, 32 channels, K = 512, random Hermitian G
    N, K, B = 2048, 512, 32
    g = torch.Generator(device=DEV).manual_seed(84)
    A = torch.randn(B, N, N, 2, device=DEV, generator=g)
    Gc = torch.view_as_complex(A)
    Gc = (Gc + Gc.conj().transpose(1, 2)) / 2
    dG = torch.view_as_real(Gc.contiguous()).contiguous()
    qc = oracle.gaussian_qc(85, B, N, K)
    dV = torch.from_numpy(qc.reshape(-1)).to(DEV)
    out = torch.empty(B, N, K, 2, device=DEV)
    with Correlator() as c:
        c.herk_adjoint(dG, dV, out, N, K, B)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    V = voltages(qc)
    for f in (0, 13, 31):
        Gf = Gc[f].cpu().numpy().astype(np.complex128)
        ref = (Gf + Gf.conj().T) @ V[f]
        o = out[f].cpu().numpy()
        got = o[..., 0] + 1j * o[..., 1]
        assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-4, f
