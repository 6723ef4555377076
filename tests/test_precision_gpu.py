"""Precision modes on float complex voltages (per-channel-scaled FP8 and the
hi+lo split-FP8 mode) against the FP64 oracle, and Kahan accumulation across
integration dumps.  Errors are measured as |dR_ij| / sqrt(R_ii R_jj) (scale
free; the bound is written in each test)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from oracle import oracle  # noqa: E402

from ftd_b200 import Correlator, tri_size  # noqa: E402
from ftd_b200._lib import (COMPUTE_FP8, COMPUTE_FP8_SPLIT, IN_FP32, IN_INT4,  # noqa: E402
                           OUT_FP32)

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def run_float(v, compute, store_mode=None):
    """store_mode 0 / 2 picks the NVFP4 single-CTA / pair kernel (None: tuned)."""
    B, N, K = v.shape
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    with Correlator() as c:
        if store_mode is not None:
            c.set_strategy(store_mode, 0)
        c.herk(A, C, N, K, B, input=IN_FP32, compute=compute, output=OUT_FP32,
               tune=store_mode is None)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    return C.cpu().numpy()


@pytest.fixture(scope="module")
def workload():
    B, N, K = 4, 256, 1024
    v = oracle.workload4_voltages(404, B, N, K)
    return v, oracle.herk_c128(v.astype(np.complex128), N, K, B)


def test_fp8_scaled_error(workload):
    v, ref = workload
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP8), ref, v.shape[1])
    print("fp8", err)
    # E4M3 keeps 4 significant bits: ~3% per sample, averaged over K samples
    assert err["max_norm"] < 3e-2 and err["rms_norm"] < 3e-3
    assert err["max_auto_rel"] < 3e-2


def test_split_fp8_error(workload):
    v, ref = workload
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP8_SPLIT), ref, v.shape[1])
    print("split", err)
    # hi + lo carries ~8 significant bits; the dropped lo.lo^H term biases R_ii by ~3e-4
    assert err["max_norm"] < 3e-3 and err["rms_norm"] < 3e-4
    err8 = oracle.correlation_errors(run_float(v, COMPUTE_FP8), ref, v.shape[1])
    assert err["rms_norm"] < err8["rms_norm"] / 8


def test_scale_invariance():
    # per-channel scaling: channels differing only by a power-of-two factor give
    # results differing by exactly that factor squared
    B, N, K = 2, 130, 256
    v = oracle.workload4_voltages(405, 1, N, K)
    v2 = np.concatenate([v, v * np.float32(8.0)], axis=0)
    out = run_float(v2, COMPUTE_FP8)
    assert np.array_equal(out[1], out[0] * 64.0)


def test_kahan_accumulation_across_dumps():
    N, K, B, dumps = 128, 1024, 2, 800
    rng = np.random.default_rng(9)
    S = torch.zeros(B, tri_size(N), 2, device=DEV)
    comp = torch.zeros_like(S)
    naive = torch.zeros_like(S)
    exact = np.zeros((B, tri_size(N), 2), dtype=np.int64)
    with Correlator() as c:
        for d in range(dumps):
            qc = oracle.gaussian_qc(int(rng.integers(1 << 30)), B, N, K, sigma=5.0)
            exact += oracle.herk_qc(qc, N, K, B)
            dq = torch.from_numpy(qc.reshape(-1)).to(DEV)
            c.herk_kahan(dq, S, comp, N, K, B, input=IN_INT4, compute=COMPUTE_FP8)
            c.herk(dq, naive, N, K, B, input=IN_INT4, output=OUT_FP32, beta=1.0, tune=False)
        assert c.device_status() == 0
    torch.cuda.synchronize()
    # the compensation holds minus the low-order part lost from the sum
    tot = S.double().cpu().numpy() - comp.double().cpu().numpy()
    err_k = np.abs(tot - exact).max()
    err_n = np.abs(naive.double().cpu().numpy() - exact).max()
    print("kahan max abs err", err_k, "naive", err_n, "max |total|", np.abs(exact).max())
    assert np.abs(exact).max() > 2 ** 24          # beyond FP32's exact-integer range
    assert err_k <= 2.0                            # compensated: ~exact
    assert err_n > 4 * max(err_k, 0.5)             # plain FP32 accumulation drifts


# ---------------------------------------------------------------- NVFP4
E2M1 = np.array([0.0, 0.5, 1.0, 1.5, 2.0, 3.0, 4.0, 6.0])


# NVFP4 kernels: store mode 0 single CTA, 2 CTA pair
@pytest.mark.parametrize("store_mode", [0, 2])
def test_nvfp4_exactly_representable_input_is_exact(store_mode):
    # Every block of 8 complex samples holds E2M1 values times a per-block power
    # of two, with one component at 6 x that power: the quantiser's block scales
    # come out exact (448, 224, 112 in UE4M3) and so does every element, so the
    # only error left is FP32 rounding (of the accumulation and of the channel
    # scale g^2, which is not a power of two): rtol 1e-6.  Any mistake in the
    # packing, scale-factor layout or tile walk shows up as O(1) errors.
    from ftd_b200._lib import COMPUTE_FP4
    rng = np.random.default_rng(90)
    B, N, K = 2, 600, 256  # several tiles per channel on both kernels
    e = rng.choice(E2M1, size=(B, N, K, 2)) * rng.choice([-1.0, 1.0], size=(B, N, K, 2))
    blocks = e.reshape(B, N, K // 8, 16)
    blocks[..., 0] = 6.0                              # the block maximum
    pw = 2.0 ** rng.integers(-2, 1, size=(B, N, K // 8, 1))
    pw[:, 0, 0, 0] = 1.0                              # channel max = 6
    v = (blocks * pw).reshape(B, N, K, 2)
    vc = (v[..., 0] + 1j * v[..., 1]).astype(np.complex64)
    got = run_float(vc, COMPUTE_FP4, store_mode)
    ref = oracle.herk_c128(vc.astype(np.complex128), N, K, B)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("nvfp4 exact-input max rel err", store_mode, err)
    assert err < 1e-6


def test_nvfp4_error(workload):
    # E2M1 with block-16 scales chosen by squared error: ~15% RMS quantisation
    # noise per sample, ~0.15 sqrt(2/K) per normalised cross-correlation.  The
    # time samples carrying 20-sigma bursts are moved to the last stage and
    # carry a lo residual there, so the burst pairs no longer set the worst
    # case (6e-2 without it).  Autocorrelations are exact.
    from ftd_b200._lib import COMPUTE_FP4
    v, ref = workload
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP4), ref, v.shape[1])
    print("nvfp4", err)
    assert err["rms_offdiag_norm"] < 5e-3 and err["max_offdiag_norm"] < 2e-2
    assert err["max_auto_rel"] < 1e-5


def test_nvfp4_error_without_rfi():
    from ftd_b200._lib import COMPUTE_FP4
    B, N, K = 4, 256, 1024
    v = oracle.workload4_voltages(406, B, N, K, rfi_time_frac=0.0, rfi_input_frac=0.0)
    ref = oracle.herk_c128(v.astype(np.complex128), N, K, B)
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP4), ref, N)
    print("nvfp4 no-rfi", err)
    assert err["rms_offdiag_norm"] < 5e-3 and err["max_offdiag_norm"] < 2e-2


def _config4_voltages(seed, B, N, K, dev):
    """The precision configuration on the device: complex Gaussian voltages
    [B][N][K][2] float32, per-channel RMS log-uniform in [0.1, 10], and in
    each channel 1% of the time samples carry 20-sigma bursts (random phase)
    on 5% of the inputs."""
    g = torch.Generator(device=dev).manual_seed(seed)
    rms = torch.exp(torch.empty(B, device=dev).uniform_(float(np.log(0.1)), float(np.log(10.0)),
                                                        generator=g))
    V = torch.randn(B, N, K, 2, device=dev, generator=g) * (rms.view(B, 1, 1, 1) / 2 ** 0.5)
    n_rfi, t_rfi = max(1, N // 20), max(1, K // 100)
    for b in range(B):
        ins = torch.randperm(N, device=dev, generator=g)[:n_rfi]
        ts = torch.randperm(K, device=dev, generator=g)[:t_rfi]
        ph = torch.rand(n_rfi, t_rfi, device=dev, generator=g) * (2 * np.pi)
        amp = 20.0 * rms[b]
        V[b, ins[:, None], ts[None, :]] = torch.stack([amp * torch.cos(ph), amp * torch.sin(ph)], -1)
    return V


def full_channel_errors(V, C):
    """max and RMS over all channels of |dR_ij| / sqrt(R_ii R_jj), cross- and
    autocorrelations, against FP64 products computed on the device."""
    B, N = V.shape[0], V.shape[1]
    ii, jj = torch.tril_indices(N, N, device=V.device)
    order = torch.argsort(ii * N + jj)
    ii, jj = ii[order], jj[order]
    off = ii != jj
    mx = mxa = 0.0
    ss = 0.0
    cnt = 0
    for b in range(B):
        Vb = torch.view_as_complex(V[b].double().contiguous())
        R = Vb @ Vb.conj().T
        auto = torch.diagonal(R).real
        got = torch.view_as_complex(C[b].double().contiguous())
        ref = R[ii, jj]
        e = (got - ref).abs() / torch.sqrt(auto[ii] * auto[jj])
        mx = max(mx, float(e[off].max()))
        mxa = max(mxa, float(e[~off].max()))
        ss += float(e[off].pow(2).sum())
        cnt += int(off.sum())
        del R, ref, got, e
    return {"max_cross": mx, "rms_cross": (ss / cnt) ** 0.5, "max_auto": mxa}


def test_nvfp4_config4_full_channels():
    # The precision configuration at full size: 4096 inputs x 64 channels x
    # K = 1024 with the RFI bursts; every element of every channel against
    # FP64.  NVFP4 (E2M1, UE4M3 block-16 scales, burst samples permuted into a
    # last stage that carries a lo residual): max <= 2e-2 over all 5.4e8
    # normalised cross-correlations; the hi + lo split mode far below it.
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    B, N, K = 64, 4096, 1024
    V = _config4_voltages(2026, B, N, K, DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    with Correlator() as c:
        for compute, bound in ((COMPUTE_FP4, 2e-2), (COMPUTE_FP4_SPLIT, 1e-2)):
            c.herk(V, C, N, K, B, input=IN_FP32, compute=compute, output=OUT_FP32, tune=False)
            assert c.device_status() == 0
            err = full_channel_errors(V, C)
            print("config 4 full channels", compute, err)
            assert err["max_cross"] <= bound and err["max_auto"] < 1e-5


@pytest.mark.parametrize("store_mode", [0, 2])
def test_nvfp4_split_exactly_representable_input_is_exact(store_mode):
    # input that NVFP4 holds exactly: the residual is zero, every lo block scale
    # is zero, and the split mode gives the plain NVFP4 result (same rtol 1e-6)
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    rng = np.random.default_rng(91)
    B, N, K = 2, 600, 256
    e = rng.choice(E2M1, size=(B, N, K, 2)) * rng.choice([-1.0, 1.0], size=(B, N, K, 2))
    blocks = e.reshape(B, N, K // 8, 16)
    blocks[..., 0] = 6.0
    pw = 2.0 ** rng.integers(-2, 1, size=(B, N, K // 8, 1))
    pw[:, 0, 0, 0] = 1.0
    v = (blocks * pw).reshape(B, N, K, 2)
    vc = (v[..., 0] + 1j * v[..., 1]).astype(np.complex64)
    ref = oracle.herk_c128(vc.astype(np.complex128), N, K, B)
    got = run_float(vc, COMPUTE_FP4_SPLIT, store_mode)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("nvfp4 split exact-input max rel err", store_mode, err)
    assert err < 1e-6
    assert np.array_equal(got, run_float(vc, COMPUTE_FP4, store_mode))


def test_nvfp4_split_error(workload):
    # hi + lo: the residual of each block is quantised again with its own block
    # scale, so a sample keeps ~2x the bits of plain NVFP4; hi.hi + hi.lo + lo.hi
    # enter the sum (lo.lo, ~1/64 of the signal, is left out; autocorrelations
    # are exact row powers).  The 20-sigma bursts that set plain NVFP4's worst
    # case (~6e-2) keep their small component now: the 2e-2 bound holds on the
    # burst workload (numpy emulation of the same quantiser: 5.2e-3).
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    v, ref = workload
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP4_SPLIT), ref, v.shape[1])
    err4 = oracle.correlation_errors(run_float(v, COMPUTE_FP4), ref, v.shape[1])
    print("nvfp4 split", err, "plain", err4)
    assert err["max_offdiag_norm"] < 2e-2
    assert err["rms_offdiag_norm"] < err4["rms_offdiag_norm"] / 4
    assert err["max_auto_rel"] < 1e-5


def test_nvfp4_split_batch_and_ragged():
    # N not a multiple of the 64 x 128 tile, K not a multiple of the 128-sample
    # k-block, several channels: each channel against its own FP64 product
    from ftd_b200._lib import COMPUTE_FP4_SPLIT
    B, N, K = 3, 200, 200
    v = oracle.workload4_voltages(407, B, N, K)
    ref = oracle.herk_c128(v.astype(np.complex128), N, K, B)
    err = oracle.correlation_errors(run_float(v, COMPUTE_FP4_SPLIT), ref, N)
    print("nvfp4 split ragged", err)
    assert err["max_offdiag_norm"] < 3e-2 and err["max_auto_rel"] < 1e-5


@pytest.mark.parametrize("compute_name", ["COMPUTE_FP4", "COMPUTE_FP4_SPLIT"])
def test_nvfp4_pair_equals_single_cta(compute_name):
    # the two NVFP4 kernels quantise alike and differ only in the order of
    # the FP32 accumulation: equal to FP32 rounding of the sums (rtol 1e-5 of
    # the largest correlation), on ragged sizes across several channels
    import ftd_b200._lib as L
    compute = getattr(L, compute_name)
    B, N, K = 3, 600, 200
    v = oracle.workload4_voltages(408, B, N, K)
    a = run_float(v, compute, 0)
    b = run_float(v, compute, 2)
    assert np.isfinite(b).all()
    assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max()


@pytest.mark.parametrize("N,K,B", [(1, 1, 1), (50, 8, 2), (113, 129, 1), (257, 64, 2)])
@pytest.mark.parametrize("store_mode", [0, 2])
def test_nvfp4_edge_sizes(N, K, B, store_mode):
    # fewer inputs than one tile, one sample, sizes one past the tile and
    # k-block edges: every element written, autocorrelations exact, the
    # cross terms within NVFP4's bound of the FP64 product
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    rng = np.random.default_rng(N * 1000 + K)
    v = (rng.normal(size=(B, N, K)) + 1j * rng.normal(size=(B, N, K))).astype(np.complex64)
    ref = oracle.herk_c128(v.astype(np.complex128), N, K, B)
    # worst single-sample case: a component near 5 in block-scale units rounds
    # by 1 (E2M1 spacing 2 above 4), ~20% of the sample, twice in a product
    for compute, bound in ((COMPUTE_FP4, 0.5), (COMPUTE_FP4_SPLIT, 0.1)):
        got = run_float(v, compute, store_mode)
        assert np.isfinite(got).all()
        err = oracle.correlation_errors(got, ref, N)
        assert err["max_auto_rel"] < 1e-5
        assert err["max_offdiag_norm"] < bound, (compute, err)


@pytest.mark.parametrize("store_mode", [0, 2])
@pytest.mark.parametrize("kind", ["rfi", "gauss"])
def test_nvfp4_matches_restated_quantiser(store_mode, kind):
    # the GPU result against oracle.herk_nvfp4: the same quantised operands
    # (row scale, rounded-up UE4M3 block scales, E2M1 round-to-nearest-even;
    # split: the fused residual), products summed in FP64.  What is left is
    # the FP32 accumulation of the MMAs and the FP32 epilogue scaling (measured
    # 1e-8..6e-7 of the largest element): bound 1e-6 plain, 1e-5 split (room
    # for a lo code flipped by the residual's last-bit rounding, one lo
    # quantum).  Autocorrelations: float32 of FP64 sums.
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    B, N, K = 2, 300, 256
    if kind == "rfi":
        v = oracle.workload4_voltages(410, B, N, K)
    else:
        rng = np.random.default_rng(411)
        v = (rng.normal(size=(B, N, K)) + 1j * rng.normal(size=(B, N, K))).astype(np.complex64)
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    diag = (i[order] == j[order])
    for compute, split, tol in ((COMPUTE_FP4, False, 1e-6), (COMPUTE_FP4_SPLIT, True, 1e-5)):
        got = run_float(v, compute, store_mode).astype(np.float64)
        ref = oracle.herk_nvfp4(v, split)
        scale = np.abs(ref).max()
        err = np.abs(got - ref)
        print(kind, store_mode, split, "max rel err vs restated quantiser",
              err[:, ~diag].max() / scale)
        assert err[:, ~diag].max() <= tol * scale
        np.testing.assert_allclose(got[:, diag, 0], ref[:, diag, 0], rtol=1e-6)


@pytest.mark.parametrize("store_mode", [0, 2])
def test_fp8_float_modes_match_restated_quantiser(store_mode):
    # per-channel-scaled E4M3 (and hi + lo split) of float voltages against
    # oracle.herk_fp8_scaled: the same quantised operands summed in FP64; the
    # rest is FP32 accumulation and the FP32 scale 1 / s^2 (bound 1e-6 of the
    # largest element, 1e-5 split)
    B, N, K = 2, 300, 256
    v = oracle.workload4_voltages(412, B, N, K)
    for compute, split, tol in ((COMPUTE_FP8, False, 1e-6), (COMPUTE_FP8_SPLIT, True, 1e-5)):
        got = run_float(v, compute, store_mode).astype(np.float64)
        ref = oracle.herk_fp8_scaled(v, split)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        print("fp8", store_mode, split, "max rel err vs restated quantiser", err)
        assert err <= tol


@pytest.mark.parametrize("store_mode", [0, 2])
def test_fp8_float_channel_scales_graph_replay(store_mode):
    # nine channels whose amplitudes span 1e-3 .. 1e3 (one of them all zero),
    # an odd K (8-byte loads, a ragged last unit) and a row count that splits
    # unevenly over the promotion's blocks: every channel against the restated
    # quantiser at 1e-6 of its own largest element, and graph capture plus
    # two replays give the direct call's bits
    B, N, K = 9, 130, 203
    rng = np.random.default_rng(414)
    v = (rng.standard_normal((B, N, K)) + 1j * rng.standard_normal((B, N, K))).astype(np.complex64)
    v *= (10.0 ** np.linspace(-3, 3, B)).astype(np.float32)[:, None, None]
    v[4] = 0
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    ref = oracle.herk_fp8_scaled(v, False)
    outs = []
    with Correlator() as c:
        c.set_strategy(store_mode, 0)
        for graph in (False, True, True):
            c.set_graph_mode(graph)
            C = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
            c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP32, tune=False)
            torch.cuda.synchronize()
            outs.append(C.cpu().numpy())
        assert c.graph_count() >= 1
        assert c.device_status() == 0
    got = outs[0].astype(np.float64)
    for b in range(B):
        scale = max(np.abs(ref[b]).max(), 1e-30)
        assert np.abs(got[b] - ref[b]).max() <= 1e-6 * scale, b
    assert not np.any(outs[0][4])
    assert np.array_equal(outs[1], outs[0]) and np.array_equal(outs[2], outs[0])


@pytest.mark.parametrize("B,N,K,store_mode", [(1, 64, 128, 0), (40, 16, 64, 2), (3, 129, 1024, 0)])
def test_fp8_float_promotion_step_edges(B, N, K, store_mode):
    # one channel (one amax step, one quantisation step), forty small
    # channels (forty waits between blocks; the CTA pair's -Re plane), and
    # rows that split unevenly over the promotion's blocks: the restated
    # quantiser (exact operands, FP64 sums) within the FP32 accumulation of
    # K products, bounded by 1e-6 per 256 of K of each channel's largest
    # element (measured 1.1e-6 at K = 1024)
    rng = np.random.default_rng(415 + B)
    v = (rng.standard_normal((B, N, K)) + 1j * rng.standard_normal((B, N, K))).astype(np.complex64)
    v *= rng.uniform(0.01, 100.0, size=(B, 1, 1)).astype(np.float32)
    got = run_float(v, COMPUTE_FP8, store_mode).astype(np.float64)
    ref = oracle.herk_fp8_scaled(v, False)
    tol = 1e-6 * max(1.0, K / 256)
    for b in range(B):
        assert np.abs(got[b] - ref[b]).max() <= tol * np.abs(ref[b]).max(), b


@pytest.mark.parametrize("store_mode", [0, 2])
def test_fp8_float_fp16_output_is_rounded_fp32_output(store_mode):
    # FP32 voltages, per-channel-scaled FP8, FP16 packed output: the epilogue
    # rounds the same scaled FP32 sums to half (nearest even), so the FP16
    # triangles equal the FP32 ones rounded by torch, bit for bit
    from ftd_b200._lib import OUT_FP16
    B, N, K = 3, 200, 256
    rng = np.random.default_rng(416)
    v = (rng.standard_normal((B, N, K)) + 1j * rng.standard_normal((B, N, K))).astype(np.complex64)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    C32 = torch.full((B, tri_size(N), 2), float("nan"), device=DEV)
    C16 = torch.full((B, tri_size(N), 2), float("nan"), dtype=torch.float16, device=DEV)
    with Correlator() as c:
        c.set_strategy(store_mode, 0)
        c.herk(A, C32, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP32, tune=False)
        c.herk(A, C16, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP16, tune=False)
        assert c.device_status() == 0
    assert torch.equal(C16, C32.half())


@pytest.mark.parametrize("store_mode", [0, 2])
def test_fp8_float_alpha_beta(store_mode):
    # C = alpha * (per-channel-scaled FP8 product) + beta * C_old, with the
    # diagonal's Im of the product zero before beta (the reference's store
    # rule); FP32 accumulation and scaling: 1e-6 of the largest element
    B, N, K = 2, 160, 256
    rng = np.random.default_rng(417)
    v = (rng.standard_normal((B, N, K)) + 1j * rng.standard_normal((B, N, K))).astype(np.complex64)
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    old = torch.randn(B, tri_size(N), 2, device=DEV)
    C = old.clone()
    with Correlator() as c:
        c.set_strategy(store_mode, 0)
        c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP32, alpha=0.5,
               beta=-2.0, tune=False)
        assert c.device_status() == 0
    ref = 0.5 * oracle.herk_fp8_scaled(v, False) - 2.0 * old.double().cpu().numpy()
    got = C.double().cpu().numpy()
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_nvfp4_rfi_at_independent_times_and_handle_reuse():
    # bursts at each input's own random times (the union of flagged samples is
    # ~10x the shared-time case: F ~ 120 of K = 1024, still one lo stage), a
    # channel with no bursts, and a silent input: the GPU equals the restated
    # quantiser, the error stays within 2e-2, and calls alternating plain /
    # split / plain on one handle give the plain result both times (the lo
    # extent of every channel is rewritten by each call)
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT
    rng = np.random.default_rng(412)
    B, N, K = 3, 256, 1024
    v = oracle.workload4_voltages(413, B, N, K, rfi_time_frac=0.0)
    for b in (0, 1):  # channel 2 keeps no bursts
        amp = 20.0 * np.sqrt(np.mean(np.abs(v[b]) ** 2))
        for i in rng.choice(N, size=N // 20, replace=False):
            ts = rng.choice(K, size=K // 100, replace=False)
            v[b, i, ts] = (amp * np.exp(2j * np.pi * rng.uniform(size=ts.size))).astype(np.complex64)
    v[1, 7] = 0  # a silent input
    order, nflag = oracle.nvfp4_time_order(v)
    assert nflag[0] > 50 and nflag[1] > 50 and nflag[2] == 0
    A = torch.from_numpy(np.ascontiguousarray(v).view(np.float32).reshape(B, N, K, 2)).to(DEV)
    C = torch.empty(B, tri_size(N), 2, device=DEV)
    outs = []
    with Correlator() as c:
        c.set_strategy(2, 0)
        for compute in (COMPUTE_FP4, COMPUTE_FP4_SPLIT, COMPUTE_FP4):
            c.herk(A, C, N, K, B, input=IN_FP32, compute=compute, output=OUT_FP32, tune=False)
            assert c.device_status() == 0
            outs.append(C.cpu().numpy().astype(np.float64))
    assert np.array_equal(outs[0], outs[2])
    ref = oracle.herk_nvfp4(v)
    scale = np.abs(ref).max()
    assert np.abs(outs[0] - ref).max() <= 1e-6 * scale
    exact = oracle.herk_c128(v.astype(np.complex128), N, K, B)
    err = oracle.correlation_errors(outs[0], exact, N)
    print("nvfp4 independent-time rfi", err)
    assert err["max_offdiag_norm"] < 2e-2 and err["max_auto_rel"] < 1e-5
    assert np.all(outs[0][1][tri_size(7) + 7] == 0)  # the silent input's autocorrelation
