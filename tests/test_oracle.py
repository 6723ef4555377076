"""The oracle against the reference's own host correlator and the golden
fixtures made from it (CPU only)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle


def _golden(golden_dir):
    return sorted(glob.glob(os.path.join(golden_dir, "*.npz")))


def test_codec_roundtrip_all_codes():
    # every QC byte decodes to the integer pair the reference's decode_qc_byte
    # yields (tests/visibility_pipeline_test.cpp:42-53); encode is its inverse
    # on [-7, 7] (test_herk_int4.cu:41-45)
    codes = np.arange(256, dtype=np.uint8)
    re, im = oracle.decode_qc(codes)
    for b in range(256):
        hr, lr = b >> 4, b & 15
        assert re[b] == (-(hr & 7) if hr & 8 else hr & 7)
        assert im[b] == (-(lr & 7) if lr & 8 else lr & 7)
    v = np.arange(-7, 8, dtype=np.int32)
    R, I = np.meshgrid(v, v, indexing="ij")
    back = oracle.decode_qc(oracle.encode_qc(R, I))
    assert np.array_equal(back[0], R) and np.array_equal(back[1], I)


def test_oracle_matches_golden(golden_dir):
    files = _golden(golden_dir)
    assert len(files) >= 8
    for f in files:
        z = np.load(f)
        N, K, B = int(z["N"]), int(z["K"]), int(z["batch"])
        got = oracle.herk_qc(z["qc"], N, K, B)
        assert np.array_equal(got, z["tri"].astype(np.int64)), os.path.basename(f)


def test_oracle_rows_subset_matches_full():
    qc = oracle.gaussian_qc(5, 2, 70, 33)
    full = oracle.herk_qc(qc, 70, 33, 2)
    part = oracle.herk_qc_rows(qc, 70, 33, 1, 20, 45)
    P0, P1 = 20 * 21 // 2, 45 * 46 // 2
    assert np.array_equal(part, full[1, P0:P1])


def test_oracle_float_matches_int():
    qc = oracle.gaussian_qc(6, 2, 40, 17)
    re, im = oracle.decode_qc(qc)
    a = re.astype(np.float64) + 1j * im.astype(np.float64)
    assert np.array_equal(oracle.herk_c128(a, 40, 17, 2), oracle.herk_qc(qc, 40, 17, 2).astype(np.float64))


def test_oracle_hermitian_identity():
    # diagonal = sum |a|^2 (real), trace identity, conjugate symmetry via numpy
    qc = oracle.gaussian_qc(8, 1, 33, 50)
    re, im = oracle.decode_qc(qc)
    a = (re + 1j * im).astype(np.complex128)[0]
    R = a @ a.conj().T
    got = oracle.herk_qc(qc, 33, 50, 1)[0]
    i, j = np.tril_indices(33)
    order = np.lexsort((j, i))
    ref = R[i[order], j[order]]
    assert np.array_equal(got[:, 0], np.rint(ref.real).astype(np.int64))
    im_ref = np.where(i[order] == j[order], 0, np.rint(ref.imag)).astype(np.int64)
    assert np.array_equal(got[:, 1], im_ref)


@pytest.mark.skipif(oracle.ref_lib() is None, reason="reference host code not built here")
def test_oracle_matches_reference_cpu_herk_fresh_inputs():
    rng = np.random.default_rng(2024)
    for (N, K, B) in [(3, 2, 2), (65, 129, 2), (130, 64, 1)]:
        qc = rng.integers(0, 256, size=B * N * K, dtype=np.uint8)
        ref = oracle.ref_cpu_herk(qc, N, K, B)
        assert np.array_equal(oracle.herk_qc(qc, N, K, B).astype(np.float64), ref)


# ------------------------------------------------ raw packet-ordered input
def _ftd_golden(golden_dir):
    return sorted(glob.glob(os.path.join(golden_dir, "ftd", "*.npz")))


def test_ftd_corner_turn_matches_golden(golden_dir):
    # the oracle's corner turn + int64 HERK against cpu_herk_ftd's triangles
    files = _ftd_golden(golden_dir)
    assert len(files) >= 2
    for f in files:
        z = np.load(f)
        a, c, p = int(z["n_ant"]), int(z["n_chan"]), int(z["n_pol"])
        ti, t = int(z["n_time_inner"]), int(z["n_time"])
        bf = oracle.ftd_to_batch_first(z["raw"], a, c, p, t, ti, oracle.LAYOUT_TIME_ANT_CHAN_POL)
        got = oracle.herk_qc(bf, a, t // ti, bf.shape[0])
        assert np.array_equal(got, z["tri"].astype(np.int64)), os.path.basename(f)


def test_ftd_corner_turn_matches_reference_fresh_inputs():
    if oracle.ref_lib() is None or not hasattr(oracle.ref_lib(), "ref_cpu_herk_ftd"):
        pytest.skip("reference host correlator not built")
    rng = np.random.default_rng(77)
    for (a, c, p, ti, K) in [(9, 4, 2, 3, 17), (16, 1, 1, 1, 64), (5, 2, 3, 2, 5)]:
        t = K * ti
        raw = rng.integers(0, 256, size=t * a * c * p, dtype=np.uint8)
        bf = oracle.ftd_to_batch_first(raw, a, c, p, t, ti, oracle.LAYOUT_TIME_ANT_CHAN_POL)
        R = oracle.herk_qc(bf, a, K, bf.shape[0]).astype(np.float32)
        for b in range(bf.shape[0]):
            assert np.array_equal(R[b], oracle.ref_cpu_herk_ftd(raw, b, a, c, p, ti, t)), (a, b)


def test_ftd_chan_pol_ant_time_index_map():
    # [chan][pol][ant][t], t = ti*K + k: restates the index arithmetic of
    # qc_pol_gather_transpose_kernel (lib/bench_pipeline.cu:321-330), which
    # writes pol p of (ch, t_inner, ant, k) from
    # qc[ch*2*n_ant*n_time + p*n_ant*n_time + ant*n_time + t_inner*K + k]
    a, c, p, ti, K = 6, 3, 2, 2, 9
    t = ti * K
    raw = np.random.default_rng(3).integers(0, 256, size=c * p * a * t, dtype=np.uint8)
    bf = oracle.ftd_to_batch_first(raw, a, c, p, t, ti, oracle.LAYOUT_CHAN_POL_ANT_TIME)
    for ch in range(c):
        for pol in range(p):
            for tin in range(ti):
                for ant in range(a):
                    for k in range(K):
                        src = ch * p * a * t + pol * a * t + ant * t + tin * K + k
                        b = (ch * p + pol) * ti + tin
                        assert bf[b, ant, k] == raw[src]


def test_ftd_pol_sum_is_sum_over_pols():
    # pol_sum concatenates the pols along the sample axis: its HERK equals the
    # sum of the per-pol HERKs (the reference adds pol 1 with beta = 1)
    a, c, p, ti, K = 11, 2, 2, 2, 20
    t = ti * K
    rng = np.random.default_rng(4)
    for layout in (oracle.LAYOUT_TIME_ANT_CHAN_POL, oracle.LAYOUT_CHAN_POL_ANT_TIME):
        raw = rng.integers(0, 256, size=c * p * a * t, dtype=np.uint8)
        per = oracle.ftd_to_batch_first(raw, a, c, p, t, ti, layout)
        summed = oracle.ftd_to_batch_first(raw, a, c, p, t, ti, layout, pol_sum=True)
        Rp = oracle.herk_qc(per, a, K, per.shape[0]).reshape(c, p, ti, -1, 2)
        Rs = oracle.herk_qc(summed, a, p * K, summed.shape[0]).reshape(c, ti, -1, 2)
        assert np.array_equal(Rs, Rp.sum(axis=1))


# ------------------------------------------------ imaging
def _tri(i, j):
    return i * (i + 1) // 2 + j


def test_imaging_point_and_mirror():
    # test_gridding_scatter_fp32_grid (lib/test_imaging.cu:109-160): baseline
    # (1, 0) at u = 2 lambda, v = 3 lambda, cell 1, vis (1, 0.5) lands at
    # (Ng/2 + 2, Ng/2 + 3) and its conjugate at (Ng/2 - 2, Ng/2 - 3)
    n, ng, f = 4, 32, 1.0e9
    lam = oracle.C_LIGHT / f
    uv = np.zeros((n * (n + 1) // 2, 2), dtype=np.float32)
    uv[_tri(1, 0)] = [2.0 * lam, 3.0 * lam]
    vis = np.zeros((1, 1, n * (n + 1) // 2, 2), dtype=np.float32)
    vis[0, 0, _tri(1, 0)] = [1.0, 0.5]
    g = oracle.image_grid(vis, uv, np.array([f]), n, ng, 1.0)
    h = ng // 2
    assert g[0, h + 3, h + 2] == 1.0 + 0.5j and g[0, h - 3, h - 2] == 1.0 - 0.5j
    assert np.count_nonzero(g) == 2  # the other baselines carry zero visibility


def test_imaging_auto_not_mirrored_and_pol_sum():
    # test_conjugate_symmetry (lib/test_imaging.cu:163-217): an auto-correlation
    # at u = 5 appears once, a cross-correlation at u = 3 at +-3 (conjugated)
    n, ng, f = 3, 32, 1.0e9
    lam = oracle.C_LIGHT / f
    uv = np.zeros((6, 2), dtype=np.float32)
    uv[_tri(1, 1), 0] = 5.0 * lam
    uv[_tri(2, 0), 0] = 3.0 * lam
    vis = np.zeros((1, 2, 6, 2), dtype=np.float32)
    vis[0, 0, _tri(1, 1)] = [2.0, 1.0]
    vis[0, 0, _tri(2, 0)] = [4.0, 2.0]
    vis[0, 1, _tri(2, 0)] = [1.0, 1.0]      # second pol adds before gridding
    g = oracle.image_grid(vis, uv, np.array([f]), n, ng, 1.0)
    h = ng // 2
    assert g[0, h, h + 5] == 2.0 + 1.0j and g[0, h, h - 5] == 0
    assert g[0, h, h + 3] == 5.0 + 3.0j and g[0, h, h - 3] == 5.0 - 3.0j


def test_imaging_beams_and_fft_definition():
    # test_beam_extraction_fp32 (lib/test_imaging.cu:624-660): |3+4i|^2 / Ng^2 etc.
    ng = 16
    img = np.zeros((1, ng, ng), dtype=np.complex128)
    img[0, 4, 5], img[0, 7, 8], img[0, 0, 0] = 3 + 4j, 1, 2j
    b = oracle.beam_intensity(img, [(4, 5), (7, 8), (0, 0), (-1, 3)])
    assert np.allclose(b[0], [25 / ng**2, 1 / ng**2, 4 / ng**2, 0])
    # a unit point at the grid centre transforms to |image| = 1 everywhere
    # (test_fft_roundtrip_fp32, lib/test_imaging.cu:287-323)
    g = np.zeros((1, 32, 32), dtype=np.complex128)
    g[0, 16, 16] = 1
    assert np.allclose(np.abs(oracle.image_from_grid(g)), 1.0)


def test_imaging_roundf_halves_away_from_zero():
    x = np.array([0.5, 1.5, 2.5, -0.5, -1.5, 0.49999997], dtype=np.float32)
    assert list(oracle._roundf(x)) == [1, 2, 3, -1, -2, 0]


# ------------------------------------------------ XEngine conventions
def test_xengine_twos_complement_decode():
    # promote_to_float (tests/xengine_test.cpp:162-167): low nibble Re, high
    # nibble Im, each a sign-extended 4-bit two's complement value
    b = np.arange(256, dtype=np.uint8)
    re, im = oracle.decode_twos(b)
    for x in range(256):
        lo, hi = x & 15, x >> 4
        assert re[x] == (lo - 16 if lo >= 8 else lo) and im[x] == (hi - 16 if hi >= 8 else hi)


def test_xengine_upper_packing_and_hermitian():
    rng = np.random.default_rng(2)
    n, K, B = 5, 7, 2
    p = rng.integers(0, 256, size=B * K * n, dtype=np.uint8)
    full = oracle.xengine(p, n, K, B, 0)
    tri = oracle.xengine(p, n, K, B, 1)
    assert np.allclose(full, np.conj(np.transpose(full, (0, 2, 1))))
    k = 0
    for r in range(n):          # row-major upper: (r, c >= r) at r*n - r(r-1)/2 + c - r
        for c in range(r, n):
            assert k == r * n - r * (r - 1) // 2 + c - r
            assert tri[0, k] == full[0, r, c]
            k += 1


def test_nvfp4_restatement_exact_on_representable_input():
    # E2M1 values times per-block powers of two with a 6 in every block: the
    # restated quantiser returns the input up to the rounding of the float32
    # row scale g = amax / 2688 (codes x block scale exact), and the split
    # residual is that rounding alone
    rng = np.random.default_rng(5)
    B, N, K = 2, 9, 32
    e = rng.choice(oracle.E2M1_GRID, size=(B, N, K, 2)) * rng.choice([-1.0, 1.0], size=(B, N, K, 2))
    blocks = e.reshape(B, N, K // 8, 16)
    blocks[..., 0] = 6.0
    blocks *= 2.0 ** rng.integers(-2, 1, size=(B, N, K // 8, 1))
    v = blocks.reshape(B, N, K, 2)
    vc = (v[..., 0] + 1j * v[..., 1]).astype(np.complex64)
    hi, lo, g = oracle.nvfp4_quantize(vc, split=True)
    deq = hi * g[..., None].astype(np.float64)
    assert np.abs(deq - vc).max() <= 1e-6 * np.abs(vc).max()
    assert np.abs(lo).max() <= 1e-5 * np.abs(hi).max()
    got = oracle.herk_nvfp4(vc)
    ref = oracle.herk_c128(vc.astype(np.complex128), N, K, B)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def test_nvfp4_restatement_rounding_rules():
    x = np.array([0.25, 0.75, 1.25, 1.75, 2.5, 3.5, 5.0, 7.0, -0.75, 0.2, 0.3], np.float32)
    assert np.array_equal(oracle.e2m1_rne(x),
                          np.array([0, 1, 1, 2, 2, 4, 4, 6, -1, 0, 0.5], np.float32))
    v = np.array([0.0, 1.0, 1.01, 447.0, 500.0, 0.001], np.float32)
    assert np.array_equal(oracle.ue4m3_ceil(v),
                          np.array([0, 1, 1.125, 448, 448, 2.0 ** -9], np.float32))


def test_nvfp4_block_scale_by_squared_error():
    # the block scale is the better of the rounded-up UE4M3 scale (no element
    # saturates) and the next smaller code (the largest may saturate at 6, the
    # rest land on finer steps): never worse than the rounded-up scale, and
    # strictly better for a good share of Gaussian blocks
    f32 = np.float32
    rng = np.random.default_rng(3)
    xs = (rng.normal(size=(2000, 16)) * np.exp(rng.normal(size=(2000, 1)))).astype(f32)[None]
    q, codes, gb = oracle._nvfp4_pass(xs, np.ones((1, 1, 1), f32))
    amax = np.abs(xs).max(-1, keepdims=True)
    b0 = oracle.ue4m3_ceil((amax / f32(6)).astype(f32)).astype(np.float64)
    q0 = oracle.e2m1_rne((xs * (f32(1) / b0.astype(f32))).astype(f32)) * b0
    e, e0 = ((q - xs) ** 2).sum(-1), ((q0 - xs) ** 2).sum(-1)
    assert np.all(e <= e0 * (1 + 1e-6))
    smaller = gb[..., 0] < b0[..., 0].astype(f32)
    assert 0.1 < smaller.mean() < 0.9 and np.all(e[smaller] < e0[smaller])
    assert np.abs(codes[smaller]).max() == 6.0  # saturated elements occur


def test_nvfp4_time_order_moves_bursts_last():
    # flagged samples (|v|^2 > 25 x the row's mean power in any row) go to the
    # end of the channel's time axis in order; the lo residual covers the
    # stages from floor((K - F) / 128) on
    B, N, K = 2, 40, 300
    v = oracle.workload4_voltages(12, B, N, K, rfi_time_frac=0.02)  # 6 burst samples
    order, nflag = oracle.nvfp4_time_order(v)
    for b in range(B):
        assert sorted(order[b]) == list(range(K))
        F = int(nflag[b])
        assert F == 6
        burst = set(np.nonzero((np.abs(v[b]) > 10 * np.abs(v[b]).std()).any(0))[0])
        assert set(order[b][K - F:]) == burst
        assert np.all(np.diff(order[b][:K - F]) > 0) and np.all(np.diff(order[b][K - F:]) > 0)
        assert oracle.nvfp4_lo_stages(K, F, False) == 3 - (K - F) // 128 == 1
    assert oracle.nvfp4_lo_stages(K, 0, False) == 0 and oracle.nvfp4_lo_stages(K, 0, True) == 3
    g = oracle.workload4_voltages(13, 1, 64, 512, rfi_time_frac=0.0)
    assert oracle.nvfp4_time_order(g)[1][0] == 0  # Gaussian voltages: nothing flagged


def test_nvfp4_restated_accuracy_on_the_burst_workload():
    # the quantiser alone (FP64 products of its operands) on the precision
    # configuration's distribution: plain NVFP4 within 2e-2, split within 5e-3
    B, N, K = 2, 256, 1024
    v = oracle.workload4_voltages(21, B, N, K)
    ref = oracle.herk_c128(v.astype(np.complex128), N, K, B)
    plain = oracle.correlation_errors(oracle.herk_nvfp4(v), ref, N)
    split = oracle.correlation_errors(oracle.herk_nvfp4(v, split=True), ref, N)
    assert plain["max_offdiag_norm"] < 2e-2 and split["max_offdiag_norm"] < 5e-3


def test_e4m3_restatement_rounding_rules():
    # ties to the even code, saturation at 448, subnormals (spacing 2^-9)
    x = np.array([1.0625, 1.1875, 448.0, 480.0, 1000.0, 2.0 ** -10, 3 * 2.0 ** -10, -1.0625, 0.0],
                 np.float32)
    want = np.array([1.0, 1.25, 448.0, 448.0, 448.0, 0.0, 2.0 ** -8, -1.0, 0.0], np.float32)
    assert np.array_equal(oracle.e4m3_rne(x), want)


# ------------------------------------------------ pinned to the reference's own helpers
# DataPromote, HermToTri, tri_decode and uv_cell are device code of the
# reference; oracle/build_ref.sh extracts them and ref_harness.cpp compiles
# them for the host, so the restatements below are checked against the
# reference's own arithmetic, not against a reading of it.
needs_ref_kernels = pytest.mark.skipif(oracle.ref_kernels() is None,
                                       reason="reference helpers not built here")


@needs_ref_kernels
def test_decode_twos_pinned_to_data_promote_all_bytes():
    b = np.arange(256, dtype=np.uint8)
    re, im = oracle.decode_twos(b)
    for host_test in (False, True):  # the kernel functor and the test's host decode
        rr, ri = oracle.ref_data_promote(b, host_test=host_test)
        assert np.array_equal(re.astype(np.float64), rr)
        assert np.array_equal(im.astype(np.float64), ri)


@needs_ref_kernels
def test_xengine_oracle_pinned_to_promote_and_herm_to_tri():
    # the reference XEngine chain: promoteData (DataPromote) -> C = M^H M per
    # block -> triangulateFromHerm (HermToTri, packed upper, row-major)
    rng = np.random.default_rng(31)
    for (n, K, B) in [(1, 1, 1), (5, 7, 2), (33, 20, 3), (64, 9, 2)]:
        p = rng.integers(0, 256, size=B * K * n, dtype=np.uint8)
        re, im = oracle.ref_data_promote(p)
        M = (re + 1j * im).reshape(B, K, n)
        full = np.einsum("btr,btc->brc", np.conj(M), M)
        tri = oracle.ref_herm_to_tri(full)
        assert np.array_equal(oracle.xengine(p, n, K, B, 1), tri)
        assert np.array_equal(oracle.xengine(p, n, K, B, 0), full)


@needs_ref_kernels
def test_tri_rows_cols_pinned_to_tri_decode():
    # every packed index of a 2048-input triangle (2,098,176 entries): the
    # reference's float decode and the oracle's exact one agree there
    n = 2048
    r, c = oracle.ref_tri_decode(n * (n + 1) // 2)
    i, j = oracle.tri_rows_cols(n)
    assert np.array_equal(r, i) and np.array_equal(c, j)


@needs_ref_kernels
def test_uv_cells_pinned_to_uv_cell():
    # random baselines over and beyond a 4096 grid, and baselines placed within
    # float resolution of a cell boundary (u / cell + Ng/2 = k + 1/2)
    rng = np.random.default_rng(5)
    ng, f, cell = 4096, 1.4e9, 1.0 / 3000.0
    lam = oracle.C_LIGHT / f
    uv = rng.uniform(-1.2, 1.2, size=(20000, 2)) * (ng / 2) * cell * lam
    k = rng.integers(-ng // 2, ng // 2, size=(4000, 2)) + 0.5
    edge = (k * cell * lam).astype(np.float32)
    nudged = np.concatenate([edge, np.nextafter(edge, np.float32(np.inf)),
                             np.nextafter(edge, np.float32(-np.inf))])
    uv = np.concatenate([uv.astype(np.float32), nudged, np.zeros((1, 2), np.float32)])
    iu, iv, iuc, ivc = oracle.uv_cells(uv, f, cell, ng)
    riu, riv, ul, vl = oracle.ref_uv_cell(uv, f, cell, ng)
    assert np.array_equal(iu, riu) and np.array_equal(iv, riv)
    # the mirror cell, as the scatter kernel forms it from uv_cell's u_lam
    c, h = np.float32(cell), np.float32(0.5 * ng)
    assert np.array_equal(iuc, oracle._roundf((-ul / c).astype(np.float32) + h))
    assert np.array_equal(ivc, oracle._roundf((-vl / c).astype(np.float32) + h))


@needs_ref_kernels
def test_reference_tri_decode_misassigns_large_indices():
    # beyond ~10.6 M entries (inputs > 4607) the reference's float decode puts
    # some diagonal entries on the next row with column -1; the library's
    # gridding decodes exactly, so its cells follow tri_rows_cols there
    n = 4700
    r, c = oracle.ref_tri_decode(n * (n + 1) // 2)
    i, j = oracle.tri_rows_cols(n)
    bad = np.nonzero((r != i) | (c != j))[0]
    assert bad.size > 0 and bad[0] == 10619135
    assert (r[bad[0]], c[bad[0]]) == (4608, -1) and (i[bad[0]], j[bad[0]]) == (4607, 4607)
