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
