"""CPU oracle for the correlator -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module, and only as the checker or the timed CPU
baseline; the product (``ftd_b200``) never does.

* ``liboracle.so`` (``herk_oracle.c``): our C restatement of the reference's
  host correlator ``cpu_herk`` (cutlass_interface/test_herk_int4.cu:51-70)
  with exact int64 accumulation for QC int4 input and FP64 for float input.
* ``_ref/libref_herk.so`` (``build_ref.sh`` + ``ref_harness.cpp``): the
  reference's own ``cpu_herk``, ``encode_int4``, ``decode_qc_byte``,
  ``cpu_herk_batch_first`` and ``cpu_herk_ftd`` compiled from the reference
  tree, used to pin the restatement and as the timed CPU baseline.
* ``ftd_to_batch_first``: the corner turn of raw packet-ordered QC input
  into per-(channel, pol, time_inner) antenna rows, restating the index maps
  of cpu_herk_ftd (tests/visibility_pipeline_test.cpp:55-96) and of
  qc_pol_gather_transpose_kernel (lib/bench_pipeline.cu:306-331).
* Seeded input generators for the workloads the correlator is measured on.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_herk.so")

_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)
_f32p = ctypes.POINTER(ctypes.c_float)

_lib = None
_ref = None


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (if missing/stale)."""
    src = os.path.join(HERE, "herk_oracle.c")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)
    return LIB_PATH


def build_ref() -> str | None:
    """Compile the reference's host correlator into _ref/ (needs the reference tree)."""
    r = subprocess.run(["bash", os.path.join(HERE, "build_ref.sh")], capture_output=True, text=True)
    return REF_PATH if r.returncode == 0 else None


def _p(a, t):
    return a.ctypes.data_as(t)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_encode_qc.argtypes = [_i32p, _i32p, ctypes.c_int64, _u8p]
        L.oracle_decode_qc.argtypes = [_u8p, ctypes.c_int64, _i32p, _i32p]
        L.oracle_herk_qc.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p]
        L.oracle_herk_qc_rows.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, _i64p]
        L.oracle_herk_c128.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def ref_lib():
    """The reference's own host correlator, or None when it was not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_PATH):
            return None
        L = ctypes.CDLL(REF_PATH)
        L.ref_gen_int4.argtypes = [ctypes.c_uint32, ctypes.c_int64, _u8p]
        L.ref_encode.argtypes = [_i32p, _i32p, ctypes.c_int64, _u8p]
        L.ref_cpu_herk.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f64p]
        L.ref_cpu_herk_batch_first.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p]
        if hasattr(L, "ref_cpu_herk_ftd"):
            L.ref_cpu_herk_ftd.argtypes = [_u8p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, _f32p]
        L.ref_num_threads.restype = ctypes.c_int
        if hasattr(L, "ref_data_promote"):
            L.ref_data_promote.argtypes = [_u8p, ctypes.c_int64, _f64p]
            L.ref_promote_to_float.argtypes = [_u8p, ctypes.c_int64, _f64p]
            L.ref_herm_to_tri.argtypes = [_f64p, ctypes.c_int, ctypes.c_int, _f64p]
            L.ref_tri_decode.argtypes = [ctypes.c_int64, _i32p, _i32p]
            L.ref_uv_cell.argtypes = [_f32p, _f32p, ctypes.c_int64, ctypes.c_double,
                                      ctypes.c_float, ctypes.c_float, _f32p, _f32p, _i32p, _i32p]
        _ref = L
    return _ref


def ref_kernels():
    """The reference's XEngine / imaging helpers compiled for the host (None
    when oracle/_ref was built without them)."""
    L = ref_lib()
    return L if L is not None and hasattr(L, "ref_data_promote") else None


def ref_data_promote(b: np.ndarray, host_test: bool = False):
    """(re, im) float64 of QC bytes through the reference's DataPromote functor
    (or, host_test, the XEngine test's promote_to_float)."""
    b = np.ascontiguousarray(b, dtype=np.uint8).reshape(-1)
    out = np.empty(2 * b.size, dtype=np.float64)
    f = ref_kernels().ref_promote_to_float if host_test else ref_kernels().ref_data_promote
    f(_p(b, _u8p), b.size, _p(out, _f64p))
    return out[0::2], out[1::2]


def ref_herm_to_tri(full: np.ndarray) -> np.ndarray:
    """Packed upper triangles [batch, n(n+1)/2] (complex128) of full
    [batch, n, n] matrices through the reference's HermToTri functor."""
    full = np.ascontiguousarray(full, dtype=np.complex128)
    b, n = full.shape[0], full.shape[1]
    out = np.zeros((b, n * (n + 1) // 2), dtype=np.complex128)
    ref_kernels().ref_herm_to_tri(_p(full.view(np.float64), _f64p), n, b,
                                  _p(out.view(np.float64), _f64p))
    return out


def ref_tri_decode(count: int):
    """(row, col) of packed lower indices 0..count-1 by the reference's tri_decode."""
    r = np.empty(count, dtype=np.int32)
    c = np.empty(count, dtype=np.int32)
    ref_kernels().ref_tri_decode(count, _p(r, _i32p), _p(c, _i32p))
    return r, c


def ref_uv_cell(uv_m: np.ndarray, freq_hz: float, cell: float, ng: int):
    """(iu, iv, u_lam, v_lam) of baselines uv_m [n, 2] (metres) by the
    reference's uv_cell."""
    u = np.ascontiguousarray(uv_m[:, 0], dtype=np.float32)
    v = np.ascontiguousarray(uv_m[:, 1], dtype=np.float32)
    n = u.size
    ul, vl = np.empty(n, np.float32), np.empty(n, np.float32)
    iu, iv = np.empty(n, np.int32), np.empty(n, np.int32)
    ref_kernels().ref_uv_cell(_p(u, _f32p), _p(v, _f32p), n, float(freq_hz), float(cell),
                              float(0.5 * ng), _p(ul, _f32p), _p(vl, _f32p), _p(iu, _i32p),
                              _p(iv, _i32p))
    return iu, iv, ul, vl


# ----------------------------------------------------------------- codecs
def encode_qc(re: np.ndarray, im: np.ndarray) -> np.ndarray:
    re = np.ascontiguousarray(re, dtype=np.int32)
    im = np.ascontiguousarray(im, dtype=np.int32)
    out = np.empty(re.shape, dtype=np.uint8)
    lib().oracle_encode_qc(_p(re, _i32p), _p(im, _i32p), re.size, _p(out, _u8p))
    return out


def decode_qc(qc: np.ndarray):
    qc = np.ascontiguousarray(qc, dtype=np.uint8)
    re = np.empty(qc.shape, dtype=np.int32)
    im = np.empty(qc.shape, dtype=np.int32)
    lib().oracle_decode_qc(_p(qc, _u8p), qc.size, _p(re, _i32p), _p(im, _i32p))
    return re, im


# ----------------------------------------------------------------- correlators
def tri_size(n: int) -> int:
    return n * (n + 1) // 2


def herk_qc(qc: np.ndarray, N: int, K: int, batch: int) -> np.ndarray:
    """Exact packed lower triangles, int64 array [batch, N(N+1)/2, 2]."""
    qc = np.ascontiguousarray(qc, dtype=np.uint8).reshape(-1)
    assert qc.size == batch * N * K
    out = np.empty((batch, tri_size(N), 2), dtype=np.int64)
    lib().oracle_herk_qc(_p(qc, _u8p), N, K, batch, _p(out, _i64p))
    return out


def herk_qc_rows(qc: np.ndarray, N: int, K: int, b: int, i0: int, i1: int) -> np.ndarray:
    """Rows [i0, i1) of channel b, int64 [sum_i (i+1), 2] (rows back to back)."""
    qc = np.ascontiguousarray(qc, dtype=np.uint8).reshape(-1)
    n = tri_size(i1) - tri_size(i0)
    out = np.empty((n, 2), dtype=np.int64)
    lib().oracle_herk_qc_rows(_p(qc, _u8p), N, K, b, i0, i1, _p(out, _i64p))
    return out


def herk_c128(a: np.ndarray, N: int, K: int, batch: int) -> np.ndarray:
    """FP64 packed lower triangles for complex input a[batch, N, K] -> [batch, P, 2]."""
    a = np.ascontiguousarray(np.asarray(a, dtype=np.complex128).reshape(batch, N, K))
    av = a.view(np.float64)
    out = np.empty((batch, tri_size(N), 2), dtype=np.float64)
    lib().oracle_herk_c128(_p(av, _f64p), N, K, batch, _p(out, _f64p))
    return out


def ref_cpu_herk(qc: np.ndarray, N: int, K: int, batch: int) -> np.ndarray:
    """The reference's cpu_herk (compiled from its source) -> float64 [batch, P, 2]."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference host correlator not built (oracle/build_ref.sh)")
    qc = np.ascontiguousarray(qc, dtype=np.uint8).reshape(-1)
    out = np.empty((batch, tri_size(N), 2), dtype=np.float64)
    L.ref_cpu_herk(_p(qc, _u8p), N, K, batch, _p(out, _f64p))
    return out


def ref_cpu_herk_ftd(raw: np.ndarray, batch_idx: int, n_ant: int, n_chan: int, n_pol: int,
                     n_time_inner: int, n_time: int) -> np.ndarray:
    """The reference's cpu_herk_ftd for one batch -> float32 [P, 2]."""
    L = ref_lib()
    if L is None or not hasattr(L, "ref_cpu_herk_ftd"):
        raise RuntimeError("reference host correlator not built (oracle/build_ref.sh)")
    raw = np.ascontiguousarray(raw, dtype=np.uint8).reshape(-1)
    out = np.empty((tri_size(n_ant), 2), dtype=np.float32)
    L.ref_cpu_herk_ftd(_p(raw, _u8p), batch_idx, n_ant, n_chan, n_pol, n_time_inner, n_time,
                       _p(out, _f32p))
    return out


# layouts of raw packet-ordered input
LAYOUT_TIME_ANT_CHAN_POL, LAYOUT_CHAN_POL_ANT_TIME = 0, 1


def ftd_to_batch_first(raw: np.ndarray, n_ant: int, n_chan: int, n_pol: int, n_time: int,
                       n_time_inner: int, layout: int, pol_sum: bool = False) -> np.ndarray:
    """Raw QC bytes -> batch-first [batch, n_ant, K'] rows.

    layout 0, [t][ant][chan][pol] with t = k*n_time_inner + ti
      (cpu_herk_ftd, tests/visibility_pipeline_test.cpp:65-75);
    layout 1, [chan][pol][ant][t] with t = ti*K + k
      (qc_pol_gather_transpose_kernel, lib/bench_pipeline.cu:321-330).
    batch b = (chan*n_pol + pol)*n_time_inner + ti, K' = K; with pol_sum the
    pols are concatenated along the sample axis (column pol*K + k), b =
    chan*n_time_inner + ti and K' = n_pol*K.
    """
    K = n_time // n_time_inner
    raw = np.ascontiguousarray(raw, dtype=np.uint8).reshape(-1)
    if layout == LAYOUT_TIME_ANT_CHAN_POL:
        a = raw.reshape(K, n_time_inner, n_ant, n_chan, n_pol)   # [k, ti, ant, chan, pol]
        a = a.transpose(3, 4, 1, 2, 0)                            # [chan, pol, ti, ant, k]
    elif layout == LAYOUT_CHAN_POL_ANT_TIME:
        a = raw.reshape(n_chan, n_pol, n_ant, n_time_inner, K)   # [chan, pol, ant, ti, k]
        a = a.transpose(0, 1, 3, 2, 4)                            # [chan, pol, ti, ant, k]
    else:
        raise ValueError(layout)
    if pol_sum:
        a = a.transpose(0, 2, 3, 1, 4)                            # [chan, ti, ant, pol, k]
        return np.ascontiguousarray(a).reshape(n_chan * n_time_inner, n_ant, n_pol * K)
    return np.ascontiguousarray(a).reshape(n_chan * n_pol * n_time_inner, n_ant, K)


def num_threads() -> int:
    return lib().oracle_num_threads()


# ----------------------------------------------------------------- generators
def gaussian_int4(rng: np.random.Generator, shape, sigma: float = 2.5):
    """Re and Im each round(N(0, sigma^2)) clipped to [-7, 7] (int32 arrays)."""
    re = np.clip(np.rint(rng.normal(0.0, sigma, size=shape)), -7, 7).astype(np.int32)
    im = np.clip(np.rint(rng.normal(0.0, sigma, size=shape)), -7, 7).astype(np.int32)
    return re, im


def gaussian_qc(seed: int, batch: int, N: int, K: int, sigma: float = 2.5) -> np.ndarray:
    """Seeded QC bytes [batch, N, K] with the Gaussian int4 distribution."""
    rng = np.random.default_rng(seed)
    re, im = gaussian_int4(rng, (batch, N, K), sigma)
    return encode_qc(re, im)


# ----------------------------------------------------------------- precision study
def workload4_voltages(seed: int, batch: int, N: int, K: int, rfi_time_frac: float = 0.01,
                       rfi_input_frac: float = 0.05, rfi_sigma: float = 20.0) -> np.ndarray:
    """Complex Gaussian voltages [batch, N, K] (complex64): per-channel RMS
    log-uniform in [0.1, 10]; on `rfi_input_frac` of the inputs, a fraction
    `rfi_time_frac` of the time samples carries a burst of `rfi_sigma` sigma."""
    rng = np.random.default_rng(seed)
    rms = np.exp(rng.uniform(np.log(0.1), np.log(10.0), size=batch))
    v = (rng.normal(size=(batch, N, K)) + 1j * rng.normal(size=(batch, N, K))) / np.sqrt(2.0)
    v *= rms[:, None, None]
    for b in range(batch):
        if rfi_time_frac <= 0 or rfi_input_frac <= 0:
            break
        ins = rng.choice(N, size=max(1, int(round(rfi_input_frac * N))), replace=False)
        ts = rng.choice(K, size=max(1, int(round(rfi_time_frac * K))), replace=False)
        phase = np.exp(2j * np.pi * rng.uniform(size=(len(ins), len(ts))))
        v[b][np.ix_(ins, ts)] = rfi_sigma * rms[b] * phase
    return v.astype(np.complex64)


def correlation_errors(got: np.ndarray, ref: np.ndarray, N: int) -> dict:
    """Errors of packed triangles [batch, P, 2] against an FP64 reference:
    elementwise |dR_ij| / sqrt(R_ii R_jj) (normalised by the autocorrelations,
    the scale-free measure for correlation products) -- max and RMS -- and the
    relative error of the autocorrelations R_ii themselves."""
    g = got[..., 0].astype(np.float64) + 1j * got[..., 1].astype(np.float64)
    r = ref[..., 0] + 1j * ref[..., 1]
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    diag = np.arange(N) * (np.arange(N) + 1) // 2 + np.arange(N)
    auto = r[:, diag].real
    norm = np.sqrt(np.maximum(auto[:, i] * auto[:, j], 1e-300))
    e = np.abs(g - r) / norm
    de = np.abs(g[:, diag].real - auto) / np.maximum(auto, 1e-300)
    off = e[:, i != j]
    return {"max_norm": float(e.max()), "rms_norm": float(np.sqrt(np.mean(e ** 2))),
            "max_offdiag_norm": float(off.max()) if off.size else 0.0,
            "rms_offdiag_norm": float(np.sqrt(np.mean(off ** 2))) if off.size else 0.0,
            "max_auto_rel": float(de.max()), "rms_auto_rel": float(np.sqrt(np.mean(de ** 2)))}


# ----------------------------------------------------------------- gain calibration
def unpack_tri(tri: np.ndarray, N: int) -> np.ndarray:
    """Packed lower triangle [P, 2] (or complex [P]) -> full Hermitian N x N complex128."""
    t = np.asarray(tri)
    if t.ndim == 2 and t.shape[-1] == 2:
        t = t[..., 0].astype(np.float64) + 1j * t[..., 1].astype(np.float64)
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    M = np.zeros((N, N), dtype=np.complex128)
    M[i, j] = t
    M[j, i] = np.conj(t)
    return M


def unpack_tri_real(tri: np.ndarray, N: int) -> np.ndarray:
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    M = np.zeros((N, N), dtype=np.float64)
    M[i, j] = tri
    M[j, i] = tri
    return M


def gain_loss_grad(robs: np.ndarray, rmod: np.ndarray, w: np.ndarray, g: np.ndarray, N: int):
    """FP64 loss and gradient of sum_f ||W o (R_obs - g R_mod g^H)||_F^2 over
    full Hermitian matrices; grad_k = dL/dRe g_k + i dL/dIm g_k
    = -4 sum_f sum_j W_kj E_kj conj(R_mod,kj) g_j."""
    g = np.asarray(g, dtype=np.complex128)
    L = 0.0
    grad = np.zeros(N, dtype=np.complex128)
    for f in range(robs.shape[0]):
        Ro, Rm, W = unpack_tri(robs[f], N), unpack_tri(rmod[f], N), unpack_tri_real(w[f], N)
        E = Ro - g[:, None] * Rm * np.conj(g)[None, :]
        L += float(np.sum(W * np.abs(E) ** 2))
        grad += -4.0 * (W * E * np.conj(Rm)) @ g
    return L, grad


# ----------------------------------------------------------------- imaging
C_LIGHT = 299792458.0


def _roundf(x: np.ndarray) -> np.ndarray:
    """C roundf (halves away from zero) of float32 values, evaluated exactly."""
    x = x.astype(np.float64)
    return (np.sign(x) * np.floor(np.abs(x) + 0.5)).astype(np.int64)


def tri_rows_cols(n: int):
    """Row i and column j of every packed lower-triangle index, in order."""
    i = np.repeat(np.arange(n), np.arange(1, n + 1))
    j = np.arange(n * (n + 1) // 2) - i * (i + 1) // 2
    return i, j


def uv_cells(uv_m: np.ndarray, freq_hz: float, cell: float, ng: int):
    """Cell of each baseline and of its mirror, with the float32 arithmetic of
    uv_cell (include/kernels/imaging_kernels.cuh:37-47): u_lam = float(u / lambda),
    iu = roundf(u_lam / cell + Ng/2); mirror roundf(-u_lam / cell + Ng/2)."""
    lam = C_LIGHT / float(freq_hz)
    ul = (uv_m[:, 0].astype(np.float64) / lam).astype(np.float32)
    vl = (uv_m[:, 1].astype(np.float64) / lam).astype(np.float32)
    c, h = np.float32(cell), np.float32(0.5 * ng)
    iu = _roundf((ul / c).astype(np.float32) + h)
    iv = _roundf((vl / c).astype(np.float32) + h)
    iuc = _roundf((-ul / c).astype(np.float32) + h)
    ivc = _roundf((-vl / c).astype(np.float32) + h)
    return iu, iv, iuc, ivc


def image_grid(vis: np.ndarray, uv_m: np.ndarray, freq_hz: np.ndarray, n_ant: int, ng: int,
               cell: float, taper: np.ndarray | None = None) -> np.ndarray:
    """Pillbox gridding (pillbox_grid_scatter_fp32_fp32grid_kernel,
    include/kernels/imaging_kernels.cuh:219-268) of vis [n_chan, n_pol, n_bl, 2]
    float32, the pols summed first (in pol order, float32) and each
    contribution weighted by the taper at its cell; auto-correlations (i == j)
    are not mirrored.  Returns complex128 [n_chan, Ng, Ng] (exact sums)."""
    n_chan, n_pol = vis.shape[0], vis.shape[1]
    v = vis[:, 0].astype(np.float32).copy()
    for p in range(1, n_pol):
        v = (v + vis[:, p]).astype(np.float32)
    vc = v[..., 0].astype(np.float64) + 1j * v[..., 1].astype(np.float64)
    i, j = tri_rows_cols(n_ant)
    cross = i != j
    w = np.ones((ng, ng)) if taper is None else taper.astype(np.float64).reshape(ng, ng)
    grid = np.zeros((n_chan, ng, ng), dtype=np.complex128)
    for f in range(n_chan):
        iu, iv, iuc, ivc = uv_cells(uv_m, freq_hz[f], cell, ng)
        ok = (iu >= 0) & (iu < ng) & (iv >= 0) & (iv < ng)
        np.add.at(grid[f], (iv[ok], iu[ok]), vc[f][ok] * w[iv[ok], iu[ok]])
        okc = cross & (iuc >= 0) & (iuc < ng) & (ivc >= 0) & (ivc < ng)
        np.add.at(grid[f], (ivc[okc], iuc[okc]), np.conj(vc[f][okc]) * w[ivc[okc], iuc[okc]])
    return grid


def image_from_grid(grid: np.ndarray) -> np.ndarray:
    """Unnormalised inverse 2-D DFT over the last two axes (cuFFT CUFFT_INVERSE)."""
    ng = grid.shape[-1]
    return np.fft.ifft2(grid, axes=(-2, -1)) * (ng * ng)


def beam_intensity(image: np.ndarray, pixels: np.ndarray) -> np.ndarray:
    """|image(row, col)|^2 / Ng^2 per beam, 0 outside the image
    (extract_beam_intensity_kernel, include/kernels/imaging_kernels.cuh:332-361)."""
    ng = image.shape[-1]
    out = np.zeros((image.shape[0], len(pixels)))
    for b, (r, c) in enumerate(pixels):
        if 0 <= r < ng and 0 <= c < ng:
            out[:, b] = np.abs(image[:, r, c]) ** 2 / (ng * ng)
    return out


# ----------------------------------------------------------------- XEngine
def decode_twos(b: np.ndarray):
    """(4,4)b two's complement bytes -> (re, im) int: low nibble Re, high nibble
    Im, each sign-extended (promote_to_float, tests/xengine_test.cpp:162-167)."""
    b = np.asarray(b, dtype=np.uint8)
    re = ((b & 0x0F).astype(np.int16) << 12).astype(np.int16) >> 12
    im = (b.astype(np.int16) << 8).astype(np.int16) >> 12
    return re.astype(np.int64), im.astype(np.int64)


def xengine(payload: np.ndarray, n_ant: int, K: int, batch: int, mat_format: int) -> np.ndarray:
    """verifyXEngine's reference (tests/xengine_test.cpp:242-310): per block
    M [K][n_ant], C = M^H M; mat_format 1 = upper triangle packed row-major,
    0 = full matrix.  Exact (float64 of integer sums)."""
    re, im = decode_twos(np.asarray(payload).reshape(batch, K, n_ant))
    M = re.astype(np.float64) + 1j * im.astype(np.float64)
    C = np.einsum("btr,btc->brc", np.conj(M), M)
    if mat_format == 0:
        return C
    r, c = np.triu_indices(n_ant)
    return C[:, r, c]


# ----------------------------------------------------------------- NVFP4
# A restatement of the library's NVFP4 quantisation (its own format; the
# reference has none) in IEEE float32 steps, so that the GPU result can be
# checked against the same quantised operands to FP32 accumulation rounding.
#  * Per input row: an FP32 scale g = amax_row / (6 * 448) (1 for an empty
#    row) and the FP64 power P = sum_t |v_t|^2.
#  * Block scale of 16 values (8 complex samples, Re/Im interleaved): the
#    candidate UE4M3 codes c0 = the smallest E4M3 value >= amax_blk / (6 g)
#    (at most 448) and c0 - 1 (a code >= 1 only); for each, gb = g b and
#    inv = 1 / gb in float32, codes E2M1(x * inv) (round to nearest, ties to
#    the even code, saturating at 6), d = fma(-code, gb, x) and
#    err = sum of fl(d * d) in float32 in element order; c0 - 1 is kept only
#    on a strictly smaller err.
#  * A lo residual r = fma(-code, gb, x) is quantised the same way with its
#    own block scale (same g) where the mode carries one:
#      split: every stage (128 samples);
#      plain: a channel's time samples t with |v_t|^2 > 25 P / K in any row
#      (FP64 comparison) are flagged; the channel's time axis is permuted to
#      the unflagged samples in order followed by the flagged ones in order
#      (a correlation is invariant under a common permutation of time), and
#      the stages from floor((K - F) / 128) on carry a lo residual (F flagged
#      samples; none when F = 0).
#  * The product is g_i g_j sum (hi_i + lo_i)(hi_j + lo_j)^* without lo lo.
E2M1_GRID = np.array([0.0, 0.5, 1.0, 1.5, 2.0, 3.0, 4.0, 6.0])
NVFP4_STAGE = 128          # samples per correlator stage (K granularity of the lo residual)
NVFP4_RFI_THRESHOLD = 25.0  # |v_t|^2 > 25 x the row's mean power flags sample t


def _e4m3_positive() -> np.ndarray:
    vals = []
    for e in range(16):
        for m in range(8):
            if e == 15 and m == 7:
                continue  # NaN
            vals.append(m / 8 * 2.0 ** -6 if e == 0 else (1 + m / 8) * 2.0 ** (e - 7))
    return np.array(sorted(set(vals)))


_E4M3 = _e4m3_positive()  # index = E4M3 code of each non-negative value


def ue4m3_ceil(v: np.ndarray) -> np.ndarray:
    """Smallest E4M3 value >= v (float32 in), 448 at most, 0 for v <= 0."""
    return _E4M3[ue4m3_ceil_code(v)].astype(np.float32)


def ue4m3_ceil_code(v: np.ndarray) -> np.ndarray:
    """Code of the smallest E4M3 value >= v, 0x7E (448) at most, 0 for v <= 0."""
    v = np.asarray(v, dtype=np.float64)
    idx = np.minimum(np.searchsorted(_E4M3, v, side="left"), len(_E4M3) - 1)
    return np.where(v > 0, idx, 0)


def e2m1_rne(x: np.ndarray) -> np.ndarray:
    """E2M1 value of float32 x: nearest grid value, ties to the even code,
    saturating at +-6."""
    a = np.minimum(np.abs(np.asarray(x, dtype=np.float64)), 6.0)
    d = np.abs(a[..., None] - E2M1_GRID)
    best = d.min(axis=-1, keepdims=True)
    cand = d == best
    codes = np.arange(8)
    # among equally near codes take the even one (ties), else the only one
    score = np.where(cand, np.where(codes % 2 == 0, 0, 1), 9)
    q = E2M1_GRID[np.argmin(score, axis=-1)]
    return np.copysign(q, x).astype(np.float32)


def _fma32(a, b, c):
    """float32 fma(a, b, c): exact in float64 for the operands used here
    (a an E2M1 value, b and c float32 of comparable magnitude or a = 0), then
    rounded once."""
    return (np.asarray(a, np.float64) * np.asarray(b, np.float64)
            + np.asarray(c, np.float64)).astype(np.float32)


def _nvfp4_pass(x: np.ndarray, g: np.ndarray):
    """Quantise float32 values x[..., nblk, 16] under row scales g[..., 1, 1]:
    (codes x block scale as float64, codes float32, g b float32), with the
    block scale picked between two candidates by squared error."""
    f32 = np.float32
    x = x.astype(f32)
    amax = np.abs(x).max(axis=-1, keepdims=True).astype(f32)
    c0 = ue4m3_ceil_code((amax / (f32(6.0) * g)).astype(f32))
    best_q = best_codes = best_gb = best_err = None
    for d in (0, 1):
        c = c0 - d
        valid = (c >= 1) if d > 0 else np.ones_like(c, dtype=bool)
        b = _E4M3[np.maximum(c, 0)].astype(f32)
        gb = (g * b).astype(f32)
        with np.errstate(divide="ignore"):
            inv = np.where(b > 0, f32(1.0) / gb, f32(0.0)).astype(f32)
        codes = e2m1_rne((x * inv).astype(f32))
        dd = _fma32(-codes, gb, x)
        err = np.zeros(dd.shape[:-1] + (1,), dtype=f32)
        for k in range(16):
            err = (err + (dd[..., k:k + 1] * dd[..., k:k + 1]).astype(f32)).astype(f32)
        q = codes.astype(np.float64) * b.astype(np.float64)
        if best_q is None:
            best_q, best_codes, best_gb, best_err = q, codes, np.broadcast_to(gb, codes.shape), err
            continue
        take = valid & (err < best_err)
        best_q = np.where(take, q, best_q)
        best_codes = np.where(take, codes, best_codes)
        best_gb = np.where(take, gb, best_gb)
        best_err = np.where(take, err, best_err)
    return best_q, best_codes, best_gb.astype(f32)


def nvfp4_time_order(v: np.ndarray):
    """Plain-mode time order of each channel of complex64 voltages
    [batch, N, K]: (order [batch, K] source sample of each position,
    flagged count [batch])."""
    B, N, K = v.shape
    e = v.real.astype(np.float64) ** 2 + v.imag.astype(np.float64) ** 2
    p = e.sum(axis=-1, keepdims=True)
    flag = (e > NVFP4_RFI_THRESHOLD * p / K).any(axis=1)
    order = np.empty((B, K), dtype=np.int64)
    for b in range(B):
        order[b] = np.concatenate([np.nonzero(~flag[b])[0], np.nonzero(flag[b])[0]])
    return order, flag.sum(axis=1)


def nvfp4_lo_stages(K: int, flagged: int, split: bool) -> int:
    """Number of trailing correlator stages that carry a lo residual."""
    stages = (K + NVFP4_STAGE - 1) // NVFP4_STAGE
    if split:
        return stages
    return 0 if flagged == 0 else stages - (K - flagged) // NVFP4_STAGE


def nvfp4_quantize(v: np.ndarray, split: bool = False):
    """Complex64 voltages [batch, N, K] -> (hi, lo, g): the dequantised
    operands (code x block scale, without the row scale) as complex128 in the
    quantiser's time order (plain mode permutes flagged samples to the end),
    lo zero where no residual is carried, and the float32 row scales g."""
    f32 = np.float32
    B, N, K = v.shape
    if not split:
        order, nflag = nvfp4_time_order(v)
        v = np.take_along_axis(v, order[:, None, :], axis=-1)
    else:
        nflag = np.zeros(B, dtype=np.int64)
    kp = (K + NVFP4_STAGE - 1) // NVFP4_STAGE * NVFP4_STAGE
    x = np.zeros((B, N, kp, 2), dtype=f32)
    x[:, :, :K, 0] = v.real
    x[:, :, :K, 1] = v.imag
    m = np.abs(x).reshape(B, N, -1).max(axis=-1).astype(f32)
    g = np.where((m > 0) & (m < f32(3.0e38)), m / f32(6.0 * 448.0), f32(1.0)).astype(f32)
    xb = x.reshape(B, N, kp // 8, 16)
    gb = g[:, :, None, None]
    hi, codes, step = _nvfp4_pass(xb, gb)
    resid = _fma32(-codes, step, xb)
    lo, _, _ = _nvfp4_pass(resid, gb)
    for b in range(B):  # keep the residual only in the stages that carry it
        first = kp // 8 - nvfp4_lo_stages(K, int(nflag[b]), split) * (NVFP4_STAGE // 8)
        lo[b, :, :first] = 0.0

    def cplx(a):
        a = a.reshape(B, N, kp, 2)[:, :, :K]
        return a[..., 0] + 1j * a[..., 1]
    return cplx(hi), cplx(lo), g


def herk_nvfp4(v: np.ndarray, split: bool = False) -> np.ndarray:
    """Packed lower triangles [batch, P, 2] (float64) of the NVFP4 product:
    g_i g_j sum_t (hi_i hi_j^* + lo_i hi_j^* + hi_i lo_j^*) over the quantised
    operands, autocorrelations the exact sum |v|^2 rounded to float32."""
    B, N, K = v.shape
    hi, lo, g = nvfp4_quantize(v, split)
    R = np.einsum("bik,bjk->bij", hi, hi.conj())
    R += np.einsum("bik,bjk->bij", lo, hi.conj()) + np.einsum("bik,bjk->bij", hi, lo.conj())
    gg = g.astype(np.float64)
    R *= gg[:, :, None] * gg[:, None, :]
    pw = (v.real.astype(np.float64) ** 2 + v.imag.astype(np.float64) ** 2).sum(axis=-1)
    pw = pw.astype(np.float32)
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    out = np.stack([R[:, i, j].real, R[:, i, j].imag], axis=-1)
    d = i == j
    out[:, d, 0] = pw[:, i[d]]
    out[:, d, 1] = 0.0
    return out


# ----------------------------------------------------------------- FP8 (float input)
# The per-channel-scaled E4M3 quantisation of float voltages (compute modes
# FP8 and FP8 split): s = 448 / amax_channel (1 for an empty channel);
# hi = E4M3(v s), round to nearest with ties to the even code, saturating at
# 448 (subnormals down to 2^-9); split: lo = E4M3(v s - hi) in float32.
# The result is scaled by 1 / (s s).
def _e4m3_table():
    vals, codes = [], []
    for c in range(127):  # positive finite codes (0x7F is NaN)
        e, m = c >> 3, c & 7
        vals.append(m / 8 * 2.0 ** -6 if e == 0 else (1 + m / 8) * 2.0 ** (e - 7))
        codes.append(c)
    return np.array(vals), np.array(codes)


_E4M3_VALS, _E4M3_CODES = _e4m3_table()


def e4m3_rne(x: np.ndarray) -> np.ndarray:
    """E4M3 value of float32 x: nearest, ties to the even code, saturating at
    +-448."""
    x = np.asarray(x, dtype=np.float64)
    a = np.minimum(np.abs(x), 448.0)
    idx = np.clip(np.searchsorted(_E4M3_VALS, a), 1, len(_E4M3_VALS) - 1)
    lo, hi = _E4M3_VALS[idx - 1], _E4M3_VALS[idx]
    dlo, dhi = a - lo, hi - a
    pick_hi = (dhi < dlo) | ((dhi == dlo) & (_E4M3_CODES[idx] % 2 == 0))
    q = np.where(pick_hi, hi, lo)
    q = np.where(a == 0, 0.0, q)
    return np.copysign(q, x).astype(np.float32)


def herk_fp16_narrowed(v: np.ndarray) -> np.ndarray:
    """The reference's stridedBatchGEMMCutlass HERK arithmetic
    (lib/cutlass_interface.cu:333-367) on complex64 voltages [batch, N, K]:
    each FP32 component narrowed to FP16 (round to nearest), FP16 -> E4M3
    unscaled (round to nearest, saturating at 448;
    cutlass_interface/shared/cast_kernels_common.hpp:34-37), products summed
    in FP64 (equal to the FP32 accumulation whenever every partial sum is
    exact in FP32), Im of the diagonal 0, each result rounded to FP16 and
    widened: packed lower triangles [batch, P, 2] float32."""
    re = e4m3_rne(np.asarray(v.real, dtype=np.float32).astype(np.float16).astype(np.float32))
    im = e4m3_rne(np.asarray(v.imag, dtype=np.float32).astype(np.float16).astype(np.float32))
    B, N, K = v.shape
    out = herk_c128(re.astype(np.float64) + 1j * im.astype(np.float64), N, K, B)
    return out.astype(np.float16).astype(np.float32)


def herk_fp8_scaled(v: np.ndarray, split: bool = False) -> np.ndarray:
    """Packed lower triangles [batch, P, 2] (float64) of the per-channel-scaled
    E4M3 product of complex64 voltages [batch, N, K] (split: hi hi + lo hi +
    hi lo), Im of the diagonal 0."""
    f32 = np.float32
    B, N, K = v.shape
    re = v.real.astype(f32)
    im = v.imag.astype(f32)
    m = np.maximum(np.abs(re), np.abs(im)).reshape(B, -1).max(axis=-1).astype(f32)
    s = np.where((m > 0) & (m < f32(3.0e38)), f32(448.0) / m, f32(1.0)).astype(f32)
    out_scale = (f32(1.0) / (s * s).astype(f32)).astype(f32)
    sb = s[:, None, None]
    xr, xi = (re * sb).astype(f32), (im * sb).astype(f32)
    hr, hi_ = e4m3_rne(xr), e4m3_rne(xi)
    h = hr.astype(np.float64) + 1j * hi_.astype(np.float64)
    R = np.einsum("bik,bjk->bij", h, h.conj())
    if split:
        lr, li = e4m3_rne((xr - hr).astype(f32)), e4m3_rne((xi - hi_).astype(f32))
        lo = lr.astype(np.float64) + 1j * li.astype(np.float64)
        R += np.einsum("bik,bjk->bij", lo, h.conj()) + np.einsum("bik,bjk->bij", h, lo.conj())
    R *= out_scale.astype(np.float64)[:, None, None]
    i, j = np.tril_indices(N)
    order = np.lexsort((j, i))
    i, j = i[order], j[order]
    out = np.stack([R[:, i, j].real, R[:, i, j].imag], axis=-1)
    out[:, i == j, 1] = 0.0
    return out
