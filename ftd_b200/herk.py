"""Python host mirror of the reference's HERK interface, over the C ABI.

``Correlator`` mirrors ``cutlass_gemm_api::CutlassComplexGemm``
(cutlass_interface/cutlass_gemm_api.h:157-789): ``herk``, ``init_herk``,
``end_herk``.  The module functions mirror the GGP engine boundary
(lib/cutlass_interface.cu:150-307): ``herk_batched_cutlass_qc`` (FP32 packed
output), ``herk_batched_cutlass_qc_fp16`` and ``herk_batched_cutlass_fp16``.

Arguments are device buffers: torch CUDA tensors or raw device addresses
(int).  Streams are ``torch.cuda.Stream`` objects, raw handles (int) or None
(the current torch stream when torch is in use, else the legacy stream).
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import (COMPUTE_FP8, COMPUTE_FP8_SPLIT, FORMAT_PACKED_TRIANGLE, IN_FP16, IN_FP32,  # noqa: F401
                   IN_INT4, OUT_FP16, OUT_FP32, FtdxError, check, load)

__all__ = ["Correlator", "herk_batched_cutlass_qc", "herk_batched_cutlass_qc_fp16",
           "herk_batched_cutlass_fp16", "init_cutlass_api", "tri_size", "FtdxError",
           "IN_FP16", "IN_INT4", "OUT_FP16", "OUT_FP32", "COMPUTE_FP8"]


def tri_size(n: int) -> int:
    return n * (n + 1) // 2


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_cuda") and not x.is_cuda:
            raise FtdxError(1, "tensor is not on a CUDA device")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x)!r}")


def _stream(s) -> int:
    if s is None:
        try:
            import torch
            if torch.cuda.is_available() and torch.cuda.is_initialized():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return 0
    if isinstance(s, int):
        return s
    return s.cuda_stream


class Correlator:
    """One handle of the correlator library (not thread-safe; one per thread)."""

    def __init__(self, device: int = -1, verbosity: int = 0, tune_cache: str | None = None):
        L = load()
        cfg = _lib.Config()
        cfg.device = device
        cfg.verbosity = verbosity
        cfg.tune_cache = tune_cache.encode() if tune_cache else None
        h = ctypes.c_void_p()
        st = L.ftdx_create(ctypes.byref(h), ctypes.byref(cfg))
        check(None, st, "ftdx_create")
        self._h = h
        self._L = L

    @property
    def handle(self) -> int:
        return self._h.value

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.ftdx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------ HERK
    def herk(self, A, C, N: int, K: int, batch: int, input: int = IN_FP16,
             compute: int = COMPUTE_FP8, output: int = OUT_FP16,
             format: int = FORMAT_PACKED_TRIANGLE, alpha: float = 1.0, beta: float = 0.0,
             stream=None, tune: bool = True) -> None:
        """C = alpha * A A^H + beta * C (batched, packed lower triangle).

        Defaults follow CutlassComplexGemm::herk (cutlass_gemm_api.h:750-760)."""
        st = self._L.ftdx_herk(self._h, _ptr(A), _ptr(C), N, K, batch, input, compute, output,
                               format, float(alpha), float(beta), _stream(stream), int(bool(tune)))
        check(self._h, st, "ftdx_herk")

    def herk_batched_v(self, channels, output: int = OUT_FP32, alpha: float = 1.0,
                       beta: float = 0.0, stream=None, tune: bool = False) -> None:
        """Uneven / flagged channels in one launch.  `channels` is a list of dicts
        with keys A, C, n_inputs, K and optionally lda, active (device buffers).
        Untuned calls follow set_strategy (store modes 0-3; 2 and 3 run the
        CTA-pair kernel); tune=True times modes 0-3 once per descriptor set."""
        arr = (_lib.ChannelDesc * len(channels))()
        for k, ch in enumerate(channels):
            arr[k].A = _ptr(ch["A"])
            arr[k].C = _ptr(ch["C"])
            arr[k].n_inputs = int(ch["n_inputs"])
            arr[k].K = int(ch["K"])
            arr[k].lda = int(ch.get("lda", 0))
            arr[k].active = _ptr(ch.get("active"))
        st = self._L.ftdx_herk_batched_v(self._h, ctypes.cast(arr, ctypes.c_void_p), len(channels),
                                         output, float(alpha), float(beta), _stream(stream),
                                         int(bool(tune)))
        check(self._h, st, "ftdx_herk_batched_v")

    def herk_ftd(self, raw, C, n_ant: int, n_chan: int, n_pol: int, n_time: int,
                 n_time_inner: int = 1, layout: int = _lib.LAYOUT_TIME_ANT_CHAN_POL,
                 pol_sum: bool = False, output: int = OUT_FP32, alpha: float = 1.0,
                 beta: float = 0.0, stream=None) -> None:
        """Correlate raw packet-ordered QC voltages with the corner turn fused
        into the promotion pass.  Output batch b = (chan*n_pol + pol)*n_time_inner
        + ti (pol_sum: chan*n_time_inner + ti, pols summed); see ftdx_herk_ftd."""
        d = _lib.FtdDesc(n_ant, n_chan, n_pol, n_time, n_time_inner, layout, int(bool(pol_sum)))
        st = self._L.ftdx_herk_ftd(self._h, _ptr(raw), _ptr(C), ctypes.byref(d), output,
                                   float(alpha), float(beta), _stream(stream))
        check(self._h, st, "ftdx_herk_ftd")

    def image_beams(self, vis, beams, n_ant: int, n_chan: int, n_pol: int, n_grid: int,
                    cell_size_rad: float, baseline_uv_m, freq_hz, taper=None, beam_pixels=None,
                    n_beam: int = 0, chan_tile: int = 0, output_stage: int = 0, grid_out=None,
                    stream=None) -> None:
        """Grid the packed triangles (pols summed, taper fused), inverse FFT and
        extract beam intensities (ftdx_image_beams).  output_stage 1 / 2 write
        the UV grid / image of every channel to grid_out instead."""
        cfg = _lib.ImagingConfig(n_ant, n_chan, n_pol, n_grid, n_beam, chan_tile,
                                 float(cell_size_rad), _ptr(baseline_uv_m), _ptr(freq_hz),
                                 _ptr(taper), _ptr(beam_pixels), output_stage)
        st = self._L.ftdx_image_beams(self._h, ctypes.byref(cfg), _ptr(vis), _ptr(beams),
                                      _ptr(grid_out), _stream(stream))
        check(self._h, st, "ftdx_image_beams")

    def wait_selftest(self, timeout_ms: int = 50, stream=None) -> None:
        """Make one bounded device wait run out (ftdx_wait_selftest); the next
        device_status() reports the timeout."""
        check(self._h, self._L.ftdx_wait_selftest(self._h, timeout_ms, _stream(stream)),
              "ftdx_wait_selftest")

    def xengine(self, payload, out, n_ant: int, K: int, batch: int, mat_format: int = 1,
                output: int = OUT_FP32, stream=None) -> None:
        """XEngine correlation of [batch][K][n_ant] two's-complement (4,4)b
        payload blocks: packed upper triangles (mat_format 1) or full matrices
        (0) of C = M^H M (ftdx_xengine)."""
        st = self._L.ftdx_xengine(self._h, _ptr(payload), _ptr(out), n_ant, K, batch, mat_format,
                                  output, _stream(stream))
        check(self._h, st, "ftdx_xengine")

    def strided_batch_gemm(self, A, B, C, m: int, n: int, k: int, trans_a: int, trans_b: int,
                           batch: int, data_type: int, stream=None) -> int:
        """quda::stridedBatchGEMMCutlass's HERK branch: flop count, or -1."""
        return int(self._L.ftdx_strided_batch_gemm(self._h, _ptr(A), _ptr(B), _ptr(C), m, n, k,
                                                   trans_a, trans_b, batch, data_type,
                                                   _stream(stream)))

    def peak_probe(self, kind: int, iters: int = 20000, reps: int = 3) -> float:
        """Measured dense tensor-core TFLOPS: kind 0 FP8 E4M3 and 1 NVFP4 (CTA-pair
        MMAs on zero tiles); 2 and 3 the CTA-pair and single-CTA correlators'
        FP8 MMA streams on QC-valued operands."""
        out = ctypes.c_double(0.0)
        check(self._h, self._L.ftdx_peak_probe(self._h, kind, iters, reps, ctypes.byref(out)),
              "ftdx_peak_probe")
        return float(out.value)

    def set_strided_mode(self, mode: int) -> None:
        """Arithmetic of strided_batch_gemm: 0 the reference's FP16 narrowing
        (default), 1 per-channel-scaled FP8 with FP32 output."""
        check(self._h, self._L.ftdx_set_strided_mode(self._h, mode), "ftdx_set_strided_mode")

    def herk_kahan(self, A, S, comp, N: int, K: int, batch: int, input: int = IN_INT4,
                   compute: int = COMPUTE_FP8, stream=None) -> None:
        """S += A A^H with Kahan compensation kept in `comp` (both packed complex64)."""
        st = self._L.ftdx_herk_kahan(self._h, _ptr(A), _ptr(S), _ptr(comp), N, K, batch, input,
                                     compute, _stream(stream))
        check(self._h, st, "ftdx_herk_kahan")

    def herk_adjoint(self, G, V, dV, N: int, K: int, batch: int, input: int = IN_INT4,
                     stream=None) -> None:
        """dV = (G + G^H) V per channel (G complex64 [batch][N][N], V QC int4)."""
        st = self._L.ftdx_herk_adjoint(self._h, _ptr(G), _ptr(V), _ptr(dV), N, K, batch, input,
                                       _stream(stream))
        check(self._h, st, "ftdx_herk_adjoint")

    def gain_gradient(self, R_obs, R_mod, W, g, N: int, n_chans: int, grad, loss,
                      stream=None) -> None:
        """Gain-calibration loss (double) and gradient (complex128 [N]) on the device."""
        st = self._L.ftdx_gain_gradient(self._h, _ptr(R_obs), _ptr(R_mod), _ptr(W), _ptr(g), N,
                                        n_chans, _ptr(grad), _ptr(loss), _stream(stream))
        check(self._h, st, "ftdx_gain_gradient")

    def init_herk(self, N: int, K: int, batch: int, stream=None) -> None:
        check(self._h, self._L.ftdx_init_herk(self._h, N, K, batch, _stream(stream)),
              "ftdx_init_herk")

    def end_herk(self) -> None:
        check(self._h, self._L.ftdx_end_herk(self._h), "ftdx_end_herk")

    # ------------------------------------------------------------ tuning / graphs
    def set_tune_cache(self, path: str | None) -> None:
        check(self._h, self._L.ftdx_set_tune_cache(self._h, path.encode() if path else None),
              "ftdx_set_tune_cache")

    def tune(self, A, C, N: int, K: int, batch: int, input: int = IN_INT4,
             output: int = OUT_FP32, stream=None) -> dict:
        """Time every launch strategy for this shape; returns the winner."""
        sm, g, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        st = self._L.ftdx_tune(self._h, _ptr(A), _ptr(C), N, K, batch, input, output,
                               _stream(stream), ctypes.byref(sm), ctypes.byref(g),
                               ctypes.byref(ms))
        check(self._h, st, "ftdx_tune")
        return {"store_mode": sm.value, "grid": g.value, "ms": ms.value}

    def lookup_tuned(self, N: int, K: int, batch: int, input: int = IN_INT4,
                     output: int = OUT_FP32, compute: int = COMPUTE_FP8):
        """The cached strategy for a shape and compute mode, or None."""
        sm, g, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        st = self._L.ftdx_lookup_tuned_compute(self._h, N, K, batch, input, compute, output,
                                               ctypes.byref(sm), ctypes.byref(g),
                                               ctypes.byref(ms))
        if st != _lib.FTDX_OK:
            return None
        return {"store_mode": sm.value, "grid": g.value, "ms": ms.value}

    def set_strategy(self, store_mode: int = 0, grid: int = 0, splits: int | None = None) -> None:
        """Strategy of untuned calls (ftdx_set_strategy): store_mode 0 direct,
        1 bulk, 2 CTA pair, 3 CTA pair with bulk stores; + 4 FP6 operands,
        2 / 3 + 8 the pair on INT8 operands (INT4 input); 16 the single-CTA
        kernel with the INT4 promotion fused into it.  grid=-1 is a plain
        one-tile-per-CTA launch; splits = split-K ranges (None leaves it
        unchanged)."""
        check(self._h, self._L.ftdx_set_strategy(self._h, store_mode, grid), "ftdx_set_strategy")
        if splits is not None:
            check(self._h, self._L.ftdx_set_split_k(self._h, splits), "ftdx_set_split_k")

    def tuned_split_k(self, N: int, K: int, batch: int, input: int = IN_INT4,
                      output: int = OUT_FP32) -> int:
        """Split-K count the autotuner recorded for this shape (-1: none)."""
        return int(self._L.ftdx_tuned_split_k(self._h, N, K, batch, input, output))

    def set_graph_mode(self, enable: bool) -> None:
        check(self._h, self._L.ftdx_set_graph_mode(self._h, int(bool(enable))),
              "ftdx_set_graph_mode")

    def graph_count(self) -> int:
        return int(self._L.ftdx_graph_count(self._h))

    def set_profiling(self, enable: bool) -> None:
        check(self._h, self._L.ftdx_set_profiling(self._h, int(bool(enable))), "ftdx_set_profiling")

    def profile_read(self) -> dict:
        """Summed CUDA-event device time (ms) and launch counts per kernel kind."""
        hm, pm = ctypes.c_double(0), ctypes.c_double(0)
        hn, pn = ctypes.c_int(0), ctypes.c_int(0)
        st = self._L.ftdx_profile_read(self._h, ctypes.byref(hm), ctypes.byref(hn),
                                       ctypes.byref(pm), ctypes.byref(pn))
        check(self._h, st, "ftdx_profile_read")
        return {"herk_ms": hm.value, "herk_launches": hn.value,
                "prep_ms": pm.value, "prep_launches": pn.value}

    def device_status(self, stream=None) -> int:
        """Synchronise the stream and return (and clear) the device status bits."""
        bits = ctypes.c_uint32(0)
        st = self._L.ftdx_device_status(self._h, _stream(stream), ctypes.byref(bits))
        if st not in (_lib.FTDX_OK, 7):
            check(self._h, st, "ftdx_device_status")
        return bits.value


# ---------------------------------------------------------------- GGP boundary
_api: Correlator | None = None
_tune_enabled = False


def _host_ptr(x) -> int:
    """Address of a host buffer: a CPU torch tensor (pinned or not) or a
    C-contiguous numpy array."""
    if hasattr(x, "data_ptr"):
        if getattr(x, "is_cuda", False):
            raise FtdxError(1, "pipeline buffers are host memory")
        if not x.is_contiguous():
            raise FtdxError(1, "pipeline buffer is not contiguous")
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        if not x.flags["C_CONTIGUOUS"]:
            raise FtdxError(1, "pipeline buffer is not C-contiguous")
        return x.ctypes.data
    raise TypeError(f"cannot take a host pointer of {type(x)!r}")


class Pipeline:
    """Host-to-host correlation of a stream of payloads (ftdx_pipeline_*):
    H2D, correlation and D2H overlapped across payloads.  Replaces
    VisibilityPipeline::correlate / correlate_pipelined (CUTLASS branch)."""

    def __init__(self, corr: Correlator, N: int = 0, K: int = 0, batch: int = 0,
                 output: int = OUT_FP32, ftd: dict | None = None, host_threads: int = 0):
        self._corr = corr
        self._L = corr._L
        self._ftd = None
        if ftd is not None:
            self._ftd = _lib.FtdDesc(ftd["n_ant"], ftd["n_chan"], ftd["n_pol"], ftd["n_time"],
                                     ftd.get("n_time_inner", 1),
                                     ftd.get("layout", _lib.LAYOUT_TIME_ANT_CHAN_POL),
                                     int(bool(ftd.get("pol_sum", False))))
        cfg = _lib.PipelineConfig(N, K, batch, output,
                                  ctypes.pointer(self._ftd) if self._ftd is not None else None,
                                  host_threads)
        h = ctypes.c_void_p()
        check(corr._h, self._L.ftdx_pipeline_create(corr._h, ctypes.byref(cfg), ctypes.byref(h)),
              "ftdx_pipeline_create")
        self._p = h

    @property
    def sizes(self) -> tuple[int, int]:
        a, b = ctypes.c_size_t(), ctypes.c_size_t()
        check(self._corr._h, self._L.ftdx_pipeline_sizes(self._p, ctypes.byref(a), ctypes.byref(b)),
              "ftdx_pipeline_sizes")
        return a.value, b.value

    def correlate(self, vis_outputs, raw_inputs) -> None:
        """Correlate every payload; returns when all outputs are in host memory."""
        n = len(raw_inputs)
        if len(vis_outputs) != n:
            raise FtdxError(1, "as many outputs as inputs are needed")
        outs = (ctypes.c_void_p * max(n, 1))(*[_host_ptr(v) for v in vis_outputs])
        ins = (ctypes.c_void_p * max(n, 1))(*[_host_ptr(r) for r in raw_inputs])
        check(self._corr._h, self._L.ftdx_pipeline_correlate(self._p, outs, ins, n),
              "ftdx_pipeline_correlate")

    def close(self):
        if self._p:
            self._L.ftdx_pipeline_destroy(self._p)
            self._p = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _get_api() -> Correlator:
    global _api
    if _api is None:
        _api = Correlator()
    return _api


def init_cutlass_api(kernel_tune_verbosity: int = 0, kernel_tune_cache_path: str | None = None,
                     strategy_tune_cache_path: str | None = None, herk_tune: bool = False,
                     strategy_tune_verbosity: int = 1) -> None:
    """Mirror of ggp::initCutlassApi (lib/cutlass_interface.cu:150-169)."""
    global _api, _tune_enabled
    if _api is not None:
        _api.close()
    _api = Correlator(verbosity=strategy_tune_verbosity if strategy_tune_verbosity > 1 else 0,
                      tune_cache=strategy_tune_cache_path)
    _tune_enabled = bool(herk_tune)


def herk_batched_cutlass_qc(qc, tri, N: int, K: int, batch: int, stream=None) -> int:
    """Mirror of ggp::herkBatchedCutlassQC (lib/cutlass_interface.cu:178-231): QC int4
    [batch][N][K] -> FP32 packed triangle.  Returns 0 on success (raises otherwise)."""
    _get_api().herk(qc, tri, N, K, batch, IN_INT4, COMPUTE_FP8, OUT_FP32,
                    stream=stream, tune=_tune_enabled)
    return 0


def herk_batched_cutlass_qc_fp16(qc, tri, N: int, K: int, batch: int, stream=None) -> int:
    """Mirror of ggp::herkBatchedCutlassQC_FP16 (lib/cutlass_interface.cu:243-289)."""
    _get_api().herk(qc, tri, N, K, batch, IN_INT4, COMPUTE_FP8, OUT_FP16,
                    stream=stream, tune=_tune_enabled)
    return 0


def herk_batched_cutlass_fp16(a16, tri, N: int, K: int, batch: int, stream=None) -> int:
    """Mirror of ggp::herkBatchedCutlassFP16 (lib/cutlass_interface.cu:292-307)."""
    _get_api().herk(a16, tri, N, K, batch, IN_FP16, COMPUTE_FP8, OUT_FP16,
                    stream=stream, tune=_tune_enabled)
    return 0
