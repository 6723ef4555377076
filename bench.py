#!/usr/bin/env python
"""Benchmark of the B200 correlator on the DSA-2000-scale workload.

Workload (one step): 2048 antennas x 2 pol = 4096 inputs, 64 channels,
K = 1024 time samples of QC int4 voltages (Re, Im each round(N(0, 2.5^2))
clipped to [-7, 7], seeded, generated on the device), correlated to packed
lower triangles of complex64 (8,390,656 entries per channel).  Metric:
effective TFLOPS = sum_f 8 * N(N+1)/2 * K / t (the FLOP convention of the
correlator's specification).

Arms
  (default)          the library through its C ABI, inputs resident in HBM;
                     `e2e` repeats the step through the same C ABI with host
                     buffers (pinned H2D of the QC input and D2H of every
                     packed triangle inside the timed region, pipelined over
                     channel chunks on two streams).
  --impl reference   the reference's own host correlator (cpu_herk,
                     cutlass_interface/test_herk_int4.cu:51-70, compiled from
                     its source into oracle/_ref/) on all host threads, on a
                     bounded sample of the same workload.

Multi-GPU (torchrun): every rank correlates its own 64 channels (weak
scaling, no collective on the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "HERK eff. TFLOPS & % FP8/FP4 peak vs plain FP8 path, same B200, stated error"
UNIT = "TFLOPS"
NOMINAL_FP8_TFLOPS = 4500.0  # datasheet dense FP8 (context only)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--inputs", type=int, default=4096, help="N (antennas x pols)")
    p.add_argument("--channels", type=int, default=64)
    p.add_argument("--k", type=int, default=1024, help="time samples per channel")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-peak", action="store_true")
    p.add_argument("--no-extra", action="store_true", help="skip the extra workload legs")
    p.add_argument("--no-sustained", action="store_true",
                   help="skip the few-second sustained run of the main step")
    p.add_argument("--leg", default=None,
                   choices=["nvfp4", "nvfp4split", "raw", "imaging", "xengine", "splitk",
                            "precision", "imaging_visbf", "batched", "xengine", "peaks",
                            "config1", "diff"],
                   help="run one extra workload alone and print its JSON (profiling cases); "
                        "nvfp4 and nvfp4split use --inputs/--channels/--k")
    p.add_argument("--strategy", default=None,
                   help="STORE_MODE,GRID: fix the correlator strategy instead of autotuning "
                        "(0 direct stores, 1 bulk stores, 2 CTA-pair kernel)")
    return p.parse_args()


def herk_flops(N, K, B):
    return 8.0 * (N * (N + 1) // 2) * K * B


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling around the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.t0 = time.time()
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(gpu_index), "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        self.marks = []

    def mark(self):
        self.marks.append(time.time())

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [ln.strip().split(", ") for ln in self.f if ln.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return None
        # Samples are ~100 ms apart; keep the ones taken inside the timed window
        # (estimated from sample order), else all samples under load.
        n = len(rows)
        t_end = time.time()
        dt = (t_end - self.t0) / max(n, 1)
        self.series = [(self.t0 + k * dt, rows[k][1]) for k in range(n)]
        sel = rows
        if len(self.marks) >= 2:
            a, b = self.marks[0], self.marks[1]
            idx = [k for k in range(n) if a - dt <= self.t0 + k * dt <= b + dt]
            if idx:
                sel = [rows[k] for k in idx]
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [v for v in (num(r[1]) for r in sel) if v is not None]
        smax = [v for v in (num(r[2]) for r in sel) if v is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in sel for k in range(4) if "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(sel),
                "power_w_max": max((num(r[3]) or 0.0) for r in sel)}


def run_sustained(torch, step, stream, gpu_index, flops, seconds=2.5, chunk=50):
    """About `seconds` of back-to-back steps (the power-capped steady state of
    a long run, not a burst): TFLOPS over the whole run, the median SM clock
    sampled during it, and the per-chunk TFLOPS grouped by the SM clock seen
    while that chunk ran (100 MHz bins)."""
    clocks = ClockSampler(gpu_index)
    time.sleep(0.3)
    torch.cuda.synchronize()
    chunks = []
    t_start = time.time()
    clocks.mark()
    while time.time() - t_start < seconds:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        h0 = time.time()
        e0.record(stream)
        for _ in range(chunk):
            step()
        e1.record(stream)
        e1.synchronize()
        chunks.append((h0, time.time(), e0.elapsed_time(e1) / chunk))
    clocks.mark()
    clk = clocks.stop() or {}
    series = getattr(clocks, "series", [])
    total_ms = sum(c[2] for c in chunks) * chunk
    bins = {}
    for h0, h1, ms in chunks:
        mhz = [float(v) for t, v in series if h0 - 0.05 <= t <= h1 + 0.05
               and v.replace(".", "", 1).isdigit()]
        if not mhz:
            continue
        key = str(int(statistics.median(mhz) // 100 * 100))
        bins.setdefault(key, []).append(flops / (ms * 1e-3) / 1e12)
    return {"seconds": round(total_ms / 1e3, 3), "steps": len(chunks) * chunk,
            "value": flops * len(chunks) * chunk / (total_ms * 1e-3) / 1e12, "unit": UNIT,
            "ms_per_step": total_ms / (len(chunks) * chunk),
            "sm_mhz_median": clk.get("sm_mhz"), "reasons": clk.get("reasons"),
            "power_w_max": clk.get("power_w_max"),
            "by_sm_clock_bin_mhz": {k: {"chunks": len(v), "tflops_median": statistics.median(v)}
                                    for k, v in sorted(bins.items())}}


def load_reference_direct():
    """The reference's own direct mma.sync HERK kernel with its INT4 -> FP8
    cast (baseline/build_direct_ref.sh builds it from the reference's
    sources into baseline/_ref/), or None when it was not built."""
    import ctypes
    path = os.path.join(ROOT, "baseline", "_ref", "libref_direct_herk.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    L.ref_direct_herk_staging_bytes.restype = ctypes.c_size_t
    L.ref_direct_herk_staging_bytes.argtypes = [ctypes.c_int] * 3
    L.ref_direct_herk_qc.restype = ctypes.c_int
    L.ref_direct_herk_qc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    return L


def run_reference_direct_leg(torch, dev, qc, C_ours, N, K, B, steps):
    """The reference's Blackwell direct HERK path on the same GPU and the same
    resident QC input: its INT4 -> interleaved-FP8 cast + herk_direct_fp8_precast
    kernel (mma.sync m16n8k32, 32 x 32 antenna tiles, grid = lower-triangle
    blocks x channels), FP32 packed lower triangles.  Timed with CUDA events;
    its triangles compared with the library's (both exact for QC input)."""
    L = load_reference_direct()
    if L is None:
        return None
    import ctypes
    from ftd_b200 import tri_size
    stream = torch.cuda.current_stream(dev)
    fp8 = torch.empty(int(L.ref_direct_herk_staging_bytes(N, K, B)), dtype=torch.uint8, device=dev)
    C = torch.empty(B, tri_size(N), 2, device=dev)

    def call():
        rc = L.ref_direct_herk_qc(ctypes.c_void_p(qc.data_ptr()), ctypes.c_void_p(fp8.data_ptr()),
                                  ctypes.c_void_p(C.data_ptr()), N, K, B,
                                  ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise RuntimeError(f"reference direct HERK launch failed ({rc})")
    ms = _timed(torch, call, reps=max(3, min(steps, 10)), warm=2)
    same = bool(torch.equal(C, C_ours))
    del fp8, C
    flops = herk_flops(N, K, B)
    return {"what": "reference herk_direct_fp8_precast_kernel (mma.sync) + "
                    "cast_int4_to_fp8_interleaved, built from its sources for sm_100a",
            "value": flops / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
            "bit_exact_vs_library": same}


def load_reference_api():
    """The reference's own public HERK API (cutlass_gemm_api::CutlassComplexGemm,
    its CUTLASS tcgen05 sub-GEMM baseline and direct kernels), compiled
    unmodified from its sources by baseline/build_cutlass_ref.sh into
    baseline/_ref/, or None when it was not built."""
    import ctypes
    path = os.path.join(ROOT, "baseline", "_ref", "libref_cutlass_api.so")
    if not os.path.exists(path):
        return None
    L = ctypes.CDLL(path)
    vp, i = ctypes.c_void_p, ctypes.c_int
    L.ref_api_create.restype = vp
    L.ref_api_destroy.argtypes = [vp]
    L.ref_api_init_herk.restype = i
    L.ref_api_init_herk.argtypes = [vp, i, i, i, vp]
    L.ref_api_herk_qc_fp32.restype = i
    L.ref_api_herk_qc_fp32.argtypes = [vp, vp, vp, i, i, i, i, vp]
    L.ref_api_herk.restype = i
    L.ref_api_herk.argtypes = [vp, vp, vp, i, i, i, i, i, ctypes.c_float, ctypes.c_float, i, vp]
    L.ref_api_set_tile_config.restype = i
    L.ref_api_set_tile_config.argtypes = [vp, i]
    return L


class _StdoutToStderr:
    """Sends what a C library prints to stdout to stderr meanwhile, so that
    the bench's stdout stays one JSON line."""

    def __enter__(self):
        import ctypes
        sys.stdout.flush()
        self.libc = ctypes.CDLL(None)
        self.saved = os.dup(1)
        os.dup2(2, 1)
        return self

    def __exit__(self, *exc):
        self.libc.fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        return False


def run_reference_api_leg(torch, dev, qc, C_ours, N, K, B, steps):
    """The reference's GPU HERK through its own public API on the same GPU and
    resident QC input (INT4 -> FP8 compute -> FP32 packed triangles, tune =
    false): its default K-adaptive dispatch (HerkMode::Auto) and its CUTLASS
    tcgen05 baseline (HerkMode::ForceBaseline: cast, sub-GEMMs, pack).  Timed
    with CUDA events after init_herk; triangles compared with the library's."""
    L = load_reference_api()
    if L is None:
        return None
    import ctypes
    from ftd_b200 import tri_size
    stream = torch.cuda.current_stream(dev)
    out = {"what": "reference cutlass_gemm_api::CutlassComplexGemm::herk, built unmodified "
                   "from its sources for sm_100a (nvcc 12.9, CUTLASS 4.5 headers, 1x1 clusters)"}
    with _StdoutToStderr():
        h = L.ref_api_create()
        if not h:
            return {**out, "unavailable": "CutlassComplexGemm construction failed"}
        try:
            if L.ref_api_init_herk(h, N, K, B, ctypes.c_void_p(stream.cuda_stream)) != 0:
                return {**out, "unavailable": "init_herk failed"}
            C = torch.empty(B, tri_size(N), 2, device=dev)
            # its default tile configuration, then the other single-CTA-cluster
            # ones its autotuner could pick (GemmOptimal, WideN, SmallTile)
            runs = [("auto", 0, 0), ("cutlass_baseline", 2, 0), ("cutlass_baseline_gemm_optimal", 2, 2),
                    ("cutlass_baseline_wide_n", 2, 3), ("cutlass_baseline_small_tile", 2, 6)]
            for name, mode, cfg in runs:
                if L.ref_api_set_tile_config(h, cfg) != 0:
                    out[name] = {"unavailable": f"tile configuration {cfg} refused"}
                    continue
                def call():
                    rc = L.ref_api_herk_qc_fp32(h, ctypes.c_void_p(qc.data_ptr()),
                                                ctypes.c_void_p(C.data_ptr()), N, K, B, mode,
                                                ctypes.c_void_p(stream.cuda_stream))
                    if rc != 0:
                        raise RuntimeError(f"reference herk failed ({rc})")
                C.fill_(float("nan"))
                try:
                    ms = _timed(torch, call, reps=max(3, min(steps, 10)), warm=2)
                except RuntimeError as e:
                    out[name] = {"unavailable": str(e)}
                    continue
                out[name] = {"value": herk_flops(N, K, B) / (ms * 1e-3) / 1e12, "unit": UNIT,
                             "ms_per_step": ms, "bit_exact_vs_library": bool(torch.equal(C, C_ours))}
            L.ref_api_set_tile_config(h, 0)
            best = [v for k, v in out.items() if k.startswith("cutlass_baseline")
                    and isinstance(v, dict) and "value" in v]
            if best:
                out["cutlass_baseline_best"] = max(best, key=lambda v: v["value"])
            del C
        finally:
            torch.cuda.synchronize()
            L.ref_api_destroy(h)
    return out


def run_fp16_output_leg(torch, dev, qc, N, K, B, world):
    """The DSA-2000 workload with FP16 packed triangles (herkBatchedCutlassQC_FP16's
    form): half the output bytes of the FP32 line.  Tuned, graph-replayed,
    CUDA events; beside it (one-GPU runs) the reference's own API on the same
    output form (default dispatch and CUTLASS baseline), each checked
    bit-exact against this library's triangles."""
    import ctypes
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP16
    C = torch.empty(B, tri_size(N), 2, dtype=torch.float16, device=dev)
    stream = torch.cuda.current_stream(dev)
    with Correlator(device=dev.index) as corr:
        corr.init_herk(N, K, B)
        corr.tune(qc, C, N, K, B, input=IN_INT4, output=OUT_FP16, stream=stream)
        corr.set_graph_mode(True)
        ms = _timed(torch, lambda: corr.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP16,
                                             stream=stream, tune=True), reps=20, warm=3)
        tuned = corr.lookup_tuned(N, K, B, input=IN_INT4, output=OUT_FP16)
    flops = herk_flops(N, K, B)
    out = {"workload": f"{N} inputs x {B} channels x K={K}, QC int4 -> packed FP16 triangles",
           "value": flops / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
           "output_bytes_per_step": int(C.numel() * 2), "tuned": tuned}
    L = load_reference_api() if world == 1 else None
    if L is not None:
        R = torch.empty_like(C)
        with _StdoutToStderr():
            h = L.ref_api_create()
            try:
                if h and L.ref_api_init_herk(h, N, K, B, ctypes.c_void_p(stream.cuda_stream)) == 0:
                    for name, mode in (("reference_default", 0), ("reference_cutlass_baseline", 2)):
                        def call():
                            rc = L.ref_api_herk(h, ctypes.c_void_p(qc.data_ptr()),
                                                ctypes.c_void_p(R.data_ptr()), N, K, B, 1, 0,
                                                1.0, 0.0, mode, ctypes.c_void_p(stream.cuda_stream))
                            if rc != 0:
                                raise RuntimeError(f"reference herk failed ({rc})")
                        try:
                            rms = _timed(torch, call, reps=5, warm=2)
                        except RuntimeError as e:
                            out[name] = {"unavailable": str(e)}
                            continue
                        out[name] = {"value": flops / (rms * 1e-3) / 1e12, "unit": UNIT,
                                     "ms_per_step": rms,
                                     "bit_exact_vs_library": bool(torch.equal(R, C))}
            finally:
                torch.cuda.synchronize()
                if h:
                    L.ref_api_destroy(h)
        del R
    del C
    return out


def run_config1_leg(torch, dev, N=128, K=256, B=32, seed=8):
    """The small plain configuration (64 antennas x 2 pols = 128 inputs, 32
    channels, K = 256): latency of one call, tuned and graph-replayed, and
    launched directly without graphs; exact against the oracle on the side."""
    import numpy as np
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP32
    qc = make_qc(torch, B, N, K, dev, seed=seed)
    C = torch.empty(B, tri_size(N), 2, device=dev)
    flops = herk_flops(N, K, B)
    with Correlator(device=dev.index) as c:
        c.init_herk(N, K, B)
        c.tune(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32)
        def call():
            c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, tune=True)
        ms_direct = _timed(torch, call, reps=200, warm=20)
        c.set_graph_mode(True)
        ms_graph = _timed(torch, call, reps=200, warm=20)
        if c.device_status() != 0:
            raise RuntimeError("device status after the config-1 leg")
    from oracle import oracle
    exact = bool(np.array_equal(C.cpu().numpy(),
                                oracle.herk_qc(qc.cpu().numpy(), N, K, B).astype(np.float32)))
    return {"workload": f"{N} inputs x {B} channels x K={K}, QC int4 -> packed complex64",
            "graph_replay": {"us_per_call": ms_graph * 1e3,
                             "value": flops / (ms_graph * 1e-3) / 1e12, "unit": UNIT},
            "direct_launch": {"us_per_call": ms_direct * 1e3,
                              "value": flops / (ms_direct * 1e-3) / 1e12, "unit": UNIT},
            "bit_exact_vs_oracle": exact}


# ------------------------------------------------------------------ inputs
def make_qc(torch, B, N, K, device, seed=1):
    """Seeded QC int4 voltages on the device: [B, N, K] uint8."""
    g = torch.Generator(device=device).manual_seed(seed)
    out = torch.empty(B, N, K, dtype=torch.uint8, device=device)
    for b in range(B):  # per channel to bound temporary memory
        re = torch.clamp(torch.round(torch.randn(N, K, device=device, generator=g) * 2.5), -7, 7)
        im = torch.clamp(torch.round(torch.randn(N, K, device=device, generator=g) * 2.5), -7, 7)
        re = re.to(torch.int32)
        im = im.to(torch.int32)
        nr = torch.where(re < 0, 8 | (-re), re)
        ni = torch.where(im < 0, 8 | (-im), im)
        out[b] = ((nr << 4) | ni).to(torch.uint8)
    return out


def measure_fp8_peak(torch, device):
    """Dense FP8 E4M3 matmul throughput of cuBLASLt (torch._scaled_mm), 8192^3,
    best of 20 back-to-back launches after warm-up: the FP8 roofline denominator."""
    M = 8192
    a = torch.randn(M, M, device=device).to(torch.float8_e4m3fn)
    b = torch.randn(M, M, device=device).to(torch.float8_e4m3fn).t()
    one = torch.tensor(1.0, device=device)
    for _ in range(5):
        torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(20):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._scaled_mm(a, b, scale_a=one, scale_b=one, out_dtype=torch.bfloat16)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * M ** 3 / best / 1e9


def measure_tcgen05_peaks(device_index, iters=20000, reps=3):
    """Dense tcgen05 throughput (TFLOPS) of the MMA shapes the correlators use,
    from ftdx_peak_probe, no loads or stores: M = N = 256 CTA-pair MMAs on
    zero tiles (FP8 E4M3, K = 32, and NVFP4 block16, K = 64), and the two FP8
    correlators' own MMA streams on QC-valued operands (CTA pair: two
    M = N = 256 MMAs per 32 samples; single CTA: four M = N = 128)."""
    from ftd_b200 import Correlator
    with Correlator(device=device_index) as c:
        return {"fp8_e4m3": c.peak_probe(0, iters, reps), "nvfp4": c.peak_probe(1, iters, reps),
                "fp8_qc_data_pair": c.peak_probe(2, iters, reps),
                "fp8_qc_data_single_cta": c.peak_probe(3, iters, reps),
                "what": f"{iters} back-to-back tcgen05.mma per SM pair (cta_group::2, M=N=256) "
                        f"or per SM (fp8_qc_data_single_cta: cta_group::1, M=N=128), best of "
                        f"{reps} launches; fp8_e4m3 / nvfp4 on zero tiles, fp8_qc_data_* on "
                        f"E4M3 codes of random integers -7..7"}


def measure_int8_peak(torch, device):
    """Dense INT8 matmul throughput of cuBLASLt (torch._int_mm, int32 out),
    8192^3, best of 20 launches after warm-up."""
    M = 8192
    a = torch.randint(-7, 8, (M, M), device=device, dtype=torch.int8)
    b = torch.randint(-7, 8, (M, M), device=device, dtype=torch.int8)
    for _ in range(5):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(20):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch._int_mm(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * M ** 3 / best / 1e9


# ------------------------------------------------------------------ CPU baseline
class CpuSample:
    """The reference's cpu_herk (cutlass_interface/test_herk_int4.cu:51-70,
    compiled from its source into oracle/_ref/) on all host threads, over the
    first n inputs of one channel of the workload, n sized once so that one
    run takes about `target_s`.  Falls back to the oracle port (kind "port")
    when the reference was not built."""

    def __init__(self, N, K, target_s):
        import numpy as np
        from oracle import oracle
        self.oracle = oracle
        self.kind = "reference" if oracle.ref_lib() is not None else "port"
        self.N, self.K = N, K
        self.rng = np.random.default_rng(5)
        n = 256
        dt = self._run(n)
        while dt < target_s / 3 and n < N:
            n = min(N, int(n * min(4.0, max(1.3, (target_s / max(dt, 1e-3)) ** 0.5))))
            dt = self._run(n)
        self.n = n
        self.cores = (oracle.ref_lib().ref_num_threads() if self.kind == "reference"
                      else oracle.num_threads())

    def _run(self, n):
        o = self.oracle
        re, im = o.gaussian_int4(self.rng, (1, n, self.K))
        qc = o.encode_qc(re, im)
        t = time.perf_counter()
        if self.kind == "reference":
            o.ref_cpu_herk(qc, n, self.K, 1)
        else:
            o.herk_qc(qc, n, self.K, 1)
        return time.perf_counter() - t

    def tflops(self):
        dt = self._run(self.n)
        return herk_flops(self.n, self.K, 1) / dt / 1e12, dt

    def describe(self, dt):
        fl = herk_flops(self.n, self.K, 1)
        return {"unit": UNIT, "cores": int(self.cores), "kind": self.kind,
                "sample": f"one channel, first {self.n} of {self.N} inputs, K={self.K} "
                          f"({fl / 1e9:.1f} GFLOP in {dt:.2f} s); FP64 complex cpu_herk, OpenMP "
                          f"over rows"}


def cpu_reference_sample(N, K, target_s=3.0):
    cs = CpuSample(N, K, target_s)
    v, dt = cs.tflops()
    return {"value": v, **cs.describe(dt)}


# ------------------------------------------------------------------ arms
def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import oracle
    N, K = args.inputs, args.k
    cs = CpuSample(N, K, target_s=2.0)
    samples = []
    dt = 0.0
    for s_ in range(args.warmup + args.steps):
        v_, dt = cs.tflops()
        if s_ >= args.warmup:
            samples.append(v_)
    v = statistics.median(samples)
    info = cs.describe(dt)
    full_flop = herk_flops(N, K, args.channels)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": full_flop / (v * 1e12) * 1e3,
            "extrapolated": {"ms_per_step": True,
                             "measured": f"each step times one sample of {cs.n} of {N} inputs of "
                                         f"one channel (K={K}); ms_per_step is the whole "
                                         f"{args.channels}-channel step at that rate",
                             "flop_multiplier": full_flop / herk_flops(cs.n, K, 1)},
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian int4, sigma 2.5)",
            "config": {"workload": f"DSA-2000 correlator: {N} inputs x {args.channels} channels x "
                                   f"K={K}, QC int4 -> packed complex triangle",
                       "inputs": N, "channels": args.channels, "k": K},
            "cpu_baseline": {"value": v, **info},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if oracle.ref_lib() is None:
        line["note"] = "reference host code not built; timed the oracle port"
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, rank, world, dist):
    import torch
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP32
    from ftd_b200.shard import max_over_ranks

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    N, K, B = args.inputs, args.k, args.channels
    P = tri_size(N)
    flops = herk_flops(N, K, B)

    qc = make_qc(torch, B, N, K, dev, seed=1 + rank)
    C = torch.empty(B, P, 2, dtype=torch.float32, device=dev)
    corr = Correlator(device=local)
    corr.init_herk(N, K, B)
    stream = torch.cuda.current_stream(dev)
    # autotune this shape (strategy sweep, outside the timed region), then
    # replay each call as a captured CUDA graph
    if args.strategy:
        sm, gr = (int(x) for x in args.strategy.split(","))
        corr.set_strategy(sm, gr)
        tuned = {"store_mode": sm, "grid": gr, "ms": None, "fixed": True}
    else:
        tuned = corr.tune(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, stream=stream)
    corr.set_graph_mode(True)
    use_tuner = not args.strategy

    def step():
        corr.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32, stream=stream, tune=use_tuner)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if corr.device_status() != 0:
        raise RuntimeError("device wait timed out during warm-up")

    clocks = ClockSampler(local)
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    clocks.mark()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()
    # Per-kernel CUDA-event times of the same calls: graph replays carry no
    # events, so the timed steps are repeated once more launched directly.
    corr.set_graph_mode(False)
    corr.set_profiling(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    prof = corr.profile_read()
    corr.set_profiling(False)
    herk_ms = prof["herk_ms"] / max(prof["herk_launches"], 1)
    prep_ms = prof["prep_ms"] / max(prof["prep_launches"], 1)
    if corr.device_status() != 0:
        raise RuntimeError("device wait timed out in the timed region")

    ms_max = max_over_ranks(ms, dist, dev)  # the slowest rank sets the step time
    value = flops * world / (ms_max * 1e-3) / 1e12

    # --- the same step sustained for a few seconds of graph replays
    sustained = None
    if not args.no_sustained:
        corr.set_graph_mode(True)
        sustained = run_sustained(torch, step, stream, local, flops)  # this rank's GPU

    # --- plain per-channel path: the same kernels launched per channel, one
    # CTA per tile (no persistence), no graph, no tuning
    plain = None
    if not args.no_plain:
        pc = Correlator(device=local)
        pc.set_strategy(0, -1)
        pc.init_herk(N, K, 1)

        def plain_step():
            for b in range(B):
                pc.herk(qc[b], C[b], N, K, 1, input=IN_INT4, output=OUT_FP32, stream=stream,
                        tune=False)
        for _ in range(2):
            plain_step()
        torch.cuda.synchronize()
        reps = max(3, min(args.steps, 10))
        e0.record(stream)
        for _ in range(reps):
            plain_step()
        e1.record(stream)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1) / reps
        pc.close()
        plain = {"value": flops / (pms * 1e-3) / 1e12, "ms_per_step": pms,
                 "what": f"{B} launches of batch=1 per step, one CTA per tile (not persistent), "
                         f"no graph, no tuning"}

    # --- the reference's own Blackwell direct kernel on the same input
    ref_direct = ref_api = None
    if not args.no_plain:
        step()
        torch.cuda.synchronize()
        ref_direct = run_reference_direct_leg(torch, dev, qc, C, N, K, B, args.steps)
        if world == 1:  # the reference's CUTLASS kernels: one-GPU runs only
            ref_api = run_reference_api_leg(torch, dev, qc, C, N, K, B, args.steps)

    # --- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(torch, args, dev, qc, N, K, B, flops, world, dist)

    batched = precision = differentiation = raw_layout = imaging = xengine = splitk = None
    imaging_visbf = config1 = fp16_out = nvfp4_gauss = None
    if not args.no_extra:
        config1 = run_config1_leg(torch, dev)
        fp16_out = run_fp16_output_leg(torch, dev, qc, N, K, B, world)
        nvfp4_gauss = run_nvfp4_case(torch, dev, N, K, B)
        batched = run_batched_leg(torch, dev)
        raw_layout = run_ftd_leg(torch, dev)
        imaging = run_imaging_leg(torch, dev)
        imaging_visbf = run_imaging_visbf_leg(torch, dev)
        xengine = run_xengine_leg(torch, dev)
        splitk = run_splitk_leg(torch, dev)
        precision = run_precision_leg(torch, dev)
        differentiation = run_diff_leg(torch, dev)

    peak = probes = None
    if not args.no_peak:
        peak = measure_fp8_peak(torch, dev)
        probes = measure_tcgen05_peaks(local)

    if rank != 0:
        return 0
    achieved = flops / (herk_ms * 1e-3) / 1e12
    mode = int(tuned.get("store_mode") or 0)  # + 4: packed FP6 planes; + 8: int8 planes
    peak_source = "cuBLASLt dense FP8 e4m3 GEMM 8192^3 (torch._scaled_mm), measured in this run"
    if peak and mode & 8:
        # the int8 kernel is held to the larger of the FP8 and INT8 library rates
        try:
            p8 = measure_int8_peak(torch, dev)
        except Exception as exc:  # noqa: BLE001 -- the FP8 figure still stands
            p8 = None
            peak_source += f"; INT8 peak not measured ({type(exc).__name__})"
        if p8:
            peak_source = (f"max of cuBLASLt dense FP8 e4m3 ({peak:.0f}) and INT8 "
                           f"(torch._int_mm, {p8:.0f}) GEMMs 8192^3, measured in this run")
            peak = max(peak, p8)
    kernel_name = "herk_fp8_pair_kernel" if (mode & 3) >= 2 else "herk_fp8_tc_kernel"
    prep_name = ("qc_to_planes6_kernel" if mode & 4 else
                 "qc_to_planes_s8_kernel" if mode & 8 else "qc_to_planes_kernel")
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "herk_fp8_traffic.json")
    if os.path.exists(tfile):
        t = json.load(open(tfile))
        entry = t.get(kernel_name, t)
        if entry.get("workload") == [N, K]:
            traffic = entry["bytes_per_channel"] * B
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("int8 (int32 accumulate)" if mode & 8 else
                  "fp6_e3m2 (fp32 accumulate)" if mode & 4 else "fp8_e4m3 (fp32 accumulate)"),
        "data": "synthetic (seeded Gaussian int4 voltages, sigma 2.5, generated on device)",
        "config": {"workload": f"DSA-2000 correlator: {N} inputs x {B} channels x K={K}, "
                               f"QC int4 -> packed complex64 lower triangle",
                   "inputs": N, "channels": B, "k": K, "per_gpu_channels": B,
                   "l2": (f"inputs {B * N * K / 1e6:.0f} MB, outputs {B * P * 8 / 1e9:.2f} GB "
                          f"({'both exceed' if B * N * K > 126e6 else 'the outputs exceed'} "
                          f"the 126 MB L2); no flush needed"),
                   "parallelism": f"replicas x{world} (independent channels)"},
        "roofline": {"bound": "tensor", "achieved": achieved,
                     "peak": peak, "unit": UNIT,
                     "frac": (achieved / peak) if peak else None,
                     "traffic": traffic,
                     "kernel": kernel_name,
                     "kernel_ms": herk_ms,
                     "peak_source": peak_source,
                     "frac_of_nominal_4500": achieved / NOMINAL_FP8_TFLOPS,
                     "tcgen05_probe_peaks": probes,
                     "frac_of_fp8_probe": (achieved / probes["fp8_e4m3"]) if probes else None,
                     # against this kernel's own MMA stream on QC-valued operands
                     "frac_of_own_mma_stream_probe": (
                         achieved / probes["fp8_qc_data_pair" if (mode & 3) >= 2
                                           else "fp8_qc_data_single_cta"]) if probes else None},
        "kernels": {kernel_name + "_ms": herk_ms, prep_name + "_ms": prep_ms},
        "gpu_launches": 2 * args.steps,
        "strategy": {"tuned": tuned, "graph_replay": True},
        "sustained": sustained,
        "config1_small": config1,
        "fp16_output": fp16_out,
        "nvfp4_gaussian": nvfp4_gauss,
        "config3_batched_uneven": ({"value": batched["value"], "unit": UNIT,
                                    "ms_per_step": batched["ms_per_step"],
                                    "frac_of_fp8_cublaslt": (batched["value"] / peak)
                                    if peak else None,
                                    "frac_of_fp8_probe": (batched["value"] / probes["fp8_e4m3"])
                                    if probes else None} if batched else None),
        "plain_per_channel": plain,
        "speedup_vs_plain": (value / world / plain["value"]) if plain else None,
        "reference_direct_mma_sync": ref_direct,
        "vs_direct_mma_sync": (value / world / ref_direct["value"]) if ref_direct else None,
        "reference_api_gpu": ref_api,
        "vs_reference_api_default": ((value / ref_api["auto"]["value"])
                                     if ref_api and "value" in ref_api.get("auto", {}) else None),
        "vs_reference_cutlass_baseline": (
            (value / ref_api["cutlass_baseline_best"]["value"])
            if ref_api and "value" in ref_api.get("cutlass_baseline_best", {}) else None),
        "e2e": e2e,
        "batched_uneven_flagged": batched,
        "raw_layout_fused_corner_turn": raw_layout,
        "imaging_from_triangles": imaging,
        "imaging_at_reference_visbf_sizes": imaging_visbf,
        "xengine_upper_triangle": xengine,
        "split_k_long_integration": splitk,
        "precision_modes": precision,
        "adjoint_and_gain_gradient": differentiation,
        "clocks": clk,
    }
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_reference_sample(N, K, target_s=10.0)
    print(json.dumps(line), flush=True)
    corr.close()
    return 0


def run_batched_leg(torch, dev, seed=3, n_chans=96, inputs=4096):
    """Uneven-K, flagged-input workload in one call: 96 channels, K uniform in
    {128, 192, ..., 2048}, active inputs uniform in [1536, 4096] after seeded
    random flagging of 4096 inputs, Gaussian int4 voltages.  Returns its
    effective TFLOPS (sum over channels of 8 N(N+1)/2 K / t)."""
    import numpy as np
    from ftd_b200 import Correlator, tri_size
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev).manual_seed(seed)
    chans, flops = [], 0.0
    for _ in range(n_chans):
        K = int(rng.integers(2, 33)) * 64
        n = int(rng.integers(1536, inputs + 1))
        active = np.sort(rng.choice(inputs, size=n, replace=False)).astype(np.int32)
        qc = make_qc(torch, 1, inputs, K, dev, seed=int(rng.integers(1 << 30)))[0]
        chans.append({"A": qc, "C": torch.empty(tri_size(n), 2, device=dev), "n_inputs": n,
                      "K": K, "active": torch.from_numpy(active).to(dev)})
        flops += herk_flops(n, K, 1)
    with Correlator(device=dev.index) as c:
        c.herk_batched_v(chans, tune=True)
        c.set_graph_mode(True)
        for _ in range(3):
            c.herk_batched_v(chans, tune=True)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        reps = 10
        e0.record()
        for _ in range(reps):
            c.herk_batched_v(chans, tune=True)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        # each fixed strategy (untuned calls, graph replay): 0 direct, 1 bulk
        # stores, 2 CTA pair, 3 CTA pair with bulk stores
        by_mode = {}
        for mode in (0, 1, 2, 3):
            c.set_strategy(mode, 0)
            for _ in range(3):
                c.herk_batched_v(chans)
            torch.cuda.synchronize()
            e0.record()
            for _ in range(reps):
                c.herk_batched_v(chans)
            e1.record()
            torch.cuda.synchronize()
            by_mode[str(mode)] = round(e0.elapsed_time(e1) / reps, 4)
        if c.device_status() != 0:
            raise RuntimeError("device wait timed out in the batched leg")
    return {"workload": f"{n_chans} channels, K in [128, 2048] step 64, {inputs} inputs with "
                        f"1536..{inputs} active after flagging, one call (tuned, graph replay)",
            "value": flops / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
            "tflop_per_step": flops / 1e12, "ms_by_store_mode": by_mode}


def run_ftd_leg(torch, dev, n_ant=2048, n_chan=64, n_pol=2, K=1024, seed=6):
    """Raw packet-ordered input [t][ant][chan][pol] (2048 antennas x 64
    channels x 2 pols x 1024 samples, 268 MB of QC bytes): the fused corner
    turn + correlator (ftdx_herk_ftd, one triangle per (channel, pol)) against
    the same correlation after a separate batch-first reorder pass."""
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, LAYOUT_TIME_ANT_CHAN_POL, OUT_FP32
    nb = n_chan * n_pol
    raw = make_qc(torch, 1, K, n_ant * n_chan * n_pol, dev, seed=seed).reshape(-1)
    C = torch.empty(nb, tri_size(n_ant), 2, device=dev)
    flops = herk_flops(n_ant, K, nb)
    with Correlator(device=dev.index) as c:
        c.init_herk(n_ant, K, nb)
        fused = _timed(torch, lambda: c.herk_ftd(raw, C, n_ant, n_chan, n_pol, K, 1,
                                                  layout=LAYOUT_TIME_ANT_CHAN_POL), reps=10)
        bf = torch.empty(nb, n_ant, K, dtype=torch.uint8, device=dev)

        def separate():
            bf.view(n_chan, n_pol, n_ant, K).copy_(raw.view(K, n_ant, n_chan, n_pol)
                                                   .permute(2, 3, 1, 0))
            c.herk(bf, C, n_ant, K, nb, input=IN_INT4, output=OUT_FP32, tune=False)
        sep = _timed(torch, separate, reps=10)
        if c.device_status() != 0:
            raise RuntimeError("device wait timed out in the raw-layout leg")
    return {"workload": f"raw [t][ant][chan][pol] QC: {n_ant} antennas x {n_chan} channels x "
                        f"{n_pol} pols x K={K} -> {nb} triangles",
            "value": flops / (fused * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": fused,
            "separate_reorder_then_herk": {"value": flops / (sep * 1e-3) / 1e12,
                                           "ms_per_step": sep}}


def run_imaging_leg(torch, dev, n_ant=2048, n_chan=64, n_pol=2, ng=2048, n_beam=4096, seed=8):
    """Imaging from the packed triangles of 2048 antennas x 64 channels x 2
    pols (FP32, 2.15 GB): pillbox gridding with the pols summed and a taper
    fused, 2048^2 inverse FFTs (cuFFT), 4096 beam pixels per channel."""
    from ftd_b200 import Correlator, tri_size
    g = torch.Generator(device=dev).manual_seed(seed)
    n_bl = tri_size(n_ant)
    vis = torch.randn(n_chan, n_pol, n_bl, 2, device=dev, generator=g)
    freq = 1.0e9 + 1.0e6 * torch.arange(n_chan, device=dev, dtype=torch.float64)
    lam = 299792458.0 / 1.0e9
    uv = ((torch.rand(n_bl, 2, device=dev, generator=g) - 0.5) * ng * lam).contiguous()
    taper = torch.rand(ng, ng, device=dev, generator=g) * 0.8 + 0.2
    pix = torch.randint(0, ng, (n_beam, 2), device=dev, generator=g, dtype=torch.int32)
    beams = torch.empty(n_chan, n_beam, device=dev)
    with Correlator(device=dev.index) as c:
        def call():
            c.image_beams(vis, beams, n_ant, n_chan, n_pol, ng, 1.0, uv, freq, taper=taper,
                          beam_pixels=pix, n_beam=n_beam)
        ms = _timed(torch, call, reps=5)
        if c.device_status() != 0:
            raise RuntimeError("device status after the imaging leg")
    vis_bytes = n_chan * n_pol * n_bl * 8
    return {"workload": f"imaging: {n_ant} antennas x {n_chan} channels x {n_pol} pols packed "
                        f"triangles (FP32) -> {ng}^2 grids -> {n_beam} beams",
            "ms_per_step": ms, "visibility_bytes": vis_bytes,
            "visibility_read_gbs": vis_bytes / (ms * 1e-3) / 1e9,
            "note": "gridding (pols summed, taper fused, FP32 atomics in L2) + cuFFT C2C "
                    "inverse + beam extraction, per grid tile of the channels that fit in 64 MiB"}


# The reference's own VisBF benchmark (pol_mode A) on GH200: 1664 antennas,
# Nf_eff = n_ch * n_time_inner = 16 * 2 = 32 visibility sets, 4096^2 grids,
# 6,000,000 beams, FP16 FFT; per-stage mean times in ms
# (scripts/bench_results_GH200/stages.csv, visbf_16ch_K128; config from
# raw_visbf_16ch_K128_20260306_115016.log).
VISBF_GH200_MS = {"pol_reduce": 0.49, "img_scatter": 1.81, "img_fft": 11.80, "img_beam": 5.29}


def run_imaging_visbf_leg(torch, dev):
    """Imaging at the reference VisBF benchmark's sizes (1664 antennas, 32
    visibility sets x 2 pols, 4096^2 grids, 6,000,000 beams), beside the
    reference's published GH200 stage times for the same stages (pol sum,
    scatter, FFT, beams; different hardware, FP16 FFT there, FP32 here)."""
    out = run_imaging_leg(torch, dev, n_ant=1664, n_chan=32, n_pol=2, ng=4096,
                          n_beam=6_000_000, seed=18)
    ref = sum(VISBF_GH200_MS.values())
    out["reference_gh200_ms"] = {**VISBF_GH200_MS, "sum": ref}
    out["speedup_vs_reference_gh200"] = ref / out["ms_per_step"]
    return out


def run_xengine_leg(torch, dev, n_ant=2048, K=1024, batch=128, seed=9):
    """XEngine-compatible path: [batch][K][n_ant] two's-complement (4,4)b
    blocks (2048 antennas x K=1024 x 128 = 268 MB) -> packed upper triangles
    of C = M^H M (the XEngine's triangular format)."""
    from ftd_b200 import Correlator, tri_size
    g = torch.Generator(device=dev).manual_seed(seed)
    p = torch.randint(0, 256, (batch * K * n_ant,), device=dev, dtype=torch.uint8, generator=g)
    C = torch.empty(batch, tri_size(n_ant), 2, device=dev)
    with Correlator(device=dev.index) as c:
        by_mode = {}
        for mode in (2, 0):  # CTA pair, single-CTA kernel
            c.set_strategy(mode, 0)
            ms = _timed(torch, lambda: c.xengine(p, C, n_ant, K, batch, mat_format=1), reps=10)
            # per-kernel CUDA-event times of 5 more calls: corner turn + promotion, correlator
            c.set_profiling(True)
            for _ in range(5):
                c.xengine(p, C, n_ant, K, batch, mat_format=1)
            torch.cuda.synchronize()
            prof = c.profile_read()
            c.set_profiling(False)
            by_mode[str(mode)] = {
                "ms_per_step": ms,
                "corner_turn_promotion_ms": prof["prep_ms"] / max(prof["prep_launches"], 1),
                "correlator_ms": prof["herk_ms"] / max(prof["herk_launches"], 1)}
        if c.device_status() != 0:
            raise RuntimeError("device status after the XEngine leg")
    ms = by_mode["0"]["ms_per_step"]  # the default strategy: single-CTA kernel
    return {"workload": f"XEngine: {batch} blocks of [K={K}][{n_ant}] two's-complement (4,4)b "
                        f"-> packed upper triangles (FP32), single-CTA kernel",
            "value": herk_flops(n_ant, K, batch) / (ms * 1e-3) / 1e12, "unit": UNIT,
            "ms_per_step": ms, "by_store_mode": by_mode}


def run_splitk_leg(torch, dev, N=256, K=65536, B=4, seed=10):
    """Few inputs, long integration (256 inputs x 4 channels x K = 65536: 12
    tiles for 148 SMs): the plain persistent launch against the autotuned
    strategy, which splits K."""
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP32
    qc = make_qc(torch, B, N, K, dev, seed=seed)
    C = torch.empty(B, tri_size(N), 2, device=dev)
    flops = herk_flops(N, K, B)
    with Correlator(device=dev.index) as c:
        plain = _timed(torch, lambda: c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32,
                                             tune=False), reps=10)
        c.tune(qc, C, N, K, B)
        splits = c.tuned_split_k(N, K, B)
        tuned = _timed(torch, lambda: c.herk(qc, C, N, K, B, input=IN_INT4, output=OUT_FP32,
                                             tune=True), reps=10)
        if c.device_status() != 0:
            raise RuntimeError("device status after the split-K leg")
    return {"workload": f"split-K: {N} inputs x {B} channels x K={K}",
            "value": flops / (tuned * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": tuned,
            "tuned_splits": splits,
            "unsplit": {"value": flops / (plain * 1e-3) / 1e12, "ms_per_step": plain}}


def _timed(torch, fn, reps=5, warm=2):
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_precision_leg(torch, dev, N=4096, B=64, K=1024, seed=4):
    """Float complex voltages, 4096 inputs x 64 channels x K=1024: per-channel
    RMS log-uniform in [0.1, 10]; 1% of time samples carry 20-sigma bursts on
    5% of the inputs.  Throughput of each compute mode, and its error against
    FP64 correlations (torch, on the device) of every element of every
    channel: |dR_ij| / sqrt(R_ii R_jj), cross- and auto-correlations."""
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import (COMPUTE_FP4, COMPUTE_FP4_SPLIT, COMPUTE_FP8, COMPUTE_FP8_SPLIT,
                               IN_FP32, OUT_FP32)
    g = torch.Generator(device=dev).manual_seed(seed)
    rms = torch.exp(torch.empty(B, device=dev).uniform_(float(__import__("math").log(0.1)),
                                                         float(__import__("math").log(10.0)),
                                                         generator=g))
    V = torch.randn(B, N, K, 2, device=dev, generator=g) * (rms.view(B, 1, 1, 1) / 2 ** 0.5)
    n_rfi, t_rfi = max(1, N // 20), max(1, K // 100)
    for b in range(B):
        ins = torch.randperm(N, device=dev, generator=g)[:n_rfi]
        ts = torch.randperm(K, device=dev, generator=g)[:t_rfi]
        ph = torch.rand(n_rfi, t_rfi, device=dev, generator=g) * (2 * 3.141592653589793)
        amp = 20.0 * rms[b]
        sub = torch.stack([amp * torch.cos(ph), amp * torch.sin(ph)], -1)
        V[b, ins[:, None], ts[None, :]] = sub
    C = torch.empty(B, tri_size(N), 2, device=dev)
    flops = herk_flops(N, K, B)
    out = {}
    with Correlator(device=dev.index) as c:
        for name, mode in [("fp8_channel_scaled", COMPUTE_FP8), ("fp8_hi_lo_split", COMPUTE_FP8_SPLIT),
                           ("nvfp4_block16", COMPUTE_FP4),
                           ("nvfp4_hi_lo_split", COMPUTE_FP4_SPLIT)]:
            def step():  # autotuned per mode: the sweep runs in the first (untimed) call
                c.herk(V, C, N, K, B, input=IN_FP32, compute=mode, output=OUT_FP32, tune=True)
            ms = _timed(torch, step)
            if c.device_status() != 0:
                raise RuntimeError("device wait timed out in the precision leg")
            e = full_channel_errors(torch, V, C)
            out[name] = {"value": flops / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
                         "max_rel_err_cross": e["max_cross"], "rms_rel_err_cross": e["rms_cross"],
                         "max_rel_err_auto": e["max_auto"]}
    del V, C
    out["workload"] = (f"{N} inputs x {B} channels x K={K}, float complex Gaussian, RMS "
                       f"log-uniform [0.1, 10], 1% of samples 20-sigma bursts on 5% of inputs; "
                       f"errors |dR_ij|/sqrt(R_ii R_jj) vs FP64 over every element of all {B} "
                       f"channels")
    return out


def full_channel_errors(torch, V, C):
    """max / RMS over all channels of |dR_ij| / sqrt(R_ii R_jj) between the
    packed triangles C [B][P][2] and FP64 products of V [B][N][K][2] computed
    on the device (cross-correlations i != j, and autocorrelations)."""
    B, N = V.shape[0], V.shape[1]
    ii, jj = torch.tril_indices(N, N, device=V.device)
    order = torch.argsort(ii * N + jj)
    ii, jj = ii[order], jj[order]
    off = ii != jj
    mx = mxa = ss = 0.0
    cnt = 0
    for b in range(B):
        Vb = torch.view_as_complex(V[b].double().contiguous())
        R = Vb @ Vb.conj().T
        auto = torch.diagonal(R).real
        e = (torch.view_as_complex(C[b].double().contiguous()) - R[ii, jj]).abs() / \
            torch.sqrt(auto[ii] * auto[jj])
        mx = max(mx, float(e[off].max()))
        mxa = max(mxa, float(e[~off].max()))
        ss += float(e[off].pow(2).sum())
        cnt += int(off.sum())
        del R, e
    return {"max_cross": mx, "rms_cross": (ss / max(cnt, 1)) ** 0.5, "max_auto": mxa}


def run_diff_leg(torch, dev, N=2048, B=32, K=512, seed=5):
    """Adjoint dV = (G + G^H) V (G random Hermitian complex64, V int4) and the
    gain-calibration gradient, 2048 inputs x 32 channels x K=512."""
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import IN_INT4, OUT_FP32
    g = torch.Generator(device=dev).manual_seed(seed)
    qc = make_qc(torch, B, N, K, dev, seed=seed)
    qm = make_qc(torch, B, N, K, dev, seed=seed + 1)
    A = torch.view_as_complex(torch.randn(B, N, N, 2, device=dev, generator=g))
    G = torch.view_as_real(((A + A.conj().transpose(1, 2)) / 2).contiguous()).contiguous()
    del A
    dV = torch.empty(B, N, K, 2, device=dev)
    P = tri_size(N)
    Ro = torch.empty(B, P, 2, device=dev)
    Rm = torch.empty_like(Ro)
    W = torch.rand(B, P, device=dev, generator=g)
    ph = torch.rand(N, device=dev, generator=g) * 6.283185307179586
    mag = 1.0 + (torch.rand(N, device=dev, generator=g) - 0.5) * 0.2
    gains = torch.stack([mag * torch.cos(ph), mag * torch.sin(ph)], -1).contiguous()
    grad = torch.empty(N, 2, dtype=torch.float64, device=dev)
    loss = torch.empty(1, dtype=torch.float64, device=dev)
    with Correlator(device=dev.index) as c:
        c.herk(qc, Ro, N, K, B, input=IN_INT4, output=OUT_FP32)
        c.herk(qm, Rm, N, K, B, input=IN_INT4, output=OUT_FP32)
        ms_adj = _timed(torch, lambda: c.herk_adjoint(G, qc, dV, N, K, B))
        ms_gg = _timed(torch, lambda: c.gain_gradient(Ro, Rm, W, gains, N, B, grad, loss))
        if c.device_status() != 0:
            raise RuntimeError("device wait timed out in the differentiation leg")
    adj_flops = 8.0 * N * N * K * B
    gg_bytes = float(B) * P * (8 + 8 + 4)
    peaks = measured_peaks()
    adj_pipe = 2.0 * adj_flops / (ms_adj * 1e-3) / 1e12  # hi + lo passes on the tensor pipe
    gg_gbs = gg_bytes / (ms_gg * 1e-3) / 1e9
    return {"workload": f"{N} inputs x {B} channels x K={K}",
            "adjoint": {"value": adj_flops / (ms_adj * 1e-3) / 1e12, "unit": UNIT,
                        "ms_per_step": ms_adj,
                        "note": "8 N^2 K per channel; executed as bf16 hi + lo (2x that on "
                                "the tensor cores), plus the G + G^H split pass",
                        "roofline": {"bound": "tensor", "achieved": adj_pipe, "unit": "TFLOPS",
                                     "peak": peaks.get("bf16_tflops"),
                                     "frac": (adj_pipe / peaks["bf16_tflops"])
                                     if peaks.get("bf16_tflops") else None,
                                     "peak_source": peaks.get("source")}},
            "gain_gradient": {"value": gg_gbs, "unit": "GB/s",
                              "ms_per_step": ms_gg, "bytes_per_step": gg_bytes,
                              "roofline": {"bound": "hbm", "achieved": gg_gbs, "unit": "GB/s",
                                           "peak": peaks.get("hbm_gbs"),
                                           "frac": (gg_gbs / peaks["hbm_gbs"])
                                           if peaks.get("hbm_gbs") else None,
                                           "peak_source": peaks.get("source")}}}


def measured_peaks():
    """HBM GB/s and dense bf16 TFLOPS (burst) of this pool's B200s from
    MEASURED_PEAKS.json when present, else the pool's earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]),
                "source": "MEASURED_PEAKS.json (measured)"}
    except (OSError, ValueError, KeyError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def run_e2e(torch, args, dev, qc_dev, N, K, B, flops, world, dist):
    """Same workload end to end through the host-to-host pipeline API
    (ftdx_pipeline_correlate, the VisibilityPipeline::correlate_pipelined
    replacement): every step copies the QC input host->device, correlates, and
    copies every packed triangle device->host (pinned buffers); payload p's
    D2H overlaps payload p+1's H2D and correlation.  Host wall time of the
    blocking call, divided by the payloads it carried."""
    from ftd_b200 import Correlator, Pipeline, tri_size
    from ftd_b200.shard import max_over_ranks
    P = tri_size(N)
    h_in = torch.empty(B * N * K, dtype=torch.uint8, pin_memory=True)
    h_in.copy_(qc_dev.reshape(-1).cpu())
    h_out = [torch.empty(B, P, 2, dtype=torch.float32, pin_memory=True) for _ in range(2)]
    steps = max(3, min(args.steps, 6))
    with Correlator(device=dev.index) as c, Pipeline(c, N, K, B) as pipe:
        pipe.correlate([h_out[0]], [h_in])  # warm-up (tuning, graph capture)
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        pipe.correlate([h_out[i % 2] for i in range(steps)], [h_in] * steps)
        ms = (time.perf_counter() - t0) * 1e3 / steps
    ms = max_over_ranks(ms, dist, dev)
    return {"value": flops * world / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
            "h2d_bytes_per_step": int(B * N * K), "d2h_bytes_per_step": int(B * P * 8),
            "steps": steps,
            "path": "ftdx_pipeline_correlate on pinned host buffers (H2D, correlation and D2H "
                    "on separate streams, D2H over two copy engines, two device buffer sets); "
                    "host wall time"}


def run_nvfp4_case(torch, dev, N, K, B, reps=5, seed=1, split=False, store_mode=None):
    """NVFP4 correlation of seeded Gaussian FP32 complex voltages [B][N][K]:
    reps calls, the whole FP4 path (statistics, quantisation, correlator)
    timed with CUDA events.  split: the hi + lo mode (three products).
    store_mode 0 / 2: single-CTA / CTA-pair kernel (None: autotuned)."""
    from ftd_b200 import Correlator, tri_size
    from ftd_b200._lib import COMPUTE_FP4, COMPUTE_FP4_SPLIT, COMPUTE_FP8, IN_FP32, OUT_FP32
    mode = COMPUTE_FP4_SPLIT if split else COMPUTE_FP4
    g = torch.Generator(device=dev).manual_seed(seed)
    A = torch.randn(B, N, K, 2, device=dev, generator=g)
    C = torch.empty(B, tri_size(N), 2, device=dev)
    with Correlator(device=dev.index) as c:
        if store_mode is not None:
            c.set_strategy(store_mode, 0)
        tune = store_mode is None
        c.herk(A, C, N, K, B, input=IN_FP32, compute=mode, output=OUT_FP32, tune=tune)
        ms = _timed(torch, lambda: c.herk(A, C, N, K, B, input=IN_FP32, compute=mode,
                                          output=OUT_FP32, tune=tune), reps=reps)
        tuned = (c.lookup_tuned(N, K, B, input=IN_FP32, output=OUT_FP32, compute=mode)
                 if tune else None)
        # the FP8 path on the same FP32 input (per-channel scale), for comparison
        c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP8, output=OUT_FP32, tune=tune)
        fp8_ms = _timed(torch, lambda: c.herk(A, C, N, K, B, input=IN_FP32, compute=COMPUTE_FP8,
                                              output=OUT_FP32, tune=tune), reps=reps)
        c.herk(A, C, N, K, B, input=IN_FP32, compute=mode, output=OUT_FP32, tune=tune)
        # per-phase CUDA-event times of the same calls (quantiser, correlator)
        c.set_profiling(True)
        for _ in range(reps):
            c.herk(A, C, N, K, B, input=IN_FP32, compute=mode, output=OUT_FP32, tune=tune)
        torch.cuda.synchronize()
        prof = c.profile_read()
        c.set_profiling(False)
        if c.device_status() != 0:
            raise RuntimeError("device status after the NVFP4 case")
    kernel = ("herk_fp4_pair_kernel" if (store_mode if store_mode is not None else
                                         (tuned or {}).get("store_mode", 0)) == 2
              else "herk_fp4_tc_kernel")
    return {"workload": f"NVFP4{' hi+lo' if split else ''}: {N} inputs x {B} channels x K={K}, "
                        f"Gaussian FP32 complex", "kernel": kernel,
            "value": herk_flops(N, K, B) / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
            "quantiser_ms": prof["prep_ms"] / max(prof["prep_launches"], 1),
            "correlator_ms": prof["herk_ms"] / max(prof["herk_launches"], 1),
            "fp8_channel_scaled_same_input_ms": fp8_ms,
            "speedup_vs_fp8_same_input": fp8_ms / ms}


def run_leg(args):
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    if args.leg == "config1":
        out = run_config1_leg(torch, dev)
    elif args.leg == "diff":
        out = run_diff_leg(torch, dev)
    elif args.leg == "peaks":
        out = measure_tcgen05_peaks(dev.index)
        out["fp8_cublaslt_8192"] = measure_fp8_peak(torch, dev)
    elif args.leg == "nvfp4":
        sm = int(args.strategy.split(",")[0]) if args.strategy else None
        out = run_nvfp4_case(torch, dev, args.inputs, args.k, args.channels, store_mode=sm)
    elif args.leg == "nvfp4split":
        sm = int(args.strategy.split(",")[0]) if args.strategy else None
        out = run_nvfp4_case(torch, dev, args.inputs, args.k, args.channels, split=True,
                             store_mode=sm)
    elif args.leg == "raw":
        out = run_ftd_leg(torch, dev)
    elif args.leg == "imaging":
        out = run_imaging_leg(torch, dev)
    elif args.leg == "splitk":
        out = run_splitk_leg(torch, dev)
    elif args.leg == "precision":
        out = run_precision_leg(torch, dev)
    elif args.leg == "imaging_visbf":
        out = run_imaging_visbf_leg(torch, dev)
    elif args.leg == "batched":
        out = run_batched_leg(torch, dev)
    else:
        out = run_xengine_leg(torch, dev)
    print(json.dumps(out), flush=True)
    return 0


def main():
    args = parse()
    if args.leg:
        return run_leg(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        return run_ours(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
