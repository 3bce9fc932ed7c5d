"""Benchmark of the batched receive path: beamformed px/s on config 1 (64 frames of three linear
probes per launch, DAS + complex IQ, persistent CUDA-graph-captured kernel).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). N > 1 runs N independent replicas (one batch per GPU, no collective
on the data path; torch.distributed is used only for the barrier and the max-over-ranks time).
--impl reference times the CPU restatement of the reference's semantics (the oracle) on the host
cores over a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "beamformed px/s"
UNIT = "px/s"
WORKLOAD = ("c1 batched DAS+IQ: 64 frames/launch (22x P64/1024 smp, 21x P128/2048, 21x P192/3072), 0.3 mm, "
            "fs 40 MHz, 64-ch aperture, F#1 Hann, int16 in; IQ 5 MHz mix, 32-tap LPF, /4, complex64 out")
# DRAM bytes per beamformed pixel of batchPackKernel (8 frames per pack, the autotuner's shape) measured
# by ncu on a 24-frame case of this workload ((dram__bytes_read.sum + dram__bytes_write.sum) / pixels
# = 916.7 MB / 7,249,920 px), scaled by pixels; profiles/batchPackKernel_c1_24frames_full.md has the capture.
TRAFFIC_BYTES_PER_PX = 126.4


def peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # the timed region starts once nvidia-smi reports (its start-up can take longer than the region)
            t0 = time.time()
            while not self.lines and time.time() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_kind() -> str:
    """"reference" when the reference's own per-sample DAS reducers are built for the CPU (oracle/_ref),
    else "port" (the oracle's restatement)."""
    from oracle import oracle as O
    return "reference" if O.ref_lib() is not None else "port"


def cpu_reference_step(geoms, rfs, threads):
    """One bounded step on the host cores: DAS of one frame of each probe through the reference's own
    sampleBeamform2D (oracle/_ref, scanlines in parallel; the oracle's restatement when it is absent),
    then the complex IQ stage (an extension without a reference counterpart: the oracle's FP64-checked
    restatement). Returns beamformed pixels."""
    from oracle import oracle as O
    use_ref = O.ref_lib() is not None
    px = 0
    for g, rf in zip(geoms, rfs):
        img = O.das(g, rf, 1.0, window=1, ref=True) if use_ref else O.das(g, rf, 1.0, window=1, threads=threads)
        img = np.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
        O.iq_complex(img.astype(np.float32), 40e6, 5e6, 2.5e6, 32, 4, threads=threads)
        px += g.num_rx * g.num_depths
    return px


def cpu_sample(threads):
    from supra_b200.workloads import c1_frame, c1_geometries
    geoms = c1_geometries()
    rfs = [c1_frame(g, 2000 + i, device="cpu").numpy() for i, g in enumerate(geoms)]
    return geoms, rfs


def cpu_rows(res):
    """The reference's CPU path beside the library's GPU time for the other configurations, on the box's
    host cores: c0 2D DAS and c2 3D DAS through the reference's own sampleBeamform2D/3D (oracle/_ref; the
    oracle's restatement when it is absent), c3 MV through the oracle's FP32 restatement of
    RxBeamformerMV on 16 of the 128 scanlines, scaled to the full c3 (the reference has no CPU MV)."""
    import torch
    from oracle import oracle as O
    from supra_b200 import synth
    from supra_b200 import workloads as W
    use_ref = O.ref_lib() is not None
    threads = os.cpu_count() or 1
    out = {"cores": threads, "kind": "reference" if use_ref else "port"}

    def timed(fn, reps):
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            best = min(best, time.perf_counter() - t0)
        return best * 1e3

    def row(name, cpu_ms, what):
        gpu_ms = (res or {}).get(name, {}).get("ms")
        out[name] = {"cpu_ms": cpu_ms, "gpu_ms": gpu_ms, "speedup": (cpu_ms / gpu_ms) if gpu_ms else None, "what": what}

    g0, rf0 = synth.c0_frame(0, device="cpu")
    rf0 = rf0.numpy()
    ms = timed(lambda: O.das(g0, rf0, 1.0, window=1, ref=use_ref, threads=threads), 3)
    row("das_c0", ms, "2D DAS of the c0 frame (128 lines x 2048 depths)")
    g2 = W.c2_geometry()
    rf2 = W.c2_volume(g2, device="cpu").numpy()
    ms = timed(lambda: O.das(g2, rf2, 1.0, window=1, ref=use_ref, threads=threads), 1)
    row("das3d_c2", ms, "3D DAS of the c2 volume (32 x 32 lines x 1024 depths)")
    del rf2
    _, x3 = W.c3_raw_delayed()
    x16 = x3[:16].cpu().numpy()
    del x3
    torch.cuda.empty_cache()
    ms = timed(lambda: O.mv(x16, W.C3_L, W.C3_T, 1.5, W.C3_LOADING, threads=threads), 1) * (128 / 16)
    row("mv_c3", ms, "complex MV of c3, timed on 16 of 128 scanlines and scaled by 8 (oracle FP32 restatement)")
    return out


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    geoms, rfs = cpu_sample(threads)
    for _ in range(args.warmup):
        cpu_reference_step(geoms, rfs, threads)
    t0 = time.perf_counter()
    px = 0
    for _ in range(args.steps):
        px += cpu_reference_step(geoms, rfs, threads)
    dt = time.perf_counter() - t0
    value = px / dt
    sample = ("per step: DAS (the reference's sampleBeamform2D on the host cores) + complex IQ of one frame of "
              "each probe (P64, P128, P192) = 917504 px") if cpu_kind() == "reference" else \
        "per step: DAS + complex IQ of one frame of each probe (P64, P128, P192) = 917504 px"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": cpu_kind(), "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def _graph_ms(fn, n, warm=2):
    """Device time of fn (a sequence of library launches) captured once in a CUDA graph and replayed n
    times, so the host's launch overhead stays out of the measurement."""
    import torch
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(warm):
            fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        fn()
    g.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(n):
        g.replay()
    b.record()
    torch.cuda.synchronize()
    del g
    return a.elapsed_time(b) / n


def _event_ms(fn, n, warm=2, reps=3):
    """Mean time of n back-to-back calls (CUDA events on the current stream), the smallest of `reps`
    repetitions, as the reference rows are timed: back-to-back runs of a multi-millisecond kernel were
    seen to spread by tens of percent on one box."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b) / n)
    return best


def chain_rows(g0, o0, hbm_row):
    """The processing after the beamformer. (1) c0's chain on its own 2048 x 128 frame: 64-tap Hilbert
    envelope, 50 dB log compression to uint8, 0.1 mm scan conversion, and the fused env -> log -> scan
    kernel (these frames sit in L2: latency figures). (2) The same kernels on inputs above the 126 MB
    L2 for their HBM rates: a 16384 x 2048 float image (128 MB) for the envelope, the IQ magnitude
    (51-tap filters, decimation 4) and the log compression; the c0 scanlines converted at 0.01 mm
    (13 B of tables per output pixel) for the scan conversion. Graph-replayed device time."""
    import torch
    from supra_b200.api import HilbertFirEnvelope, IQDemodulator, LogCompressor, ScanConverter
    res = {}
    img0 = torch.nan_to_num(o0, nan=0.0, posinf=0.0, neginf=0.0)
    hil = HilbertFirEnvelope(64)
    logc = LogCompressor()
    env0 = hil.demodulate(img0)
    in_max = float(env0.max())
    sc0 = ScanConverter(g0.scanlines, g0.rx_layout, g0.num_depths, g0.depth_mm, 0.1)
    row = {"env_ms": _graph_ms(lambda: hil.demodulate(img0), 20),
           "log_ms": _graph_ms(lambda: logc.compress(env0, 50.0, 1.0, in_max, out_dtype=torch.uint8), 20),
           "scan_ms": _graph_ms(lambda: sc0.convert(env0, torch.uint8), 20),
           "fused_env_log_scan_ms": _graph_ms(lambda: sc0.env_log_convert(hil, img0, 50.0, 1.0, in_max, torch.uint8), 20),
           "image": list(sc0.image_size[:2])}
    res["chain_c0"] = row
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    big = torch.randn((16384, 2048), generator=gen, device="cuda") * 1000.0
    n = big.numel()
    ms = _graph_ms(lambda: hil.demodulate(big), 10)
    res["hilbert_env_large"] = {"ms": ms, "px_per_s": n / ms * 1e3, **hbm_row(8 * n, ms)}
    iq = IQDemodulator(40e6, 2.5e6, 51, 51, (7e6,), (1e6,), (1.0,))
    ms = _graph_ms(lambda: iq.demodulate_magnitude(big, 4), 10)
    res["iq_magnitude_large"] = {"ms": ms, "px_per_s": n / ms * 1e3, **hbm_row(4 * n + 4 * (n // 4), ms)}
    iq3 = IQDemodulator(40e6, 2.5e6, 51, 51, (7e6, 5e6, 9e6), (1e6, 2e6, 2e6), (1.0, 0.5, 0.5))
    ms = _graph_ms(lambda: iq3.demodulate_magnitude(big, 4), 5)
    res["iq_magnitude_3f_large"] = {"ms": ms, "px_per_s": n / ms * 1e3, "filters": 3, **hbm_row(4 * n + 4 * (n // 4), ms)}
    ms = _graph_ms(lambda: logc.compress(big, 50.0, 1.0, 4000.0, out_dtype=torch.uint8), 10)
    res["logcompress_large"] = {"ms": ms, "px_per_s": n / ms * 1e3, **hbm_row(5 * n, ms)}
    del big
    scf = ScanConverter(g0.scanlines, g0.rx_layout, g0.num_depths, g0.depth_mm, 0.01)
    npx = scf.numel
    ms = _graph_ms(lambda: scf.convert(env0, torch.uint8), 10)
    res["scan_large"] = {"ms": ms, "image": list(scf.image_size[:2]), "px_per_s": npx / ms * 1e3,
                         **hbm_row(14 * npx + 4 * env0.numel(), ms)}
    ms = _graph_ms(lambda: scf.env_log_convert(hil, img0, 50.0, 1.0, in_max, torch.uint8), 10)
    res["fused_env_log_scan_large"] = {"ms": ms, "px_per_s": npx / ms * 1e3, **hbm_row(14 * npx + 4 * img0.numel(), ms)}
    return res


def extras(wl, plans):
    """Secondary measurements of the other rows (N = 1 only; device time with CUDA events)."""
    import torch
    from supra_b200.api import RxBeamformer, iq_complex, mv_beamform
    from supra_b200 import workloads as W
    res = {}
    hbm, peak_kind = peaks()
    # FP32 FMA peak of the SIMT pipes at the measured maximum SM clock (148 SMs x 128 lanes x 2 flop)
    fp32_tflops = 148 * 128 * 2 * 1.965e9 / 1e12

    def hbm_row(nbytes, ms):
        gbs = nbytes / ms / 1e6
        return {"gb_per_s": gbs, "hbm_frac": gbs / hbm, "peak": f"{hbm:.1f} GB/s {peak_kind}", "bytes": nbytes}
    # plain per-frame GPU path on the same 64 frames: per-frame DAS kernel + IQ kernel, one frame at a time
    outs = [torch.empty((wl.geometries[p].num_depths, wl.geometries[p].num_rx), device="cuda") for p in wl.frame_probe]

    def per_frame():
        for k, p in enumerate(wl.frame_probe):
            plans[p].beamform(wl.rf[k], 1.0, window_type=1, out=outs[k])
            iq_complex(outs[k], 40e6, 5e6, 2.5e6, 32, 4)
    ms = _graph_ms(per_frame, 3)
    res["per_frame_path"] = {"px_per_s": wl.beamformed_px / ms * 1e3, "frames_per_s": len(wl.rf) / ms * 1e3,
                             "ms_per_batch": ms,
                             "what": "same 64 frames, per-frame DAS + IQ launches (device time, graph-captured)"}
    # c0: one 128-line x 2048-depth frame through the per-frame DAS path
    from supra_b200 import synth
    g0, rf0 = synth.c0_frame(0, device="cuda")
    bf0 = RxBeamformer(g0)
    o0 = torch.empty((g0.num_depths, g0.num_rx), device="cuda")
    ms = _graph_ms(lambda: bf0.beamform(rf0, 1.0, window_type=1, out=o0), 20)
    res["das_c0"] = {"px_per_s": g0.num_rx * g0.num_depths / ms * 1e3, "frames_per_s": 1e3 / ms, "ms": ms,
                     **hbm_row(rf0.numel() * 2 + o0.numel() * 4, ms)}
    # c2: 3D volume, 32 x 32 lines x 1024 depths from 1024 transmits x 256 channels x 1024 samples
    g2 = W.c2_geometry()
    rf2 = W.c2_volume(g2)
    bf2 = RxBeamformer(g2)
    o2 = torch.empty((g2.num_depths, g2.num_rx), device="cuda")
    ms = _event_ms(lambda: bf2.beamform(rf2, 1.0, window_type=1, out=o2), 3, warm=1)
    res["das3d_c2"] = {"vox_per_s": g2.num_rx * g2.num_depths / ms * 1e3, "volumes_per_s": 1e3 / ms, "ms": ms,
                       **hbm_row(rf2.numel() * 2 + o2.numel() * 4, ms)}
    del rf2
    # c2's processing after DAS: 65-tap envelope, 50 dB log, 3D scan conversion to a 0.25 mm grid
    from supra_b200.api import HilbertFirEnvelope, ScanConverter
    v2 = torch.nan_to_num(o2, nan=0.0, posinf=0.0, neginf=0.0)
    hil2 = HilbertFirEnvelope(65)
    sc2 = ScanConverter(g2.scanlines, g2.rx_layout, g2.num_depths, g2.depth_mm, 0.25)
    env2 = hil2.demodulate(v2)
    in_max2 = float(env2.max())
    res["chain_c2"] = {"env_ms": _graph_ms(lambda: hil2.demodulate(v2), 20),
                       "scan_ms": _graph_ms(lambda: sc2.convert(env2, torch.uint8), 20),
                       "env_log_scan_ms": _graph_ms(lambda: sc2.env_log_convert(hil2, v2, 50.0, 1.0, in_max2, torch.uint8), 20),
                       "grid": list(sc2.image_size), "voxels": sc2.numel}
    # c3: complex MV, 128 x 2048 systems of 32 x 32, FP64 re-solve above 1e6
    g3, x3 = W.c3_raw_delayed()
    ms = _event_ms(lambda: mv_beamform(x3, W.C3_L, W.C3_T, 1.5, False, W.C3_LOADING, 1e6, with_stats=False), 5, warm=3)
    _, st = mv_beamform(x3, W.C3_L, W.C3_T, 1.5, False, W.C3_LOADING, 1e6)
    res["mv_c3"] = {"px_per_s": x3.shape[0] * x3.shape[2] / ms * 1e3, "frames_per_s": 1e3 / ms, "ms": ms,
                    "fp64_systems": int(st.fp64_systems), "max_condition_estimate": float(st.max_condition_estimate)}
    del x3
    # RawDelay of the c0 frame: [128 lines][64 channels][2048 depths] float out (67 MB)
    ms = _graph_ms(lambda: bf0.raw_delay(rf0, 1.0, window_type=1), 10)
    res["rawdelay_c0"] = {"ms": ms, **hbm_row(rf0.numel() * 2 + g0.num_rx * g0.num_channels * g0.num_depths * 4, ms)}
    # the other sample beamformers on the c0 frame (per-frame kernels, reference float semantics)
    for name in ("DelayAndStdDev", "CoherenceFactorDelayAndSum"):
        ms = _graph_ms(lambda: bf0.beamform(rf0, 1.0, window_type=1, out=o0, beamformer=name), 10)
        res["das_" + name] = {"px_per_s": g0.num_rx * g0.num_depths / ms * 1e3, "ms": ms,
                              **hbm_row(rf0.numel() * 2 + o0.numel() * 4, ms)}
    # MV with the PCG solve on the c0 frame's raw-delayed data (real, 128 lines x 64 channels x 2048)
    from supra_b200.api import HilbertEnvelope, mv_beamform_pcg, temporal_filter
    raw0 = bf0.raw_delay(rf0, 1.0, window_type=1)
    raw0[~(raw0.abs() < 1e30)] = 0.0
    ms = _event_ms(lambda: mv_beamform_pcg(raw0, 32, 5), 5, warm=3)
    res["mv_pcg_c0"] = {"px_per_s": raw0.shape[0] * raw0.shape[2] / ms * 1e3, "ms": ms, "L": 32, "T": 5}
    del raw0
    # analytic-signal envelope (HilbertEnvelope) of the c0 image. 2048 samples take the FFT path: two
    # complex transforms of N points per pair of scanlines, 5 N log2 N flops per scanline
    env = HilbertEnvelope(g0.num_depths)
    ms = _event_ms(lambda: env.envelope(o0), 10)
    n_env = g0.num_depths
    fft_path = n_env >= 64 and n_env <= 16384 and (n_env & (n_env - 1)) == 0
    flops = (5.0 * n_env * math.log2(n_env) if fft_path else 2.0 * n_env ** 2) * g0.num_rx
    tf = flops / ms / 1e9
    res["analytic_env_c0"] = {"ms": ms, "path": "fft" if fft_path else "circulant", "tflops": tf,
                              "fp32_frac": tf / fp32_tflops, "peak": f"{fp32_tflops:.1f} TFLOP/s nominal FP32 FMA",
                              "bytes": o0.numel() * 8, "note": "input and output (2 MB) stay in L2: latency-bound"}
    # temporal filter over 3 float images of 4096 x 4096 (192 MB in + 64 MB out, above the 126 MB L2)
    ims = [torch.randn((4096, 4096), device="cuda") for _ in range(3)]
    ms = _event_ms(lambda: temporal_filter(ims), 10)
    res["temporal_filter"] = {"ms": ms, "images": 3, **hbm_row(4 * 4096 * 4096 * 4, ms)}
    del ims
    res.update(chain_rows(g0, o0, hbm_row))
    # c4: differentiable DAS, 16 frames: adjoint (all three gradients) vs forward
    g4, rf4 = W.c4_batch()
    bf4 = RxBeamformer(g4)
    apod = torch.ones(g4.num_elements, device="cuda")
    c = g4.speed_of_sound_mm_s
    fwd = bf4.forward_apod(rf4, apod, c)
    gout = torch.randn_like(fwd)
    ms_f = _event_ms(lambda: bf4.forward_apod(rf4, apod, c), 5)
    ms_a = _event_ms(lambda: bf4.adjoint(rf4, apod, gout, c, forward_out=fwd), 5)
    res["adjoint_c4"] = {"forward_ms": ms_f, "adjoint_ms": ms_a, "adjoint_to_forward": ms_a / ms_f,
                         "frames": int(rf4.shape[0])}
    return res


def reference_gpu_rows(res):
    """The reference's own kernels on this GPU: the reference's sources built with its
    production flags (--use_fast_math, release), oracle/_ref/libsupra_ref_gpu_fast.so, each called as its
    node calls it per frame (kernels + pooled output allocation), CUDA-event time per call on the call's
    stream. Beside each: the library's time for the same input from `res` and the speed-up. Even FIR
    lengths read one tap past the reference's filter buffer, so the envelope comparison uses 65 taps."""
    import ctypes as C
    import torch
    from oracle import oracle as O
    from supra_b200 import synth
    from supra_b200 import workloads as W
    from supra_b200.api import HilbertFirEnvelope, mv_beamform
    lib = O.refgpu_fast_lib()
    if lib is None:
        return {"unavailable": "oracle/_ref/libsupra_ref_gpu_fast.so not built (make -C oracle refgpu)"}
    out = {"build": "reference sources, nvcc --use_fast_math -O2, NDEBUG (SupraLib/CMakeLists.txt:65)",
           "timing": "CUDA events around back-to-back calls of the reference's class method on its stream; "
                     "smallest of 5 repetitions"}

    def row(name, ref_ms, ours_ms, what):
        out[name] = {"reference_ms": ref_ms, "ours_ms": ours_ms,
                     "speedup": (ref_ms / ours_ms) if (ref_ms and ours_ms and ref_ms > 0) else None, "what": what}

    def geo(g):
        return g.ctypes()

    g0, rf0 = synth.c0_frame(0, device="cpu")
    x0 = np.ascontiguousarray(rf0.numpy())
    gc = geo(g0)
    # the library's MV timings first: the reference's container pool frees buffers from a background
    # thread (cudaFree synchronises the device), which would stall launches timed after its calls
    from supra_b200.api import RxBeamformer, mv_beamform_pcg
    raw = RxBeamformer(g0).raw_delay(rf0.cuda(), 1.0, window_type=1)
    raw[~(raw.abs() < 1e30)] = 0.0
    raw = raw[:, :, :2000].contiguous()
    rh = np.ascontiguousarray(raw.cpu().numpy())
    ours_mv = _event_ms(lambda: mv_beamform(raw, 32, 5, 1.5, False, 1.0, 1e6, with_stats=False), 5, warm=2)
    ours_pcg = _event_ms(lambda: mv_beamform_pcg(raw, 32, 5, convergence_threshold=1e-4), 5, warm=2)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    big = torch.randn((16384, 2048), generator=gen, device="cuda") * 1000.0  # 128 MB, above L2
    hil = HilbertFirEnvelope(65)
    ours_hil = _graph_ms(lambda: hil.demodulate(big), 10)
    hb = np.ascontiguousarray(big.cpu().numpy())
    del big
    ms = lib.refg_time_das(C.byref(gc), C.c_void_p(x0.ctypes.data), C.c_double(1.0),
                           C.c_double(g0.speed_of_sound_mm_s), 1, 0, C.c_double(g0.depth_mm), 20)
    row("das_c0", ms, res.get("das_c0", {}).get("ms"), "2D DAS, c0 frame (128 lines x 2048 depths, int16 in)")
    for bf, name in ((1, "das_DelayAndStdDev"), (2, "das_CoherenceFactorDelayAndSum")):
        ms = lib.refg_time_das(C.byref(gc), C.c_void_p(x0.ctypes.data), C.c_double(1.0),
                               C.c_double(g0.speed_of_sound_mm_s), 1, bf, C.c_double(g0.depth_mm), 10)
        row(name, ms, res.get(name, {}).get("ms"), "sample beamformer on the c0 frame")
    ms = lib.refg_time_rawdelay(C.byref(gc), C.c_void_p(x0.ctypes.data), C.c_double(1.0),
                                C.c_double(g0.speed_of_sound_mm_s), 1, C.c_double(g0.depth_mm), 10)
    row("rawdelay_c0", ms, res.get("rawdelay_c0", {}).get("ms"), "RawDelay of the c0 frame")
    g2 = W.c2_geometry()
    x2 = np.ascontiguousarray(W.c2_volume(g2).cpu().numpy())
    gc2 = geo(g2)
    ms = lib.refg_time_das(C.byref(gc2), C.c_void_p(x2.ctypes.data), C.c_double(1.0),
                           C.c_double(g2.speed_of_sound_mm_s), 1, 0, C.c_double(g2.depth_mm), 3)
    row("das3d_c2", ms, res.get("das3d_c2", {}).get("ms"), "3D DAS, c2 volume (32 x 32 lines x 1024 depths)")
    del x2
    # envelope chain on a 16384 x 2048 float image (128 MB, above L2)
    ms = lib.refg_time_hilbert(C.c_void_p(hb.ctypes.data), C.c_uint32(2048), C.c_uint32(16384), C.c_uint32(65), 10)
    row("hilbert_env_large_65taps", ms, ours_hil, "Hilbert FIR envelope, 65 taps, 16384 x 2048 float image")
    f = np.array([7e6]), np.array([1e6]), np.array([1.0])
    fa = [np.ascontiguousarray(v, np.float64) for v in f]
    ms = lib.refg_time_iq(C.c_void_p(hb.ctypes.data), C.c_uint32(2048), C.c_uint32(16384), C.c_double(40e6),
                          C.c_double(7e6), C.c_double(2.5e6), C.c_uint32(51), C.c_uint32(51), C.c_uint32(4),
                          C.c_uint32(1), *(C.c_void_p(v.ctypes.data) for v in fa), 10)
    row("iq_magnitude_large", ms, res.get("iq_magnitude_large", {}).get("ms"),
        "IQ magnitude, 51-tap filters, decimation 4, 16384 x 2048 float image")
    f3 = [np.ascontiguousarray(v, np.float64) for v in ((7e6, 5e6, 9e6), (1e6, 2e6, 2e6), (1.0, 0.5, 0.5))]
    ms = lib.refg_time_iq(C.c_void_p(hb.ctypes.data), C.c_uint32(2048), C.c_uint32(16384), C.c_double(40e6),
                          C.c_double(7e6), C.c_double(2.5e6), C.c_uint32(51), C.c_uint32(51), C.c_uint32(4),
                          C.c_uint32(3), *(C.c_void_p(v.ctypes.data) for v in f3), 3)
    row("iq_magnitude_3f_large", ms, res.get("iq_magnitude_3f_large", {}).get("ms"),
        "IQ magnitude with frequency compounding (3 filters), decimation 4, 16384 x 2048 float image")
    ms = lib.refg_time_logcompress(C.c_void_p(hb.ctypes.data), C.c_uint32(2048), C.c_uint32(16384), C.c_double(50.0),
                                   C.c_double(1.0), C.c_double(4000.0), 10)
    row("logcompress_large", ms, res.get("logcompress_large", {}).get("ms"),
        "log compression to uint8, 16384 x 2048 float image")
    del hb
    # scan conversion of the c0 envelope at 0.1 mm
    img0 = np.abs(np.random.Generator(np.random.PCG64(3)).standard_normal((g0.num_depths, g0.num_rx))).astype(np.float32)
    rs = O.RefScan(g0.scanlines, g0.rx_layout, g0.num_depths, g0.depth_mm, 0.1, lib=lib)
    ms = lib.refg_time_scan(rs.h, C.c_void_p(img0.ctypes.data), 20)
    row("scan_c0", ms, res.get("chain_c0", {}).get("scan_ms"), "2D scan conversion of the c0 frame to 0.1 mm, uint8")
    del rs
    # FFT envelope of the c0 image, temporal filter of 3 x 64 MB
    ms = lib.refg_time_fft_env(C.c_void_p(img0.ctypes.data), C.c_uint32(g0.num_rx), C.c_uint32(g0.num_depths), 10)
    row("analytic_env_c0", ms, res.get("analytic_env_c0", {}).get("ms"), "FFT (analytic-signal) envelope, c0 image")
    t = np.random.Generator(np.random.PCG64(4)).standard_normal((4096, 4096)).astype(np.float32)
    ms = lib.refg_time_temporal(C.c_void_p(t.ctypes.data), C.c_uint32(3), C.c_uint32(4096), C.c_uint32(4096), 10)
    row("temporal_filter", ms, res.get("temporal_filter", {}).get("ms"), "temporal filter of 3 float 4096 x 4096 images")
    del t
    # minimum variance on the c0 frame's raw-delayed data (real), 2000 depths (the reference's MV
    # handles at most 2000 samples), L 32, +-5; the library with the reference's loading trace/L
    ms = lib.refg_time_mv(C.c_void_p(rh.ctypes.data), C.c_uint32(128), C.c_uint32(64), C.c_uint32(2000), C.c_uint32(32),
                          C.c_uint32(5), C.c_double(1.5), 1)
    row("mv_c0_2000", ms, ours_mv, "MV (real, loading trace/L), c0 raw-delayed 128 lines x 64 channels x 2000 depths, L 32, +-5")
    ms = lib.refg_time_mvpcg(C.c_void_p(rh.ctypes.data), C.c_uint32(128), C.c_uint32(64), C.c_uint32(2000),
                             C.c_uint32(32), C.c_uint32(5), C.c_double(1e-4), C.c_double(1.5), 2)
    row("mv_pcg_c0_2000", ms, ours_pcg, "MV-PCG (convergence threshold 1e-4, the node's default), same input")
    return out


def profile_case(case: str):
    """One small invocation for an ncu capture (no timing)."""
    import torch
    from supra_b200.api import BatchedDasIq, RxBeamformer, mv_beamform
    from supra_b200.workloads import c1_workload
    if case == "batch":
        wl = c1_workload(num_frames=24, device="cuda")  # 8 frames per probe: packs of 8 frames are full
        plans = [RxBeamformer(g) for g in wl.geometries]
        b = BatchedDasIq([(plans[p], rf) for p, rf in zip(wl.frame_probe, wl.rf)], ctas_per_sm=4, depth_tile=256,
                         frames_per_pack=8)
        for _ in range(2):
            b.run(use_graph=False)
    elif case == "mv":
        x = torch.randn((16, 128, 2048), dtype=torch.complex64, device="cuda")
        mv_beamform(x, 32, 5, 1.5, False, 0.01, 1e6)
    elif case == "pcg":
        x = torch.randn((16, 64, 2048), device="cuda") * 1000.0
        from supra_b200.api import mv_beamform_pcg
        mv_beamform_pcg(x, 32, 5)
    elif case == "chain":
        # the envelope-chain kernels on inputs above L2: 16384 x 2048 float image (128 MB)
        from supra_b200.api import HilbertFirEnvelope, IQDemodulator, LogCompressor
        gen = torch.Generator(device="cuda")
        gen.manual_seed(7)
        big = torch.randn((16384, 2048), generator=gen, device="cuda") * 1000.0
        HilbertFirEnvelope(64).demodulate(big)
        IQDemodulator(40e6, 2.5e6, 51, 51, (7e6,), (1e6,), (1.0,)).demodulate_magnitude(big, 4)
        IQDemodulator(40e6, 2.5e6, 51, 51, (7e6, 5e6, 9e6), (1e6, 2e6, 2e6), (1.0, 0.5, 0.5)).demodulate_magnitude(big, 4)
        LogCompressor().compress(big, 50.0, 1.0, 4000.0, out_dtype=torch.uint8)
    elif case == "misc":
        # one launch each: c0 DAS (single-frame pack kernel), DelayAndStdDev on c0, the FFT envelope of
        # the c0 image, scan conversion of the c0 envelope at 0.01 mm, temporal filter of 3 x 64 MB
        from supra_b200 import synth
        from supra_b200.api import HilbertEnvelope, HilbertFirEnvelope, ScanConverter, temporal_filter
        g0, rf0 = synth.c0_frame(0, device="cuda")
        bf0 = RxBeamformer(g0)
        img = bf0.beamform(rf0, 1.0, window_type=1)
        bf0.beamform(rf0, 1.0, window_type=1, beamformer="DelayAndStdDev")
        img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
        HilbertEnvelope(g0.num_depths).envelope(img)
        env = HilbertFirEnvelope(64).demodulate(img)
        ScanConverter(g0.scanlines, g0.rx_layout, g0.num_depths, g0.depth_mm, 0.01).convert(env, torch.uint8)
        temporal_filter([torch.randn((4096, 4096), device="cuda") for _ in range(3)])
    elif case == "das3d":
        from supra_b200 import workloads as W
        g2 = W.c2_geometry()
        rf2 = W.c2_volume(g2)
        RxBeamformer(g2).beamform(rf2, 1.0, window_type=1)
    elif case == "refgpu":
        # the reference's own kernels (production flags) on the rows' inputs, for their launch list
        print(json.dumps(reference_gpu_rows({}), default=str)[:200])
    elif case == "adjoint":
        from supra_b200 import workloads as W
        g4, rf4 = W.c4_batch(frames=2)
        bf4 = RxBeamformer(g4)
        apod = torch.ones(g4.num_elements, device="cuda")
        fwd = bf4.forward_apod(rf4, apod, g4.speed_of_sound_mm_s)
        bf4.adjoint(rf4, apod, torch.randn_like(fwd), g4.speed_of_sound_mm_s, forward_out=fwd)
    torch.cuda.synchronize()
    print("profile case done:", case)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # defaults: 200 GPU steps (about 0.2 s timed, so nvidia-smi's 0.1 s samples fall inside), or 3 CPU
    # steps of about 10 s each for the reference arm
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's own GPU kernels")
    ap.add_argument("--no-extras", action="store_true", help="skip the secondary measurements (c0, c2, c3, c4)")
    ap.add_argument("--frames", type=int, default=64, help="frames per launch (64 = the named workload)")
    ap.add_argument("--profile-case", choices=["batch", "mv", "adjoint", "das3d", "pcg", "chain", "misc", "refgpu"],
                    help="run one small case for ncu and exit")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 3 if args.impl == "reference" else 200
    if args.warmup is None:
        args.warmup = 1 if args.impl == "reference" else 5
    if args.profile_case:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        return profile_case(args.profile_case)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from supra_b200.api import BatchedDasIq, RxBeamformer, check_device_errors
    from supra_b200.replicas import job_rate
    from supra_b200.workloads import c1_workload

    wl = c1_workload(num_frames=args.frames, device="cuda", seed0=1000 + 100 * rank)
    plans = [RxBeamformer(g) for g in wl.geometries]
    frames = [(plans[p], rf) for p, rf in zip(wl.frame_probe, wl.rf)]
    batch = BatchedDasIq(frames, 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4)
    shape = batch.autotune(os.path.join(HERE, "supra_b200", "lib", "autotune_cache.txt"))
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(max(args.warmup, 3)):
        batch.run(use_graph=True)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local) as clk:
        evs[0].record(stream)
        for i in range(args.steps):
            batch.run(use_graph=True)
            evs[i + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    check_device_errors()
    per = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    px = wl.beamformed_px
    value, total_ms = job_rate(px, args.steps, total_ms, device="cuda")
    kern_ms = statistics.mean(per)
    alg_bytes = wl.rf_bytes + wl.iq_bytes(4)
    hbm, peak_kind = peaks()
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    traffic = None if TRAFFIC_BYTES_PER_PX is None else TRAFFIC_BYTES_PER_PX * px

    # end to end through the public API: pinned host RF -> device, batch, IQ -> pinned host. Steps
    # alternate between two streams, each with its own device RF set and batch, so one step's batch and
    # IQ read-back (the other PCIe direction) overlap the next step's RF upload, as a streaming
    # acquisition would run; every step still uploads its inputs and reads back its result.
    host_rf = [r.cpu().pin_memory() for r in wl.rf]
    host_iq = [[torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in batch.outputs] for _ in range(2)]
    h2d = sum(h.numel() * h.element_size() for h in host_rf)
    d2h = sum(h.numel() * h.element_size() for h in host_iq[0])
    rf_b = [torch.empty_like(r) for r in wl.rf]
    batch_b = BatchedDasIq([(plans[p], r) for p, r in zip(wl.frame_probe, rf_b)], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4,
                           ctas_per_sm=shape[0], depth_tile=shape[1], frames_per_pack=shape[2], staged=shape[3])
    lanes = [(torch.cuda.Stream(), wl.rf, batch, host_iq[0]), (torch.cuda.Stream(), rf_b, batch_b, host_iq[1])]

    def e2e_step(i):
        st, rfs, bt, hiq = lanes[i % 2]
        with torch.cuda.stream(st):
            for h, d in zip(host_rf, rfs):
                d.copy_(h, non_blocking=True)
            bt.run(use_graph=True)
            for h, d in zip(hiq, bt.outputs):
                h.copy_(d, non_blocking=True)

    for i in range(2):
        e2e_step(i)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for st, _, _, _ in lanes:
        st.wait_stream(stream)
    for i in range(args.e2e_steps):
        e2e_step(i)
    for st, _, _, _ in lanes:
        stream.wait_stream(st)
    b.record(stream)
    torch.cuda.synchronize()
    e2e_value, _ = job_rate(px, args.e2e_steps, a.elapsed_time(b), device="cuda")
    del batch_b, rf_b

    extra = None
    if world == 1 and not args.no_extras:
        extra = extras(wl, plans)
        extra["per_frame_path"]["batched_speedup"] = value / extra["per_frame_path"]["px_per_s"]

    # baseline leg (rank 0, one GPU): the reference's own GPU kernels on this GPU beside the library's
    # rows, and the reference's CPU path on the host cores
    ref_gpu = None
    if rank == 0 and world == 1 and extra is not None and not args.no_ref_gpu:
        ref_gpu = reference_gpu_rows(extra)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        geoms, rfs = cpu_sample(threads)
        cpu_reference_step(geoms, rfs, threads)
        t0 = time.perf_counter()
        n = 0
        while time.perf_counter() - t0 < 10.0:
            n += cpu_reference_step(geoms, rfs, threads)
        kind = cpu_kind()
        cpu = {"value": n / (time.perf_counter() - t0), "unit": UNIT, "cores": threads, "kind": kind,
               "sample": ("the reference's sampleBeamform2D" if kind == "reference" else "oracle DAS (reference FP32 "
                          "semantics)") + " + complex IQ (oracle), one frame per probe per step, ~10 s"}
        if extra is not None:
            extra["cpu"] = cpu_rows(extra)

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_launch": len(wl.rf), "beamformed_px_per_launch": px,
                       "parallelism": f"replicas x{world}", "l2": "inputs 2.47 GB per launch > L2, no flush",
                       "tile_shape": {"ctas_per_sm": shape[0], "depth_tile": shape[1], "frames_per_pack": shape[2],
                                      "staged": shape[3]},
                       "graph_captured": True},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": ("batchPackStagedKernel" if shape[3] else "batchPackKernel") if shape[2] > 1
                         else "batchDasIqKernel",
                         "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": kern_ms},
            "cpu_baseline": cpu,
            "reference_gpu": ref_gpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "rows": extra,
        }
        print(json.dumps(out), flush=True)
    del batch
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
