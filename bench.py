#!/usr/bin/env python
"""Benchmark: Gsamp/s correlated through the FX hot path.

Workload (default): 16 stations; 2-bit real VDIF at 2 Gbps/station
(2 pol x 8 subbands x 32 MHz, 16 bands); 256 channels per subband (512-point
FFTs); 1% seeded invalid frames per station; seeded quadratic delay models
(|tau| <= 20 ms, rates <= 3 us/s); fringe rotation order 1; all four polarisation
products on all 120 baselines plus autocorrelations.  One step = one 0.2 s
subint (25 000 FFT blocks per station, 3.28 Gsamples = station x band time
samples).  The input (0.8 GB of VDIF per step) is larger than L2, so no L2
flush is needed between steps.

Arms:
  default            gxcorr: value = device-resident gx_subint_device steps timed
                     with CUDA events; e2e = gx_subint with pinned host buffers
                     (H2D of the raw VDIF and D2H of the result array inside the
                     timed region).
  --impl reference   the reference correlator's own CPU path (oracle/_ref, compiled
                     from its sources: Configuration/Mode/Core::processdata) on
                     every host core, on a bounded sample of the same workload.

Multi-GPU (torchrun): each rank correlates its own subints (the reference's
time-division axis); no collective on the data path; value = all ranks'
samples / max-over-ranks time (weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from difx_b200 import capi, synth  # noqa: E402
from difx_b200.jobfiles import JobSpec, Subband, write_job  # noqa: E402

METRIC = "Gsamp/s correlated"
UNIT = "Gsamp/s"


def workload_spec(name="c2", subint_ns=200_000_000, threads=1) -> JobSpec:
    if name == "c2":
        return JobSpec(name=f"bench_{name}", nstations=16,
                       subbands=[Subband(8200.0 + 32 * i, 32.0, "U", 256) for i in range(8)],
                       nbits=2, payload_bytes=8000, subint_ns=subint_ns, execute_seconds=20, int_time=1.0,
                       max_delay_us=20000.0, max_rate_us_per_s=3.0, seed=2026)
    if name == "c1":
        return JobSpec(name=f"bench_{name}", nstations=4,
                       subbands=[Subband(8400.0 + 16 * i, 16.0, "U", 128) for i in range(4)],
                       nbits=2, payload_bytes=8000, subint_ns=subint_ns, execute_seconds=20, int_time=0.5,
                       max_delay_us=20000.0, max_rate_us_per_s=3.0, seed=2025)
    raise ValueError(name)


def samples_per_subint(spec: JobSpec) -> float:
    return spec.nstations * spec.nbands * spec.samples_per_second * spec.subint_ns * 1e-9


def build_input(spec: JobSpec, sub_start_ns: int, rho=0.02, invalid_frac=0.01, tile_ms=2.0):
    """Station buffers for one subint: a correlated segment repeated over the window."""
    tile_frames = max(1, int(tile_ms * 1e-3 * spec.frames_per_second))
    streams = []
    for s in range(spec.nstations):
        f0, nf = synth.subint_window(spec, s, sub_start_ns)
        streams.append(synth.make_station_stream_tiled(spec, s, f0, nf, tile_frames, rho=rho, seed=spec.seed,
                                                       invalid_frac=invalid_frac))
    return synth.build_subint(spec, streams, sub_start_ns)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def reference_rate(spec_name: str, target_s: float = 15.0, max_subints: int = 50):
    """The reference's own CPU path on every host core over a bounded sample."""
    from oracle import pyoracle
    if not pyoracle.reference_available():
        return None, "reference harness not built (oracle/_ref/libdifxref.so)"
    ncores = os.cpu_count() or 1
    spec = workload_spec(spec_name, subint_ns=4_000_000 if spec_name == "c2" else 8_000_000)
    d = tempfile.mkdtemp(prefix="gxref_")
    paths = write_job(spec, d)
    with open(paths["threads"], "w") as f:
        f.write(f"{'NUMBER OF CORES:':<20}1\n{ncores}\n")
    ref = pyoracle.Reference(paths["input"])
    si = build_input(spec, 100_000_000, tile_ms=2.0)
    ref.process(si)  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        ref.process(si)
        n += 1
        el = time.perf_counter() - t0
        if el >= target_s or n >= max_subints:
            break
    rate = n * samples_per_subint(spec) / el / 1e9
    sample = (f"{n} subints of {spec.subint_ns / 1e6:g} ms ({spec.blocks_per_send} FFT blocks) of the same workload, "
              f"{ref.nthreads} process threads, {el:.1f} s")
    return {"value": rate, "unit": UNIT, "cores": int(ref.nthreads), "kind": "reference", "sample": sample}, None


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    steps = []
    base, err = None, None
    for _ in range(max(1, args.steps)):
        base, err = reference_rate(args.config, target_s=max(3.0, 15.0 / max(1, args.steps)))
        if base is None:
            break
        steps.append(base["value"])
    if base is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    v = statistics.median(steps)
    base["value"] = v
    spec = workload_spec(args.config)
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": samples_per_subint(spec) / (v * 1e9) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded correlated VDIF)", "impl": "reference",
            "config": config_dict(spec, args), "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def config_dict(spec: JobSpec, args):
    return {"workload": f"{args.config.upper()}: {spec.nstations} stations, {spec.nbits}-bit real VDIF, "
                        f"{len(spec.subbands)} subbands x {len(spec.pols)} pol x {spec.bw_mhz:g} MHz, "
                        f"{spec.nchan} ch/subband, 1% invalid frames, {spec.subint_ns / 1e6:g} ms subints",
            "stations": spec.nstations, "bands_per_station": spec.nbands, "nchan": spec.nchan,
            "fft_points": spec.fftchannels, "subint_ms": spec.subint_ns / 1e6,
            "samples_per_step": samples_per_subint(spec), "xstep": args.xstep,
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"subint-parallel x{args.gpus}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gxcorr", choices=["gxcorr", "reference"])
    ap.add_argument("--config", default="c2", choices=["c2", "c1"])
    ap.add_argument("--xstep", default="fp32", choices=["fp32", "tc"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--subint-ms", type=float, default=200.0,
                    help="subint length (default 200 ms); smaller values give small profiling cases")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    from difx_b200.gxcorr import Correlator

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    spec = workload_spec(args.config, subint_ns=int(round(args.subint_ms * 1e6)))
    xstep = capi.GX_XSTEP_FP32 if args.xstep == "fp32" else capi.GX_XSTEP_TC_FP16
    d = tempfile.mkdtemp(prefix=f"gxbench{rank}_")
    paths = write_job(spec, d)
    # each rank correlates its own subint of the job
    t_sub = 200_000_000 + rank * spec.subint_ns
    si = build_input(spec, t_sub)
    jd = capi.job_desc_from_spec(spec, xstep=xstep, max_data_bytes=max(len(x) for x in si.data))
    corr = Correlator.from_desc(jd, device=local)
    model = Correlator.from_input(paths["input"], device=-1)
    interp = np.array([model.interpolator(s, 0, si.sec, si.ns) for s in range(spec.nstations)])
    model.close()

    # device-resident inputs
    dev = [torch.from_numpy(x).to(f"cuda:{local}") for x in si.data]
    dres = torch.zeros(2 * corr.result_length, dtype=torch.float32, device=f"cuda:{local}")
    sd_dev = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in dev], [len(x) for x in si.data],
                             [x.ctypes.data for x in si.control], len(si.control[0]), interp)
    stream = torch.cuda.Stream(device=local)
    sptr = stream.cuda_stream
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        corr.subint_device(sd_dev, dres.data_ptr(), sptr)
    stream.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches = 0
    stage = np.zeros(3)
    with ClockSampler(local) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            corr.subint_device(sd_dev, dres.data_ptr(), sptr)
            launches += corr.launch_count()
        ev1.record(stream)
        ev1.synchronize()
        dev_ms = ev0.elapsed_time(ev1)
        stage = corr.stage_times()     # last step's per-stage device time
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
        t = torch.tensor([dev_ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_ms = float(t.item())
    total_samples = samples_per_subint(spec) * args.steps * world
    value = total_samples / (dev_ms * 1e-3) / 1e9

    # end to end through the public host-buffer entry point, pinned host memory
    pinned = [torch.from_numpy(x).pin_memory() for x in si.data]
    res_host = torch.zeros(2 * corr.result_length, dtype=torch.float32).pin_memory()
    sd_host = capi.SubintDesc(si.scan, si.sec, si.ns, 0.0, [t.data_ptr() for t in pinned],
                              [len(x) for x in si.data], [x.ctypes.data for x in si.control],
                              len(si.control[0]), interp)
    out_np = res_host.numpy().view(np.complex64)
    for _ in range(2):
        corr.subint(sd_host, out=out_np)
    lat = []
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        a = time.perf_counter()
        corr.subint(sd_host, out=out_np)
        lat.append((time.perf_counter() - a) * 1e3)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = total_samples / e2e_s / 1e9

    # roofline of the dominant kernel (from the last device step's stage times)
    info = corr.info
    chunks = -(-spec.blocks_per_send // 4096)
    nblk_total = spec.blocks_per_send
    f_ms, x_ms = float(stage[0]), float(stage[1])
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    in_bytes = nblk_total * spec.nstations * spec.fftchannels * (spec.bits_per_timesample // 8)
    spec_bytes = nblk_total * spec.nstations * spec.nbands * spec.nchan * 8
    f_bytes = in_bytes + spec_bytes
    if f_ms >= x_ms:
        achieved = f_bytes / (f_ms * 1e-3) / 1e9
        roof = {"kernel": "fstep_kernel", "bound": "hbm", "achieved": achieved, "peak": hbm_peak,
                "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": None, "peak_source": peak_src,
                "algorithmic_bytes_per_subint": f_bytes, "stage_ms": {"F": f_ms, "X": x_ms, "finalise": float(stage[2])}}
    else:
        ncross = spec.nstations * spec.nbands
        cmacs = nblk_total * len(spec.subbands) * spec.nchan * (ncross // len(spec.subbands)) * \
            (ncross // len(spec.subbands) + 1) / 2
        achieved = 8 * cmacs / (x_ms * 1e-3) / 1e12
        fp32_peak = 148 * 128 * 2 * (peaks.get("sm_max_mhz", 1965.0) * 1e6) / 1e12
        roof = {"kernel": "xmac_fp32_kernel", "bound": "fp32-core", "achieved": achieved, "peak": fp32_peak,
                "unit": "TFLOP/s", "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": "nominal FP32 CUDA-core peak (148 SM x 128 FMA/clk x 1965 MHz)",
                "stage_ms": {"F": f_ms, "X": x_ms, "finalise": float(stage[2])}}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded correlated VDIF, 2 ms correlated segment repeated; random-init delay models)",
            "config": config_dict(spec, args),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(sum(len(x) for x in si.data)),
                    "d2h_bytes_per_step": int(corr.result_length * 8)},
            "latency_ms": {"p50": statistics.median(lat), "p99": float(np.percentile(lat, 99)),
                           "subint_ms": spec.subint_ns / 1e6},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        base, err = reference_rate(args.config)
        line["cpu_baseline"] = base if base else {"unavailable": err}
    corr.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
