#!/usr/bin/env python3
"""Benchmark of the decode hot path: LTE turbo decoding on the GPU.

Workload (one "step"): one batch of 1024 LTE turbo frames, K = 6144, rate 1/3,
8-state RSC (13, 15 octal) with trellis termination and the LTE QPP interleaver,
BPSK over AWGN at Eb/N0 = 0.7 dB, FP32 L-values, max-log-MAP (Approximate),
6 iterations, serial scheduling; synthetic seeded frames.

value      decoded info Mbit/s with the L-values resident in device memory (each rank
           decodes its own batch; whole-job bits / max-over-ranks device time).
e2e        the same metric through the public decode call with pinned host buffers:
           host->device copy of the L-values and device->host copy of the bits inside
           the timed region.
roofline   the dominant kernel against the measured HBM copy bandwidth, with the
           algorithmic bytes of one decode (algorithmic_bytes_per_frame: L-values once,
           per half-iteration the systematic, parity and a-priori reads and the
           extrinsic write, one byte per decoded bit) over the decode's device time.

`--impl reference` times the reference FeCl decoder compiled from its sources
(oracle/_ref) on this machine's host cores on the same workload.
"""
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

METRIC = "decoded info Mbit/s at matched FER vs plain GPU path; p50/p99 latency"
K = 6144
FRAMES = 1024
ITERATIONS = 6
EBN0_DB = 0.7
SEED = 2024


def workload_config(n_gpus):
    return {
        "workload": "LTE turbo decode, K=6144 x 1024 frames per GPU, rate 1/3 RSC(13,15) + QPP, "
                    "max-log-MAP, 6 iterations, serial, Eb/N0 0.7 dB, FP32 L-values",
        "K": K, "frames_per_gpu": FRAMES, "iterations": ITERATIONS, "algorithm": "Approximate (max-log-MAP)",
        "scheduling": "Serial", "ebn0_db": EBN0_DB, "llr_dtype": "f32",
        "l2": "flushed between timed steps (256 MiB write); inputs 75.5 MB per GPU",
        "parallelism": "frame shards, replicas per GPU" if n_gpus > 1 else "single GPU",
    }


def algorithmic_bytes_per_frame(k=K, iters=ITERATIONS, s_llr=4, s_ext=4):
    """Minimal traffic of one frame decode: the L-values once, then per
    half-iteration the systematic + parity + a-priori reads and the extrinsic
    write, then one byte per decoded bit."""
    return (3 * k + 12) * s_llr + iters * 2 * ((2 * k + 3) * s_llr + 2 * (k + 3) * s_ext) + k


def make_inputs(code, frames, seed):
    import numpy as np
    from fecl_b200 import channel as ch
    msg = ch.random_bits(frames * code.msgSize(), seed)
    cw = code.encode(msg)
    llr = ch.awgn_llr(cw, EBN0_DB, code.msgSize() / code.paritySize(), seed, np.float32)
    return msg, llr


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def kernels_per_decode(run):
    """The library's kernel launches in one call of `run` (outside any timed region),
    counted from the CUDA activity trace of torch's profiler; None if the trace is not
    available."""
    import torch
    try:
        from torch.profiler import ProfilerActivity, profile
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            run()
            torch.cuda.synchronize()
        names = [e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
        n = sum(1 for s in names if "turbo_lte" in s)
        return n or None
    except Exception:
        return None


def profiled_traffic():
    """DRAM bytes per decode of the dominant kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "turbo_lte_traffic.json")) as f:
            return json.load(f).get("dram_bytes_per_decode")
    except Exception:
        return None


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region.  NVML is polled
    from a thread every 2 ms (one sample also on entry and on exit), so even a timed
    region of a tenth of a second has tens of samples; where NVML cannot be loaded,
    nvidia-smi samples every 200 ms instead."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock event reason bits (nvmlClocksEventReason*) of the reasons reported
    REASON_BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
                   ("sw_power_cap", 0x4))

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.nvml = None
        self.handle = None
        self.max_mhz = None
        self.f = None
        self.p = None
        self.thread = None
        self.stop = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            pr = torch.cuda.get_device_properties(self.index)
            bus = "%08X:%02X:%02X.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.index)

    def _sample(self):
        n = self.nvml
        try:
            sm = n.nvmlDeviceGetClockInfo(self.handle, n.NVML_CLOCK_SM)
            get = getattr(n, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                n.nvmlDeviceGetCurrentClocksThrottleReasons
            self.rows.append((float(sm), int(get(self.handle))))
        except Exception:
            pass

    def _poll(self):
        while not self.stop.wait(0.002):
            self._sample()

    def __enter__(self):
        try:
            import threading
            self.nvml, self.handle = self._nvml_handle()
            self.max_mhz = float(self.nvml.nvmlDeviceGetMaxClockInfo(self.handle, self.nvml.NVML_CLOCK_SM))
            self._sample()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.thread is not None:
            self._sample()
            self.stop.set()
            self.thread.join(timeout=5)
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if self.nvml is not None:
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "source": "nvml"}
            reasons = sorted({name for _, mask in self.rows for name, bit in self.REASON_BITS if mask & bit})
            return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                    "reasons": reasons, "samples": len(self.rows), "source": "nvml"}
        try:
            self.f.seek(0)
            rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
            os.unlink(self.f.name)
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "source": "nvidia-smi"}


def channel_module():
    """The seeded channel model (fecl_b200/channel.py, plain numpy), loaded from its
    file so that the reference arm imports nothing that loads the GPU library."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("_fecl_channel", os.path.join(ROOT, "fecl_b200", "channel.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


APPROXIMATE, SERIAL = 2, 0  # fec::DecoderAlgorithm::Approximate, fec::SchedulingType::Serial


def reference_lte_codec(workgroup):
    """The reference's LTE turbo codec (oracle/_ref): RSC (13, 15) twice, the QPP
    interleaver of its own Lte3Gpp table, Tail termination, max-log-MAP, serial."""
    import numpy as np
    from oracle import ref
    return ref.RefCodec.turbo([([4], [[0o15]], [0o13])], [np.arange(K), ref.lte_interleaver(K)], 0,
                              APPROXIMATE, SERIAL, ITERATIONS, workgroup=workgroup)


def cpu_reference(frames_sample, llr, code_sizes):
    """Time the reference FeCl decoder (oracle/_ref) with all host threads on a
    bounded sample of the workload.  Falls back to the C restatement of the oracle."""
    import numpy as np
    from oracle import ref
    cores = os.cpu_count() or 1
    n = frames_sample
    x = np.ascontiguousarray(llr[: n * code_sizes["parity"]], dtype=np.float64)
    if ref.available():
        rc = reference_lte_codec(cores)
        t = time.perf_counter()
        bits = rc.decode(x)
        dt = time.perf_counter() - t
        kind = "reference"
    else:
        from oracle import restated
        if not restated.available():
            return None, None
        t = time.perf_counter()
        bits, _ = restated.turbo_lte_decode(K, APPROXIMATE, ITERATIONS, SERIAL, x, threads=cores)
        dt = time.perf_counter() - t
        kind = "port"
    return {"value": n * K / dt / 1e6, "unit": "Mbit/s", "cores": cores, "kind": kind,
            "sample": "%d frames of the workload, one decode, %d threads, %.2f s wall" % (n, cores, dt)}, bits


def hard_parity(bits, ref_bits, msg, k):
    """The hard-decision parity rule against the reference decoder: in every frame the
    reference decodes the decisions are equal bit for bit, and the same frames fail.
    In a failed frame the decisions follow FP32 rounding, so a few may differ; their
    count is reported."""
    import numpy as np
    b = np.asarray(bits).reshape(-1, k)
    r = np.asarray(ref_bits).reshape(-1, k)
    m = np.asarray(msg).reshape(-1, k)
    ok = ~np.any(r != m, axis=1)
    gpu_ok = ~np.any(b != m, axis=1)
    diff = np.sum(b != r, axis=1)
    return {"frames": int(len(ok)), "decoded_by_reference": int(ok.sum()),
            "equal_in_decoded_frames": bool(np.all(diff[ok] == 0)),
            "same_failed_frames": bool(np.array_equal(ok, gpu_ok)),
            "bits_differing_in_failed_frames": int(diff[~ok].sum()),
            "all_frames_equal": bool(np.all(diff == 0))}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_reference_arm(args):
    """The reference's own decoder (compiled from its sources into oracle/_ref) on the
    host cores.  The inputs come from the reference's encoder and interleaver and the
    numpy channel model, so this arm loads nothing of this repository's library."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libfecl_ref.so was not built on this machine"}))
        return 0
    ch = channel_module()
    parity = 3 * K + 12
    sizes = {"parity": parity}
    cores = os.cpu_count() or 1
    sample = max(8, min(FRAMES, cores * 8))
    msg = ch.random_bits(sample * K, SEED)
    cw = reference_lte_codec(cores).encode(msg)
    llr = ch.awgn_llr(cw, EBN0_DB, K / parity, SEED, np.float32)
    vals = []
    for i in range(args.warmup + args.steps):
        cb, _ = cpu_reference(sample, llr, sizes)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "Mbit/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sample * K / v / 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": workload_config(world), "cpu_baseline": cb,
        "e2e": {"value": round(v, 3), "unit": "Mbit/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---- LDPC workloads (--workload ldpc-short | ldpc-normal) ----------------------------

LDPC_WORKLOADS = {
    # DVB-S2 short frame, nominal rate 1/2 (K = 7200), Exact BP, at most 20 iterations
    # with the syndrome stop, FP64 L-values; outputs hard bits and a-posteriori L-values.
    "ldpc-short": {"codes": [(16200, (1, 2), 64, 1.5)], "algorithm": "Exact", "iterations": 20, "scaling": 1.0,
                   "llr": "f64", "soft": True,
                   "text": "DVB-S2 short n=16200 r=1/2 x 64 frames, Exact BP, <=20 iterations with syndrome stop, "
                           "Eb/N0 1.5 dB, FP64 L-values, hard bits + a-posteriori L-values"},
    # DVB-S2 normal frames at rates 1/2, 3/4, 9/10, 512 frames each, normalised min-sum
    # (0.75), at most 50 iterations; message storage set by --precision.
    "ldpc-normal": {"codes": [(64800, (1, 2), 512, 1.5), (64800, (3, 4), 512, 2.75), (64800, (9, 10), 512, 3.75)],
                    "algorithm": "Approximate", "iterations": 50, "scaling": 0.75, "llr": "f32", "soft": False,
                    "text": "DVB-S2 normal n=64800 r=1/2, 3/4, 9/10 x 512 frames each (Eb/N0 1.5, 2.75, 3.75 dB), "
                            "normalised min-sum 0.75, <=50 iterations with syndrome stop, FP32 L-values"},
}
PRECISIONS = {"f32": 0, "f16": 1, "i8": 2}


def run_ldpc(args, embedded=False):
    """LDPC workloads; with `embedded` the line is returned instead of printed."""
    import numpy as np
    import torch
    from fractions import Fraction
    import fecl_b200 as F
    from fecl_b200 import channel as ch

    w = LDPC_WORKLOADS[args.workload]
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    prec = PRECISIONS[args.precision]
    np_llr = {"f64": np.float64, "f32": np.float32, "f16": np.float16}[w["llr"]]
    alg = getattr(F, w["algorithm"])
    jobs = []
    for n, (num, den), frames, ebn0 in w["codes"]:
        frames = args.frames or frames
        H = F.Ldpc.DvbS2.matrix(n, Fraction(num, den))
        code = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(alg).iterations(w["iterations"])
                      .scalingFactor(w["scaling"]).precision(prec))
        code.setKernel(args.kernel)
        if args.cluster or args.threads:
            code.setClusterShape(args.cluster, args.threads)
        if args.wave:
            code.setWave(args.wave)
        if args.persist is not None:
            code.setPersistent(args.persist)
        Kc, Nc = code.msgSize(), code.paritySize()
        msg = ch.random_bits(frames * Kc, SEED + rank)
        llr = ch.awgn_llr(code.encode(msg), ebn0, Kc / Nc, SEED + rank, np_llr)
        d_llr = torch.from_numpy(llr).cuda()
        out = torch.empty(frames * Kc, dtype=torch.float64 if w["soft"] else torch.uint8, device="cuda")
        jobs.append({"H": H, "code": code, "K": Kc, "N": Nc, "E": code.stateSize(), "frames": frames, "msg": msg,
                     "llr": llr, "d_llr": d_llr, "out": out, "rate": "%d/%d" % (num, den), "ebn0": ebn0})
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step(j, host=False):
        src = j["h_llr"] if host else j["d_llr"]
        dst = j["h_out"] if host else j["out"]
        if w["soft"]:
            j["code"].soDecode(F.Codec.Input().parity(src), F.Codec.Output().msg(), out={"msg": dst})
        else:
            j["code"].decode(src, out=dst)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if args.profile_decodes:
        for _ in range(args.profile_decodes):
            for j in jobs:
                step(j)
        torch.cuda.synchronize()
        return 0
    for _ in range(max(args.warmup, 3)):
        for j in jobs:
            step(j)
    barrier()
    times = []
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for j in jobs:
                step(j)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
    clocks = clk.summary()
    ms = statistics.mean(times)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    info_bits = sum(j["frames"] * j["K"] for j in jobs)
    value = world * info_bits / (ms * 1e-3) / 1e6

    # per-code FER and iterations, and the algorithmic bytes of one step
    alg_bytes = 0
    per_code = []
    s_llr = np.dtype(np_llr).itemsize
    s_msg = {0: 4, 1: 2, 2: 1}[prec]
    for j in jobs:
        bits, its = j["code"].decode(j["d_llr"], iterations=True)
        bits = bits.cpu().numpy().reshape(j["frames"], j["K"])
        its = its.cpu().numpy()
        fer = float(np.mean(np.any(bits != j["msg"].reshape(j["frames"], j["K"]), axis=1)))
        alg_bytes += j["frames"] * (j["N"] * s_llr + (j["K"] * 8 if w["soft"] else j["K"])) + \
            int(its.sum()) * (2 * j["E"] * s_msg + 2 * j["N"] * 4)
        per_code.append({"n": j["N"], "rate": j["rate"], "frames": j["frames"], "ebn0_db": j["ebn0"], "fer": fer,
                         "iterations_mean": round(float(its.mean()), 2), "iterations_max": int(its.max())})
        j["bits"] = bits

    # end to end with pinned host buffers
    for j in jobs:
        j["h_llr"] = torch.from_numpy(j["llr"]).pin_memory()
        j["h_out"] = torch.empty(j["out"].shape, dtype=j["out"].dtype).pin_memory()
        step(j, host=True)
    e2e = []
    barrier()
    for _ in range(max(2, args.steps // 2)):
        t0 = time.perf_counter()
        for j in jobs:
            step(j, host=True)
        e2e.append(time.perf_counter() - t0)
    barrier()
    e2e_s = statistics.mean(e2e)
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mbit/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {0: "f32", 1: "f16", 2: "i8"}[prec], "data": "synthetic",
        "config": {"workload": w["text"], "message_storage": args.precision, "kernel": args.kernel, "codes": per_code,
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": "frame shards, replicas per GPU" if world > 1 else "single GPU"},
        "latency_ms": {"p50": round(statistics.median(times), 4),
                       "p99": round(sorted(times)[min(len(times) - 1, int(0.99 * len(times)))], 4)},
        "e2e": {"value": round(world * info_bits / e2e_s / 1e6, 2), "unit": "Mbit/s",
                "h2d_bytes_per_step": int(sum(j["llr"].nbytes for j in jobs)),
                "d2h_bytes_per_step": int(sum(j["out"].numel() * j["out"].element_size() for j in jobs))},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                     "kernel": {"auto": "lane-batched BP (check and bit kernels) per step",
                                "cluster": "cluster-resident BP (ldpc_cluster_kernel) per step",
                                "lanes": "lane-batched BP (check and bit kernels) per step"}[args.kernel],
                     "algorithmic_bytes_per_step": int(alg_bytes)},
        "gpu_launches": None,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], line["matched_hard_decisions_vs_reference"] = ldpc_cpu_reference(w, jobs)
    if embedded:
        return line
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def ldpc_cpu_reference(w, jobs, sample_frames=16):
    """The reference BP decoder (oracle/_ref, else the C restatement) on the first
    `sample_frames` frames of each code of the workload, all host threads."""
    import numpy as np
    import fecl_b200 as F
    from oracle import ref
    cores = os.cpu_count() or 1
    alg = getattr(F, w["algorithm"])
    total_bits, total_s, match = 0, 0.0, True
    kind = "reference" if ref.available() else "port"
    for j in jobs:
        n = min(sample_frames, j["frames"])
        x = np.ascontiguousarray(j["llr"][: n * j["N"]], dtype=np.float64)
        H = j["H"]
        if kind == "reference":
            rc = ref.RefCodec.ldpc(H.rows(), H.cols(), H.row_ptr, H.col_idx, alg, w["iterations"], (w["scaling"],),
                                   workgroup=cores)
            t = time.perf_counter()
            bits = rc.decode(x)
            total_s += time.perf_counter() - t
        else:
            from oracle import restated
            t = time.perf_counter()
            bits, _ = restated.ldpc_decode(H, alg, w["iterations"], w["scaling"], x, threads=cores)
            total_s += time.perf_counter() - t
        total_bits += n * j["K"]
        match = match and bool(np.array_equal(np.asarray(bits).ravel(), j["bits"][:n].ravel()))
    return ({"value": total_bits / total_s / 1e6, "unit": "Mbit/s", "cores": cores, "kind": kind,
             "sample": "first %d frames of each code, one decode each, %d threads, %.2f s wall"
                       % (sample_frames, cores, total_s)}, match)


# ---- mixed batch (--workload mixed) ---------------------------------------------------

MIXED_RATES = [(1, 2), (3, 5), (2, 3), (3, 4), (4, 5), (5, 6)]


def mixed_requests(total, seed):
    """The mixed batch of 4096 frames: 50 % LTE turbo frames with K uniform over the 188
    QPP sizes, 40 % DVB-S2 short and 10 % DVB-S2 normal LDPC frames with the rate
    uniform over MIXED_RATES; Eb/N0 uniform in 0.5-3.0 dB per frame (seeded)."""
    import numpy as np
    import fecl_b200 as F
    rng = np.random.default_rng(seed)
    sizes = F.Turbo.Lte3Gpp.sizes()
    kinds = rng.choice(3, size=total, p=[0.5, 0.4, 0.1])
    reqs = []
    for k in kinds:
        ebn0 = float(rng.uniform(0.5, 3.0))
        if k == 0:
            reqs.append(("turbo", int(sizes[rng.integers(len(sizes))]), ebn0))
        else:
            reqs.append(("ldpc", (16200 if k == 1 else 64800, MIXED_RATES[rng.integers(len(MIXED_RATES))]), ebn0))
    return reqs


class MixedCodes:
    """One codec per code of the mix: LTE turbo (max-log-MAP, 6 iterations) and DVB-S2
    LDPC (normalised min-sum 0.75, at most 50 iterations with the syndrome stop) with the
    given LDPC message precision."""

    def __init__(self, precision):
        self.precision = precision
        self.codes = {}

    def get(self, key):
        import fecl_b200 as F
        from fractions import Fraction
        if key not in self.codes:
            kind, p = key
            if kind == "turbo":
                self.codes[key] = F.Turbo.lte(p, F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(6)
                                              .scheduling(F.Serial))
            else:
                n, (a, b) = p
                H = F.Ldpc.DvbS2.matrix(n, Fraction(a, b))
                self.codes[key] = F.Ldpc(F.Ldpc.EncoderOptions(H), F.Ldpc.DecoderOptions().algorithm(F.Approximate)
                                         .iterations(50).scalingFactor(0.75).precision(self.precision))
        return self.codes[key]


def mixed_inputs(reqs, codes, seed):
    """Per request: codec key, message bits and FP16 L-values (seeded per request)."""
    import numpy as np
    from fecl_b200 import channel as ch
    out = []
    for i, (kind, p, ebn0) in enumerate(reqs):
        key = (kind, p)
        code = codes.get(key)
        msg = ch.random_bits(code.msgSize(), seed * 100003 + i)
        llr = ch.awgn_llr(code.encode(msg), ebn0, code.msgSize() / code.paritySize(), seed * 100003 + i, np.float16)
        out.append((key, msg, llr))
    return out


def build_mixed_batch(inputs, codes, autotune=True, shared_ldpc=None):
    """One F.Batch over mixed requests: one job per code, its frames' L-values
    contiguous in one device buffer, decisions and iteration counts likewise."""
    import numpy as np
    import torch
    import fecl_b200 as F
    by_key = {}
    for idx, (key, msg, llr) in enumerate(inputs):
        by_key.setdefault(key, []).append(idx)
    keys = sorted(by_key, key=str)
    llr_host = np.concatenate([inputs[i][2] for k in keys for i in by_key[k]])
    msg_ref = [np.concatenate([inputs[i][1] for i in by_key[k]]) for k in keys]
    d_llr = torch.from_numpy(llr_host).cuda()
    n_bits_out = sum(codes.get(k).msgSize() * len(by_key[k]) for k in keys)
    d_msg = torch.zeros(n_bits_out, dtype=torch.uint8, device="cuda")
    d_its = torch.zeros(len(inputs), dtype=torch.int32, device="cuda")
    jobs, lo, mo, fo = [], 0, 0, 0
    for k in keys:
        c, n = codes.get(k), len(by_key[k])
        jobs.append((c, d_llr[lo:lo + n * c.paritySize()], d_msg[mo:mo + n * c.msgSize()], d_its[fo:fo + n]))
        lo += n * c.paritySize()
        mo += n * c.msgSize()
        fo += n
    t0 = time.perf_counter()
    batch = F.Batch(jobs, autotune=autotune, shared_ldpc=shared_ldpc)
    build_s = time.perf_counter() - t0
    return {"by_key": by_key, "keys": keys, "llr_host": llr_host, "msg_ref": msg_ref, "d_llr": d_llr, "d_msg": d_msg,
            "d_its": d_its, "n_bits_out": n_bits_out, "batch": batch, "build_s": build_s}


def batch_frame_errors(mb, codes):
    """Frames of a mixed batch whose decisions differ from their message bits."""
    import numpy as np
    bits = mb["d_msg"].cpu().numpy()
    errs, mo = 0, 0
    for k, ref in zip(mb["keys"], mb["msg_ref"]):
        K, n = codes.get(k).msgSize(), len(mb["by_key"][k])
        errs += int(np.sum(np.any(bits[mo:mo + n * K].reshape(n, K) != ref.reshape(n, K), axis=1)))
        mo += n * K
    return errs


def run_mixed(args):
    import numpy as np
    import torch
    import fecl_b200 as F

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    total = args.frames or 4096
    prec = PRECISIONS[args.precision if args.precision != "f32" else "f16"]
    reqs = mixed_requests(total, SEED + rank)
    codes = MixedCodes(prec)
    inputs = mixed_inputs(reqs, codes, SEED + rank)
    mb = build_mixed_batch(inputs, codes, autotune=not args.no_autotune, shared_ldpc=args.shared_ldpc)
    by_key, keys, llr_host, msg_ref = mb["by_key"], mb["keys"], mb["llr_host"], mb["msg_ref"]
    d_llr, d_msg, d_its, n_bits_out = mb["d_llr"], mb["d_msg"], mb["d_its"], mb["n_bits_out"]
    batch, build_s = mb["batch"], mb["build_s"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if args.profile_decodes:
        for _ in range(args.profile_decodes):
            batch.run()
        torch.cuda.synchronize()
        return 0
    for _ in range(max(args.warmup, 3)):
        batch.run()
    barrier()
    times = []
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.run()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
    clocks = clk.summary()
    ms = statistics.mean(times)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    info_bits = sum(codes.get(k).msgSize() * len(by_key[k]) for k in keys)
    value = world * info_bits / (ms * 1e-3) / 1e6

    # FER per family and the algorithmic bytes of one step (iterations as run)
    bits = d_msg.cpu().numpy()
    its = d_its.cpu().numpy()
    fam = {"turbo": [0, 0], "ldpc16200": [0, 0], "ldpc64800": [0, 0]}
    alg_bytes = 0
    mo = fo = 0
    s_msg = {0: 4, 1: 2, 2: 1}[prec]
    for k, ref in zip(keys, msg_ref):
        c, n = codes.get(k), len(by_key[k])
        K = c.msgSize()
        got = bits[mo:mo + n * K].reshape(n, K)
        bad = np.any(got != ref.reshape(n, K), axis=1)
        name = "turbo" if k[0] == "turbo" else "ldpc%d" % k[1][0]
        fam[name][0] += int(bad.sum())
        fam[name][1] += n
        if k[0] == "turbo":
            alg_bytes += n * algorithmic_bytes_per_frame(K, 6, 2, 4)
        else:
            alg_bytes += n * (c.paritySize() * 2 + K) + int(its[fo:fo + n].sum()) * (2 * c.stateSize() * s_msg + 2 * c.paritySize() * 4)
        mo += n * K
        fo += n

    # end to end: pinned host L-values in, decisions out, every step
    h_llr = torch.from_numpy(llr_host).pin_memory()
    h_msg = torch.empty(n_bits_out, dtype=torch.uint8).pin_memory()
    e2e = []
    barrier()
    for _ in range(max(3, args.steps // 2)):
        t1 = time.perf_counter()
        d_llr.copy_(h_llr, non_blocking=True)
        batch.run()
        h_msg.copy_(d_msg, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        e2e.append(time.perf_counter() - t1)
    barrier()
    e2e_s = statistics.mean(e2e)

    # the plain per-request FP32 GPU decoder on a sample of the same requests: one
    # decode call per frame, FP32 messages, device-resident L-values
    plain = None
    if rank == 0 and not args.no_plain:
        sample = inputs[: min(len(inputs), args.plain_sample)]
        pcodes = MixedCodes(0)
        d_in = [torch.from_numpy(llr).cuda() for _, _, llr in sample]
        torch.cuda.synchronize()
        for (key, _, _), x in zip(sample[:8], d_in[:8]):
            pcodes.get(key).decode(x)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        outs = [pcodes.get(key).decode(x) for (key, _, _), x in zip(sample, d_in)]
        torch.cuda.synchronize()
        pt = time.perf_counter() - t1
        perr = sum(int(np.any(o.cpu().numpy() != m)) for o, (_, m, _) in zip(outs, sample))
        sbits = sum(m.size for _, m, _ in sample)
        # the batch's errors on the same requests
        berr = 0
        pos = {}
        mo = 0
        for k in keys:
            K = codes.get(k).msgSize()
            for j, i in enumerate(by_key[k]):
                pos[i] = mo + j * K
            mo += len(by_key[k]) * K
        for i, (key, m, _) in enumerate(sample):
            berr += int(np.any(bits[pos[i]:pos[i] + m.size] != m))
        plain = {"value": round(sbits / pt / 1e6, 2), "unit": "Mbit/s", "frames": len(sample), "fer": perr / len(sample),
                 "batch_fer_same_frames": berr / len(sample),
                 "what": "one decode call per frame, FP32 messages, L-values in device memory, same requests"}

    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mbit/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16", "data": "synthetic",
        "config": {"workload": "mixed batch of %d frames: 50%% LTE turbo (K uniform over the 188 QPP sizes, max-log-MAP, "
                               "6 iterations), 40%% DVB-S2 short and 10%% DVB-S2 normal LDPC (rates 1/2..5/6, "
                               "normalised min-sum 0.75, <=50 iterations), Eb/N0 U(0.5, 3.0) dB per frame, FP16 L-values, "
                               "one CUDA graph" % total,
                   "ldpc_message_storage": {0: "f32", 1: "f16", 2: "i8"}[prec], "codes": len(keys),
                   "autotune": not args.no_autotune, "shared_ldpc_launch": args.shared_ldpc,
                   "build_s": round(build_s, 3),
                   "fer": {k: (v[0] / v[1] if v[1] else None) for k, v in fam.items()},
                   "l2": "flushed between timed steps (256 MiB write)",
                   "parallelism": "frame shards, replicas per GPU" if world > 1 else "single GPU"},
        "latency_ms": {"p50": round(statistics.median(times), 4),
                       "p99": round(sorted(times)[min(len(times) - 1, int(0.99 * len(times)))], 4)},
        "e2e": {"value": round(world * info_bits / e2e_s / 1e6, 2), "unit": "Mbit/s",
                "h2d_bytes_per_step": int(llr_host.nbytes), "d2h_bytes_per_step": int(n_bits_out)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None, "peak_source": peak_kind,
                     "kernel": "mixed batch graph (turbo_lte_batch_kernel + LDPC kernels) per step",
                     "algorithmic_bytes_per_step": int(alg_bytes)},
        "plain_per_request_fp32": plain,
        "gpu_launches": None,
        "clocks": clocks,
    }
    if plain:
        line["speedup_vs_plain_per_request"] = round(value / plain["value"], 1)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---- serving (--workload serving) -----------------------------------------------------

SERVING_RATES = [1000, 5000, 20000, 50000, 100000, 200000]


def run_serving(args, embedded=False):
    """Poisson request streams at SERVING_RATES frames/s against the decode server
    (one frame per request, the mix of the mixed batch: 50 % LTE turbo, 40 % DVB-S2
    short, 10 % DVB-S2 normal, Eb/N0 U(0.5, 3.0), FP16 L-values, 40 GiB admission
    budget).  Requests cycle over a pool of distinct frames; each rate replays
    `--serve-seconds` of arrivals and waits for the last completion."""
    import numpy as np
    import torch
    import fecl_b200 as F

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1 and rank != 0:
        return 0
    pool_n = args.frames or 2048
    reqs = mixed_requests(pool_n, SEED + 7)
    codes = MixedCodes(1)
    pool = mixed_inputs(reqs, codes, SEED + 7)
    srv = F.Server(device_budget=40 << 30, max_batch_frames=args.serve_batch, slots=args.serve_slots)
    # warm-up: every code once
    seen = {}
    for key, _, llr in pool:
        if key not in seen:
            seen[key] = srv.submit(codes.get(key), llr)
    for t in seen.values():
        srv.wait(t)
    rows = []
    rng = np.random.default_rng(SEED + 11)
    peak = None
    rates = [int(r) for r in args.serve_rates.split(",")] if args.serve_rates else SERVING_RATES
    for rate in rates:
        n = max(200, int(rate * args.serve_seconds))
        arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n))
        order = rng.integers(0, len(pool), size=n)
        batch = [(codes.get(pool[i][0]), pool[i][2]) for i in order]
        srv.reset_stats()
        t0 = time.perf_counter()
        outs, lat = srv.replay(arrivals, batch)
        wall = time.perf_counter() - t0
        rep = srv.report()
        errs = sum(int(np.any(o != pool[i][1])) for o, i in zip(outs, order))
        bits = sum(pool[i][1].size for i in order)
        row = {"offered_frames_per_s": rate, "requests": n, "sustained_info_mbps": round(bits / rep["wall_s"] / 1e6, 2),
               "completed_frames_per_s": round(n / rep["wall_s"], 1), "p50_ms": round(1e3 * float(np.median(lat)), 3),
               "p99_ms": round(1e3 * float(np.quantile(lat, 0.99)), 3), "batches": rep["batches"],
               "fer": round(errs / n, 4), "replay_wall_s": round(wall, 3),
               "batch_frames_mean": round(rep["batch_frames"], 1), "batch_gpu_ms_mean": round(1e3 * rep["batch_gpu_s"], 3),
               "batch_host_ms_mean": round(1e3 * rep["batch_host_s"], 3)}
        rows.append(row)
        if peak is None or row["sustained_info_mbps"] > peak["sustained_info_mbps"]:
            peak = row
    srv.close()

    # the plain per-request FP32 GPU decoder: one decode call per frame, host L-values
    sample = pool[: min(len(pool), args.plain_sample)]
    pcodes = MixedCodes(0)
    for key, _, llr in sample[:8]:
        pcodes.get(key).decode(llr)
    t1 = time.perf_counter()
    pouts = [pcodes.get(key).decode(llr) for key, _, llr in sample]
    pt = time.perf_counter() - t1
    perr = sum(int(np.any(o != m)) for o, (_, m, _) in zip(pouts, sample))
    plain = {"value": round(sum(m.size for _, m, _ in sample) / pt / 1e6, 2), "unit": "Mbit/s", "frames": len(sample),
             "fer": round(perr / len(sample), 4), "what": "one decode call per frame, FP32 messages, host L-values"}

    # the same pool decoded as one batch with FP32 LDPC messages (not served): what
    # batching alone gives at FP32, against which the FP16 server is also compared
    mb = build_mixed_batch(pool, pcodes, autotune=False)
    mb["batch"].run()
    torch.cuda.synchronize()
    bts = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        mb["batch"].run()
        e1.record()
        e1.synchronize()
        bts.append(e0.elapsed_time(e1))
    pool_bits = sum(m.size for _, m, _ in pool)
    batched = {"value": round(pool_bits / (statistics.median(bts) * 1e-3) / 1e6, 2), "unit": "Mbit/s",
               "frames": len(pool), "fer": round(batch_frame_errors(mb, pcodes) / len(pool), 4),
               "what": "the whole pool as one batch (one CUDA graph), FP32 LDPC messages, device-resident L-values"}
    del mb
    line = {
        "metric": METRIC, "value": peak["sustained_info_mbps"], "unit": "Mbit/s", "n_gpus": 1, "steps": len(rates),
        "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f16", "data": "synthetic",
        "config": {"workload": "decode server, Poisson arrivals of single-frame requests at %s frames/s: 50%% LTE turbo "
                               "(K uniform over the 188 QPP sizes), 40%% DVB-S2 short, 10%% DVB-S2 normal LDPC (rates "
                               "1/2..5/6), Eb/N0 U(0.5, 3.0) dB, FP16 L-values and LDPC messages, 40 GiB budget"
                               % rates,
                   "pool_frames": len(pool), "slots": args.serve_slots, "max_batch_frames": args.serve_batch,
                   "seconds_per_rate": args.serve_seconds},
        "serving": rows,
        "latency_ms": {"p50": peak["p50_ms"], "p99": peak["p99_ms"], "at_offered_frames_per_s": peak["offered_frames_per_s"]},
        "e2e": {"value": peak["sustained_info_mbps"], "unit": "Mbit/s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "note": "every request goes host -> device -> host through the server"},
        "plain_per_request_fp32": plain,
        "batched_fp32": batched,
        "speedup_vs_plain_per_request": round(peak["sustained_info_mbps"] / plain["value"], 1),
        "gpu_launches": None,
    }
    if embedded:
        return line
    print(json.dumps(line))
    return 0


SWEEP_SHIFTS = (0.1, 0.25)


def run_fer_sweep(args):
    """FER sweep of the DVB-S2 normal-frame decoder (fecl_b200/fer.py): rates 1/2, 3/4,
    9/10, 512 frames per point, Eb/N0 1.0-4.0 dB in 0.25 dB steps, normalised min-sum
    0.75, <= 50 iterations, FP32 / FP16 / int8 message storage, against the FP64
    reference decoder's frame failures on the same L-values (tests/golden/
    fer_sweep_oracle.json).  Each reduced-precision decoder also runs 0.1 and 0.25 dB
    above every point on the same noise draws, so "loses at most 0.1 dB" is a
    pointwise comparison (loss_check_points_over lists the points where it does not
    hold).  One GPU: under torchrun only rank 0 runs the sweep."""
    import numpy as np
    import torch
    from fecl_b200 import fer

    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    with open(os.path.join(ROOT, "tests", "golden", "fer_sweep_oracle.json")) as f:
        oracle = json.load(f)
    precs = (("f32", 0), ("f16", 1), ("i8", 2))
    stream = torch.cuda.current_stream()
    ms = {p: 0.0 for p, _ in precs}
    info_bits = 0
    report, thresholds, losses, f32_equal, llr_err = {}, {}, {}, {}, {}
    with ClockSampler(local) as clk:
        for r, (num, den) in enumerate(fer.RATES):
            name = "%d/%d" % (num, den)
            codes = {p: fer.code(r, q) for p, q in precs}
            K = codes["f32"].msgSize()
            o_fer = oracle["rates"][name]["fer"]
            curves = {p: [] for p, _ in precs}
            curves.update({"%s_shift%g" % (pn, d): [] for pn in ("f16", "i8") for d in SWEEP_SHIFTS})
            diff = []
            mid = min(range(len(o_fer)), key=lambda i: abs(o_fer[i] - 0.5))
            for p in range(len(fer.EBN0_DB)):
                msg = fer.sweep_msg(K, r, p)
                cw = codes["f32"].encode(msg)
                d_llr = torch.from_numpy(fer.sweep_llr(cw, K, r, p)).cuda()
                out = torch.empty(fer.FRAMES * K, dtype=torch.uint8, device="cuda")
                for pn, _ in precs:
                    codes[pn].decode(d_llr, out=out)  # warm-up of this shape
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    codes[pn].decode(d_llr, out=out)
                    e1.record(stream)
                    e1.synchronize()
                    ms[pn] += e0.elapsed_time(e1)
                    fails = fer.frame_fails(out.cpu().numpy(), msg, fer.FRAMES)
                    curves[pn].append(float(fails.mean()))
                    if pn == "f32":
                        ofails = fer.unpack_fails(oracle["rates"][name]["fails"][p], fer.FRAMES)
                        diff.append(int(np.sum(fails != ofails)))
                if p == mid:
                    # a-posteriori message L-values of the reduced precisions against FP32
                    import fecl_b200 as F
                    so = {pn: codes[pn].soDecode(F.Codec.Input().parity(d_llr), F.Codec.Output(np.float32).msg()).msg()
                          for pn, _ in precs}
                    ref = so["f32"].double()
                    llr_err[name] = {"ebn0_db": fer.EBN0_DB[p]}
                    for pn in ("f16", "i8"):
                        d = so[pn].double() - ref
                        llr_err[name][pn] = {
                            "rel_rms": round(float(d.pow(2).mean().sqrt() / ref.pow(2).mean().sqrt()), 5),
                            "sign_agree": round(float(((so[pn] >= 0) == (so["f32"] >= 0)).double().mean()), 6)}
                for d in SWEEP_SHIFTS:
                    s_llr = torch.from_numpy(fer.sweep_llr(cw, K, r, p, shift_db=d)).cuda()
                    for pn in ("f16", "i8"):
                        codes[pn].decode(s_llr, out=out)
                        curves["%s_shift%g" % (pn, d)].append(
                            float(fer.frame_fails(out.cpu().numpy(), msg, fer.FRAMES).mean()))
                info_bits += fer.FRAMES * K
            report[name] = {"oracle": o_fer, **{k: v for k, v in curves.items()}}
            f32_equal[name] = {"frames_differing_per_point": diff}
            thresholds[name] = {
                "fer_%g" % t: {k: (None if (x := fer.threshold_db(fer.EBN0_DB, c, t)) is None else round(x, 3))
                               for k, c in (("oracle", o_fer), ("f32", curves["f32"]), ("f16", curves["f16"]),
                                            ("i8", curves["i8"]))}
                for t in (0.1, 0.01)}
            losses[name] = {"%s_shift%g" % (pn, d): fer.loss_check(curves["%s_shift%g" % (pn, d)], o_fer)
                            for pn in ("f16", "i8") for d in SWEEP_SHIFTS}
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": round(info_bits / (ms["f16"] * 1e-3) / 1e6, 2), "unit": "Mbit/s", "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": round(ms["f16"], 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16", "data": "synthetic",
        "config": {"workload": "FER sweep: DVB-S2 normal n=64800 r=1/2, 3/4, 9/10 x 512 frames per point, Eb/N0 "
                               "1.0-4.0 dB in 0.25 dB steps, normalised min-sum 0.75, <=50 iterations with syndrome "
                               "stop, FP32 L-values; FP32/FP16/int8 messages against the FP64 reference decoder",
                   "l2": "inputs 133 MB per point (larger than L2)", "parallelism": "single GPU"},
        "mbps_by_precision": {p: round(info_bits / (ms[p] * 1e-3) / 1e6, 2) for p, _ in precs},
        "ebn0_db": list(fer.EBN0_DB), "fer": report, "f32_vs_oracle": f32_equal,
        "threshold_db": thresholds, "shifts_db": list(SWEEP_SHIFTS),
        "loss_check_points_over": losses, "llr_error_vs_f32": llr_err,
        "gpu_launches": None, "clocks": clocks,
    }
    print(json.dumps(line))
    return 0


def extra_workloads(args):
    """The other configurations of the metric, measured in the default run so that
    every one of them is on record: DVB-S2 short-frame Exact BP (64 frames, FP64
    L-values, soft output), DVB-S2 normal frames with FP16 messages (3 x 512 frames,
    normalised min-sum) and the decode server under Poisson load, each bounded to a
    few seconds of GPU time."""
    import argparse
    out = {}
    base = dict(vars(args))
    base.update(frames=0, kernel="auto", cluster=0, threads=0, wave=0, profile_decodes=0, warmup=3)
    l1 = run_ldpc(argparse.Namespace(**dict(base, workload="ldpc-short", precision="f32", steps=10)), embedded=True)
    l3 = run_ldpc(argparse.Namespace(**dict(base, workload="ldpc-normal", precision="f16", steps=5,
                                            no_cpu_baseline=True)), embedded=True)
    keep = ("value", "unit", "ms_per_step", "dtype", "config", "e2e", "roofline", "latency_ms", "clocks",
            "cpu_baseline", "matched_hard_decisions_vs_reference")
    out["ldpc"] = {"short_exact_f64_x64": {k: l1[k] for k in keep if k in l1},
                   "normal_nms_f16_3x512": {k: l3[k] for k in keep if k in l3}}
    sv = run_serving(argparse.Namespace(**dict(base, serve_seconds=0.25, serve_slots=3, serve_batch=2048,
                                               plain_sample=256)), embedded=True)
    out["serving"] = {k: sv[k] for k in ("value", "unit", "config", "serving", "latency_ms", "plain_per_request_fp32",
                                         "batched_fp32", "speedup_vs_plain_per_request") if k in sv}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="lte-turbo", choices=["lte-turbo", "mixed", "serving", "fer-sweep"] + sorted(LDPC_WORKLOADS),
                    help="lte-turbo is the headline workload; the LDPC workloads print the same line for BP")
    ap.add_argument("--frames", type=int, default=0,
                    help="LDPC workloads: frames per code instead of the workload's (small cases for ncu)")
    ap.add_argument("--precision", default="f32", choices=sorted(PRECISIONS),
                    help="LDPC message storage (f32 is the reference-parity mode)")
    ap.add_argument("--kernel", default="auto", choices=["auto", "cluster", "lanes"],
                    help="LDPC workloads: decoder kernel (auto: the lane-batched one where it applies)")
    ap.add_argument("--cluster", type=int, default=0, help="LDPC: CTAs per frame of the cluster kernel (0: built-in)")
    ap.add_argument("--threads", type=int, default=0, help="LDPC: threads per CTA of the cluster kernel (0: built-in)")
    ap.add_argument("--wave", type=int, default=0, help="LDPC: frame groups of 32 decoded together (0: built-in)")
    ap.add_argument("--persist", type=int, default=None, choices=[-1, 0, 1],
                    help="LDPC: one persistent launch for small batches (1), built-in choice (0), never (-1)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="mixed: build the batch without autotuning")
    ap.add_argument("--no-plain", action="store_true", help="mixed: skip the per-request FP32 comparison")
    ap.add_argument("--shared-ldpc", default=None, choices=["passes", "persistent"],
                    help="mixed: the FP16 LDPC jobs share their launches (per pass, or one persistent launch per class)")
    ap.add_argument("--plain-sample", type=int, default=256, help="mixed: requests decoded one by one for the comparison")
    ap.add_argument("--serve-seconds", type=float, default=0.25, help="serving: seconds of arrivals per rate")
    ap.add_argument("--serve-slots", type=int, default=3, help="serving: batches in flight")
    ap.add_argument("--serve-batch", type=int, default=2048, help="serving: frames per batch at most")
    ap.add_argument("--serve-rates", default="", help="serving: comma-separated offered rates (default: all)")
    ap.add_argument("--no-extras", action="store_true",
                    help="lte-turbo: skip the LDPC and serving figures added to the default line")
    ap.add_argument("--profile-decodes", type=int, default=0,
                    help="only run this many decodes of the workload (for ncu captures) and exit")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload in LDPC_WORKLOADS:
        return run_ldpc(args)
    if args.workload == "mixed":
        return run_mixed(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "fer-sweep":
        return run_fer_sweep(args)

    import numpy as np
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import fecl_b200 as F
    dec = F.Turbo.DecoderOptions().algorithm(F.Approximate).iterations(ITERATIONS).scheduling(F.Serial)
    code = F.Turbo.lte(K, dec)
    msg, llr = make_inputs(code, FRAMES, SEED + rank)
    d_llr = torch.from_numpy(llr).cuda()
    d_bits = torch.empty(FRAMES * K, dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    if args.profile_decodes:
        for _ in range(args.profile_decodes):
            code.decode(d_llr, out=d_bits)
        torch.cuda.synchronize()
        return 0

    for _ in range(max(args.warmup, 3)):
        code.decode(d_llr, out=d_bits)
    barrier()

    # ---- device-resident timing
    times = []
    with ClockSampler(local) as clk:
        barrier()
        for _ in range(args.steps):
            flush.fill_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            code.decode(d_llr, out=d_bits)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        barrier()
    clocks = clk.summary()
    bits = d_bits.cpu().numpy()
    fer = float(np.mean(np.any(bits.reshape(FRAMES, K) != msg.reshape(FRAMES, K), axis=1)))
    ms = statistics.mean(times)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * FRAMES * K / (ms * 1e-3) / 1e6

    # ---- end to end through the public call with pinned host buffers
    h_llr = torch.from_numpy(llr).pin_memory()
    h_bits = torch.empty(FRAMES * K, dtype=torch.uint8).pin_memory()
    code.decode(h_llr, out=h_bits)
    e2e_times = []
    barrier()
    for _ in range(max(2, args.steps // 2)):
        t0 = time.perf_counter()
        code.decode(h_llr, out=h_bits)
        e2e_times.append(time.perf_counter() - t0)
    barrier()
    e2e_s = statistics.mean(e2e_times)
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * FRAMES * K / e2e_s / 1e6

    peak, peak_kind = measured_peaks()
    alg = algorithmic_bytes_per_frame() * FRAMES
    achieved = alg / (ms * 1e-3) / 1e9
    traffic = profiled_traffic()
    per_decode = kernels_per_decode(lambda: code.decode(d_llr, out=d_bits))

    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "Mbit/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(world),
        "fer": fer, "latency_ms": {"p50": round(statistics.median(times), 4),
                                   "p99": round(sorted(times)[min(len(times) - 1, int(0.99 * len(times)))], 4)},
        "e2e": {"value": round(e2e_value, 2), "unit": "Mbit/s", "h2d_bytes_per_step": int(llr.nbytes),
                "d2h_bytes_per_step": int(FRAMES * K)},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic, "peak_source": peak_kind,
                     "kernel": "turbo_lte_kernel (+ input staging) per decode",
                     "algorithmic_bytes_per_decode": alg},
        "gpu_launches": per_decode * args.steps if per_decode else None,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, ref_bits = cpu_reference(FRAMES, llr, {"parity": code.paritySize()})
        line["cpu_baseline"] = cb
        if ref_bits is not None:
            line["parity_vs_reference"] = hard_parity(bits, ref_bits, msg, K)
    if world == 1 and not args.no_extras:
        line.update(extra_workloads(args))
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
