#!/usr/bin/env python3
"""Benchmark of the lsCOMP uint16 codec on B200 (one JSON line on rank 0).

Workload: the CSSI-like stack, 600 x 1813 x 1558 uint16 (3.39 GB, z fastest,
seeded synthetic data).  One step = compress + decompress in the lossless
mode (-b 1 1 1 1 -p 1) and compress + decompress lossy (-b 3 5 10 15 -p 0.5):
four passes over the stack.

    value  = 4 * input bytes per step / device time of the step (GB/s, 1e9),
             inputs resident in HBM, CUDA events on the launching stream;
    e2e    = the same metric through the C ABI's host-memory calls: every
             pass takes its input from pinned host memory and leaves its
             result there;
    roofline  = the dominant kernel's algorithmic bytes per launch / its mean
             launch time, against the measured HBM copy bandwidth of this
             pool's B200s;
    cpu_baseline = the C/OpenMP oracle on a bounded frame sample, all cores.

--impl reference times the reference's own CUDA build (oracle/_ref) through
its host API on the same stack and steps (e2e: the same host-buffer path as
this library's e2e); --impl reference --ref-cpu times the path on the host
cores instead (the reference has no CPU implementation, so the C/OpenMP
oracle, all threads, a bounded frame sample per step).  --gpus N (torchrun) runs N independent
replicas, one per GPU: the codec does not shard, so there is no data-path
collective; the step time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "sc25-lscomp_b200"))

DIMS = (600, 1813, 1558)
MODES = [("lossless", (1, 1, 1, 1), 1.0), ("lossy", (3, 5, 10, 15), 0.5)]
SEED = 2
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 2**20
KIND_NAMES = {"cssi": "CSSI-like", "xpcs": "XPCS-like", "small": "small (Poisson background, spots, hot pixels)"}
# the benchmark set's other plain stacks, measured beside the headline one
# (each mode: one compress and one decompress per repetition)
PER_CONFIG = [("xpcs", (512, 1024, 1024)), ("small", (64, 256, 256))]


def l2_note(nbytes):
    if nbytes > L2_BYTES:
        return f"inputs ({nbytes / 1e9:.2f} GB) larger than L2 (126 MB); no flush needed"
    return f"inputs ({nbytes / 1e6:.1f} MB) fit in L2 (126 MB): a 256 MB buffer is written between timed passes"


def data_note(kind):
    return f"synthetic (seeded {KIND_NAMES[kind]} generator)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dims", type=str, default=None, help="x,y,z (default: the CSSI-like stack)")
    ap.add_argument("--kind", default="cssi", choices=["cssi", "xpcs", "small"])
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-per-config", action="store_true",
                    help="skip the XPCS-like and small stacks measured beside the default CSSI-like one")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--serve", type=str, default="",
                    help="serving benchmark: Poisson arrivals at this many requests per second, or a comma-separated "
                         "sweep of rates (its own JSON line)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="duration of each rate of the serving run")
    ap.add_argument("--serve-max-mb", type=int, default=512, help="largest request of the serving benchmark")
    ap.add_argument("--serve-pinned", action="store_true",
                    help="serving benchmark: client buffers in page-locked host memory (copied by the device "
                         "directly) instead of pageable numpy arrays (staged by the server's copy threads)")
    ap.add_argument("--serve-arena-gb", type=int, default=120,
                    help="device arena of the serving benchmark's server (its admission cap)")
    ap.add_argument("--batch-frames", type=int, default=64, help="largest frame count of a batch stack")
    ap.add_argument("--ref-build", choices=["sm_100a", "default"], default=None,
                    help="with --impl reference: time this one build of the reference (default: each in a process of "
                         "its own, the faster reported)")
    ap.add_argument("--ref-cpu", action="store_true",
                    help="with --impl reference: the oracle on the host cores instead of the reference's CUDA build")
    ap.add_argument("--ref-step-seconds", type=float, default=1.5,
                    help="with --impl reference: CPU time of one step's sample")
    ap.add_argument("--batch", type=int, default=0,
                    help="batched-stacks benchmark over this many stacks (its own JSON line)")
    return ap.parse_args()


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples while the timed region runs: NVML
    polled in-process every few milliseconds (the device matched by PCI bus
    id), or nvidia-smi when NVML is unavailable."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event (throttle) reason bits
    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap"}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []
        self.stop_flag = False
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            h = None
            try:
                pr = torch.cuda.get_device_properties(gpu_index)
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(gpu_index)
            self.nvml, self.h = pynvml, h
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nvml = None

    def start(self):
        if self.nvml is not None:
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv = self.nvml
        while not self.stop_flag:
            try:
                clk = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                try:
                    why = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    why = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((float(clk), int(why)))
            except Exception:
                pass
            time.sleep(0.005)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag = True
            self.t.join(timeout=2)
            reasons = set()
            for _, why in self.samples:
                for bit, name in self.REASONS.items():
                    if why & bit:
                        reasons.add(name)
            sm = [c for c, _ in self.samples]
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def make_stack(kind, dims):
    import lscomp

    return getattr(lscomp, f"synth_{kind}")(dims, seed=SEED if kind == "cssi" else 1)


def cpu_baseline(kind, dims, budget_s):
    """Oracle (C/OpenMP port of the reference algorithm) on the first frames
    of the same stack, all host threads, lossless + lossy compress/decompress."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import lscomp
    from oracle import Oracle

    orc = Oracle()
    threads = orc.max_threads()
    x, y, z = dims

    def run(nf):
        d = (nf, y, z)
        a = getattr(lscomp, f"synth_{kind}")(dims, seed=SEED if kind == "cssi" else 1, frames=(0, nf))
        t0 = time.perf_counter()
        for _, bins, p in MODES:
            s, _ = orc.compress(a, d, bins, p, threads=threads)
            orc.decompress(s, d, bins, p, threads=threads)
        return time.perf_counter() - t0, a.size * 2

    nf = 2
    t, nbytes = run(nf)
    target = max(1, min(x, int(nf * budget_s / max(t, 1e-3))))
    if target > nf:
        nf = target
        t, nbytes = run(nf)
    return {"value": round(4 * nbytes / t / 1e9, 4), "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"first {nf} of {x} frames ({nbytes / 1e9:.3f} GB), lossless+lossy compress+decompress, "
                      f"{t:.1f} s"}


def dist_init(n, backend=None):
    """One process per GPU under torchrun: NCCL for the barrier and the
    max-over-ranks timing (gloo when no GPU is visible, as in the CPU tests
    of this plumbing).  A short process-group timeout ends a rank that waits
    for a dead peer with an error."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


BATCH_SETTINGS = [((1, 1, 1, 1), 1.0), ((3, 5, 10, 15), None), ((5, 10, 15, 20), None)]
BATCH_P = (0.3, 0.5, 0.8)


def batch_workload(n, max_frames, seed=11):
    """Seeded batch description: per stack dims (frames U{1..max_frames},
    frame height and width U{100..2048}, non-multiples of 8 included), data
    kind (CSSI-like or XPCS-like, alternating) and settings (bins from
    {lossless, 3 5 10 15, 5 10 15 20}; lossy stacks take p from
    {0.3, 0.5, 0.8}, lossless stacks p = 1)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        dims = (int(rng.integers(1, max_frames + 1)), int(rng.integers(100, 2049)), int(rng.integers(100, 2049)))
        kind = "cssi" if i % 2 == 0 else "xpcs"
        bins, p = BATCH_SETTINGS[int(rng.integers(0, len(BATCH_SETTINGS)))]
        if p is None:
            p = BATCH_P[int(rng.integers(0, len(BATCH_P)))]
        out.append({"dims": dims, "kind": kind, "bins": bins, "p": p, "seed": seed + i})
    return out


POOL_FRAMES = 64   # frames per kind in the device frame pools of the batch benchmark
POOL_SIDE = 2048  # their height and width (the largest a batch stack has)


def batch_pools(lscomp, dev, frames, seed=11):
    """Seeded CSSI-like and XPCS-like frames (at least POOL_FRAMES, and at
    least a stack's largest frame count, of POOL_SIDE^2 each) made by the
    host generators and kept on the device; batch stacks are cut from them
    (batch_assemble)."""
    import torch

    dims = (max(POOL_FRAMES, frames), POOL_SIDE, POOL_SIDE)
    return {k: torch.from_numpy(getattr(lscomp, f"synth_{k}")(dims, seed=seed + i).view(np.int16)).to(dev).view(dims)
            for i, k in enumerate(("cssi", "xpcs"))}


def batch_assemble(pools, d, dst):
    """Stack d (frames F, height H, width W) into dst: F consecutive pool
    frames of its kind (so the XPCS-like frames keep their frame-to-frame
    correlation), each cut to its central H x W window."""
    f, h, w = d["dims"]
    o = d["seed"] % (pools[d["kind"]].shape[0] - f + 1)
    y0, x0 = (POOL_SIDE - h) // 2, (POOL_SIDE - w) // 2
    dst.view(f, h, w).copy_(pools[d["kind"]][o:o + f, y0:y0 + h, x0:x0 + w])


def bench_batch(args, local):
    """Batched compress of many uneven stacks, each with its own bins and
    pooling threshold: one lscomp_compress_batch_ex_u16 call, and the same
    captured once as a CUDA graph (lscomp_plan_*), against one plain call
    per stack and one plain call per frame (and, for --impl reference, the
    reference's host API called per stack); then batch decompression of all
    streams against one plain call per stack.  Inputs resident in HBM.

    Stacks are cut on the device from frame pools (batch_pools), and every
    output buffer has the exact size of its stream (lscomp_stream_sizes_batch,
    a pass that writes nothing), so the configuration's 2000 stacks of up to
    64 frames fit one GPU; if they do not fit the free device memory, the
    largest leading subset that does is run, and the line says so.  The
    decodes are written over the inputs once compression is measured."""
    import torch

    import lscomp

    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    ws = lscomp.Workspace(local)
    desc = batch_workload(args.batch, args.batch_frames)
    t_setup = time.perf_counter()
    pools = batch_pools(lscomp, dev, args.batch_frames)

    def n_el(d):
        return d["dims"][0] * d["dims"][1] * d["dims"][2]

    def al16(nbytes):
        return (nbytes + 15) // 16 * 16

    # exact stream sizes, stack by stack through a bounded scratch buffer
    exact = [0] * len(desc)
    scratch_el = 4 << 30
    buf = torch.empty(scratch_el, dtype=torch.int16, device=dev)
    i = 0
    while i < len(desc):
        items, off = [], 0
        while i < len(desc) and off + al16(2 * n_el(desc[i])) // 2 <= scratch_el:
            d = desc[i]
            sl = buf[off:off + n_el(d)]
            batch_assemble(pools, d, sl)
            items.append((sl, d["dims"], None, d["bins"], d["p"]))
            off += al16(2 * n_el(d)) // 2
            i += 1
        for k, v in enumerate(lscomp.stream_sizes_batch(ws, items)):
            exact[i - len(items) + k] = v
    del buf, items
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # the largest leading subset whose inputs and exact outputs fit
    free, _ = torch.cuda.mem_get_info(dev)
    frame_scratch = max(lscomp.max_stream_bytes((1, d["dims"][1], d["dims"][2])) for d in desc)
    budget = free - (6 << 30) - frame_scratch - 2 * max(al16(lscomp.max_stream_bytes(d["dims"])) for d in desc)
    n, used = 0, 0
    while n < len(desc) and used + al16(2 * n_el(desc[n])) + al16(exact[n]) <= budget:
        used += al16(2 * n_el(desc[n])) + al16(exact[n])
        n += 1
    desc = desc[:n]
    frames = sum(d["dims"][0] for d in desc)
    nel = [n_el(d) for d in desc]
    nbytes = 2 * sum(nel)
    offs_in, offs_out, n_in, n_out = [], [], 0, 0
    for d, ne, ex in zip(desc, nel, exact):
        offs_in.append(n_in)
        n_in += al16(2 * ne) // 2
        offs_out.append(n_out)
        n_out += al16(ex)
    d_in_all = torch.empty(n_in, dtype=torch.int16, device=dev)
    d_out_all = torch.zeros(n_out, dtype=torch.uint8, device=dev)
    items = []
    for d, ne, oi, oo, ex in zip(desc, nel, offs_in, offs_out, exact):
        d_in = d_in_all[oi:oi + ne]
        batch_assemble(pools, d, d_in)
        items.append((d_in, d["dims"], d_out_all[oo:oo + ex], d["bins"], d["p"]))
    del pools
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    config = {"workload": f"{len(desc)} stacks, frames U{{1..{args.batch_frames}}}, frame height and width "
                          f"U{{100..2048}} uint16, CSSI-like and XPCS-like alternating; per stack bins from "
                          f"{{lossless, 3 5 10 15, 5 10 15 20}} and p from {{0.3, 0.5, 0.8}} (lossless: p 1)",
              "stacks": len(desc), "stacks_asked": args.batch, "frames": frames, "input_bytes": nbytes,
              "stream_bytes": int(sum(exact[:n])),
              "data": f"stacks cut on the device from {POOL_FRAMES} seeded frames per kind "
                      f"({POOL_SIDE}x{POOL_SIDE}, host generators): consecutive frames, central window",
              "output_buffers": "exact stream sizes from lscomp_stream_sizes_batch_u16",
              "setup_s": round(t_setup, 1)}
    if n < args.batch:
        config["subset"] = (f"the first {n} of {args.batch} stacks: their inputs and exact outputs fill the "
                            "free device memory")

    def timed(fn, reps, name=None):
        # name: an NVTX range around the timed calls (not the warm-up), so a
        # profiler can select exactly those launches (ncu --nvtx-include)
        for _ in range(max(args.warmup, 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts = []
        if name:
            torch.cuda.nvtx.range_push(name)
        for _ in range(reps):
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        if name:
            torch.cuda.nvtx.range_pop()
        return float(np.median(ts))

    def fps(ms):
        return round(frames / ms * 1e3, 1)

    if args.impl == "reference":
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        from oracle import RefLib

        ref = RefLib()

        def loop_ref():
            for d_in, dims, d_out, bins, p in items:
                ref.compress(d_in.data_ptr(), d_out.data_ptr(), dims, bins, p, stream=stream.cuda_stream)

        ms = timed(loop_ref, args.steps)
        print(json.dumps({"metric": "batched compress frames per second (reference host API, one call per stack)",
                          "value": fps(ms), "unit": "frames/s", "impl": "reference", "higher_is_better": True,
                          "per_stack_calls_ms": round(ms, 3), "config": config}))
        return

    t0 = time.perf_counter()
    lscomp.stream_sizes_batch(ws, items)
    t_sizes = (time.perf_counter() - t0) * 1e3
    got = lscomp.compress_batch_mixed(ws, items)
    assert [sl for sl, _ in got] == exact[:n], "size pass differs from the written streams"
    step = max(1, len(items) // 24)
    chk = torch.empty(max(lscomp.max_stream_bytes(it[1]) for it in items[::step]), dtype=torch.uint8, device=dev)
    for it, (sl, rs) in zip(items[::step], got[::step]):
        d_in, dims, d_out, bins, p = it
        assert lscomp.compress_into(ws, d_in, dims, bins, p, chk) == (sl, rs)
        assert torch.equal(chk[:sl], d_out[:sl]), "batch stream differs from the single-stack stream"
    t_batch = timed(lambda: lscomp.compress_batch_mixed(ws, items), args.steps)
    plan = lscomp.Plan(ws, items)
    assert plan.run() == got, "graph plan sizes differ from the batch call"
    t_plan = timed(plan.run, args.steps, "graph_plan")
    plan.close()

    def loop_stack():
        for d_in, dims, d_out, bins, p in items:
            lscomp.compress_into(ws, d_in, dims, bins, p, d_out)

    t_stack = timed(loop_stack, args.steps)
    # one plain call per frame, each frame a stack of its own; every frame
    # writes the same scratch stream buffer (only the time is kept)
    scratch = torch.empty(frame_scratch, dtype=torch.uint8, device=dev)

    def loop_frame():
        for d_in, dims, d_out, bins, p in items:
            fsz = dims[1] * dims[2]
            for f in range(dims[0]):
                lscomp.compress_into(ws, d_in[f * fsz:(f + 1) * fsz], (1, dims[1], dims[2]), bins, p, scratch)

    t_frame = timed(loop_frame, max(1, args.steps // 2))
    del scratch
    # decode every stream: first the sampled stacks into a scratch buffer,
    # checked (lossless: the input; lossy: the single-stack decode), then
    # all of them over the inputs (no longer needed), one batch call against
    # one plain call per stack
    dchk = torch.empty(max(it[0].numel() for it in items[::step]), dtype=torch.int16, device=dev)
    for (d_in, dims, d_out, bins, p), (sl, _) in zip(items[::step], got[::step]):
        ne = d_in.numel()
        lscomp.decompress_batch(ws, [(d_out, sl, dims, dchk[:ne], bins, p)])
        if bins == (1, 1, 1, 1):
            assert torch.equal(dchk[:ne], d_in), "batch decode differs from the input (lossless)"
        one = torch.empty_like(d_in)
        lscomp.decompress_into(ws, d_out, sl, dims, bins, p, one)
        assert torch.equal(dchk[:ne], one), "batch decode differs from the single-stack decode"
    del dchk
    ditems = [(d_out, sl, dims, d_in, bins, p) for (d_in, dims, d_out, bins, p), (sl, _) in zip(items, got)]
    t_dbatch = timed(lambda: lscomp.decompress_batch(ws, ditems), args.steps, "batch_decompress")

    def loop_dstack():
        for d_s, sl, dims, d_o, bins, p in ditems:
            lscomp.decompress_into(ws, d_s, sl, dims, bins, p, d_o)

    t_dstack = timed(loop_dstack, args.steps)
    res = {"batch_call_ms": round(t_batch, 3), "graph_plan_ms": round(t_plan, 3),
           "size_pass_ms": round(t_sizes, 3),
           "decompress_batch_call_ms": round(t_dbatch, 3), "decompress_per_stack_calls_ms": round(t_dstack, 3),
           "decompress_frames_per_s": {"batch_call": fps(t_dbatch), "per_stack_calls": fps(t_dstack)},
           "decompress_output_gbs_batch_call": round(nbytes / t_dbatch / 1e6, 1),
           "per_stack_calls_ms": round(t_stack, 3), "per_frame_calls_ms": round(t_frame, 3),
           "frames_per_s": {"graph_plan": fps(t_plan), "batch_call": fps(t_batch), "per_stack_calls": fps(t_stack),
                            "per_frame_calls": fps(t_frame)},
           "input_gbs_graph_plan": round(nbytes / t_plan / 1e6, 1),
           "speedup_graph_plan_vs_per_frame": round(t_frame / t_plan, 2),
           "speedup_graph_plan_vs_per_stack": round(t_stack / t_plan, 2)}
    print(json.dumps({"metric": "batched compress frames per second (one graph replay of the mixed-settings "
                                "batch launch)",
                      "value": fps(t_plan), "unit": "frames/s", "higher_is_better": True, "results": res,
                      "config": config, "tuned": tuned_summary(lscomp, ("batch",)),
                      "timing": f"CUDA events around each call, median of {args.steps}; sizes read back to the "
                                "host inside every batch call, graph replay and plain call"}))


def tuned_summary(lscomp, kinds=("compress", "batch", "decompress")):
    """The tuner's choices so far: key -> chosen shape/tile size and the
    candidates' measured ms per call."""
    shapes = {-1: "rule", 0: "2x8", 1: "2x7", 2: "2x13", 3: "2x8n"}
    out = []
    for e in lscomp.tune_table():
        if e["kind"] not in kinds:
            continue
        out.append({"kind": e["kind"], "es": e["es"], "layout": e["layout"], "pool": e["pool"], "bzb": e["bzb"],
                    "chosen": f"{shapes[e['shape']]}/{e['tile_blocks']}",
                    "ms": {f"{shapes[t['shape']]}/{t['tile_blocks']}": t["ms"] for t in e["times"]}})
    return out


def bench_serve(args, local):
    """Serving loop under Poisson arrivals: requests of log-uniform size
    (256 KB .. --serve-max-mb of 1024x1024 or 1813x1558 uint16 frames), 70%
    compress / 30% decompress, 60% lossless / 40% lossy (-b 3 5 10 15
    -p 0.5), host buffers in and out.  Latency = queue + service time per
    request.  --serve-pinned puts every client buffer in page-locked host
    memory, which the server copies directly; otherwise the buffers are
    pageable and go through its staging."""
    import torch

    import lscomp

    def client(a):
        # a client buffer equal to a: pageable numpy, or a numpy view of a
        # page-locked tensor (which it keeps alive)
        if not args.serve_pinned:
            return a
        v = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype).reshape(a.shape)
        v[...] = a
        return v

    rng = np.random.default_rng(5)
    pool = []
    max_bytes = int(args.serve_max_mb) << 20
    for i in range(32):
        size = float(np.exp(rng.uniform(np.log(256 << 10), np.log(max_bytes))))
        h, w = (1024, 1024) if i % 2 else (1813, 1558)
        frames = max(1, int(round(size / (2 * h * w))))
        if size < 2 * h * w:
            h = max(8, int(size / (2 * w)))
        dims = (frames, h, w)
        kind = "xpcs" if i % 2 else "cssi"
        pool.append((dims, client(getattr(lscomp, f"synth_{kind}")(dims, seed=100 + i).reshape(dims))))
    modes = [("lossless", (1, 1, 1, 1), 1.0), ("lossy", (3, 5, 10, 15), 0.5)]
    arena = int(args.serve_arena_gb) << 30
    srv = lscomp.Server(local, arena_bytes=arena)
    # containers of every pool stack in both modes, for the decompress requests
    conts = {}
    for k, (dims, a) in enumerate(pool):
        for name, bins, p in modes:
            o = np.zeros(64 + lscomp.max_stream_bytes(dims), dtype=np.uint8)
            r = srv.wait(srv.submit_compress(a, dims, bins, p, o))
            conts[(k, name)] = client(o[: r["out_len"]].copy())
    import queue as qmod

    # one output buffer per pool stack and direction, written before use, so
    # the run measures the server and not page faults on fresh client memory
    # (requests for the same stack may share one: their bytes are not checked)
    outs = {k: (client(np.ones(64 + lscomp.max_stream_bytes(dims), dtype=np.uint8)), client(np.ones_like(a)))
            for k, (dims, a) in enumerate(pool)}

    def run_rate(rate, dur):
        pending = qmod.Queue()
        lat, nbytes_done, failed = [], [0], []

        def waiter():
            while True:
                item = pending.get()
                if item is None:
                    return
                rid, nb = item
                r = srv.wait(rid)
                if r["status"] != 0:
                    failed.append(r)
                lat.append((r["queued_ns"] + r["service_ns"]) / 1e6)
                nbytes_done[0] += nb

        st0 = srv.stats()
        wt = threading.Thread(target=waiter)
        wt.start()
        t0 = time.perf_counter()
        t_next = t0
        n_sub = 0
        while True:
            t_next += float(rng.exponential(1.0 / rate))
            if t_next - t0 > dur:
                break
            while time.perf_counter() < t_next:
                pass
            k = int(rng.integers(0, len(pool)))
            dims, a = pool[k]
            name, bins, p = modes[0] if rng.random() < 0.6 else modes[1]
            if rng.random() < 0.7:
                rid = srv.submit_compress(a, dims, bins, p, outs[k][0])
            else:
                rid = srv.submit_decompress(conts[(k, name)], outs[k][1])
            pending.put((rid, a.nbytes))
            n_sub += 1
        pending.put(None)
        wt.join()
        elapsed = time.perf_counter() - t0
        if failed:
            raise SystemExit(f"request failed: {failed[0]}")
        st = srv.stats()
        lat_a = np.array(lat)
        return {"offered_req_per_s": rate, "achieved_req_per_s": round(n_sub / elapsed, 1), "requests": n_sub,
                "p50_ms": round(float(np.percentile(lat_a, 50)), 3),
                "p99_ms": round(float(np.percentile(lat_a, 99)), 3), "mean_ms": round(float(lat_a.mean()), 3),
                "input_gb_per_s": round(nbytes_done[0] / elapsed / 1e9, 2),
                "launch_rounds": st["rounds"] - st0["rounds"], "batches": st["batches"] - st0["batches"],
                "batched_requests": st["batched_requests"] - st0["batched_requests"]}

    rates = [float(v) for v in str(args.serve).split(",")]
    sweep = [run_rate(r, args.serve_seconds) for r in rates]
    srv.close()
    head = sweep[0]
    print(json.dumps({"metric": "serving latency p99 (Poisson arrivals, host buffers in and out)",
                      "value": head["p99_ms"], "unit": "ms", "higher_is_better": False, **head,
                      "sweep": sweep if len(sweep) > 1 else None,
                      "config": {"workload": f"32 seeded stacks, log-uniform 256 KB..{args.serve_max_mb} MB, "
                                             "1024x1024 (XPCS-like) or 1813x1558 (CSSI-like) uint16 frames; 70/30 "
                                             "compress/decompress; 60/40 lossless/lossy", "arena_bytes": arena,
                                 "duration_s_per_rate": args.serve_seconds,
                                 "client_buffers": "page-locked (direct copies)" if args.serve_pinned
                                 else "pageable (staged through the server's pinned slots)",
                                 "copy_threads_per_direction": int(os.environ.get("LSCOMP_SERVER_COPY_THREADS", 8))}}))


def main():
    args = parse()
    dims = tuple(int(v) for v in args.dims.split(",")) if args.dims else DIMS
    rank, world, local = dist_init(args.gpus)
    import torch

    if args.impl == "reference" and not (args.ref_cpu or args.ref_build or args.batch or args.serve):
        # each reference build in a process of its own; rank 0 reports
        if rank == 0:
            print(json.dumps(reference_builds(args)), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()
        return

    if args.batch:
        torch.cuda.set_device(local)
        if rank == 0:
            bench_batch(args, local)
        return
    if args.serve:
        torch.cuda.set_device(local)
        if rank == 0:
            bench_serve(args, local)
        return

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nbytes = dims[0] * dims[1] * dims[2] * 2
    hbm, peak_kind = peaks()
    stream = torch.cuda.current_stream()
    h = make_stack(args.kind, dims)
    d_in = torch.from_numpy(h.view(np.int16)).to(dev)
    cap = (lambda nb: (nb + 3) // 4 * 4 + 128 * nb)(dims[0] * ((dims[1] + 7) // 8) * ((dims[2] + 7) // 8))
    d_cmp = torch.zeros(cap, dtype=torch.uint8, device=dev)
    d_dec = torch.empty_like(d_in)
    config = {"workload": f"{KIND_NAMES[args.kind]} stack {dims[0]}x{dims[1]}x{dims[2]} uint16, z fastest",
              "modes": "lossless -b 1 1 1 1 -p 1; lossy -b 3 5 10 15 -p 0.5",
              "step": "compress+decompress in both modes (4 passes)",
              "input_bytes": nbytes, "l2": l2_note(nbytes),
              "parallelism": f"replicas{world}"}

    if args.impl == "reference":
        return bench_reference(args, dims, rank, world, dev, d_in, d_cmp, d_dec, nbytes, config, h)

    import lscomp

    ws = lscomp.Workspace(local)
    sizes = {}

    def step(ev=None):
        for i, (name, bins, p) in enumerate(MODES):
            if ev is not None:
                ev[4 * i].record(stream)
            lscomp.compress_async(ws, d_in, dims, bins, p, d_cmp)
            if ev is not None:
                ev[4 * i + 1].record(stream)
            lscomp.decompress_async(ws, d_cmp, sizes[name], dims, bins, p, d_dec)
            if ev is not None:
                ev[4 * i + 2].record(stream)

    # exact stream lengths and a correctness check before timing; the
    # device streams and decodes are kept on the host for the e2e check
    expect = {}
    for name, bins, p in MODES:
        sl, rs = lscomp.compress_into(ws, d_in, dims, bins, p, d_cmp)
        sizes[name] = sl
        sizes[name + "_ref_size"] = rs
        lscomp.decompress_into(ws, d_cmp, sl, dims, bins, p, d_dec)
        if name == "lossless" and not torch.equal(d_dec, d_in):
            raise SystemExit("lossless round trip failed")
        if args.e2e_steps > 0:
            expect[name] = (d_cmp[:sl].cpu(), d_dec.cpu())
    for _ in range(max(args.warmup, 3)):
        step()
    ws.check()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(8)] for _ in range(args.steps)]
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    launches0 = lscomp.launch_count()
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    e_start.record(stream)
    for k in range(args.steps):
        step(evs[k])
    e_end.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    launches = lscomp.launch_count() - launches0
    ws.check()
    total_ms = max_over_ranks(e_start.elapsed_time(e_end), world)
    ms_step = total_ms / args.steps
    per = {}
    for i, (name, bins, p) in enumerate(MODES):
        tc = float(np.mean([e[4 * i].elapsed_time(e[4 * i + 1]) for e in evs]))
        td = float(np.mean([e[4 * i + 1].elapsed_time(e[4 * i + 2]) for e in evs]))
        sl = sizes[name]
        per[name] = {"compress_gbs": round(nbytes / tc / 1e6, 1), "decompress_gbs": round(nbytes / td / 1e6, 1),
                     "compress_mib_per_ms": round(nbytes / 2**20 / tc, 1),
                     "decompress_mib_per_ms": round(nbytes / 2**20 / td, 1),
                     "compress_ms": round(tc, 4), "decompress_ms": round(td, 4), "stream_bytes": sl,
                     "ratio": round(nbytes / sizes[name + "_ref_size"], 4),
                     "compress_hbm_frac": round((nbytes + sl) / tc / 1e6 / hbm, 4),
                     "decompress_hbm_frac": round((nbytes + sl) / td / 1e6 / hbm, 4)}
    # dominant kernel: largest time share in the step
    shares = []
    for name, _, _ in MODES:
        shares.append((per[name]["compress_ms"], f"enc_kernel ({name})", nbytes + sizes[name]))
        shares.append((per[name]["decompress_ms"], f"dec_kernel ({name})", nbytes + sizes[name]))
    shares.sort(reverse=True)
    t_dom, k_dom, b_dom = shares[0]
    achieved = b_dom / t_dom / 1e6
    roofline = {"bound": "hbm", "kernel": k_dom, "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_kind": peak_kind,
                "traffic": None, "algorithmic_bytes_per_launch": b_dom}
    prof = os.path.join(ROOT, "profiles", "traffic.json")  # measured on the default stack only
    if os.path.exists(prof) and args.dims is None and args.kind == "cssi":
        try:
            tr = json.load(open(prof)).get(k_dom)
            if tr:
                roofline["traffic"] = tr
        except Exception:
            pass
    value = world * 4 * nbytes / (ms_step / 1e3) / 1e9

    e2e = bench_e2e(args, dims, ws, h, dev, nbytes, sizes, world, expect) if args.e2e_steps > 0 else None
    del expect
    per_config = None
    if not args.no_per_config and args.dims is None and args.kind == "cssi":
        del d_cmp, d_dec
        per_config = bench_per_config(args, lambda kind, pdims: codec_ours(ws, lscomp, pdims), local)
    out = {"metric": "lsCOMP compress+decompress throughput (lossless and lossy b=3 5 10 15 p=0.5), "
                     "uncompressed GB per second",
           "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
           "warmup": max(args.warmup, 3), "ms_per_step": round(ms_step, 4), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": data_note(args.kind),
           "config": config, "per_mode": per, "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches),
           "clocks": clk, "tuned": tuned_summary(lscomp)}
    if per_config is not None:
        out["per_config"] = per_config
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args.kind, dims, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def bench_e2e(args, dims, ws, h, dev, nbytes, sizes, world, expect):
    """Host buffers in, host buffers out, through the C ABI's host-memory
    calls (lscomp_compress_host_u16 / lscomp_decompress_host_u16): per mode
    the stack in pinned host memory is compressed into a host stream buffer,
    and that stream decompressed into a host stack buffer; every byte crosses
    PCIe inside the timed region (the calls pipeline chunks of frames so
    copies up, kernels and copies down overlap).  Before timing, one pass per
    mode is checked: its stream must equal the device-memory call's byte for
    byte (expect[mode][0]) and its decode the device decode (expect[mode][1],
    equal to the input for the lossless mode)."""
    import torch

    import lscomp

    h_in = torch.from_numpy(h.view(np.int16)).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    cap = max(sizes[m[0]] for m in MODES)
    h_cmp = torch.empty(cap, dtype=torch.uint8).pin_memory()
    stream = torch.cuda.current_stream()
    moved = {"h2d": 0, "d2h": 0}

    def step():
        moved["h2d"] = moved["d2h"] = 0
        for name, bins, p in MODES:
            sl, _ = lscomp.compress_host(ws, h_in, dims, bins, p, h_cmp)
            lscomp.decompress_host(ws, h_cmp, sl, dims, bins, p, h_out)
            moved["h2d"] += nbytes + sl  # the stack up, then the stream up
            moved["d2h"] += sl + nbytes  # the stream down, then the stack down
        torch.cuda.synchronize()

    for name, bins, p in MODES:
        sl, _ = lscomp.compress_host(ws, h_in, dims, bins, p, h_cmp)
        want_s, want_d = expect[name]
        if sl != want_s.numel() or not torch.equal(h_cmp[:sl], want_s):
            raise SystemExit(f"e2e ({name}): host-memory stream differs from the device-memory stream")
        h_out.fill_(-1)
        lscomp.decompress_host(ws, h_cmp, sl, dims, bins, p, h_out)
        if not torch.equal(h_out, want_d):
            raise SystemExit(f"e2e ({name}): host-memory decode differs from the device decode")
        if name == "lossless" and not torch.equal(h_out, h_in):
            raise SystemExit("e2e round trip failed (lossless decode differs from the input)")
    step()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.e2e_steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world) / args.e2e_steps
    # the link this box gives: one plain copy of the pinned stack each way;
    # the floor a pass can reach is its larger direction at these rates
    d_tmp = torch.empty_like(h_in, device=dev)
    rates = {}
    for way, (dst, src) in (("h2d", (d_tmp, h_in)), ("d2h", (h_out, d_tmp))):
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        e0.record(stream)
        dst.copy_(src, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        rates[way] = nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9
    del d_tmp
    floor = sum(max(nbytes / rates["h2d"], sizes[m[0]] / rates["d2h"]) +
                max(sizes[m[0]] / rates["h2d"], nbytes / rates["d2h"]) for m in MODES) / 1e6
    return {"value": round(world * 4 * nbytes / (ms / 1e3) / 1e9, 2), "unit": "GB/s",
            "h2d_bytes_per_step": int(moved["h2d"]), "d2h_bytes_per_step": int(moved["d2h"]),
            "ms_per_step": round(ms, 3), "checked": "streams and decodes equal the device-memory calls' (both modes)",
            "path": "lscomp_compress_host_u16 / lscomp_decompress_host_u16 (C ABI), pinned host buffers",
            "pcie_copy_gbs": {k: round(v, 1) for k, v in rates.items()},
            "pcie_floor_ms_per_step": round(floor, 3)}


def codec_ours(ws, lscomp, dims):
    """(compress, decompress) callables of this library for bench_per_config."""

    def comp(d_in, bins, p, d_cmp):
        lscomp.compress_async(ws, d_in, dims, bins, p, d_cmp)

    def decomp(d_cmp, sl, bins, p, d_dec):
        lscomp.decompress_async(ws, d_cmp, sl, dims, bins, p, d_dec)

    def sizes(d_in, bins, p, d_cmp):
        return lscomp.compress_into(ws, d_in, dims, bins, p, d_cmp)

    return comp, decomp, sizes


def codec_ref(ref, dims):
    """(compress, decompress) callables of the reference's host API."""

    def comp(d_in, bins, p, d_cmp):
        ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p)

    def decomp(d_cmp, sl, bins, p, d_dec):
        ref.decompress(d_dec.data_ptr(), d_cmp.data_ptr(), sl, dims, bins, p)

    def sizes(d_in, bins, p, d_cmp):
        d_cmp.zero_()
        rs = ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p)
        return rs, rs

    return comp, decomp, sizes


def bench_per_config(args, make_codec, local, reps=6):
    """The other plain stacks of the benchmark set (XPCS-like 512x1024x1024,
    small 64x256x256): per mode the median device time of one compress and
    one decompress (CUDA events around each call, inputs resident in HBM),
    GB/s of input and the fraction of the measured HBM copy bandwidth the
    algorithmic bytes reach.  A stack that fits in L2 gets a 256 MB buffer
    written before every timed call."""
    import torch

    hbm, _ = peaks()
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 2**20, dtype=torch.uint8, device=dev)
    res = {}
    for kind, dims in PER_CONFIG:
        nbytes = 2 * dims[0] * dims[1] * dims[2]
        d_in = torch.from_numpy(make_stack(kind, dims).view(np.int16)).to(dev)
        nb = dims[0] * ((dims[1] + 7) // 8) * ((dims[2] + 7) // 8)
        d_cmp = torch.zeros((nb + 3) // 4 * 4 + 128 * nb, dtype=torch.uint8, device=dev)
        d_dec = torch.empty_like(d_in)
        comp, decomp, sizes = make_codec(kind, dims)
        small = nbytes <= L2_BYTES
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def timed(fn):
            for _ in range(3):
                fn()
            ts = []
            for _ in range(reps):
                if small:
                    flush.fill_(1)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            return float(np.median(ts))

        per = {}
        for name, bins, p in MODES:
            sl, rs = sizes(d_in, bins, p, d_cmp)
            tc = timed(lambda: comp(d_in, bins, p, d_cmp))
            td = timed(lambda: decomp(d_cmp, sl, bins, p, d_dec))
            per[name] = {"compress_ms": round(tc, 4), "decompress_ms": round(td, 4),
                         "compress_gbs": round(nbytes / tc / 1e6, 1), "decompress_gbs": round(nbytes / td / 1e6, 1),
                         "compress_hbm_frac": round((nbytes + sl) / tc / 1e6 / hbm, 4),
                         "decompress_hbm_frac": round((nbytes + sl) / td / 1e6 / hbm, 4),
                         "stream_bytes": int(sl), "ratio": round(nbytes / rs, 4)}
        res[f"{KIND_NAMES[kind].split(' ')[0]} {dims[0]}x{dims[1]}x{dims[2]}"] = {
            "modes": per, "input_bytes": nbytes, "l2": l2_note(nbytes), "data": data_note(kind)}
        del d_in, d_cmp, d_dec
    return res


def bench_reference(args, dims, rank, world, dev, d_in, d_cmp, d_dec, nbytes, config, h):
    """The reference arm.  Default: the reference's own CUDA build (sm_100a)
    through its host API (cuLSZ_compression_uint16_bsize64 /
    cuLSZ_decompression_uint16_bsize64) on the same stack and steps: value
    with the stack resident in HBM, timed like the reference CLI times it
    (the whole host call); e2e through host buffers with every pass's input
    and output copied across PCIe, as the reference CLI moves them and as
    this library's e2e does.  --ref-cpu: the path on the host cores -- the
    reference has no CPU implementation of the codec, so the oracle (the same
    algorithm in C/OpenMP, streams byte-identical to the reference build's)
    with every host thread, each step one pass over a bounded sample of the
    stack's first frames."""
    import torch

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    if world > 1 and rank != 0:
        # the reference arm runs on rank 0 only
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
        return
    if args.ref_cpu:
        out = bench_reference_cpu(args, dims, config)
    else:
        out = bench_reference_gpu(args, dims, dev, d_in, d_cmp, d_dec, nbytes, config, h)
    print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def bench_reference_cpu(args, dims, config):
    import lscomp
    from oracle import Oracle

    orc = Oracle()
    threads = orc.max_threads()
    x, y, z = dims

    def sample(nf):
        return getattr(lscomp, f"synth_{args.kind}")(dims, seed=SEED if args.kind == "cssi" else 1, frames=(0, nf))

    def step(a, nf):
        d = (nf, y, z)
        t0 = time.perf_counter()
        for _, bins, p in MODES:
            s, _ = orc.compress(a, d, bins, p, threads=threads)
            orc.decompress(s, d, bins, p, threads=threads)
        return time.perf_counter() - t0

    # size the sample so one step takes about args.ref_step_seconds
    nf = 2
    t = step(sample(nf), nf)
    nf = max(1, min(x, int(nf * args.ref_step_seconds / max(t, 1e-3))))
    a = sample(nf)
    for _ in range(max(args.warmup, 3)):
        step(a, nf)
    ts = [step(a, nf) for _ in range(args.steps)]
    sec = float(np.mean(ts))
    sbytes = a.size * 2
    value = 4 * sbytes / sec / 1e9
    smp = (f"first {nf} of {x} frames ({sbytes / 1e9:.3f} GB) of the same {KIND_NAMES[args.kind]} stack per step, "
           "lossless + "
           f"lossy compress + decompress, {sec:.2f} s per step")
    return {"impl": "reference",
            "metric": "lsCOMP compress+decompress throughput (lossless and lossy b=3 5 10 15 p=0.5), "
                      "uncompressed GB per second",
            "value": round(value, 3), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(sec * 1e3, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": data_note(args.kind),
            "config": config,
            "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                             "sample": smp + "; the reference has no CPU implementation, so the oracle (its "
                                             "algorithm restated in C/OpenMP, byte-identical streams) runs"},
            "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_builds(args):
    """Both builds of the reference's CUDA sources, each timed in a process of
    its own (one reference library per process: two in one process measured
    the second one several times slower): nvcc -O3 for sm_100a, and nvcc's
    default target as the reference's own CMake builds it (PTX compiled by
    the driver on B200).  Returns the line of the faster build, with both
    builds' step times."""
    lines = {}
    for b in ("sm_100a", "default"):
        cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference", "--ref-build", b, "--steps",
               str(args.steps), "--warmup", str(args.warmup), "--e2e-steps", str(args.e2e_steps), "--kind", args.kind]
        if args.dims:
            cmd += ["--dims", args.dims]
        if args.no_per_config:
            cmd.append("--no-per-config")
        env = {k: v for k, v in os.environ.items()
               if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "LOCAL_WORLD_SIZE", "GROUP_RANK", "MASTER_ADDR",
                            "MASTER_PORT", "TORCHELASTIC_RUN_ID")}
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        for ln in reversed(r.stdout.splitlines()):
            if ln.startswith("{"):
                d = json.loads(ln)
                if "unavailable" not in d:
                    lines[b] = d
                break
    if not lines:
        return {"impl": "reference", "unavailable": "reference build missing or failed (oracle/_ref)"}
    best = min(lines, key=lambda b: lines[b]["ms_per_step"])
    out = lines[best]
    out["ms_per_step_by_build"] = {b: d["ms_per_step"] for b, d in lines.items()}
    return out


def bench_reference_gpu(args, dims, dev, d_in, d_cmp, d_dec, nbytes, config, h):
    """One build of the reference's CUDA sources (--ref-build: sm_100a, or
    the default-target PTX build) through its host API on the same stack and
    steps: value with the stack resident in HBM, e2e through host buffers,
    and the other plain stacks (per_config)."""
    import torch

    try:
        from oracle import REF_LIB, REF_LIB_DEFAULT, RefLib

        label = "sm_100a" if args.ref_build == "sm_100a" else "default arch (PTX JIT)"
        ref = RefLib(REF_LIB if args.ref_build == "sm_100a" else REF_LIB_DEFAULT)
    except Exception as e:  # the reference build is not present
        return {"impl": "reference", "unavailable": f"reference build missing: {e}"}
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def run(ref, steps, clocks=None):
        sizes = {}
        for name, bins, p in MODES:
            d_cmp.zero_()
            sizes[name] = ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p)
            torch.cuda.synchronize()

        def step(ev=None):
            for i, (name, bins, p) in enumerate(MODES):
                if ev is not None:
                    ev[3 * i].record(stream)
                ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p)
                if ev is not None:
                    ev[3 * i + 1].record(stream)
                ref.decompress(d_dec.data_ptr(), d_cmp.data_ptr(), sizes[name], dims, bins, p)
                if ev is not None:
                    ev[3 * i + 2].record(stream)

        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(6)] for _ in range(steps)]
        if clocks:
            clocks.start()
        e0.record(stream)
        for k in range(steps):
            step(evs[k])
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks else None
        # per pass, each call's own interval (the reference's calls
        # allocate, clear, free and read back inside it)
        per = {}
        for i, (name, _, _) in enumerate(MODES):
            per[name] = {"compress_ms": round(float(np.mean([e[3 * i].elapsed_time(e[3 * i + 1]) for e in evs])), 4),
                         "decompress_ms": round(float(np.mean([e[3 * i + 1].elapsed_time(e[3 * i + 2])
                                                               for e in evs])), 4)}
        return e0.elapsed_time(e1) / steps, sizes, clk, per

    ms, sizes, clk, per_mode = run(ref, args.steps, ClockSampler(torch.cuda.current_device()))
    value = 4 * nbytes / (ms / 1e3) / 1e9
    e2e = None
    if args.e2e_steps > 0:
        # host buffers in and out, as the reference CLI moves them: stack to
        # the device, compress, stream back; stream to the device,
        # decompress, stack back (pinned host memory, like this library's e2e)
        h_in = torch.from_numpy(h.view(np.int16)).pin_memory()
        h_out = torch.empty_like(h_in).pin_memory()
        h_cmp = torch.empty(max(sizes.values()), dtype=torch.uint8).pin_memory()
        moved = {"h2d": 0, "d2h": 0}

        def step_e2e():
            moved["h2d"] = moved["d2h"] = 0
            for name, bins, p in MODES:
                d_in.copy_(h_in, non_blocking=True)
                sl = ref.compress(d_in.data_ptr(), d_cmp.data_ptr(), dims, bins, p)
                h_cmp[:sl].copy_(d_cmp[:sl], non_blocking=True)
                d_cmp[:sl].copy_(h_cmp[:sl], non_blocking=True)
                ref.decompress(d_dec.data_ptr(), d_cmp.data_ptr(), sl, dims, bins, p)
                h_out.copy_(d_dec, non_blocking=True)
                moved["h2d"] += nbytes + sl
                moved["d2h"] += sl + nbytes
            torch.cuda.synchronize()

        step_e2e()
        e0.record(stream)
        for _ in range(args.e2e_steps):
            step_e2e()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1) / args.e2e_steps
        e2e = {"value": round(4 * nbytes / (ems / 1e3) / 1e9, 2), "unit": "GB/s",
               "h2d_bytes_per_step": int(moved["h2d"]), "d2h_bytes_per_step": int(moved["d2h"]),
               "ms_per_step": round(ems, 3),
               "path": "reference host API (cuLSZ_*_bsize64) with pinned host buffers copied in and out"}
    per_config = None
    if not args.no_per_config and args.dims is None and args.kind == "cssi":
        per_config = bench_per_config(args, lambda kind, pdims: codec_ref(ref, pdims), torch.cuda.current_device())
    return {"impl": "reference",
            "metric": "lsCOMP compress+decompress throughput (lossless and lossy b=3 5 10 15 p=0.5), "
                      "uncompressed GB per second",
            "value": round(value, 2), "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u16", "data": data_note(args.kind),
            "config": config, "clocks": clk, "build": label,
            "cpu_baseline": {"value": round(value, 2), "unit": "GB/s", "cores": 1, "kind": "reference",
                             "sample": f"the reference's CUDA sources ({label} build; without --ref-build the faster "
                                       "of its two builds is reported) through its host API on the full stack; "
                                       "the reference has no CPU "
                                       "implementation (bench.py --impl reference --ref-cpu times the C/OpenMP "
                                       "oracle on the host cores)"},
            "e2e": e2e, "per_mode": per_mode, "per_config": per_config}


if __name__ == "__main__":
    main()
