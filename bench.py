"""Benchmark of the TAN time-varying convolution path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 64 channels, block 512 at 48 kHz, IR 65536 samples (128 partitions),
every channel's IR replaced every 32 blocks through UpdateResponseTD with a
one-block linear crossfade; input uniform[-1, 1] noise; IRs Gaussian noise x
exp decay with RT60 ~ U[0.2, 1.5] s, unit L2 norm (seeded synthetic data; 8
pre-generated IR sets are cycled). One step = one audio block of every channel.

ours (default):
  value  GSamples/s with inputs and IRs resident in HBM (device-pointer Process
         and UpdateResponseTD), device time from CUDA events on the object's
         stream, L2 flushed before every timed step (a 256 MiB write, then
         reads of two other 256 MiB buffers, so that no dirty line of the
         flush is written back inside the step).
  e2e    the same metric through the host C ABI (tanb_convolution_process with
         host float* rows, H2D + D2H inside), wall clock per step including the
         tail kernel; p50/p99/p99.9 of the per-block latency (Process return).
reference: the oracle's C++ restatement of TAN's CPU path on all host cores.
Under torchrun each rank runs its own 64-channel replica (weak scaling, no
data-path collective); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "max real-time channels (p99 block latency < 5.33 ms) & GSamples/s vs plain FP32"
FS = 48000
C, B, L, SWAP_EVERY, N_IR_SETS = 64, 512, 65536, 32, 8
SEED = 20261203 + 1
L2_FLUSH_BYTES = 256 << 20
PROFILE_STEPS = 512  # steps of the per-kernel (roofline) pass
REF_WARM_BLOCKS = 64  # untimed blocks before the reference arm's timed steps
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=32)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--cpu-sample-s", type=float, default=10.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-capacity", action="store_true")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the sub-records of the other configurations (uneven batch, non-uniform, serving)")
    return p.parse_args()


def swap_index(k, warmup):
    """IR set loaded before step k, or None: the first IR before step 0, then a
    swap every SWAP_EVERY steps counted from the first timed step (warmup), so
    that every timed window of SWAP_EVERY or more steps contains swaps."""
    if k == 0:
        return 0
    if k >= warmup and (k - warmup) % SWAP_EVERY == 0:
        return 1 + (k - warmup) // SWAP_EVERY
    return None


def swaps_timed(steps):
    return (steps + SWAP_EVERY - 1) // SWAP_EVERY


def config_dict(P):
    return {
        "workload": "time-varying FP32 convolution: 64 ch, block 512 @ 48 kHz, IR 65536 (128 partitions), "
                    "IR swap every 32 blocks with 1-block crossfade",
        "channels": C, "block": B, "ir_length": L, "partitions": P, "swap_every_blocks": SWAP_EVERY,
        "swap_schedule": "IR swaps at timed steps 0, 32, 64, ... (the first IR before warm-up step 0)",
        "sample_rate": FS, "deadline_ms": 1000.0 * B / FS, "ir_sets_cycled": N_IR_SETS,
    }


def exp_decay_ir(g, n, rt60_s, fs=FS):
    """Gaussian noise times exp(-ln(1000) t / (RT60 fs)), unit L2 norm (float32)."""
    t = np.arange(n, dtype=np.float64)
    h = g.standard_normal(n) * np.exp(-np.log(1000.0) * t / (rt60_s * fs))
    h /= np.linalg.norm(h)
    return h.astype(np.float32)


def make_inputs(nblocks, seed=SEED):
    g = np.random.Generator(np.random.PCG64(seed))
    x = g.uniform(-1.0, 1.0, (C, nblocks * B)).astype(np.float32)
    irs = [np.stack([exp_decay_ir(g, L, float(g.uniform(0.2, 1.5))) for _ in range(C)])
           for _ in range(N_IR_SETS)]
    return x, irs


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    MIN_WINDOW_S = 1.0

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.t0 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "50",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # the timed region is short: start it once sampling is running
            t_end = time.time() + 3.0
            while not self.lines and time.time() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def keep_busy(self, step):
        """Runs step() (more of the timed workload, untimed) until the sampling
        window has lasted MIN_WINDOW_S: nvidia-smi samples every 50 ms, and a
        timed region of a few ms alone would see none."""
        n = 0
        while time.time() - self.t0 < self.MIN_WINDOW_S:
            step(n)
            n += 1
        return n

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
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [t.strip() for t in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm), "window": "timed steps, then the same workload continued to >= 1 s"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def max_over_ranks(pg, value, local):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(pg, value, local):
    if pg is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def cpu_baseline(sample_s, threads=None):
    """Oracle restatement of TAN's CPU path on the host cores, bounded sample."""
    from oracle import ref

    threads = threads or os.cpu_count()
    nb_max = 100000  # the time bound (--cpu-sample-s) ends the sample first
    x, irs = make_inputs(0)
    g = np.random.Generator(np.random.PCG64(SEED + 7))
    xb = g.uniform(-1.0, 1.0, (C, 64 * B)).astype(np.float32)
    conv = ref.RefConvolution(L, B, C, threads=threads)
    y = np.zeros((C, B), np.float32)
    done_blocks = 0
    t0 = time.perf_counter()
    while done_blocks < nb_max:
        if done_blocks % SWAP_EVERY == 0:
            conv.update_response_td(irs[(done_blocks // SWAP_EVERY) % N_IR_SETS])
        j = done_blocks % 64
        conv.process(np.ascontiguousarray(xb[:, j * B:(j + 1) * B]), None, y)
        done_blocks += 1
        if time.perf_counter() - t0 > sample_s:
            break
    dt = time.perf_counter() - t0
    conv.close()
    return {"value": C * B * done_blocks / dt / 1e9, "unit": "GSamples/s", "cores": threads, "kind": "port",
            "sample": f"{done_blocks} blocks of the workload (64 ch x 512) incl. IR swaps every 32 blocks, "
                      f"{dt:.1f} s wall", "ms_per_block": 1000.0 * dt / done_blocks}


def cpu_pipeline_chain(S=32, B=256, L=48000, blocks=100):
    """The sample pipeline's chain (int16 -> convolution -> mix per ear ->
    int16, bench_workloads.py pipeline) on the oracle restatement, per block,
    on all host cores: the CPU baseline of the fused GPU call."""
    from oracle import ref

    import bench_workloads as bw

    C = 2 * S
    src, h, group, rows_in = bw.pipeline_inputs(S, B, L, blocks)
    threads = os.cpu_count()
    conv = ref.RefConvolution(L, B, C, threads=threads)
    conv.update_response_td(h)
    lat = []
    for k in range(blocks):
        t0 = time.perf_counter()
        x = np.stack([ref.convert_s16_f32(r[2 * k * B:], 1.0, in_step=2, n=B) for r in rows_in])
        y = np.zeros_like(x)
        conv.process(x, None, y)
        for ear in range(2):
            ref.convert_f32_s16(ref.mix(y[ear::2]), 1.0)
        lat.append(1e3 * (time.perf_counter() - t0))
    conv.close()
    lat = np.asarray(lat[5:])
    return {"what": "the sample pipeline's chain on the restatement (32 int16 stereo sources, 64 channels, "
                    "1 s IRs, B = 256), per block", "cores": threads,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "gsamples_per_s": float(C * B / (lat.mean() / 1e3) / 1e9)}


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref

    ref.build()
    threads = os.cpu_count()
    x, irs = make_inputs(64)
    conv = ref.RefConvolution(L, B, C, threads=threads)
    y = np.zeros((C, B), np.float32)
    xs_blocks = [np.ascontiguousarray(x[:, j * B:(j + 1) * B]) for j in range(64)]
    # Warm-up: the OpenMP pool, first touch of every buffer and one untimed IR
    # swap, so that the timed blocks are steady-state blocks (at least
    # REF_WARM_BLOCKS of them, whatever --warmup says).
    nwarm = max(args.warmup, REF_WARM_BLOCKS)
    for k in range(nwarm):
        if k in (0, nwarm // 2):
            conv.update_response_td(irs[(k // 7) % N_IR_SETS])
        conv.process(xs_blocks[k % 64], None, y)
    times = []
    for t in range(args.steps):
        k = args.warmup + t
        si = swap_index(k, args.warmup)
        t0 = time.perf_counter()
        if si is not None:
            conv.update_response_td(irs[si % N_IR_SETS])
        conv.process(xs_blocks[k % 64], None, y)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = C * B * args.steps / total / 1e9
    lat = np.array(times) * 1e3
    swap_step = np.array([swap_index(args.warmup + t, args.warmup) is not None for t in range(args.steps)])
    P = conv.partitions
    line = {
        "metric": METRIC, "value": value, "unit": "GSamples/s", "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_dict(P),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "p999": float(np.percentile(lat, 99.9))},
        "latency_ms_without_swap_blocks": {"p50": float(np.percentile(lat[~swap_step], 50)),
                                           "p99": float(np.percentile(lat[~swap_step], 99))},
        "swap_block_ms_mean": float(lat[swap_step].mean()),
        "swaps_timed": swaps_timed(args.steps), "warmup_blocks": nwarm,
        "cpu_baseline": {"value": value, "unit": "GSamples/s", "cores": threads, "kind": "port",
                         "sample": f"{args.steps} timed blocks (64 ch x 512) incl. IR swaps every 32 blocks "
                                   f"({swaps_timed(args.steps)} timed) after {nwarm} warm-up blocks; "
                                   "oracle C++ restatement of TAN's CPU uniform-partitioned path "
                                   "(the reference needs OpenCL headers and FFTW 3.3.5, absent here)"},
        "e2e": {"value": value, "unit": "GSamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def read_traffic(name="tail_kernel_64ch_b512_ir65536.txt"):
    """dram bytes per launch of the dominant kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for ln in open(path):
        if ln.startswith("dram_bytes_per_launch_full:"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def size_floor(torch, stream, flush_l2, nbytes, dev, reps=50):
    """What one bandwidth-bound launch over `nbytes` reaches when timed like the
    partition MAC (L2 flushed before each launch, CUDA events around it on the
    same stream, median of `reps`): the library's own streaming read
    (tanb_stream_read, 16-byte loads) at its best of a few grid shapes, and a
    torch reduction over the same bytes beside it."""
    from tan_b200 import convolution as cv

    lib = cv.lib()
    nbytes = nbytes // 16 * 16
    # 4x the bytes: the same read at 1x, 2x and 4x its size gives the line below
    buf = torch.ones(4 * nbytes // 4, dtype=torch.float32, device=f"cuda:{dev}")
    acc = torch.zeros(1, dtype=torch.float32, device=f"cuda:{dev}")
    out = torch.empty((), dtype=torch.float32, device=f"cuda:{dev}")

    def timed(fn):
        ms = []
        with torch.cuda.stream(stream):
            for r in range(reps + 3):
                flush_l2()
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fn()
                b.record(stream)
                b.synchronize()
                if r >= 3:
                    ms.append(a.elapsed_time(b))
        return 1e3 * statistics.median(ms)

    def own(cps, thr):
        rc = lib.tanb_stream_read(buf.data_ptr(), nbytes, acc.data_ptr(), cps, thr, stream.cuda_stream)
        assert rc == 0, cv.last_error()

    shapes = ((1, 1024), (2, 1024), (2, 512), (4, 512), (4, 256), (8, 256))
    grids = {f"{cps} CTAs/SM x {thr}": timed(lambda: own(cps, thr)) for cps, thr in shapes}
    best = min(grids, key=grids.get)
    cps, thr = shapes[list(grids).index(best)]
    head = buf[:nbytes // 4]
    torch_us = timed(lambda: torch.sum(head, 0, out=out))
    us = grids[best]
    # the same launch over 16 bytes and over 1x, 2x and 4x the bytes: a line
    # through the sizes separates the fixed cost of one launch timed this way
    # from the rate at which its bytes stream
    empty_us = timed(lambda: lib.tanb_stream_read(buf.data_ptr(), 16, acc.data_ptr(), cps, thr, stream.cuda_stream))
    sizes = [nbytes, 2 * nbytes, 4 * nbytes]
    ts = []
    for nb in sizes:
        ts.append(timed(lambda: lib.tanb_stream_read(buf.data_ptr(), nb, acc.data_ptr(), cps, thr,
                                                     stream.cuda_stream)))
    slope, fixed = np.polyfit(np.array(sizes, float), np.array(ts), 1)
    del buf, head
    return {"bytes": nbytes, "us": us, "gbs": nbytes / (us * 1e-6) / 1e9, "grid": best,
            "what": "tanb_stream_read (the library's 16-byte streaming read) over the same bytes, best grid, "
                    "one launch, L2 flushed, CUDA events (median)",
            "grids_us": grids, "torch_sum_us": torch_us, "torch_sum_gbs": nbytes / (torch_us * 1e-6) / 1e9,
            "empty_launch_us": empty_us,
            "fit": {"sizes": sizes, "us": ts, "fixed_us": float(fixed), "marginal_gbs": float(1e-3 / slope),
                    "what": "least-squares line through the streaming read of 1x, 2x and 4x the bytes"}}


def marginal(nbytes, us, floor, peak):
    """The launch's bytes over its time less the fixed cost of one launch timed
    the same way (the streaming read's fitted line): the rate at which the
    kernel streams once running. A derived figure beside `frac`, not instead."""
    fixed = floor["fit"]["fixed_us"]
    if us <= fixed:
        return None
    gbs = nbytes / ((us - fixed) * 1e-6) / 1e9
    return {"fixed_us": fixed, "gbs": gbs, "frac": gbs / peak,
            "what": "bytes_per_launch / (avg_launch_us - size_floor.fit.fixed_us)"}


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def run_ours(args):
    import torch

    from tan_b200 import autotune
    from tan_b200 import convolution as cv

    world, rank, local, pg = dist_setup(args)
    dev = local
    torch.cuda.set_device(dev)
    nblocks = args.warmup + args.steps
    x, irs = make_inputs(min(nblocks, 256))
    xblocks = x.shape[1] // B

    ctx = cv.TANContext(dev)

    # ---- device-resident pass (value + roofline) --------------------------
    conv = autotune.tuned(ctx, cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C)
    P = conv.info()["partitions"]
    tiling = conv.tiling()[1]
    stream = torch.cuda.ExternalStream(conv.stream(), device=dev)
    x_dev = torch.from_numpy(x).to(f"cuda:{dev}")
    y_dev = torch.zeros((C, B * 2), dtype=torch.float32, device=f"cuda:{dev}")
    ir_dev = [torch.from_numpy(h).to(f"cuda:{dev}") for h in irs]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")
    flush_r2 = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{dev}")

    def flush_l2():
        # write one buffer larger than L2, then read two others: after one
        # read pass some dirty lines of the write are still in L2 and would be
        # written back inside the timed step (measured: the 66 MB streaming
        # read takes 16.4 us after write + two reads or after reads alone, and
        # 16.4 or 18.5 us after write + one read, 18.5 us after a write alone)
        with torch.cuda.stream(stream):
            flush.zero_()
            flush_r.sum()
            flush_r2.sum()
    row = x_dev.stride(0) * 4
    yrow = y_dev.stride(0) * 4
    torch.cuda.synchronize()
    import ctypes

    lib = cv.lib()
    # device row-pointer arrays built once, as a C caller would keep them
    dev_in = [(ctypes.c_void_p * C)(*[x_dev.data_ptr() + c * row + j * B * 4 for c in range(C)])
              for j in range(xblocks)]
    dev_out = [(ctypes.c_void_p * C)(*[y_dev.data_ptr() + c * yrow + p * B * 4 for c in range(C)]) for p in range(2)]
    dev_ir = [(ctypes.c_void_p * C)(*[h.data_ptr() + c * h.stride(0) * 4 for c in range(C)]) for h in ir_dev]
    dev_done = ctypes.c_size_t(0)

    def dev_step(k):
        si = swap_index(k, args.warmup)
        if si is not None:
            rc = lib.tanb_convolution_update_response_td_device(conv._h, dev_ir[si % N_IR_SETS], L, None, 0)
            assert rc == 0, cv.last_error()
        rc = lib.tanb_convolution_process_device(conv._h, dev_in[k % xblocks], dev_out[k % 2], B, None,
                                                 ctypes.byref(dev_done))
        assert rc == 0 and dev_done.value == B, cv.last_error()

    for k in range(args.warmup):
        flush_l2()
        dev_step(k)
    conv.Synchronize()
    conv.profile_read()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    # value: CUDA events around each step only (an event pair between the
    # head and tail launches would add its own overhead and keep the tail from
    # overlapping the head)
    evs = []
    with ClockSampler(dev) as clk:
        for k in range(args.warmup, nblocks):
            flush_l2()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            dev_step(k)
            b.record(stream)
            evs.append((a, b))
        conv.Synchronize()
        counts = conv.profile_read()
        # the same workload continues, untimed, so that the clock samples
        # cover at least a second of it
        nbusy = clk.keep_busy(lambda n: (flush_l2(), dev_step(nblocks + n)))
        conv.Synchronize()
    torch.cuda.synchronize()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    dev_ms = max_over_ranks(pg, dev_ms, local)
    if pg:
        pg.barrier()
    value = world * C * B * args.steps / (dev_ms / 1e3) / 1e9
    launches = counts["head"]["launches"] + counts["tail"]["launches"] + counts["ir_spectrum"]["launches"]
    # roofline: the same steps continued with an event pair around every
    # kernel launch (the tail then runs alone, after its head)
    nprof = min(args.steps, PROFILE_STEPS)
    conv.profile(True)
    for k in range(nblocks + nbusy, nblocks + nbusy + nprof):
        flush_l2()
        dev_step(k)
    conv.Synchronize()
    torch.cuda.synchronize()
    conv.profile(False)
    prof = conv.profile_read()
    tail = prof["tail"]
    tail_ms_avg = tail["ms"] / max(1, tail["timed"])
    bytes_per_tail = C * ((P - 2) * B * 16 + B * 8)  # partitions 2..P-1 of H and FDL, one tail row written
    peak, peak_kind = hbm_peak()
    achieved = bytes_per_tail / (tail_ms_avg / 1e3) / 1e9
    floor = size_floor(torch, stream, flush_l2, bytes_per_tail, dev)
    conv.Release()
    plain = {"value": value, "ms_per_step": dev_ms / args.steps, "gpu_launches": launches,
             "roofline_frac": achieved / peak, "tail_gbs": achieved}

    # ---- device-resident pass through the batched engine ---------------------
    # one 64-channel session; per block: commit of a pending IR update, head,
    # tail (persistent, over work items); IR updates from device memory with
    # BLOCK_UNTIL_READY, so the swap lands on the next block as above
    from tan_b200 import engine as eng

    e = eng.Engine(ctx, B, eng.SPECTRUM_FP32, budget_bytes=1 << 30, max_channels=C)
    rc, sess = e.open_session(C, L)
    assert rc == 0, cv.last_error()
    estream = torch.cuda.ExternalStream(e.stream(), device=dev)
    y_full = torch.zeros_like(x_dev)
    T = x_dev.shape[1]

    def eng_step(k):
        si = swap_index(k, args.warmup)
        if si is not None:
            assert sess.update_response_td_device(ir_dev[si % N_IR_SETS], block_until_ready=True) == 0
        j = k % xblocks
        assert e.process_device(x_dev.data_ptr() + j * B * 4, y_full.data_ptr() + j * B * 4, T) == 0

    def eflush():
        with torch.cuda.stream(estream):
            flush.zero_()
            flush_r.sum()
            flush_r2.sum()

    for k in range(args.warmup):
        eflush()
        eng_step(k)
    e.synchronize()
    e.profile_read()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    eevs = []
    with ClockSampler(dev) as eclk:
        for k in range(args.warmup, nblocks):
            eflush()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(estream)
            eng_step(k)
            b.record(estream)
            eevs.append((a, b))
        e.synchronize()
        ecounts = e.profile_read()
        ebusy = eclk.keep_busy(lambda n: (eflush(), eng_step(nblocks + n)))
        e.synchronize()
    torch.cuda.synchronize()
    einfo = e.info()
    eng_ms = max_over_ranks(pg, sum(a.elapsed_time(b) for a, b in eevs), local)
    eng_value = world * C * B * args.steps / (eng_ms / 1e3) / 1e9
    e.profile(True)
    for k in range(nblocks + ebusy, nblocks + ebusy + nprof):
        eflush()
        eng_step(k)
    e.synchronize()
    torch.cuda.synchronize()
    e.profile(False)
    eprof = e.profile_read()
    eng_block_us = 1000.0 * eprof["block_ms"] / max(1, eprof["timed"])
    eng_block_bytes = einfo["block_bytes"]
    eng_achieved = eng_block_bytes / (eng_block_us * 1e-6) / 1e9
    eng_floor = size_floor(torch, estream, eflush, eng_block_bytes, dev)
    engine_path = {"value": eng_value, "ms_per_step": eng_ms / args.steps,
                   "gpu_launches": ecounts["blocks"] + ecounts["commits"] + ecounts["ir_updates"],
                   "roofline_frac": eng_achieved / peak, "block_gbs": eng_achieved,
                   "block_bytes_per_launch": eng_block_bytes, "block_us": eng_block_us}
    e.release()
    del x_dev, y_dev, ir_dev, y_full

    # ---- end-to-end pass through the host C ABI ----------------------------
    conv = autotune.tuned(ctx, cv.TAN_CONVOLUTION_METHOD_FFT_UNIFORM_PARTITIONED, L, B, C)
    stream = torch.cuda.ExternalStream(conv.stream(), device=dev)
    lib = cv.lib()
    # the caller's audio buffers in page-locked host memory, as an audio
    # host keeps the buffers it hands a GPU: input blocks, output block, IRs
    pin_x = torch.from_numpy(np.ascontiguousarray(x.reshape(C, xblocks, B).transpose(1, 0, 2))).pin_memory()
    pin_y = torch.zeros((C, B), dtype=torch.float32).pin_memory()
    pin_ir = [torch.from_numpy(h).pin_memory() for h in irs]
    xs_blocks = [pin_x[j].numpy() for j in range(xblocks)]
    y = pin_y.numpy()
    # host row-pointer arrays built once, as a C caller would keep them
    in_rows = [(ctypes.c_void_p * C)(*[xb[c].ctypes.data for c in range(C)]) for xb in xs_blocks]
    out_rows = (ctypes.c_void_p * C)(*[y[c].ctypes.data for c in range(C)])
    ir_rows = [(ctypes.c_void_p * C)(*[h.numpy()[c].ctypes.data for c in range(C)]) for h in pin_ir]
    done = ctypes.c_size_t(0)

    def host_step(k):
        si = swap_index(k, args.warmup)
        if si is not None:
            rc = lib.tanb_convolution_update_response_td(conv._h, ir_rows[si % N_IR_SETS], L, None, 0)
            assert rc == 0
        rc = lib.tanb_convolution_process(conv._h, in_rows[k % xblocks], out_rows, B, None, ctypes.byref(done))
        assert rc == 0 and done.value == B

    for k in range(args.warmup):
        host_step(k)
    conv.Synchronize()
    lat, step_s = [], []
    if pg:
        pg.barrier()
    for k in range(args.warmup, nblocks):
        flush_l2()
        conv.Synchronize()
        t0 = time.perf_counter()
        host_step(k)
        t1 = time.perf_counter()
        conv.Synchronize()
        t2 = time.perf_counter()
        lat.append(t1 - t0)
        step_s.append(t2 - t0)
    e2e_s = max_over_ranks(pg, sum(step_s), local)
    e2e_value = world * C * B * args.steps / e2e_s / 1e9
    lat_ms = np.array(lat) * 1e3
    p99 = float(max_over_ranks(pg, float(np.percentile(lat_ms, 99)), local))
    e2e_in_place = conv.call_times()["in_place"]
    conv.Release()

    capacity = roofline_serving = None
    if rank == 0 and world == 1 and not args.no_capacity:
        from tan_b200 import serving

        cp = serving.capacity(ctx, "plain", 4, 48000, 256, blocks=150)
        c1 = serving.capacity(ctx, "plain_one", 4, 48000, 256, blocks=100, start=512)
        cb = serving.capacity(ctx, "batched", 4, 48000, 256, blocks=150)
        c24 = serving.capacity(ctx, "batched", 4, 48000, 256, spectrum=eng.SPECTRUM_FP24, blocks=150)
        capacity = {"what": "max channels (sessions of 4 ch, IR 48000 = 1 s, block 256 @ 48 kHz) with p99 "
                            "block latency < 5.33 ms, host buffers, FP32",
                    "plain_fp32": cp["max_realtime_channels"], "batched_fp32": cb["max_realtime_channels"],
                    "ratio": cb["max_realtime_channels"] / max(1, cp["max_realtime_channels"]),
                    "batched_fp24": c24["max_realtime_channels"],
                    "fp24_what": "IR spectra and delay line stored in 24 bits (error vs FP64 about -100 dB, "
                                 "tests/test_gpu_engine.py), FP32 accumulation",
                    "ratio_fp24": c24["max_realtime_channels"] / max(1, cp["max_realtime_channels"]),
                    "plain_one_object_fp32": c1["max_realtime_channels"],
                    "plain_one_object_what": "one drop-in TANConvolution holding every channel (host rows)",
                    "ratio_vs_one_object": cb["max_realtime_channels"] / max(1, c1["max_realtime_channels"])}
        # the MAC where its working set is far above L2: the batched engine's
        # block launch at the capacity found above
        rs = serving.mac_roofline(ctx, cb["max_realtime_channels"], 4, 48000, 256)
        roofline_serving = {"bound": "hbm", "achieved": rs["achieved_gbs"], "peak": peak, "unit": "GB/s",
                            "frac": rs["achieved_gbs"] / peak, "peak_source": f"{peak_kind} hbm_gbs",
                            "kernel": "eng_block_kernel (heads + partition MAC work items, one launch per block)",
                            "what": "batched FP32 engine at its real-time capacity (sessions of 4 ch, IR 48000, "
                                    "block 256), device I/O, CUDA events per block; working set >> L2",
                            **{k: v for k, v in rs.items() if k != "achieved_gbs"}}
    # the other configurations: the small drop-in case (cfg1), the uneven batch (cfg3, error vs FP64 for every
    # channel), the non-uniform 2^20-tap IRs (cfg4, on the engine, with its
    # autotuned schedule) and the serving loop (cfg5, FP32, FP16 and FP24)
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        import bench_workloads as bw

        configs = {"cfg1": bw.dropin_small(ctx), "cfg3": bw.engine_uneven(ctx), "cfg4": bw.nonuniform_long(ctx),
                   "cfg5": bw.serving_cfg5(ctx, seconds=10.0)}
    # several GPUs: the serving mix sharded over the ranks (sessions placed by
    # the engines' admission rule, no audio crossing GPUs), every rank its own
    # engine; latencies gathered to rank 0
    sharded = None
    if world > 1 and not args.no_configs:
        from tan_b200 import serving

        sharded = serving.serve_sharded(pg, ctx, sessions=300 * world, blocks=1000)
    # the CPU baseline loads every host core for seconds; it runs after the
    # latency measurements above, whose host-side copies it would slow down
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample_s)
        # also at the reference library's default thread count, a quarter of
        # the host's processors (FFTImpl.cpp:245-249, MathImpl.cpp:154-158)
        cpu["reference_default_threads"] = cpu_baseline(min(5.0, args.cpu_sample_s),
                                                         threads=max(1, (os.cpu_count() or 4) // 4))
        cpu["pipeline_chain"] = cpu_pipeline_chain()

    if rank == 0:
        deadline_ms = 1000.0 * B / FS
        best = engine_path if engine_path["value"] > plain["value"] else plain
        best_name = "engine" if best is engine_path else "drop-in"
        if best is engine_path:
            achieved, bytes_per_tail, tail_ms_avg = eng_achieved, eng_block_bytes, eng_block_us / 1e3
            launches, clk, floor = engine_path["gpu_launches"], eclk, eng_floor
        line = {
            "metric": METRIC, "value": best["value"], "unit": "GSamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": best["ms_per_step"], "higher_is_better": True,
            "path": best_name, "paths": {"drop-in": plain, "engine": engine_path},
            "swaps_timed": swaps_timed(args.steps),
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(P),
            "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": p99,
                           "p999": float(np.percentile(lat_ms, 99.9)), "deadline": deadline_ms,
                           "what": "host Process() call, H2D + head + D2H, per block"},
            "realtime_factor_p99": deadline_ms / p99,
            "l2": "flushed before every timed step (a 256 MiB write, then reads of two other 256 MiB buffers, "
                  "on the object's stream)",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": read_traffic("eng_block_kernel_64ch_b512_ir65536.txt" if best is engine_path
                                                 else "tail_kernel_64ch_b512_ir65536.txt"),
                         "kernel": "eng_block_kernel (heads + partition MAC work items, one launch per block)"
                         if best is engine_path else "tail_kernel (partition MAC)",
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "bytes_per_launch": bytes_per_tail, "avg_launch_us": tail_ms_avg * 1e3,
                         "launches_timed": tail["timed"], "tiling": list(tiling),
                         "size_floor": dict(floor, frac_of_peak=floor["gbs"] / peak,
                                            tail_vs_floor=achieved / floor["gbs"]),
                         "marginal": marginal(bytes_per_tail, tail_ms_avg * 1e3, floor, peak)},
            "kernel_ms": {k: v["ms"] for k, v in prof.items()},
            "e2e": {"value": e2e_value, "unit": "GSamples/s", "h2d_bytes_per_step": C * B * 4,
                    "d2h_bytes_per_step": C * B * 4,
                    "ir_h2d_bytes_per_swap": C * L * 4,
                    "rows_in_place": e2e_in_place,
                    "what": "tanb_convolution_process with host rows in page-locked memory (read and written "
                            "by the head over the bus: rows_in_place 3 = inputs and outputs) + "
                            "UpdateResponseTD from page-locked IR rows at the timed swap steps; wall clock "
                            "per block including the tail kernel"},
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if capacity:
            line["max_realtime_channels"] = capacity
        if roofline_serving:
            line["roofline_serving"] = roofline_serving
        if configs:
            line["configs"] = configs
        if sharded:
            line["serving_sharded"] = sharded
        print(json.dumps(line), flush=True)
    ctx.Release()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def main():
    args = parse()
    if args.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
