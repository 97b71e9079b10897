#!/usr/bin/env python
"""Throughput of the full compute_dmsc path on B200.

Workload: one 4096 x 4096 float32 field per GPU = 2000 Gaussian bumps
(amplitude U[-1, 1], sigma U[4, 64] px) + N(0, 0.02^2) noise, seeded; full
geometry (gradient, ridges, valleys, peaks, basins). The timed steps cycle
through the four variants (is_dual, threshold) in {False, True} x {0, 0.05}.
A step is one compute_dmsc call on one field. The field and the gradient
output (64 MiB + 256 MiB) exceed the 126 MB L2, so no flush is needed.

Metric: Mpixel/s (higher is better). ``value`` is device-timed with the
input resident in HBM; ``e2e`` is the same metric through the public API
from pinned host memory with every output read back to the host. N GPUs run
N independent replicas (one field each, weak scaling), timed as the max over
ranks.

``--impl reference`` times the reference's own CPU path (compiled from the
reference sources into oracle/_ref/ordered with an order-preserving parallel
TBB stand-in, all host threads) on the same workload.
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

import torch  # noqa: E402

METRIC = "Mpixel/s full compute_dmsc at 4096^2 (bit-exact)"
UNIT = "Mpixel/s"
VARIANTS = [(False, 0.0), (False, 0.05), (True, 0.0), (True, 0.05)]
SEED = 1234


def workload_config(size):
    return {
        "workload": f"{size}x{size} float32 bump field: {int(round(2000 * (size / 4096) ** 2))} Gaussian bumps "
                    "(a~U[-1,1], sigma~U[4,64] px) + N(0,0.02^2) noise, full geometry, steps cycle "
                    "is_dual x threshold in {F,T} x {0,0.05}",
        "image": [size, size],
        "variants": [{"is_dual": d, "threshold": t} for d, t in VARIANTS],
        "l2": "inputs larger than L2 (64 MiB field + 256 MiB gradient per call)",
        "parallelism": "replicas (one field per GPU, no collective)",
    }


def _json_line(d):
    print(json.dumps(d), flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref) -- checker and CPU baseline only
# ---------------------------------------------------------------------------
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def load_reference():
    """The reference CPU path compiled from its sources: the build with the
    order-preserving parallel TBB stand-in (oracle/_ref/ordered, all threads,
    bit-identical to the single-thread order) when present, else the serial
    stand-in build (oracle/_ref), else the C restatement (oracle/). Returns
    (kind, shim, run)."""
    for sub, shim in (("ordered", "ordered parallel TBB stand-in"), ("", "serial TBB stand-in")):
        ref_dir = os.path.join(ROOT, "oracle", "_ref", sub) if sub else os.path.join(ROOT, "oracle", "_ref")
        if os.path.exists(os.path.join(ref_dir, "dmsc_cpu.so")):
            sys.path.insert(0, ref_dir)
            import dmsc_cpu

            def run(img, thr, dual, geometry=True):
                r = dmsc_cpu.extract_dmsc(img, thr, True, dual, geometry, geometry, True, True)
                return [r[i] for i in range(19)]

            return "reference", shim, run
    from oracle import oracle

    def run(img, thr, dual, geometry=True):
        return list(oracle.run(img, thr, True, dual, geometry, geometry, True, True))

    return "port", "C restatement, one thread", run


def same_outputs(a, b):
    for x, y in zip(a, b):
        x = x.cpu()
        y = y.cpu()
        if x.shape != y.shape or x.dtype != y.dtype:
            return False
        if x.is_floating_point():
            x, y = x.view(torch.int32), y.view(torch.int32)
        if not torch.equal(x, y):
            return False
    return True


def cpu_baseline(img_cpu, gpu_outputs):
    """Reference CPU path on the same field: the four variants with all host
    threads (timed, each checked bit for bit against the GPU's outputs of the
    same variant) and one variant with one thread."""
    kind, shim, run = load_reference()
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    pix, t_tot, exact, done = 0, 0.0, True, []
    for dual, thr in VARIANTS:
        t0 = time.perf_counter()
        out = run(img_cpu, thr, dual)
        t_tot += time.perf_counter() - t0
        pix += img_cpu.numel()
        done.append(f"is_dual={dual},thr={thr}")
        g = gpu_outputs.get((dual, thr))
        exact = exact and g is not None and same_outputs(g, out)
    torch.set_num_threads(1)
    t0 = time.perf_counter()
    run(img_cpu, VARIANTS[1][1], VARIANTS[1][0])
    t1 = time.perf_counter() - t0
    torch.set_num_threads(threads)
    return {
        "value": pix / 1e6 / t_tot,
        "unit": UNIT,
        "cores": threads,
        "kind": kind,
        "shim": shim,
        "cpu_model": cpu_model(),
        "sample": f"{len(done)} full compute_dmsc calls on the same {img_cpu.shape[0]}x{img_cpu.shape[1]} field "
                  f"({'; '.join(done)}), torch threads={threads}",
        "seconds": t_tot,
        "one_thread": {"value": img_cpu.numel() / 1e6 / t1, "unit": UNIT, "seconds": t1,
                       "sample": f"one call (is_dual={VARIANTS[1][0]},thr={VARIANTS[1][1]}), torch threads=1"},
    }, exact


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from dmsc_b200.synthetic import field_4096_bumps

    size = args.size
    kind, shim, run = load_reference()
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    img = field_4096_bumps(seed=SEED, size=size)
    # bound the run to a few minutes: measure one call, shrink to a centred
    # crop when K + W full calls would not fit
    t0 = time.perf_counter()
    run(img, VARIANTS[0][1], VARIANTS[0][0])
    est = time.perf_counter() - t0
    sample = img
    if est * (args.steps + args.warmup) > 240.0:
        scale = (240.0 / (est * (args.steps + args.warmup))) ** 0.5
        c = max(256, int(size * scale) // 64 * 64)
        o = (size - c) // 2
        sample = img[o:o + c, o:o + c].contiguous()
    for w in range(max(0, args.warmup - 1)):
        d, t = VARIANTS[w % 4]
        run(sample, t, d)
    times = []
    for k in range(args.steps):
        d, t = VARIANTS[k % 4]
        t0 = time.perf_counter()
        run(sample, t, d)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = sample.numel() * args.steps / 1e6 / total
    sample_desc = (f"{'full field' if sample is img else f'centred {sample.shape[0]}x{sample.shape[1]} crop'} of the "
                   f"{size}x{size} workload per step, cycling the 4 variants")
    _json_line({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/i32",
        "data": "synthetic", "config": workload_config(size),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "shim": shim,
                         "cpu_model": cpu_model(), "sample": sample_desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_key, size):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    e = d.get(kernel_key)
    if not e:
        return None
    return e["bytes_per_launch_per_pixel"] * size * size


def b200_arm(args):
    from dmsc_b200 import _lib, compute_dmsc
    from dmsc_b200.synthetic import field_4096_bumps

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    size = args.size
    dev = torch.device("cuda", local)
    img = field_4096_bumps(seed=SEED + rank, size=size, device=dev)
    torch.cuda.synchronize()
    ctx = _lib.context(local)
    st = torch.cuda.current_stream(dev)

    def step(k):
        d, t = VARIANTS[k % 4]
        return compute_dmsc(img, t, is_dual=d)

    gpu_out = {}
    # warm-up covers every variant once, so workspace growth happens here
    warm = max(args.warmup, len(VARIANTS))
    for w in range(warm):
        ms = step(w)
        if rank == 0 and world == 1:
            gpu_out[VARIANTS[w % 4]] = [x.cpu() for x in ms]
    torch.cuda.synchronize()

    # ---- profiling pass (untimed): per-stage device times, loop counts and
    # the library's own kernel launches of the same K steps ----
    ctx.set_profiling(True)
    stage_sum = {}
    launches = 0
    loops = []
    for k in range(args.steps):
        step(k)
        for name, v in ctx.stage_times().items():
            stage_sum[name] = stage_sum.get(name, 0.0) + v
        launches += ctx.launch_count()
        loops.append(ctx.loop_counts())
    ctx.set_profiling(False)
    torch.cuda.synchronize()

    # ---- timed region: device-resident input, K plain calls ----
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for k in range(args.steps):
        step(k)
    e1.record(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms_total = e0.elapsed_time(e1)
    clk = clocks.stop()  # clocks cover the device-timed region
    t = torch.tensor([ms_total], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * args.steps * size * size / 1e6 / (ms_max / 1000.0)

    # ---- end to end through the public API from pinned host memory ----
    host = img.cpu().pin_memory()
    h2d = host.numel() * host.element_size()
    d2h = 0
    ms = None
    for w in range(2 * warm):  # warm the pinned host buffers exactly as the timed loop uses them
        d, th = VARIANTS[w % 4]
        ms = compute_dmsc(host, th, is_dual=d)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # host wall clock: the call is synchronous for a CPU caller (it returns host
    # tensors), so the wall clock covers H2D, compute, D2H and host-side work
    w0 = time.perf_counter()
    for k in range(args.steps):
        d, th = VARIANTS[k % 4]
        ms = compute_dmsc(host, th, is_dual=d)  # H2D, compute, every output back to the host
        d2h += sum(x.numel() * x.element_size() for x in ms)
    torch.cuda.synchronize()
    te = torch.tensor([1000.0 * (time.perf_counter() - w0)], device=dev)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e = world * args.steps * size * size / 1e6 / (float(te.item()) / 1000.0)

    batched = None if args.batch_images <= 0 else batched_section(args, dev, ctx, dist, world, rank)
    seg_only = segmentation_only_section(args, img, dev, ctx, dist, size)
    diff = None if args.no_diff else diff_section(args, dev, dist)
    tune = tune_section(args, img, dev, size) if (not args.no_tune and world == 1) else None
    c3 = c3_section(args, dev, ctx) if (args.c3_size > 0 and world == 1) else None

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    peak, peak_kind = measured_peak()
    # roofline of the gradient kernel: 4 B/pixel read + 16 B/index written
    grad_bytes = 4.0 * size * size + 16.0 * (size + 1) * (size + 1)
    grad_ms = stage_sum.get("gradient", 0.0) / args.steps
    achieved = grad_bytes / (grad_ms / 1000.0) / 1e9 if grad_ms > 0 else None
    traffic = ncu_traffic("gradient_kernel", size)
    # shapes 3 and 4 run the TMA-staged persistent kernel on one image
    grad_kernel = "gradient_tma_kernel" if ctx.get_tuning().grad_shape >= 3 else "gradient_batch_kernel"
    # segmentation (basins + peaks) kernels
    seg_bytes = 8.0 * (size + 1) ** 2 + 4.0 * size * size + 4.0 * (size + 1) ** 2
    lab_ms = stage_sum.get("labels", 0.0) / args.steps
    seg = seg_bytes / (lab_ms / 1000.0) / 1e9 if lab_ms > 0 else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": warm, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/i32", "data": "synthetic",
        "config": workload_config(size),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h // args.steps,
                "timing": "host wall clock around K public-API calls from pinned host memory, max over ranks"},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": grad_kernel, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "algorithmic_bytes": grad_bytes, "avg_ms": grad_ms,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                     else "fallback 6.65 TB/s"},
        "roofline_segmentation": {"bound": "hbm", "kernel": "label stage (label_tile_kernel + label_exit_kernel x2)", "achieved": seg, "peak": peak,
                                  "unit": "GB/s", "frac": (seg / peak) if seg else None,
                                  "traffic_label_tile_kernel": ncu_traffic("label_tile_kernel", size),
                                  "algorithmic_bytes": seg_bytes, "avg_ms": lab_ms},
        "stage_ms_per_step": {k: v / args.steps for k, v in stage_sum.items()},
        "device_loops_per_variant": {f"dual={d},thr={t}": loops[k] for k, (d, t) in enumerate(VARIANTS) if k < len(loops)},
        "clocks": clk,
    }
    if batched is not None:
        line["batched"] = batched
    line["segmentation_only"] = seg_only
    if diff is not None:
        line["differentiation"] = diff
    if tune is not None:
        line["tuning"] = tune
    if c3 is not None:
        line["worst_case_uniform"] = c3
    if world == 1 and not args.no_cpu_baseline:
        cb, exact = cpu_baseline(img.cpu(), gpu_out)
        line["cpu_baseline"] = cb
        line["bit_exact_vs_reference"] = exact
    _json_line(line)
    if dist:
        dist.destroy_process_group()


def _same(a, b):
    """Bitwise equality of two 19-field complexes (float32 compared by bits)."""
    for x, y in zip(a, b):
        if x.shape != y.shape or x.dtype != y.dtype:
            return False
        if x.dtype == torch.float32:
            x, y = x.view(torch.int32), y.view(torch.int32)
        if not torch.equal(x, y):
            return False
    return True


def batched_section(args, dev, ctx, dist, world, rank):
    """Uneven batch: ``args.batch_images`` images, H and W log-uniform in
    [64, 2048], bump count area / 8000, sigma U[4, 32], noise N(0, 0.03^2),
    threshold U[0.02, 0.2], is_dual ~ Bernoulli(0.5); images resident in HBM.
    One compute_dmsc_batched call over all of them against one plain
    compute_dmsc call per image, both timed by the host wall clock around the
    whole pass (each ends with a device synchronisation), max over ranks.
    Every image's batched outputs are checked bit for bit against its plain
    call."""
    from dmsc_b200 import compute_dmsc, compute_dmsc_batched
    from dmsc_b200.synthetic import batch_uneven

    n = args.batch_images
    imgs, thr, dual = batch_uneven(n, seed=SEED + 17 * rank, device=dev)
    px = sum(x.numel() for x in imgs)
    torch.cuda.synchronize()

    def plain_pass():
        return [compute_dmsc(x, t, is_dual=d) for x, t, d in zip(imgs, thr, dual)]

    def batched_pass():
        return compute_dmsc_batched(imgs, thr, dual)

    ref = plain_pass()
    got = batched_pass()
    torch.cuda.synchronize()
    exact = all(_same(a, b) for a, b in zip(got, ref))
    del ref, got
    ctx.set_profiling(True)
    batched_pass()
    stages = ctx.stage_times()
    launches = ctx.launch_count()
    ctx.set_profiling(False)

    def timed(fn, reps):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        t = torch.tensor([(time.perf_counter() - t0) / reps], device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    t_plain = timed(plain_pass, 1)
    t_batch = timed(batched_pass, 3)
    return {
        "workload": f"{n} images per GPU, H and W log-uniform in [64, 2048], bumps area/8000 (sigma U[4,32]) + "
                    "N(0,0.03^2) noise, threshold U[0.02,0.2], is_dual Bernoulli(0.5), full geometry",
        "n_images": n * world, "mpixel": px * world / 1e6,
        "images_per_s": n * world / t_batch, "plain_images_per_s": n * world / t_plain,
        "speedup_vs_plain_calls": t_plain / t_batch,
        "ms_per_pass": 1000.0 * t_batch, "plain_ms_per_pass": 1000.0 * t_plain,
        "bit_exact_vs_plain_calls": exact,
        "device_batch_stage_ms": stages, "device_batch_launches": launches,
        "form": "one device batch per pass (every stage once over the union of the images); "
                "host wall clock, inputs resident in HBM",
    }


def segmentation_only_section(args, img, dev, ctx, dist, size):
    """Segmentation-only preset (the reference's basins/peaks use:
    return_gradient=False, no ridges or valleys): the same field and variant
    cycle, K device-timed calls. Its label stage reads the 1-byte flow codes
    and writes the two label maps; no gradient is written and no arc is
    traced."""
    from dmsc_b200 import compute_dmsc

    def step(k):
        d, t = VARIANTS[k % 4]
        return compute_dmsc(img, t, return_gradient=False, is_dual=d, trace_valleys=False, trace_ridges=False)

    for w in range(max(args.warmup, len(VARIANTS))):
        step(w)
    ctx.set_profiling(True)
    stage_sum = {}
    for k in range(args.steps):
        step(k)
        for name, v in ctx.stage_times().items():
            stage_sum[name] = stage_sum.get(name, 0.0) + v
    ctx.set_profiling(False)
    st = torch.cuda.current_stream(dev)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for k in range(args.steps):
        step(k)
    e1.record(st)
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item()) / args.steps
    world = dist.get_world_size() if dist else 1
    return {
        "workload": "same field and variants; return_gradient=False, trace_ridges=False, trace_valleys=False",
        "value": world * size * size / 1e6 / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms,
        "stage_ms_per_step": {k: v / args.steps for k, v in stage_sum.items()},
    }


def diff_section(args, dev, dist):
    """Differentiation workload: 64 float32 512 x 512 fields (200 bumps,
    sigma U[4,32], noise N(0,0.05^2), plus 1e-6 * permutation rank / N), loss
    = sum of p^2 over pairs with ppairs != -1 and 0 <= p < 0.1. A step is the
    forward (persistence pairs of the batch) and the backward (the
    deterministic scatter kernel) of that loss; host wall clock around K
    steps ending with a device synchronisation, max over ranks. The backward
    kernel alone is timed with CUDA events."""
    from dmsc_b200.autograd import persistence_pairs, scatter_pair_grads
    from dmsc_b200.synthetic import bump_field

    n, size = 64, 512
    fields = []
    for i in range(n):
        f = bump_field(size, size, 200, 4.0, 32.0, 0.05, SEED + 101 * i, device=dev)
        g = torch.Generator().manual_seed(SEED + 101 * i + 1)
        rank = torch.randperm(size * size, generator=g).reshape(size, size).float().to(dev)
        fields.append(f + 1e-6 * rank / (size * size))
    x0 = torch.stack(fields).contiguous()

    def step():
        x = x0.detach().requires_grad_(True)
        pp = persistence_pairs(x, -1.0)
        p = pp.persistence
        keep = (pp.ppairs != -1) & (p >= 0) & (p < 0.1)
        (p * p * keep).sum().backward()
        return x.grad, pp

    g1, pp = step()
    g2, _ = step()
    deterministic = bool(torch.equal(g1.view(torch.int32), g2.view(torch.int32)))
    steps = max(3, args.steps)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    torch.cuda.synchronize()
    t = torch.tensor([(time.perf_counter() - t0) / steps], device=dev)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    # the backward kernel alone, on this batch's pairs
    base = (pp.image * (size * size)).to(torch.int32)
    plus = torch.where(pp.plus_pixel >= 0, pp.plus_pixel + base, pp.plus_pixel)
    minus = torch.where(pp.minus_pixel >= 0, pp.minus_pixel + base, pp.minus_pixel)
    gp = torch.ones_like(pp.persistence)
    st = torch.cuda.current_stream(dev)
    for _ in range(3):
        scatter_pair_grads(plus, minus, gp, x0.shape)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(10):
        scatter_pair_grads(plus, minus, gp, x0.shape)
    e1.record(st)
    torch.cuda.synchronize()
    return {
        "workload": "64 x 512^2 float32 bump fields (200 bumps, sigma U[4,32], noise N(0,0.05^2)) + 1e-6*rank/N; "
                    "loss = sum p^2 over pairs with ppairs != -1 and 0 <= p < 0.1",
        "ms_per_forward_backward": 1000.0 * float(t.item()),
        "images_per_s": n / float(t.item()),
        "pairs": int(pp.persistence.numel()),
        "backward_kernel_ms": e0.elapsed_time(e1) / 10,
        "backward_deterministic": deterministic,
        "timing": "host wall clock around K forward+backward steps, inputs resident in HBM",
    }


C3_DIGESTS = os.path.join(ROOT, "tests", "golden", "uniform16384_digests.json")


def _digests(outs):
    import hashlib

    names = ("shape max_pts min_pts sad_pts e_max e_min p_max p_min ppairs_max ppairs_min grad_indices peaks ridges "
             "ridge_offsets ridge_arc_offsets basins valleys valley_offsets valley_arc_offsets").split()
    d = {}
    for n, t in zip(names, outs):
        a = t.contiguous().cpu().numpy()
        d[n] = {"shape": list(a.shape), "dtype": str(a.dtype), "sha256": hashlib.sha256(a.tobytes()).hexdigest()}
    return d


def c3_section(args, dev, ctx):
    """Worst-case critical-point density: one size x size i.i.d. U[0, 1)
    float32 field (seed 1234, CPU generator), primal, thresholds 0 and 0.5.
    At 0 every output is produced and checked against the digests of the
    reference CPU path's outputs on the same field
    (tests/golden/uniform16384_digests.json, made by
    tests/golden/make_uniform_digests.py). At 0.5 almost every pair cancels
    and the simplified arcs exceed int32 offsets, where the reference fails;
    the full call must raise the same overflow, and the call without arcs
    (gradient, lists, pairs, labels) is timed and checked. Device time by CUDA
    events around whole calls, input resident in HBM."""
    import hashlib

    from dmsc_b200 import extract_dmsc
    from dmsc_b200.synthetic import field_uniform

    size = args.c3_size
    img_cpu = field_uniform(size, seed=SEED)
    in_sha = hashlib.sha256(img_cpu.numpy().tobytes()).hexdigest()
    img = img_cpu.to(dev)
    del img_cpu
    ref = None
    if os.path.exists(C3_DIGESTS):
        with open(C3_DIGESTS) as f:
            ref = json.load(f)
        if ref.get("size") != size or ref.get("input_sha256") != in_sha:
            ref = None
    st = torch.cuda.current_stream(dev)
    out = {"workload": f"{size}x{size} i.i.d. U[0,1) float32 (seed {SEED}), primal", "input_sha256": in_sha,
           "runs": {}}
    for thr, geom in ((0.0, True), (0.5, False), (0.5, True)):
        ent = {}
        try:
            r = extract_dmsc(img, thr, True, False, geom, geom, True, True)  # warm-up (workspace growth)
            del r
            torch.cuda.synchronize()
            times = []
            for _ in range(2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                r = extract_dmsc(img, thr, True, False, geom, geom, True, True)
                e1.record(st)
                torch.cuda.synchronize()
                times.append(e0.elapsed_time(e1))
            ms = min(times)
            ent.update({"ms_per_call": ms, "value": size * size / 1e6 / (ms / 1000.0), "unit": UNIT,
                        "loops": ctx.loop_counts(),
                        "sizes": {"max_pts": int(r[1].numel()), "min_pts": int(r[2].numel()),
                                  "sad_pts": int(r[3].numel()), "ridges": int(r[12].numel()),
                                  "valleys": int(r[16].numel())}})
            free, total = torch.cuda.mem_get_info(dev)
            ent["device_memory_used_gb"] = (total - free) / 1e9
            rk = str(thr) if geom else f"{thr}_noarcs"
            if ref is not None and rk in ref and "fields" in ref[rk]:
                dg = _digests(r)
                ent["bit_exact_vs_reference"] = all(dg[n] == ref[rk]["fields"][n] for n in dg)
                ent["reference_seconds"] = ref[rk].get("seconds")
            del r
        except RuntimeError as e:
            ent["error"] = str(e)
            if ref is not None and "0.5" in ref and "error" in ref["0.5"]:
                ent["reference_error"] = ref["0.5"]["error"]
        out["runs"][f"thr={thr},arcs={geom}"] = ent
        torch.cuda.empty_cache()
    del img
    torch.cuda.empty_cache()
    return out


def tune_section(args, img, dev, size):
    """The launch-shape tuner (dmsc_b200.tuning) on this workload: one
    variant (is_dual=False, threshold 0.05) of the field, median of 5 runs per
    candidate; the report gives the default and tuned whole-call device times.
    The choice stays cached for the rest of the run (the timed steps above
    ran before it, with the default shapes)."""
    from dmsc_b200 import compute_dmsc, tuning

    rep = tuning.tune(lambda: compute_dmsc(img, 0.05), size * size, reps=5)
    return {"workload": f"{size}x{size} field, is_dual=False, threshold 0.05", "choice": rep["choice"],
            "default_ms": rep["default_ms"], "tuned_ms": rep["tuned_ms"], "stage_medians_ms": rep["stages"]}


def profile_workload(args):
    """Workload for profiler captures (prints no measurement): the bump field
    of --size generated on the host, one warm-up call of three variants, then
    --profile-calls calls of variant --profile-variant (default 1: is_dual=False,
    threshold 0.05). A capture that skips the launches of the warm-up calls sees
    exactly the profiled calls."""
    from dmsc_b200 import compute_dmsc
    from dmsc_b200.synthetic import field_4096_bumps

    img = field_4096_bumps(seed=SEED, size=args.size).cuda()
    for d, t in ((False, 0.0), (True, 0.05), (False, 0.05)):
        compute_dmsc(img, t, is_dual=d)
    torch.cuda.synchronize()
    d, t = VARIANTS[args.profile_variant]
    for _ in range(args.profile_calls):
        compute_dmsc(img, t, is_dual=d)
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=4096)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-images", type=int, default=512, help="uneven-batch images per GPU (0: skip)")
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiation workload")
    ap.add_argument("--c3-size", type=int, default=16384, help="worst-case U[0,1) field size (0: skip)")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape tuner section")
    ap.add_argument("--profile-calls", type=int, default=0,
                    help="run the profiler workload (warm-up, then this many calls) and exit")
    ap.add_argument("--profile-variant", type=int, default=1, choices=range(4),
                    help="variant of the profiled calls (index into the bench's (is_dual, threshold) variants)")
    args = ap.parse_args()
    if args.profile_calls > 0:
        profile_workload(args)
        return
    if args.impl == "reference":
        reference_arm(args)
    else:
        b200_arm(args)


if __name__ == "__main__":
    main()
