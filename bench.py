#!/usr/bin/env python3
"""Frame-pairs/s of the per-frame measurement path on B200 (one JSON line on rank 0).

Workload (default ``c2``): 3840x2160 10-bit 4:2:0, one source and three encodes per frame step (3 frame pairs), seeded
synthetic frames (es_synth: dark gradients with grain, blurred / de-grained / requantised encodes). A step is one
es_frame_queue + es_frame_collect of a whole frame step: unpack, CAMBI of the source and every encode, window and
lasting-texture figures, PSNR and color, and the per-frame reduction into per-segment accumulators.

* ``value``: frame pairs/s with the input frames resident in HBM (a pool of distinct steps, 100 MB of input per step,
  so consecutive steps do not hit L2), timed with CUDA events on the queueing stream; a step's done event also waits
  for the CAMBI streams.
* ``e2e``: the same through the C ABI with the inputs in pinned host memory, copied host-to-device every step on a copy
  stream (three input slots, each step's copy queued one step ahead) and the figures read back, inside the timed
  region.
* ``roofline``: the kernel with the most device time in a frame step: its algorithmic bytes per step (every launch
  of it in the step; algorithmic_bytes) over its event-timed duration per step, against the measured HBM copy
  bandwidth; ``step`` gives the same for the whole step (inputs read once, per-window outputs written once) over the
  timed ms per step, and ``issue`` the kernel's instruction-issue roofline from a one-kernel ncu capture
  (profiles/issue.json). Durations come from a pass over the pool after the timed region with every kernel alone on
  the stream and bracketed by CUDA events (``kernels`` lists them all, each with its own HBM fraction).
* ``cpu_baseline``: the CPU oracle (plain-C restatement of the reference) on the host cores, rank 0 at N = 1 only:
  strips of a real frame step (13 distinct source frames for the lasting texture, host collect included), one strip
  per process side by side for the all-core rate (median of 5 rounds) and one process alone for ``value_1_core``.
* ``c3``: the uneven batch of 16 source / encode pairs per frame step, plain (16 es_frame) against batched (one
  es_batch), as extra figures (``--workload c3`` makes it the headline instead).

``--impl reference`` times the reference's CPU path instead: the CPU oracle port over all host cores (the reference's
own CPU implementation of this path is its numpy module plus libvmaf's CAMBI, neither of which exists on the GPU
hosts), printing the same metric and config.

Multi-GPU: one process per GPU (torchrun), each scoring its own source; scaling is weak and the time is the max over
ranks.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "encode-score_b200"))

METRIC = "4K10 frame-pairs/s (1 source + 3 encodes per frame step)"
UNIT = "frame-pairs/s"
WORKLOADS = {
    "c2": dict(w=3840, h=2160, pd=10, n_enc=3, gen="c2_step", desc="3840x2160 10-bit 4:2:0, 1 source + 3 encodes (blur 0.8/1.5/2.5, "
               "de-grain, requantised rectangles) per frame step"),
    "c1": dict(w=1920, h=1080, pd=8, n_enc=1, gen="c1_step", desc="1920x1080 8-bit 4:2:0, 1 source + 1 encode per frame step"),
}


def scale_pixels(w: int, h: int) -> list[int]:
    out = []
    for _ in range(5):
        out.append(w * h)
        w, h = (w + 1) >> 1, (h + 1) >> 1
    return out


def algorithmic_bytes(name: str, wl: dict) -> float | None:
    """Bytes the launches of `name` in one frame step must move at least: inputs read once, outputs written once."""
    w, h, e = wl["w"], wl["h"], wl["n_enc"]
    n, windows, pics = w * h, (w // 16) * (h // 16), 1 + wl["n_enc"]
    sp = scale_pixels(w, h)
    table = {
        "cambi_cvalues": 2.0 * sum(sp) * pics,              # every picture's 5 scale planes (16-bit words)
        "cambi_prep0": (2.0 * n + 2.0 * n) * pics,          # plane in, scale-0 words out
        "cambi_decimate_mode": 4.0 * sum(sp[1:]) * pics,    # scale s - 1's even rows in, scale s out
        "window_stats": 2.0 * n * (1 + e) + 32.0 * windows * e,
        "persist_stats": 2.0 * n * (2 + 4 + 2 + e) + 20.0 * windows * e,
        "pair_sums": 3.0 * n * (1 + e),
        "frame_unpack": (1.5 * n * 2) * (1 + e) + 3.0 * n * (1 + e),
        "frame_collect": 32.0 * windows * e + 20.0 * windows * e + 12.0 * windows * e,
    }
    return table.get(name)


def step_algorithmic_bytes(wl: dict) -> float:
    """A whole frame step's algorithmic bytes: every input picture read once (4:2:0, 2 bytes a sample at 10 bits, 1 at
    8) plus the per-window outputs written once (8 window and 5 lasting floats per window and encode)."""
    w, h, e = wl["w"], wl["h"], wl["n_enc"]
    b = 2 if wl["pd"] == 10 else 1
    return (1 + e) * 1.5 * w * h * b + e * (w // 16) * (h // 16) * 13 * 4


def read_peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return {"hbm_gbs": float(p["hbm_gbs"]), "source": "measured"}
    except (OSError, KeyError, ValueError):
        return {"hbm_gbs": 6650.0, "source": "fallback"}


def read_issue(kernel: str, workload: str):
    """The instruction-issue roofline of a kernel from a one-kernel ncu capture (profiles/issue.json): instructions
    issued over (SMs x 4 schedulers x SM clock x duration), with the clock and duration of that capture."""
    try:
        with open(os.path.join(ROOT, "profiles", "issue.json")) as f:
            t = json.load(f)
        return t.get(workload, {}).get(kernel)
    except (OSError, ValueError):
        return None


def read_traffic(kernel: str, workload: str):
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        return t.get(workload, {}).get(kernel)
    except (OSError, ValueError):
        return None


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"es_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict | None:
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def make_pool(wl: dict, steps: int, source: int):
    import es_synth

    gen = getattr(es_synth, wl["gen"])
    out = []
    for f in range(steps):
        kw = dict(w=wl["w"], h=wl["h"], source=source)
        if wl["gen"] == "c2_step":
            kw["n_encodes"] = wl["n_enc"]
        out.append(gen(f, **kw))
    return out


STRIP_ROWS = 144   # rows of a frame step per CPU sample (1/15 of a 4K picture)
CPU_FRAME = 12     # the frame step the CPU samples measure: its lasting texture reads source frames 0 .. 12


def _cpu_frames_dir() -> str:
    import tempfile

    return tempfile.mkdtemp(prefix="es_cpu_frames_")


def cpu_make_frame(args):
    """Worker: frame step f of the workload, saved as .npy planes under `d` (the source's luma of every frame; every
    plane of the frames whose figures are measured)."""
    import numpy as np

    import es_synth

    wl_name, f, d = args
    wl = WORKLOADS[wl_name]
    step = getattr(es_synth, wl["gen"])(f, w=wl["w"], h=wl["h"])
    np.save(os.path.join(d, f"f{f}_p0_y.npy"), step.source.y)
    if f in (CPU_FRAME, CPU_FRAME - 6):
        for i, pic in enumerate([step.source] + list(step.encodes)):
            for name in ("y", "u", "v"):
                np.save(os.path.join(d, f"f{f}_p{i}_{name}.npy"), getattr(pic, name))
    return f


def cpu_strip(args):
    """A horizontal strip of frame step CPU_FRAME through the CPU oracle (the reference's algorithm restated in C):
    CAMBI of the source and of each encode (with the whole picture's window), window figures, lasting-texture figures
    over 13 real source frames, PSNR squared errors and color sums, then the host collect of the window and lasting
    figures into per-segment accumulators. Returns (frame pairs measured, as a fraction of whole pictures; seconds)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    wl_name, d, row0, rows = args
    wl = WORKLOADS[wl_name]
    f, n_enc, pd = CPU_FRAME, wl["n_enc"], wl["pd"]
    r0, r1 = row0, min(row0 + rows, wl["h"])

    def plane(frame, pic, name):
        a = np.load(os.path.join(d, f"f{frame}_p{pic}_{name}.npy"), mmap_mode="r")
        c = 1 if name == "y" else 2
        return np.ascontiguousarray(a[r0 // c:r1 // c])

    src = [plane(f, 0, n) for n in ("y", "u", "v")]
    encs = [[plane(f, 1 + e, n) for n in ("y", "u", "v")] for e in range(n_enc)]
    ring = [plane(k, 0, "y") for k in range(f - 12, f + 1)]
    centre = [plane(f - 6, 1 + e, "y") for e in range(n_enc)]
    up = 10 - pd
    p = oracle.cambi_params(wl["w"], wl["h"])
    acc = [oracle.Accum() for _ in range(n_enc)]
    t0 = time.perf_counter()
    oracle.cambi(src[0], pd, p)
    oracle.color_sums(src[1], src[2], up)
    for e in range(n_enc):
        y, u, v = encs[e]
        oracle.cambi(y, pd, p)
        _, st = oracle.window_stats(src[0], y, up)
        _, ps = oracle.persist_stats(ring, centre[e], up)
        for a, b in ((src[0], y), (src[1], u), (src[2], v)):
            oracle.plane_sse(a, b)
        oracle.color_sums(u, v, up)
        mask = oracle.collect_frame(acc[e], st)
        oracle.collect_lasting(acc[e], ps, mask)
    return n_enc * (r1 - r0) / wl["h"], time.perf_counter() - t0


class CpuSampler:
    """Spawned processes on the host cores timing strips of a real frame step (generated once by the same processes
    and kept in a temporary directory): one strip per process and round, side by side, for the all-core rate, and
    strips one at a time on one process for the 1-core rate."""

    def __init__(self, wl_name: str, processes: int):
        import multiprocessing as mp

        self.wl, self.n = wl_name, processes
        self.pool = mp.get_context("spawn").Pool(processes)
        self.dir = _cpu_frames_dir()
        self.pool.map(cpu_make_frame, [(wl_name, f, self.dir) for f in range(CPU_FRAME + 1)], chunksize=1)
        self.strips = WORKLOADS[wl_name]["h"] // STRIP_ROWS
        self.round = 0

    def sample(self) -> tuple[float, str]:
        """All cores: one strip per process in parallel (the strips of the step in turn); frame pairs / slowest."""
        jobs = [(self.wl, self.dir, ((self.round * self.n + i) % self.strips) * STRIP_ROWS, STRIP_ROWS) for i in range(self.n)]
        self.round += 1
        res = self.pool.map(cpu_strip, jobs, chunksize=1)
        busy = max(r[1] for r in res)
        pairs = sum(r[0] for r in res)
        return pairs / busy, f"{self.n} strips of {STRIP_ROWS} rows ({pairs:.3f} frame pairs) side by side, {busy:.2f} s"

    def sample_one_core(self, strips: int = 3) -> float:
        """One process, strips one after another: frame pairs / seconds."""
        pairs = secs = 0.0
        for i in range(strips):
            fp, t = self.pool.apply(cpu_strip, ((self.wl, self.dir, (i % self.strips) * STRIP_ROWS, STRIP_ROWS),))
            pairs += fp
            secs += t
        return pairs / secs

    def close(self):
        import shutil

        self.pool.close()
        self.pool.join()
        shutil.rmtree(self.dir, ignore_errors=True)


def cpu_baseline_line(args, cores: int, rounds: int, warmup: int = 1) -> dict:
    sampler = CpuSampler(args.workload, cores)
    try:
        for _ in range(warmup):
            sampler.sample()
        vals = [sampler.sample() for _ in range(rounds)]
        one = sampler.sample_one_core()
    finally:
        sampler.close()
    wl = WORKLOADS[args.workload]
    value = statistics.median(v for v, _ in vals)
    return {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "value_1_core": one, "rounds": [round(v, 4) for v, _ in vals],
            "sample": (f"frame step {CPU_FRAME} of {wl['desc']} in strips of {STRIP_ROWS} rows: CAMBI of every picture, window and "
                       "lasting-texture figures over 13 real source frames, PSNR, color and the host collect; median of "
                       f"{rounds} rounds of {vals[-1][1]}; value_1_core: 3 strips one after another on one process")}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_config(wl: dict, world: int) -> dict:
    """The workload's config, the same in both arms."""
    return {"workload": wl["desc"], "frame_pairs_per_step": wl["n_enc"],
            "l2": "inputs larger than L2: distinct frame steps of ~100 MB input cycled", "parallelism": f"replicas x{world}"}


def reference_arm(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    cores = host_cores()
    wl = WORKLOADS[args.workload]
    sampler = CpuSampler(args.workload, cores)
    for _ in range(args.warmup):
        sampler.sample()
    values, sample = [], ""
    t0 = time.perf_counter()
    for _ in range(args.steps):
        v, sample = sampler.sample()
        values.append(v)
    wall = time.perf_counter() - t0
    sampler.close()
    value = statistics.median(values)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * wall / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u16/int64", "data": "synthetic (seeded es_synth frames, no video decode)",
            "config": run_config(wl, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": (f"each step: {sample} of frame step {CPU_FRAME} (CAMBI, window and lasting figures over "
                                        "13 real source frames, PSNR, color, host collect)")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's CPU path for CAMBI is libvmaf and for texture its numpy module; neither runs on the GPU hosts, "
                    "so the plain-C oracle restating the reference's algorithm stands in, over all host cores"}
    print(json.dumps(line), flush=True)


def run_c3(args, rank: int, world: int, local: int, module=None, quiet: bool = False) -> dict | None:
    """The uneven batch: 16 source / encode pairs per frame step (6 x 1280x720 8-bit, 6 x 1920x800 10-bit cropped from
    1920x1080 frames with black bars, 4 x 3840x1600 10-bit; es_synth.c3_step), scored as 16 plain es_frame instances
    and as one es_batch (one launch per stage for all 32 pictures, graphs from frame 14, autotuned tiles). Device-
    resident inputs, pool of 2 distinct steps (1.1 GB, larger than L2); time on the device with CUDA events."""
    import numpy as np
    import torch

    import es_b200
    import es_synth

    from concurrent.futures import ThreadPoolExecutor

    torch.cuda.set_device(local)
    srcs = es_synth.C3_SOURCES
    with ThreadPoolExecutor(max_workers=min(16, host_cores())) as ex:
        made = {(f, i): ex.submit(es_synth.c3_step, f, i, w, h, d) for f in range(2) for i, (w, h, d) in enumerate(srcs)}
        made = {k: v.result() for k, v in made.items()}
    pool = []
    for f in range(2):
        step = []
        for i, (w, h, d) in enumerate(srcs):
            st = made[(f, i)]
            fw, fh = es_synth.C3_BARS.get((w, h), (w, h))
            y0 = ((fh - h) // 2) & ~1
            pics = []
            for pic in [st.source] + st.encodes:
                Y = np.zeros((fh, fw), np.uint16)
                Y[y0:y0 + h] = pic.y
                U = np.full((fh // 2, fw // 2), 0, np.uint16)
                V = U.copy()
                U[y0 // 2:y0 // 2 + h // 2], V[y0 // 2:y0 // 2 + h // 2] = pic.u, pic.v
                t = [torch.from_numpy(a.view(np.int16)).cuda() for a in (Y, U, V)]
                pics.append((t, es_b200.FrameView(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), fw * 2, fw, 0, 2, 0, d), y0))
            step.append(pics)
        pool.append(step)
    torch.cuda.synchronize()
    own_module = module is None
    if own_module:
        module = es_b200.Module()
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    pairs = len(srcs) * args.steps

    def timed(queue, collect):
        f = 0
        with torch.cuda.stream(stream):
            for _ in range(max(args.warmup, 28)):
                queue(f)
                collect(f)
                f += 1
            torch.cuda.synchronize()
            l0 = es_b200.launch_count()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for k in range(args.steps):
                queue(f)
                if k:
                    collect(f - 1)
                f += 1
            collect(f - 1)
            b.record(stream)
            b.synchronize()
        return a.elapsed_time(b), es_b200.launch_count() - l0

    frames = [es_b200.Frame(module, w, h, d, 1) for (w, h, d) in srcs]
    accs = [[es_b200.new_accum()] for _ in srcs]

    def q_plain(f):
        step = pool[f % 2]
        for i, fr in enumerate(frames):
            (ts, vs, ys), (te, ve, ye) = step[i]
            fr.queue(f, vs, [ve], sh, sx=0, sy=ys, ex=[0], ey=[ye])

    def c_plain(f):
        for i, fr in enumerate(frames):
            fr.collect(f, accs[i], accs[i])

    ms_plain, l_plain = timed(q_plain, c_plain)
    for fr in frames:
        fr.close()
    batch = es_b200.Batch(module, [(w, h, d, 1) for (w, h, d) in srcs])
    acc = [es_b200.new_accum() for _ in srcs]

    def q_batch(f):
        step = pool[f % 2]
        views = [p[1] for pics in step for p in pics]
        crops = [(0, p[2]) for pics in step for p in pics]
        batch.queue(f, views, sh, crops=crops)

    def c_batch(f):
        batch.collect(f, acc, acc)

    ms_b, l_b = timed(q_batch, c_batch)
    graphs = batch.graph_launches()
    batch.close()
    if own_module:
        module.close()
    if rank == 0:
        line = {"metric": "frame-pairs/s, 16 uneven source/encode pairs per frame step", "value": pairs / (ms_b / 1000.0),
                "unit": "frame-pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u16/int64",
                "data": "synthetic (seeded es_synth c3 frames)",
                "config": {"workload": "6 x 1280x720 8-bit, 6 x 1920x800 10-bit (cropped from 1920x1080 with bars), 4 x 3840x1600 10-bit",
                           "frame_pairs_per_step": len(srcs), "l2": "2 distinct steps of 1.1 GB input cycled",
                           "form": "batched (es_batch, graphs, autotuned c-value tiles)"},
                "forms": {"plain": {"value": pairs / (ms_plain / 1000.0), "ms_per_step": ms_plain / args.steps, "gpu_launches": int(l_plain)},
                          "batched": {"value": pairs / (ms_b / 1000.0), "ms_per_step": ms_b / args.steps, "gpu_launches": int(l_b),
                                      "graph_steps": int(graphs)}}}
        if not quiet:
            print(json.dumps(line), flush=True)
        return line
    return None


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["c3"], default="c2")
    ap.add_argument("--pool", type=int, default=6, help="distinct frame steps cycled through")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--only-head", action="store_true", help="time only the headline form (for profiling runs)")
    ap.add_argument("--no-graphs", action="store_true", help="batched forms launch every kernel (for profiling runs)")
    ap.add_argument("--no-c3", action="store_true", help="skip the 16-pair uneven batch figures")
    ap.add_argument("--profile", type=int, default=0, metavar="N",
                    help="profiling run: N untimed frame steps of the headline form, every kernel its own launch, then exit")
    ap.add_argument("--form", choices=["plain", "batched", "learned"], default=None, help="the form --profile runs")
    ap.add_argument("--budget", type=float, default=None, help="learned form: score budget of skipped tiles (default: the network's)")
    ap.add_argument("--tolerance", type=float, default=None, help="learned form: audit tolerance (default: the network's)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    if args.workload == "c3":
        run_c3(args, rank, world, local)
        return

    import numpy as np
    import torch

    import es_b200

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    wl = WORKLOADS[args.workload]
    w, h, pd, n_enc = wl["w"], wl["h"], wl["pd"], wl["n_enc"]
    pool = make_pool(wl, args.pool, source=rank)
    stream = torch.cuda.Stream()
    # device-resident frames (planar 16-bit)
    dev_pool = []
    for step in pool:
        pics = []
        for pic in [step.source] + step.encodes:
            t = [torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda() for a in (pic.y, pic.u, pic.v)]
            pics.append((t, es_b200.FrameView(t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), w * 2, w, 0, 2, 0, pic.depth)))
        dev_pool.append(pics)
    torch.cuda.synchronize()
    module = es_b200.Module()

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident legs: the plain form (es_frame) and the batched form (es_batch, CUDA graphs) -------------
    class PlainForm:
        name = "plain (es_frame queue/collect, one launch set per picture, CAMBI on per-picture streams)"

        def __init__(self):
            self.fr = es_b200.Frame(module, w, h, pd, n_enc)

        def queue(self, f, pics, sh):
            self.fr.queue(f, pics[0], pics[1:], sh)

        def collect(self, f, acc):
            self.fr.collect(f, acc, acc)

        def close(self):
            self.fr.close()

    class BatchedForm:
        name = "batched (es_batch: one launch per stage for all pictures, steps replayed from CUDA graphs)"

        def __init__(self):
            self.b = es_b200.Batch(module, [(w, h, pd, n_enc)], use_graphs=not args.no_graphs)

        def queue(self, f, pics, sh):
            self.b.queue(f, pics, sh)

        def collect(self, f, acc):
            self.b.collect(f, acc, acc)

        def close(self):
            self.b.close()

    class LearnedForm(BatchedForm):
        def __init__(self):
            super().__init__()
            import eval_proposal
            self.net, meta = eval_proposal.load_net(es_b200)
            self.threshold = meta["threshold"]
            self.budget = meta.get("skip_budget", 0.0) if args.budget is None else args.budget
            self.tolerance = meta.get("tolerance", 0.025) if args.tolerance is None else args.tolerance
            self.b.set_proposal(self.net, threshold=self.threshold, tolerance=self.tolerance, budget=self.budget)
            skip = (f"tiles predicted below {self.threshold:g}" +
                    (f" or, per picture, predicted to add at most {self.budget:g} to CAMBI" if self.budget else ""))
            self.name = ("batched + learned proposal (es_batch with es_batch_set_proposal: c-values of scales 0-1 skip the "
                         f"{skip}, except a 5%/20% audit; fallback to every tile above an estimated {self.tolerance:g} "
                         "change of CAMBI)")

        def close(self):
            super().close()
            self.net.close()

    def time_form(form, f0: int) -> tuple[float, int, dict | None, int]:
        """Warm-up, then args.steps timed steps of `form` over the device pool; returns (ms, launches, clocks, next f).
        The warm-up runs frames 0-27, so the batched forms have captured the graph of each of the 14 ring phases and only
        replay graphs in the timed region."""
        acc = [es_b200.new_accum() for _ in range(n_enc)]
        f = f0
        with torch.cuda.stream(stream):
            sh = stream.cuda_stream
            for _ in range(max(args.warmup, 28)):
                p = dev_pool[f % len(dev_pool)]
                form.queue(f, [x[1] for x in p], sh)
                form.collect(f, acc)
                f += 1
            barrier()
            torch.cuda.synchronize()
            clocks = Clocks(local)
            clocks.start()
            time.sleep(0.25)
            launches0 = es_b200.launch_count()
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for k in range(args.steps):
                p = dev_pool[f % len(dev_pool)]
                form.queue(f, [x[1] for x in p], sh)
                if k > 0:
                    form.collect(f - 1, acc)
                f += 1
            form.collect(f - 1, acc)
            end.record(stream)
            end.synchronize()
            launches = es_b200.launch_count() - launches0
            clk = clocks.stop()
        return max_over_ranks(start.elapsed_time(end)), launches, clk, f

    if args.profile:
        # a short run for a profiler: no timing, no graphs (each kernel is its own launch), two distinct steps
        args.no_graphs = True
        have = os.path.exists(os.path.join(ROOT, "encode-score_b200", "proposal_net.npy"))
        which = args.form or ("learned" if have else "batched")
        form = {"plain": PlainForm, "batched": BatchedForm, "learned": LearnedForm}[which]()
        acc = [es_b200.new_accum() for _ in range(n_enc)]
        with torch.cuda.stream(stream):
            res = []
            for f in range(args.profile):
                p = dev_pool[f % len(dev_pool)]
                form.queue(f, [x[1] for x in p], stream.cuda_stream)
                res = form.collect(f, acc) or res
        torch.cuda.synchronize()
        form.close()
        module.close()
        print(f"profile run: {args.profile} frame steps of the {which} form", flush=True)
        return

    pairs = args.steps * n_enc * world
    forms = {}
    have_net = os.path.exists(os.path.join(ROOT, "encode-score_b200", "proposal_net.npy"))
    if not (args.only_head and have_net):
        plain = PlainForm()
        ms_plain, launches_plain, clk_plain, f = time_form(plain, 0)
        forms["plain"] = {"value": pairs / (ms_plain / 1000.0), "ms_per_step": ms_plain / args.steps, "form": plain.name,
                          "gpu_launches": int(launches_plain)}
        plain.close()
        batched = BatchedForm()
        ms_b, launches_b, clk, _ = time_form(batched, 0)
        batched.close()
        forms["batched"] = {"value": pairs / (ms_b / 1000.0), "ms_per_step": ms_b / args.steps, "form": batched.name,
                            "gpu_launches": int(launches_b)}
        head = "batched"
        ms, launches = ms_b, launches_b
    if have_net:
        learned = LearnedForm()
        ms_l, launches_l, clk, _ = time_form(learned, 0)
        learned.close()
        forms["learned"] = {"value": pairs / (ms_l / 1000.0), "ms_per_step": ms_l / args.steps, "form": learned.name,
                            "gpu_launches": int(launches_l), "threshold": learned.threshold, "budget": learned.budget,
                            "tolerance": learned.tolerance}
        head = "learned"
        ms, launches = ms_l, launches_l
    value = forms[head]["value"]

    # ---- per-kernel leg: one pass over the pool with every kernel alone on the stream, each bracketed by events -
    # (in the timed region kernels of a step overlap, so an event pair there would also time its neighbours; kernel
    # timing also switches graph replay off, so each kernel is launched and timed on its own)
    kform = {"plain": PlainForm, "batched": BatchedForm, "learned": LearnedForm}[head]()
    kacc = [es_b200.new_accum() for _ in range(n_enc)]
    with torch.cuda.stream(stream):
        kf = 0
        for _ in range(14):
            p = dev_pool[kf % len(dev_pool)]
            kform.queue(kf, [x[1] for x in p], stream.cuda_stream)
            kform.collect(kf, kacc)
            kf += 1
        es_b200.kernel_timing(True, serial=True)
        for _ in range(len(dev_pool)):
            p = dev_pool[kf % len(dev_pool)]
            kform.queue(kf, [x[1] for x in p], stream.cuda_stream)
            kform.collect(kf, kacc)
            kf += 1
    times = es_b200.kernel_times()
    es_b200.kernel_timing(False)
    kform.close()
    kernel_steps = len(dev_pool)

    # ---- end-to-end leg: host frames, copies inside the timed region ------------------------------------------
    e2e = None
    if not args.no_e2e:
        # each step's twelve planes in one page-locked arena (each plane 256-byte aligned), copied with one
        # cudaMemcpyAsync per step: per-copy overheads of twelve small copies left the link idle between them
        plane_list = [(pic, a) for pic in [pool[0].source] + pool[0].encodes for a in (pic.y, pic.u, pic.v)]
        offsets, at = [], 0
        for _, a in plane_list:
            offsets.append(at)
            at += (a.size + 127) // 128 * 128
        arena_elems = at
        host_pool = []
        for step in pool:
            arena = torch.empty(arena_elems, dtype=torch.int16).pin_memory()
            planes = [a for pic in [step.source] + step.encodes for a in (pic.y, pic.u, pic.v)]
            for off, a in zip(offsets, planes):
                arena[off:off + a.size] = torch.from_numpy(np.ascontiguousarray(a).view(np.int16).ravel())
            host_pool.append(arena)
        # three input slots: step g + 1's copy is queued before step g - 1 is collected, so the copy stream never waits
        # for the host (with two slots and the copy queued after the collect, the host's collect time left the copy
        # engine idle for a fifth of each step)
        depth = 3
        slots = [torch.empty(arena_elems, dtype=torch.int16, device="cuda") for _ in range(depth)]
        views = []
        for slot in slots:
            base = slot.data_ptr()
            vs = []
            for k, pic in enumerate([pool[0].source] + pool[0].encodes):
                y, u, v = (base + 2 * offsets[3 * k + i] for i in range(3))
                vs.append(es_b200.FrameView(y, u, v, w * 2, w, 0, 2, 0, pic.depth))
            views.append(vs)
        h2d = sum(a.size * 2 for _, a in plane_list)  # the planes' bytes (the arena's alignment gaps are copied too)
        windows = (w // 16) * (h // 16)
        d2h = 8 * (3 * n_enc + 3 * (n_enc + 1)) + 136 * n_enc + 2 * 6 * windows * n_enc + 48 * (1 + n_enc)
        fr2 = {"plain": PlainForm, "batched": BatchedForm, "learned": LearnedForm}[head]()
        acc2 = [es_b200.new_accum() for _ in range(n_enc)]
        copy_stream = torch.cuda.Stream()
        copied = [torch.cuda.Event() for _ in range(depth)]
        free = [torch.cuda.Event() for _ in range(depth)]

        def copy_in(g):
            s = g % depth
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(free[s])  # the step that last read this slot is done
                slots[s].copy_(host_pool[g % len(host_pool)], non_blocking=True)
                copied[s].record(copy_stream)

        def e2e_step(g, g_first, g_end):
            """Step g of the run g_first .. g_end - 1: its frames' copy (queued one step ahead), its launches, and the
            collect of step g - 1."""
            s = g % depth
            if g == g_first:
                copy_in(g)
            if g + 1 < g_end:
                copy_in(g + 1)
            stream.wait_event(copied[s])
            fr2.queue(g, views[s], stream.cuda_stream)
            free[s].record(stream)
            if g > g_first:
                fr2.collect(g - 1, acc2)

        with torch.cuda.stream(stream):
            warm = max(args.warmup, 28)
            for g in range(warm):
                e2e_step(g, 0, warm)
            fr2.collect(warm - 1, acc2)
            barrier()
            torch.cuda.synchronize()
            t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t_start.record(stream)
            copy_stream.wait_event(t_start)
            g0 = warm
            for k in range(args.steps):  # exactly steps copies, steps launch sets and steps collects in the region
                e2e_step(g0 + k, g0, g0 + args.steps)
            fr2.collect(g0 + args.steps - 1, acc2)
            t_end.record(stream)
            t_end.synchronize()
        e2e_ms = max_over_ranks(t_start.elapsed_time(t_end))
        e2e = {"value": pairs / (e2e_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_ms / args.steps}
        fr2.close()

    # ---- roofline of the dominant kernel ------------------------------------------------------------------------
    peaks = read_peaks()
    total_kernel_ms = sum(v[0] for v in times.values()) or 1.0
    top = max(times, key=lambda k: times[k][0]) if times else None
    roofline = None
    if top:
        # per step: all launches of the kernel in one frame step (with the proposal the c-value kernel runs twice, the
        # second launch over the fallback tiles only), so bytes per step over the kernel's time per step
        ms_step = times[top][0] / kernel_steps
        launches_step = times[top][1] / kernel_steps
        alg = algorithmic_bytes(top, wl)
        achieved = alg / (ms_step / 1000.0) / 1e9 if alg else None
        step_bytes = step_algorithmic_bytes(wl)
        roofline = {"bound": "hbm", "kernel": top, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"] if achieved else None, "traffic": read_traffic(top, f"{args.workload}:{head}"),
                    "algorithmic_bytes_per_step": alg, "ms_per_step": ms_step, "launches_per_step": launches_step,
                    "peak_source": peaks["source"],
                    "step": {"algorithmic_bytes": step_bytes, "ms_per_step": ms / args.steps,
                             "achieved": step_bytes / (ms / args.steps / 1000.0) / 1e9,
                             "frac": step_bytes / (ms / args.steps / 1000.0) / 1e9 / peaks["hbm_gbs"]},
                    "issue": read_issue(top, f"{args.workload}:{head}")}
    kernels = {}
    for k, v in sorted(times.items(), key=lambda kv: -kv[1][0]):
        kms = v[0] / kernel_steps
        kb = algorithmic_bytes(k, wl)
        kernels[k] = {"ms_per_step": kms, "launches_per_step": v[1] / kernel_steps, "share": v[0] / total_kernel_ms,
                      "algorithmic_bytes_per_step": kb, "hbm_frac": kb / (kms / 1000.0) / 1e9 / peaks["hbm_gbs"] if kb else None}

    # ---- CPU baseline (rank 0, one GPU) -------------------------------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        os.environ.setdefault("OMP_NUM_THREADS", "1")
        cpu = cpu_baseline_line(args, host_cores(), rounds=5)

    # ---- the uneven batch (16 pairs per step): plain vs batched, as extra figures -------------------------------
    c3 = None
    if args.workload == "c2" and not args.no_c3 and not args.only_head:
        c3 = run_c3(args, rank, world, local, module=module, quiet=True)

    module.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "u16/int64", "data": "synthetic (seeded es_synth frames, no video decode)",
                "config": run_config(wl, world), "form": forms[head]["form"], "pool_steps": args.pool,
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": int(launches),
                "forms": forms, "kernels": kernels, "c3": c3}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
