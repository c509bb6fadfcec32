"""Benchmark of the B200 K-Litho SOCS imaging path.

Headline workload (the batched SOCS forward configuration): 384 seeded
random-rectangle binary clips -- 128 x 512^2, 192 x 1024^2, 64 x 2048^2,
1 nm pixels, 25-40 % density -- each imaged at 3 focus values with K = 24
kernels per focus (one kernel set per clip size and focus).  A step images
every clip at every focus once.  Metric: 1024^2-equivalent SOCS images per
second (total image pixels / 1024^2 / time).

`value` is device-resident throughput (masks already in HBM, images left in
HBM); `e2e` is the same metric through the public host entry point
(kl_socs_forward_host: pinned host masks in, host images out).  The roofline
object covers the kernel with the largest share of device time.
`--impl reference` times the reference's own CPU implementation of the path
(oracle/_ref, else the restated oracle) on the host cores instead.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "k-litho_b200"))
sys.path.insert(0, REPO)

METRIC = "1024^2-equivalent SOCS images/s"
UNIT = "images/s"
CLASSES = [(512, 128), (1024, 192), (2048, 64)]  # (clip size, clips)
FOCUS_NM = [-25.0, 0.0, 25.0]
NK = 24
SEED = 2024


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def peaks_tensor():
    """Dense bf16 TFLOP/s (burst figure: a kernel timed on its own)."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"])
    return 1590.0


def class_band(L):
    # the annular optics: annular 0.6/0.9 on 41^2, NA 1.35 (sigma_o = 0.9)
    import klitho as K
    src = K.createSource(41, "Annular", 0.6, 0.9)
    return K.bandSize(1.35, L, L, K.getOuterSigma(src))


def make_masks(L, n, seed):
    import synth
    rng = np.random.default_rng(seed)
    out = np.empty((n, L, L), dtype=np.float32)
    for i in range(n):
        out[i] = synth.rect_mask_fill(L, int(rng.integers(1 << 30)), float(rng.uniform(0.25, 0.40)))
    return out


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    Polls NVML every few milliseconds from a thread (so that even a timed
    region of some tens of milliseconds gets samples); falls back to
    `nvidia-smi -lms 200` where NVML cannot be loaded.  Only reads state."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, dev_index=0, period_s=0.004):
        self.dev = dev_index
        self.period = period_s
        self.proc = None
        self.th = None
        self.lines = []
        self.samples = []  # (sm_mhz, max_mhz, reasons bitmask)
        self._run = False
        self._nvml = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.dev)
            self._nvml = (pynvml, h)
            self._smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self._run = True
            self.th = threading.Thread(target=self._poll, daemon=True)
            self.th.start()
            return
        except Exception:
            self._nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except OSError:
            self.proc = None

    def _poll(self):
        pynvml, h = self._nvml
        while self._run:
            try:
                sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                rs = int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))
                self.samples.append((sm, self._smax, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def clear(self):
        self.lines.clear()
        self.samples.clear()

    def stop(self):
        if self._nvml is not None:
            self._run = False
            self.th.join(timeout=2)
            sm = [x[0] for x in self.samples]
            reasons = sorted(nm for nm, bit in self.REASONS.items() if any(x[2] & bit for x in self.samples))
            return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self._smax,
                    "reasons": reasons, "samples": len(sm), "source": "NVML polled every 4 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(max(smax)) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi -lms 200"}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch
    import klitho as K
    import synth

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    if ws > 1:
        print(f"[bench] rank {rank} of {ws} on cuda:{local}, communicator nccl "
              f"(world size {dist.get_world_size()}), {args.scaling} scaling", file=sys.stderr)

    # weak scaling: every rank images its own full batch (clips are independent);
    # strong scaling: the one batch is split over the ranks by shard.partition
    # (clips balanced by pixels), no collective on the data path
    full_px = sum(L * L * n * len(FOCUS_NM) for L, n in CLASSES)
    if args.scaling == "strong" and ws > 1:
        import shard
        sizes, cls_of = [], []
        for ci, (L, n) in enumerate(CLASSES):
            sizes += [L * L] * n
            cls_of += [ci] * n
        mine = shard.partition(sizes, ws)[rank]
        counts = [sum(1 for i in mine if cls_of[i] == ci) for ci in range(len(CLASSES))]
        CLASSES[:] = [(L, c) for (L, _), c in zip(CLASSES, counts) if c > 0]
    # kernel sets: the annular optics (annular 0.6/0.9 on 41^2, NA 1.35, water) at
    # each clip size and focus, K=24, from the GPU TCC + subspace iteration
    src = K.createSource(41, "Annular", 0.6, 0.9)
    plans, masks_d, imgs_d, masks_h, kset0, ksets = [], [], [], [], [], []
    for ci, (L, n) in enumerate(CLASSES):
        Nx, Ny = class_band(L)
        p = K.SocsPlan(L, L, Nx, Ny, NK, nsets=len(FOCUS_NM), max_clips=n)
        ksets_cur = []
        for s, f_nm in enumerate(FOCUS_NM):
            tp = K.TccPlan(src, 1.35, synth.defocus_arg(f_nm), L, L, n_medium=synth.N_WATER)
            krn, sc, _, _ = tp.topk(NK)
            tp.close()
            p.set_kernels(s, krn, sc)
            ksets_cur.append((krn, sc))
            if s == 0:
                kset0.append((krn, sc))
        m = make_masks(L, n, SEED + 1000 * ci + rank)
        masks_h.append(m)
        masks_d.append(torch.from_numpy(m).to(f"cuda:{local}"))
        imgs_d.append(torch.empty((n, len(FOCUS_NM), L, L), dtype=torch.float32,
                                  device=f"cuda:{local}"))
        plans.append(p)
        ksets.append(list(ksets_cur))
    px_per_step = sum(L * L * n * len(FOCUS_NM) for L, n in CLASSES)
    img_equiv = px_per_step / float(1024 * 1024)

    # launch shapes tuned per size class, then all classes in one graph whose
    # branches run concurrently (kl_socs_autotune + kl_socs_batch_forward);
    # the larger classes are split into CHUNKS plans over contiguous clip
    # ranges so that one chunk's on-chip stage overlaps another's memory-bound
    # stages
    tuned = [p.autotune(md, im, stream=stream) for p, md, im in zip(plans, masks_d, imgs_d)]
    bplans, bmasks, bimgs = [], [], []
    for (L, n), md, im, ks in zip(CLASSES, masks_d, imgs_d, ksets):
        nch = max(1, min(args.chunks if L >= 1024 else 1, n))
        Nx, Ny = class_band(L)
        for c in range(nch):
            a, b = n * c // nch, n * (c + 1) // nch
            bp = K.SocsPlan(L, L, Nx, Ny, NK, nsets=len(FOCUS_NM), max_clips=b - a)
            for si, (krn, sc) in enumerate(ks):
                bp.set_kernels(si, krn, sc)
            bp.autotune(md[a:b], im[a:b], stream=stream)
            bplans.append(bp)
            bmasks.append(md[a:b])
            bimgs.append(im[a:b])
    batch = K.SocsBatch(bplans)

    def step():
        batch.forward(bmasks, bimgs, stream=stream)

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks.clear()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    torch.cuda.nvtx.range_push("socs_timed")  # lets a profiler select the timed launches
    for _ in range(args.steps):
        step()
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    # per-kernel device time of the same tuned launches run one plan after
    # another (CUDA events on the launch stream): the kernels' own durations
    for p in plans:
        p.enable_timing(True)
    tsteps = min(args.steps, 20)
    for _ in range(tsteps):
        for p, md, im in zip(plans, masks_d, imgs_d):
            p.forward(md, im, stream=stream)
    stage_ms = np.zeros(3)
    stage_n = np.zeros(3, dtype=int)
    per_class = []
    for (L, n), p, (ns, spc) in zip(CLASSES, plans, tuned):
        t, c = p.stage_times()
        stage_ms += np.array(t)
        stage_n += np.array(c)
        per_class.append({"L": L, "clips": n, "fwd_ms": t[0] / max(c[0], 1), "spectral_ms": t[1] / max(c[1], 1),
                          "synthesis_ms": t[2] / max(c[2], 1), "tuned_kernel_slices": ns,
                          "tuned_strips_per_cta": spc, "synthesis": p.synthesis(n)})
        p.enable_timing(False)
    # ... and their spans inside the graph, where the size classes overlap
    # (stage events captured into a separate graph)
    batch.enable_timing(True)
    spans = [np.zeros(3) for _ in bplans]
    for _ in range(tsteps):
        step()
        for i in range(len(bplans)):
            spans[i] += np.array(batch.stage_times(i))
    branches = [{"L": bp.Lx, "clips": int(bm.shape[0]), "span_ms": [round(x / tsteps, 4) for x in sp]}
                for bp, bm, sp in zip(bplans, bmasks, spans)]
    batch.enable_timing(False)
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / args.steps
    # whole-job rate: every rank's pixels over the slowest rank's time
    total_equiv = (full_px / float(1024 * 1024)) if (args.scaling == "strong" and ws > 1) else img_equiv * ws
    value = total_equiv / (ms_per_step / 1e3)

    # roofline of the dominant kernel (largest share of device time)
    names = ["socs_forward", "socs_spectral", "socs_synthesis"]
    dom = int(np.argmax(stage_ms))
    bytes_per_step = [sum(4 * L * L * n for L, n in CLASSES),
                      0,
                      sum(4 * L * L * n * len(FOCUS_NM) for L, n in CLASSES)]
    launches_per_step = len(CLASSES)
    avg_launch_ms = stage_ms[dom] / max(stage_n[dom], 1)
    peak, peak_kind = peaks()
    roof = None
    if bytes_per_step[dom] > 0:
        achieved = bytes_per_step[dom] / launches_per_step / (avg_launch_ms / 1e3) / 1e9
        roof = {"kernel": names[dom], "bound": "hbm", "achieved": round(achieved, 1),
                "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": (int(TRAFFIC_PER_ALGORITHMIC_BYTE[names[dom]] * bytes_per_step[dom] / launches_per_step)
                            if names[dom] in TRAFFIC_PER_ALGORITHMIC_BYTE else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the k_socs_synth_tc "
                                  "captures at 2048^2 and 1024^2 (the ncu summaries of k_socs_synth_tc), scaled by pixels",
                "kernels": sorted({("k_socs_synth_tc" if c["synthesis"] == "tensor" else "k_socs_inverse")
                                   for c in per_class}),
                "algorithmic_bytes_per_launch": int(bytes_per_step[dom] / launches_per_step)}
    else:
        roof = {"kernel": names[dom], "bound": "compute", "achieved": None, "peak": None,
                "unit": None, "frac": None, "traffic": None}
    if roof.get("achieved") is not None:
        # the whole overlapped step: every algorithmic byte over the step time
        step_gbs = (bytes_per_step[0] + bytes_per_step[2]) / (ms_per_step / 1e3) / 1e9
        roof["timing"] = ("kernel durations from CUDA events around each launch of the tuned shapes run "
                          "one plan after another; in the timed graph the size classes overlap")
        roof["step_algorithmic_GBps"] = round(step_gbs, 1)
        roof["step_frac"] = round(step_gbs / peak, 4)
    # the other streaming kernel too, for context
    other = {names[i]: {"ms_per_step": round(stage_ms[i] / max(stage_n[i], 1) * len(CLASSES), 4)} for i in range(3)}
    for i in (0, 2):
        if stage_n[i]:
            lps = len(CLASSES)
            bw = bytes_per_step[i] / lps / (stage_ms[i] / stage_n[i] / 1e3) / 1e9
            other[names[i]]["GBps"] = round(bw, 1)
            other[names[i]]["frac_of_peak"] = round(bw / peak, 4)

    # end-to-end through the host entry point (pinned host buffers)
    e2e = None if args.no_e2e else run_e2e(plans, masks_h, args, total_equiv / img_equiv, img_equiv)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(max_seconds=args.cpu_seconds)

    fp64 = None
    if not args.no_secondary:
        fp64 = fp64_baseline(masks_d, imgs_d, kset0, value / ws, img_equiv)

    batch.close()
    for bp in bplans:
        bp.close()
    secondary = {}
    if not args.no_secondary:
        for p in plans:
            p.close()
        plans = []
        del masks_d, imgs_d
        torch.cuda.empty_cache()
        secondary["fwd_adj"] = bench_fwd_adj(args, stream, peaks()[0])
        secondary["socs_4096"] = bench_socs_4096(args, stream, peaks()[0])
        torch.cuda.empty_cache()
        secondary["fwd_adj_4096"] = bench_fwd_adj_4096(args, stream, peaks()[0])
        torch.cuda.empty_cache()
        secondary["tcc_eigen"] = bench_tcc_eigen(args)
        secondary["tcc_eigen_large"] = bench_tcc_eigen_large(args)
        secondary["tcc_gemm"] = bench_tcc_gemm(args)

    if rank == 0:
        out = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": args.scaling if ws > 1 else "weak", "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded random-rectangle masks; kernels from the GPU TCC + "
                    "subspace iteration of the annular NA 1.35 optics, K=24 per size and focus)",
            "config": dict(workload_config(),
                           **{"image_equiv_1024_per_step_per_gpu": img_equiv,
                              "l2": "inputs larger than L2 (1.9 GB masks, 5.8 GB images per GPU)",
                              "parallelism": f"clip sharding ({args.scaling if ws > 1 else 'weak'}), {ws} GPU(s), "
                                             f"no collective on the data path"}),
            "roofline": roof, "stages": other, "per_class": per_class, "graph_branches": branches,
            "image_err_vs_fp64_of_clear_field": (fp64 or {}).get("image_max_err_of_clear_field"),
            "clocks": clk, "e2e": e2e,
            "gpu_launches": int(3 * len(bplans) * args.steps),
            "cpu_baseline": cpu,
            "fp64_gpu_baseline": fp64,
            "secondary": secondary,
        }
        print(json.dumps(out))
    for p in plans:
        p.close()
    if dist:
        dist.destroy_process_group()


# DRAM bytes per algorithmic byte measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum): tensor-core synthesis on 48 x 2048^2 + 144 x 1024^2
# images, forward on 48 clips of 1024^2; both kernels stream their clip data
# once, so traffic scales with the pixels of a launch.
TRAFFIC_PER_ALGORITHMIC_BYTE = {"socs_synthesis": (5.847 + 746.890 + 3.649 + 546.218) / (805.31 + 603.98),
                                "socs_forward": (201.372 + 4.389) / 201.33}


def clear_field(krn, sc, Nx, Ny):
    """Clear-field intensity of a kernel set: sum_k lambda_k |H_k(0)|^2."""
    c = (2 * Ny + 1) * (2 * Nx + 1) // 2
    return float(np.sum(np.asarray(sc, np.float64) * np.abs(np.asarray(krn)[:, c].astype(np.complex128)) ** 2))


def fp64_baseline(masks_d, imgs_d, kset0, value_per_gpu, img_equiv):
    """The plain FP64 GPU path (kl_fp64_socs_forward: full FP64 FFTs, K fields
    materialised) on 8 clips of each size class (4 of 2048^2) with one kernel
    set, timed with CUDA events after a warm-up call; its 1024^2-equivalent
    rate for the same mixed workload (every clip x every focus) is the
    baseline of the fused path.  The same FP64 images give the error of the
    timed workload's images (kernel set 0) as max |fused - FP64| over the
    clear-field intensity."""
    import torch
    import klitho as K
    t_clip, errs = [], []
    for (L, n), md, im, (krn, sc) in zip(CLASSES, masks_d, imgs_d, kset0):
        Nx, Ny = class_band(L)
        kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
        sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
        nf = 4 if L >= 2048 else 8
        m = md[:nf]
        out = torch.empty((nf, L, L), dtype=torch.float64, device="cuda")
        K.fp64_socs_forward(m, Nx, Ny, kd, sd, out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(2):
            K.fp64_socs_forward(m, Nx, Ny, kd, sd, out)
        e1.record()
        torch.cuda.synchronize()
        t_clip.append(e0.elapsed_time(e1) / (2 * nf) / 1e3)
        cf = clear_field(krn, sc, Nx, Ny)
        errs.append(float((im[:nf, 0].double() - out).abs().max()) / cf)
        del out
    step_s = sum(t * n * len(FOCUS_NM) for t, (L, n) in zip(t_clip, CLASSES))
    rate = img_equiv / step_s
    return {"value": round(rate, 2), "unit": UNIT, "speedup_of_fused_path": round(value_per_gpu / rate, 2),
            "seconds_per_clip": {str(L): round(t, 6) for t, (L, n) in zip(t_clip, CLASSES)},
            "image_max_err_of_clear_field": max(errs) if errs else None,
            "image_err_per_class": {str(L): e for e, (L, n) in zip(errs, CLASSES)},
            "sample": "8 clips per size class (4 of 2048^2), one focus, 2 passes after a warm-up call, "
                      "CUDA events; step time = sum over classes of clips x focus x seconds per clip"}


def bench_fwd_adj(args, stream, peak_gbs):
    """Differentiable SOCS: 32 clips of 1024^2, continuous masks (smooth noise
    through a sigmoid), binary rectangle targets, K = 24, loss
    sum (sigmoid(50 (I - 0.225)) - target)^2; a step is one forward + adjoint
    (image, loss and dL/dmask written).  16 B/px of algorithmic traffic."""
    import torch
    import klitho as K
    import synth
    L, n, nk = 1024, (args.clips if args.part == "fwd_adj" and args.clips else 32), 24
    src = K.createSource(41, "Annular", 0.6, 0.9)
    tp = K.TccPlan(src, 1.35, 0.0, L, L, n_medium=synth.N_WATER)
    krn, sc, _, _ = tp.topk(nk)
    plan = K.SocsPlan(L, L, tp.Nx, tp.Ny, nk, max_clips=n, adjoint=True)
    plan.set_kernels(0, krn, sc)
    masks = torch.from_numpy(np.stack([synth.smooth_mask(L, seed=100 + i) for i in range(n)])).cuda()
    tgts = torch.from_numpy(np.stack([synth.rect_mask(L, 60, seed=200 + i) for i in range(n)])).cuda()
    grad = torch.empty_like(masks)
    img = torch.empty((n, 1, L, L), dtype=torch.float32, device="cuda")
    loss = torch.empty(n, dtype=torch.float64, device="cuda")
    steps = max(10, min(args.steps, 100))
    for _ in range(3):
        plan.vjp(masks, tgts, grad, loss, img, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.vjp(masks, tgts, grad, loss, img, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    bytes_step = 16 * L * L * n
    gbs = bytes_step / (ms / 1e3) / 1e9
    # source-weight gradient through the TCC factor (one call over all clips)
    gs = torch.zeros(src.size, dtype=torch.float32, device="cuda")
    t0 = time.perf_counter()
    plan.vjp_source(tp, gs)
    src_ms = (time.perf_counter() - t0) * 1e3
    # plain FP64 GPU path on 8 of the clips (same loss, one kernel set)
    nf = min(8, n)
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
    sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
    g64 = torch.empty((nf, L, L), dtype=torch.float64, device="cuda")
    l64 = torch.empty(nf, dtype=torch.float64, device="cuda")
    K.fp64_socs_vjp(masks[:nf], tgts[:nf], tp.Nx, tp.Ny, kd, sd, g64, l64)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(3):
        K.fp64_socs_vjp(masks[:nf], tgts[:nf], tp.Nx, tp.Ny, kd, sd, g64, l64)
    f1.record()
    torch.cuda.synchronize()
    fp64_rate = 3 * nf / (f0.elapsed_time(f1) / 1e3)
    gerr = float((grad[:nf].double() - g64).abs().max() / g64.abs().max())
    plan.close()
    tp.close()
    value = n / (ms / 1e3)
    return {"metric": "1024^2 fwd+adj grads/s", "value": round(value, 2),
            "unit": "grads/s", "ms_per_step": round(ms, 4), "clips_per_step": n, "K": nk,
            "GBps_algorithmic": round(gbs, 1), "frac_of_hbm_peak": round(gbs / peak_gbs, 4),
            "source_gradient_ms": round(src_ms, 3), "S": tp.S,
            "fp64_gpu_grads_per_s": round(fp64_rate, 2), "speedup_vs_fp64_gpu": round(value / fp64_rate, 2),
            "grad_max_err_vs_fp64_rel": gerr,
            "fp64_sample": f"{nf} of the clips, 3 passes, CUDA events (kl_fp64_socs_vjp)",
            "gpu_launches_per_step": 6}


QUAD4096 = dict(srcSize=81, kind="CrossQuadrupole", radius=0.12, offset=0.75)
FOCUS4096_NM = [-50.0, -25.0, 0.0, 25.0, 50.0]


def quad4096_kernels(nk=64):
    """K kernels per focus of the stress configuration (4096^2, cross-quadrupole
    0.75/0.12 on 81^2, NA 1.35 water) from the library's TCC + eigen path."""
    import klitho as K
    import synth
    src = K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75)
    sets = []
    for f_nm in FOCUS4096_NM:
        tp = K.TccPlan(src, 1.35, synth.defocus_arg(f_nm), 4096, 4096, n_medium=synth.N_WATER)
        krn, sc, _, _ = tp.topk(nk)
        Nx, Ny = tp.Nx, tp.Ny
        tp.close()
        sets.append((krn, sc))
    return src, Nx, Ny, sets


def smooth_masks_gpu(L, n, seed, sigma_px=12.0, gain=6.0):
    """Continuous masks in [0, 1] (Gaussian-filtered noise through a sigmoid,
    the construction of synth.smooth_mask) generated on the device, so that
    4096^2 inputs take no CPU minutes; setup only, never timed."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    f = torch.fft.fftfreq(L, dtype=torch.float64, device="cuda")
    filt = torch.exp(-2.0 * (np.pi * sigma_px) ** 2 * (f[:, None] ** 2 + f[None, :] ** 2))
    out = torch.empty((n, L, L), dtype=torch.float32, device="cuda")
    for i in range(n):
        noise = torch.randn((L, L), generator=g, dtype=torch.float64).cuda()
        sm = torch.fft.ifft2(torch.fft.fft2(noise) * filt).real
        sm /= sm.std() + 1e-30
        out[i] = torch.sigmoid(gain * sm).float()
    return out


def stage_report(plan):
    t, c = plan.stage_times()
    return [x / max(n, 1) for x, n in zip(t, c)]


def bench_socs_4096(args, stream, peak_gbs):
    """Stress configuration, forward: 16 seeded 4096^2 random-rectangle clips
    (25-40 % density) at 5 focus values, K = 64 kernels per focus (N = 11449,
    SOCS grid 213: the general pipeline).  A step images every clip at every
    focus; algorithmic traffic 4 B per mask pixel + 4 B per image pixel.  The
    error of clip 0 at focus 0 against the plain FP64 GPU path
    (kl_fp64_socs_forward) is reported as a fraction of clear field, and that
    path's time per image is the baseline."""
    import torch
    import klitho as K
    L, n, nk = 4096, (args.clips if args.part == "socs_4096" and args.clips else 16), 64
    nf = len(FOCUS4096_NM)
    _, Nx, Ny, sets = quad4096_kernels(nk)
    plan = K.SocsPlan(L, L, Nx, Ny, nk, nsets=nf, max_clips=n)
    for i, (k, sc) in enumerate(sets):
        plan.set_kernels(i, k, sc)
    masks = torch.from_numpy(make_masks(L, n, SEED + 4096)).cuda()
    imgs = torch.empty((n, nf, L, L), dtype=torch.float32, device="cuda")
    for _ in range(3):
        plan.forward(masks, imgs, stream=stream)
    torch.cuda.synchronize()
    steps = max(3, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.forward(masks, imgs, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    plan.enable_timing(True)
    for _ in range(3):
        plan.forward(masks, imgs, stream=stream)
    st = stage_report(plan)
    plan.enable_timing(False)
    px = L * L
    bytes_step = 4 * px * n + 4 * px * n * nf
    gbs = bytes_step / (ms / 1e3) / 1e9
    syn_gbs = 4 * px * n * nf / (st[2] / 1e3) / 1e9
    # FP64 GPU path on clip 0, focus 0
    krn, sc = sets[2]
    kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
    sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
    out = torch.empty((1, L, L), dtype=torch.float64, device="cuda")
    K.fp64_socs_forward(masks[:1], Nx, Ny, kd, sd, out)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    K.fp64_socs_forward(masks[:1], Nx, Ny, kd, sd, out)
    f1.record()
    torch.cuda.synchronize()
    t64 = f0.elapsed_time(f1) / 1e3
    err = float((imgs[0, 2].double() - out[0]).abs().max()) / clear_field(krn, sc, Nx, Ny)
    plan.close()
    del masks, imgs, out
    rate = n * nf / (ms / 1e3)
    return {"metric": "4096^2 SOCS images/s (16 clips x 5 focus, K=64)", "value": round(rate, 2),
            "unit": "images/s", "ms_per_step": round(ms, 3), "clips": n, "focus": nf, "K": nk,
            "N": (2 * Nx + 1) * (2 * Ny + 1), "engine": "general",
            "GBps_algorithmic": round(gbs, 1), "frac_of_hbm_peak": round(gbs / peak_gbs, 4),
            "stage_ms": {"row_and_column_forward": round(st[0], 4), "spectral": round(st[1], 4),
                         "column_and_row_synthesis": round(st[2], 4)},
            "synthesis_GBps": round(syn_gbs, 1), "synthesis_frac_of_hbm_peak": round(syn_gbs / peak_gbs, 4),
            "image_max_err_of_clear_field_vs_fp64": err,
            "fp64_gpu_images_per_s": round(1.0 / t64, 3), "speedup_vs_fp64_gpu": round(rate * t64, 2),
            "timing": f"CUDA events over {steps} steps after 3 warm-up steps; stages from per-launch events"}


def bench_fwd_adj_4096(args, stream, peak_gbs):
    """Stress configuration, forward + adjoint: 16 seeded 4096^2 continuous
    clips (smooth noise through a sigmoid) with binary rectangle targets at 5
    focus values, K = 64; loss sum over focus of
    sum (sigmoid(50 (I - 0.225)) - target)^2, gradient dL/dmask summed over
    focus.  Algorithmic traffic per clip pixel: mask, target read and gradient
    written (12 B) plus 4 B per image pixel written.  Checked against the plain
    FP64 GPU path (kl_fp64_socs_vjp, clip 0, the 5 focus values summed)."""
    import torch
    import klitho as K
    import synth
    L, n, nk = 4096, (args.clips if args.part == "fwd_adj_4096" and args.clips else 16), 64
    nf = len(FOCUS4096_NM)
    _, Nx, Ny, sets = quad4096_kernels(nk)
    plan = K.SocsPlan(L, L, Nx, Ny, nk, nsets=nf, max_clips=n, adjoint=True)
    for i, (k, sc) in enumerate(sets):
        plan.set_kernels(i, k, sc)
    masks = smooth_masks_gpu(L, n, SEED + 44)
    rng = np.random.default_rng(SEED + 45)
    tgts = torch.from_numpy(np.stack([synth.rect_mask_fill(L, int(rng.integers(1 << 30)), 0.3)
                                      for _ in range(n)])).cuda()
    grad = torch.empty_like(masks)
    imgs = torch.empty((n, nf, L, L), dtype=torch.float32, device="cuda")
    loss = torch.empty(n * nf, dtype=torch.float64, device="cuda")
    for _ in range(3):
        plan.vjp(masks, tgts, grad, loss, imgs, stream=stream)
    torch.cuda.synchronize()
    steps = max(3, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.vjp(masks, tgts, grad, loss, imgs, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    px = L * L
    bytes_step = 12 * px * n + 4 * px * n * nf
    gbs = bytes_step / (ms / 1e3) / 1e9
    # FP64 GPU adjoint of clip 0 for each focus, summed (after one untimed call)
    g64 = torch.zeros((1, L, L), dtype=torch.float64, device="cuda")
    l64 = torch.empty(1, dtype=torch.float64, device="cuda")
    gk = torch.empty((1, L, L), dtype=torch.float64, device="cuda")
    t64 = 0.0
    for i, (krn, sc) in enumerate(sets):
        kd = torch.from_numpy(np.stack([krn.real, krn.imag], -1).astype(np.float32).copy()).cuda()
        sd = torch.from_numpy(np.asarray(sc, dtype=np.float32)).cuda()
        if i == 0:
            K.fp64_socs_vjp(masks[:1], tgts[:1], Nx, Ny, kd, sd, gk, l64)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        K.fp64_socs_vjp(masks[:1], tgts[:1], Nx, Ny, kd, sd, gk, l64)
        f1.record()
        torch.cuda.synchronize()
        t64 += f0.elapsed_time(f1) / 1e3
        g64 += gk
    gerr = float((grad[:1].double() - g64).abs().max() / g64.abs().max())
    plan.close()
    del masks, tgts, grad, imgs, g64, gk
    rate = n * nf / (ms / 1e3)
    fp64_rate = nf / t64
    return {"metric": "4096^2 fwd+adj (clip, focus) pairs/s (16 clips x 5 focus, K=64)", "value": round(rate, 2),
            "unit": "pairs/s", "ms_per_step": round(ms, 3), "clips": n, "focus": nf, "K": nk,
            "GBps_algorithmic": round(gbs, 1), "frac_of_hbm_peak": round(gbs / peak_gbs, 4),
            "grad_max_err_vs_fp64_rel": gerr, "fp64_gpu_pairs_per_s": round(fp64_rate, 3),
            "speedup_vs_fp64_gpu": round(rate / fp64_rate, 2),
            "fp64_sample": "clip 0 at the 5 focus values (kl_fp64_socs_vjp, CUDA events, after one untimed call)",
            "timing": f"CUDA events over {steps} steps after 3 warm-up steps"}


def subspace_report(k_fast, k_ref, ev_ref):
    """Kernels of two eigensolves compared as subspaces: the largest principal
    angle (radians) at every cut m < K where the spectrum has a gap
    ((lambda_m-1 - lambda_m) / lambda_0 > 1e-4; inside near-degenerate
    clusters the basis is arbitrary), and the weighted projectors
    sum lambda v v^H (relative Frobenius error)."""
    A = np.asarray(k_fast, dtype=np.complex128).T
    B = np.asarray(k_ref, dtype=np.complex128).T
    ev = np.asarray(ev_ref, dtype=np.float64)
    qa, _ = np.linalg.qr(A)
    qb, _ = np.linalg.qr(B)
    cuts, worst = [], 0.0
    for m in range(1, A.shape[1]):
        if (ev[m - 1] - ev[m]) / ev[0] > 1e-4:
            sv = np.linalg.svd(qa[:, :m].conj().T @ qb[:, :m], compute_uv=False)
            ang = float(np.arccos(np.clip(sv.min(), -1.0, 1.0)))
            cuts.append((m, ang))
            worst = max(worst, ang)
    # weighted projectors through the K x K Gram products (no N x N matrices)
    w = np.sqrt(np.maximum(ev, 0))
    Aw, Bw = A * w[None, :], B * w[None, :]
    aa, bb, ab = Aw.conj().T @ Aw, Bw.conj().T @ Bw, Aw.conj().T @ Bw
    diff2 = np.real(np.trace(aa @ aa) + np.trace(bb @ bb) - 2 * np.trace(ab @ ab.conj().T))
    rel = float(np.sqrt(max(diff2, 0.0)) / np.sqrt(np.real(np.trace(bb @ bb))))
    return {"max_principal_angle_rad": worst, "gap_cuts": len(cuts),
            "angles_at_cuts": [[m, a] for m, a in cuts[:64]], "weighted_projector_rel_err": rel}


def bench_tcc_eigen(args):
    """TCC + top-K eigen at the larger field: 2048^2, dipole-X (0.7, 0.15) on a
    61^2 grid (98 source points), NA 1.35 water, K = 32, focus -50..50 nm in
    five steps.  Seconds per focus for
      fast (one focus per call): FP32 pupil factor, tcgen05 BF16x3 TCC, and the
        top-K by one exact Rayleigh-Ritz step on span(A) (exact Gram on the
        tensor cores + tridiagonal eigensolve on a thread-block cluster);
      fast (focus sweep): the five focus values through kl_topk_eig_batch,
        whose eigensolves share one launch (total / 5);
      plain FP64 GPU path: FP64 pupil table, FP64 TCC by direct accumulation,
        FP64 subspace iteration on the dense TCC, one focus after another.
    Each includes plan creation (source sampling, pupil factor) and the kernel
    download; the materialised TCC of the fast path (tcgen05 GEMM) is timed
    separately since the eigensolve does not need it."""
    import torch
    import klitho as K
    import synth
    L, nk = 2048, 32
    src = K.createSource(61, "Dipole", radius=0.15, offset=0.7, onXAxis=1)
    focus = [-50.0, -25.0, 0.0, 25.0, 50.0]

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    # warm-up of both paths (module load, first launches)
    w = K.TccPlan(src, 1.35, 0.0, L, L, n_medium=synth.N_WATER)
    w.topk(nk)
    w.close()
    w = K.TccPlan(src, 1.35, 0.0, L, L, n_medium=synth.N_WATER, precision=K.PREC_FP64)
    w.topk(nk)
    w.close()
    fast_t, tcc_t, fp64_t, tcc_err, ev_err, its, fast_ev, subs = [], [], [], [], [], [], [], []
    fast_plan_t, fp64_plan_t = [], []
    for f_nm in focus:
        df = synth.defocus_arg(f_nm)

        tp, tpl = timed(lambda: K.TccPlan(src, 1.35, df, L, L, n_medium=synth.N_WATER))
        (krn, sc, ev, it), t = timed(lambda: tp.topk(nk))
        fast_plan_t.append(tpl)
        fast_t.append(tpl + t)
        its.append(it)
        fast_ev.append(ev)
        T, t = timed(tp.build)
        tcc_t.append(t)

        tq, tql = timed(lambda: K.TccPlan(src, 1.35, df, L, L, n_medium=synth.N_WATER,
                                          precision=K.PREC_FP64))
        (krn64, sc64, ev64, _), t = timed(lambda: tq.topk(nk))
        fp64_plan_t.append(tql)
        fp64_t.append(tql + t)
        T64 = tq.build()
        tcc_err.append(float(torch.linalg.norm(T.double() - T64) / torch.linalg.norm(T64)))
        ev_err.append(float(np.max(np.abs(ev - ev64)) / np.max(np.abs(ev64))))
        subs.append(subspace_report(krn, krn64, ev64))
        N = tp.N
        tp.close()
        tq.close()
        del T, T64

    def sweep():
        ps = [K.TccPlan(src, 1.35, synth.defocus_arg(f), L, L, n_medium=synth.N_WATER) for f in focus]
        return ps, K.TccPlan.topk_batch(ps, nk)
    (ps, (kb, sb, eb, itb)), t_sweep = timed(sweep)
    batch_dev = max(float(np.max(np.abs(eb[i] - fast_ev[i])) / np.max(np.abs(fast_ev[i])))
                    for i in range(len(focus)))
    for p_ in ps:
        p_.close()
    f1, fs, d = float(np.median(fast_t)), t_sweep / len(focus), float(np.median(fp64_t))
    return {"metric": "TCC + top-K eigen seconds per focus (2048^2 dipole, K=32)",
            "fast_s": round(f1, 5), "fast_focus_sweep_s": round(fs, 5), "fp64_gpu_s": round(d, 5),
            "speedup_vs_fp64_gpu": round(d / f1, 2), "speedup_sweep_vs_fp64_gpu": round(d / fs, 2),
            "tcc_tcgen05_materialise_s": round(float(np.median(tcc_t)), 5),
            "fast_s_each": [round(x, 5) for x in fast_t], "fp64_gpu_s_each": [round(x, 5) for x in fp64_t],
            "fast_plan_s_each": [round(x, 5) for x in fast_plan_t],
            "fp64_plan_s_each": [round(x, 5) for x in fp64_plan_t],
            "N": N, "S": int(K.sourcePointCount(src, K.getOuterSigma(src))), "focus_nm": focus,
            "gram_solve_iterations": its, "tcc_rel_frobenius_err_vs_fp64": max(tcc_err),
            "eigenvalue_rel_err_vs_fp64": max(ev_err), "sweep_vs_single_eigenvalue_dev": batch_dev,
            "max_principal_angle_rad_vs_fp64": max(x["max_principal_angle_rad"] for x in subs),
            "weighted_projector_rel_err_vs_fp64": max(x["weighted_projector_rel_err"] for x in subs),
            "gap_cuts_checked": sum(x["gap_cuts"] for x in subs),
            "timing": "wall clock per focus (median of 5) incl. plan (source sampling, pupil factor), "
                      "eigen-solve and kernel download, synchronised; the TCC itself is not needed by "
                      "the fast eigensolve and is timed separately"}


def bench_tcc_eigen_large(args):
    """TCC + top-K eigen at the stress field: 4096^2, cross-quadrupole
    (0.75, 0.12) on an 81^2 grid (196 source points), NA 1.35 water, K = 64,
    block 96.  Fast path: FP32 factor + the one-step Rayleigh-Ritz solve on
    span(A) (exact Gram A^H A on the tensor cores, 196 x 196, eigensolved by
    Householder tridiagonalisation on a thread-block cluster, bisection and
    inverse iteration); five focus values.  Plain FP64 GPU path: FP64 TCC by direct accumulation
    (N = 11449, 2.1 GB) and FP64 subspace iteration on the dense TCC, at one
    focus value (seconds per focus)."""
    import torch
    import klitho as K
    import synth
    L, nk, blk = 4096, 64, 96
    src = K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75)
    focus = [-50.0, -25.0, 0.0, 25.0, 50.0]

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, time.perf_counter() - t0

    # warm-up of both paths at this size (memory pool growth, first launches)
    for prec in (K.PREC_FAST, K.PREC_FP64):
        w = K.TccPlan(src, 1.35, 0.0, L, L, n_medium=synth.N_WATER, precision=prec)
        w.topk(nk, block=blk)
        w.close()
    fast_t, its, evs = [], [], []
    for f_nm in focus:
        def fast():
            tp = K.TccPlan(src, 1.35, synth.defocus_arg(f_nm), L, L, n_medium=synth.N_WATER)
            r = tp.topk(nk, block=blk)
            N, S = tp.N, tp.S
            tp.close()
            return r, N, S
        ((krn, sc, ev, it), N, S), t = timed(fast)
        if f_nm == focus[2]:
            fast_k0 = krn
        fast_t.append(t)
        its.append(it)
        evs.append(ev)

    # the focus sweep in one call (kl_topk_eig_batch: the five Gram solves run
    # concurrently, one thread-block cluster each), plans included
    def sweep():
        ps = [K.TccPlan(src, 1.35, synth.defocus_arg(f_nm), L, L, n_medium=synth.N_WATER) for f_nm in focus]
        r = K.TccPlan.topk_batch(ps, nk, block=blk)
        for q in ps:
            q.close()
        return r
    sweep()
    (kb, sb, eb, itb), ts = timed(sweep)
    sweep_dev = float(max(np.max(np.abs(eb[i] - evs[i])) / np.max(np.abs(evs[i])) for i in range(len(focus))))

    def fp64():
        tq = K.TccPlan(src, 1.35, synth.defocus_arg(focus[2]), L, L, n_medium=synth.N_WATER,
                       precision=K.PREC_FP64)
        r = tq.topk(nk, block=blk)
        tq.close()
        return r
    (k64, s64, ev64, it64), t64 = timed(fp64)
    f = float(np.median(fast_t))
    sub = subspace_report(fast_k0, k64, ev64)
    return {"metric": "TCC + top-K eigen seconds per focus (4096^2 cross-quadrupole, K=64)",
            "fast_s": round(f, 4), "fast_s_each": [round(x, 4) for x in fast_t],
            "fast_focus_sweep_s": round(ts / len(focus), 5), "sweep_vs_single_eigenvalue_dev": sweep_dev,
            "fp64_gpu_s": round(t64, 4), "speedup_vs_fp64_gpu": round(t64 / f, 2),
            "N": N, "S": S, "subspace_iterations": its, "fp64_iterations": it64,
            "eigenvalue_rel_err_vs_fp64": float(np.max(np.abs(evs[2] - ev64)) / np.max(np.abs(ev64))),
            "max_principal_angle_rad_vs_fp64": sub["max_principal_angle_rad"],
            "weighted_projector_rel_err_vs_fp64": sub["weighted_projector_rel_err"],
            "gap_cuts_checked": sub["gap_cuts"],
            "timing": "wall clock per focus incl. plan, eigen-solve and kernel download, after a warm-up "
                      "solve of each path; the sweep is the five foci in one kl_topk_eig_batch call, "
                      "divided by five; FP64 at focus 0 only"}


def bench_tcc_gemm(args):
    """The TCC as a materialised matrix (kl_tcc_build: BF16x3 split + tcgen05
    GEMM, FP32 accumulate in TMEM, Hermitian mirror in the epilogue), CUDA
    events around the call on its stream, at the 2048^2 dipole field (N = 2809,
    S = 98) and the 4096^2 cross-quadrupole field (N = 11449, S = 196).
    Rooflines: tensor (8 N^2 S flop, the dense complex product counted once)
    against the measured bf16 peak, and store (N^2 x 8 B of complex64)
    against the measured HBM copy bandwidth."""
    import torch
    import klitho as K
    import synth
    out = []
    for name, L, src in (("2048^2 dipole", 2048, K.createSource(61, "Dipole", radius=0.15, offset=0.7, onXAxis=1)),
                         ("4096^2 cross-quadrupole", 4096,
                          K.createSource(81, "CrossQuadrupole", radius=0.12, offset=0.75))):
        tp = K.TccPlan(src, 1.35, synth.defocus_arg(25.0), L, L, n_medium=synth.N_WATER)
        N, S = tp.N, tp.S
        T = torch.empty((N, N, 2), dtype=torch.float32, device="cuda")
        st = torch.cuda.current_stream()
        for _ in range(2):
            K.check(K.lib().kl_tcc_build(tp._h, K._dev_ptr(T), st.cuda_stream), "kl_tcc_build")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 5
        e0.record(st)
        for _ in range(reps):
            K.check(K.lib().kl_tcc_build(tp._h, K._dev_ptr(T), st.cuda_stream), "kl_tcc_build")
        e1.record(st)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / reps / 1e3
        flop, byts = 8.0 * N * N * S, 8.0 * N * N
        bf16 = peaks_tensor()
        out.append({"case": name, "N": N, "S": S, "ms": round(t * 1e3, 4),
                    "tensor_TFLOPs": round(flop / t / 1e12, 1), "tensor_frac": round(flop / t / 1e12 / bf16, 4),
                    "store_GBps": round(byts / t / 1e9, 1), "store_frac": round(byts / t / 1e9 / peaks()[0], 4)})
        del T
        tp.close()
    return {"metric": "TCC materialisation (kl_tcc_build) device time", "cases": out,
            "peaks": {"bf16_TFLOPs": peaks_tensor(), "hbm_GBps": peaks()[0]},
            "timing": "CUDA events around kl_tcc_build (operand split + tcgen05 GEMM) on its stream, "
                      "5 calls after 2 warm-up calls; the call synchronises to check the pipeline status"}


def run_e2e(plans, masks_h, args, ws, img_equiv):
    import torch
    steps = max(1, min(args.steps, args.e2e_steps))
    pinned_in, pinned_out = [], []
    for (L, n), m in zip(CLASSES, masks_h):
        ti = torch.from_numpy(m).pin_memory()
        to = torch.empty((n, len(FOCUS_NM), L, L), dtype=torch.float32).pin_memory()
        pinned_in.append(ti)
        pinned_out.append(to)
    import klitho as K
    stream = torch.cuda.current_stream()

    def once():
        for p, ti, to in zip(plans, pinned_in, pinned_out):
            K.check(K.lib().kl_socs_forward_host(
                p._h, K.ctypes.cast(ti.data_ptr(), K._c_float_p), int(ti.shape[0]),
                K.ctypes.cast(to.data_ptr(), K._c_float_p), int(stream.cuda_stream)),
                "kl_socs_forward_host")

    once()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        once()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    h2d = sum(int(t.numel()) * 4 for t in pinned_in)
    d2h = sum(int(t.numel()) * 4 for t in pinned_out)
    return {"value": round(img_equiv * ws / dt, 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": round(dt * 1e3, 2), "steps": steps,
            "path": "kl_socs_forward_host (C ABI), pinned host buffers, copies timed"}


# ---------------------------------------------------------------------------
# CPU: the reference's own implementation of the path on the host cores
# ---------------------------------------------------------------------------

def workload_config():
    """The benchmark workload (both arms): the batched forward's clip mix and focus values."""
    return {"workload": "batched SOCS forward: 128x512^2 + 192x1024^2 + 64x2048^2 clips x 3 focus, K=24",
            "clips_per_gpu": sum(n for _, n in CLASSES), "focus_nm": FOCUS_NM}


def _cpu_task(args):
    """One reference SOCS image (FT_r2c + calcSOCS + FI) of an L^2 clip."""
    L, seed, use_ref = args
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "k-litho_b200"))
    import synth
    from oracle import oracle as O
    Nx = {512: 6, 1024: 13, 2048: 27}[L]
    krn, sc = synth.random_kernels(NK, Nx, Nx, seed=seed)
    mask = synth.rect_mask_fill(L, seed, 0.3)
    t0 = time.perf_counter()
    if use_ref:
        O.ref_socs_image(mask, krn.real, krn.imag, sc, Nx, Nx)
    else:
        O.socs_image(mask, krn.astype(np.complex128), sc, Nx, Nx)
    return time.perf_counter() - t0


def cpu_baseline_sample(max_seconds=20.0, processes=1):
    """Time the reference SOCS path on 1024^2 clips (1 focus each) for about
    `max_seconds`; returns images/s in the bench unit."""
    from oracle import oracle as O
    use_ref = O.ref_available()
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    done, t_start = 0, time.perf_counter()
    with ctx.Pool(processes) as pool:
        while time.perf_counter() - t_start < max_seconds:
            pool.map(_cpu_task, [(1024, 100 + done + i, use_ref) for i in range(processes)])
            done += processes
    wall = time.perf_counter() - t_start
    return {"value": round(done / wall, 4), "unit": UNIT, "cores": processes,
            "kind": "reference" if use_ref else "port",
            "sample": f"{done} clips of 1024^2 at one focus, K=24 "
                      f"({'reference klitho_socs.cpp compiled with the project FFT shim' if use_ref else 'restated FP64 oracle'})"
                      f", {wall:.1f} s wall"}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    nproc = os.cpu_count() or 1
    from oracle import oracle as O
    use_ref = O.ref_available()
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    # the workload's mix of clip sizes, by image count (128 : 192 : 64 clips,
    # every clip imaged at each focus, which costs the CPU path the same): a
    # step images the pattern 2 x 512^2, 3 x 1024^2, 1 x 2048^2 about nproc / 2
    # times, the pool handing out one image at a time so that the processes
    # stay busy; the rate counts 1024^2-equivalent images
    pattern = [2048, 1024, 1024, 1024, 512, 512]
    reps = max(1, nproc // 2)
    per_step = len(pattern) * reps
    times, equiv, nimg = [], 0.0, 0
    with ctx.Pool(nproc) as pool:
        for s in range(args.warmup + args.steps):
            sizes = pattern * reps
            t0 = time.perf_counter()
            pool.map(_cpu_task, [(L, 7 + s * per_step + i, use_ref) for i, L in enumerate(sizes)], chunksize=1)
            if s >= args.warmup:
                times.append(time.perf_counter() - t0)
                equiv += sum((L / 1024.0) ** 2 for L in sizes)
                nimg += len(sizes)
    dt = float(np.mean(times))
    value = equiv / float(np.sum(times))
    kind = "reference" if use_ref else "port"
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": UNIT,
           "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(dt * 1e3, 2), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(),
           "cpu_baseline": {"value": round(value, 4), "unit": UNIT, "cores": nproc, "kind": kind,
                            "sample": f"{nimg} images of the workload's size mix (2 x 512^2 : 3 x 1024^2 : "
                                      f"1 x 2048^2, K=24), {per_step} per step over {nproc} processes"},
           "e2e": {"value": round(value, 4), "unit": UNIT, "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_part(args):
    """One secondary measurement alone, printed as its own JSON object."""
    import torch
    torch.cuda.set_device(0)
    if args.part == "fwd_adj":
        r = bench_fwd_adj(args, torch.cuda.current_stream(), peaks()[0])
    elif args.part == "socs_4096":
        r = bench_socs_4096(args, torch.cuda.current_stream(), peaks()[0])
    elif args.part == "fwd_adj_4096":
        r = bench_fwd_adj_4096(args, torch.cuda.current_stream(), peaks()[0])
    elif args.part == "tcc_eigen_large":
        r = bench_tcc_eigen_large(args)
    elif args.part == "tcc_gemm":
        r = bench_tcc_gemm(args)
    else:
        r = bench_tcc_eigen(args)
    print(json.dumps(r))


def spawn_ranks(args):
    """`--gpus N` outside a launcher: start N ranks (one process per GPU) with
    torch.distributed.run on this node, bounded by a timeout; fails loudly when
    fewer GPUs are visible."""
    import socket
    import torch
    have = torch.cuda.device_count()
    if have < args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} requested but {have} GPU(s) visible")
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr", "127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__)] + sys.argv[1:]
    raise SystemExit(subprocess.call(cmd))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the fwd+adj and TCC+eigen measurements")
    ap.add_argument("--only", type=int, default=0,
                    help="restrict to one clip size (profiling cases)")
    ap.add_argument("--clips", type=int, default=0, help="clip count for --only")
    ap.add_argument("--chunks", type=int, default=1,
                    help="plans per size class (>= 1024^2) in the timed graph")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="N > 1: every rank images its own batch (weak) or the batch is split (strong)")
    ap.add_argument("--part", choices=["all", "fwd_adj", "socs_4096", "fwd_adj_4096", "tcc_eigen",
                                       "tcc_eigen_large", "tcc_gemm"], default="all",
                    help="run one secondary measurement alone (profiling cases)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        spawn_ranks(args)
        return
    if args.only:
        n = args.clips or dict(CLASSES).get(args.only, 16)
        CLASSES[:] = [(args.only, n)]
    if args.impl == "reference":
        run_reference(args)
    elif args.part != "all":
        run_part(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
