"""Benchmark: cone-beam forward projection + exact adjoint on one B200.

Workload (default, the FDK scanner): 256^3 float32 volume of
1 mm voxels holding 30 seeded ellipsoids, 360 views over 360 deg, flat
detector 512 x 384 at 1.2 mm, source-axis 600 mm, source-detector 1200 mm.
One step = forward projection (reference slab-split weights) of the volume
plus the exact transpose applied to a dense incoming gradient sinogram (what
one autograd forward+backward of the projector does; a dense gradient has no
zero rays for the adjoint to skip).

Metric: ray-voxel intersections per second, forward + adjoint (I
intersections each, I counted exactly by the count kernel).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1: launched by torchrun, one rank per GPU; every rank runs its own scan
(independent seeded phantom), no collective on the data path ("weak").
Rank 0 prints one JSON line.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CFG = dict(n=256, voxel=1.0, ellipsoids=30, seed=2, nv=360, na=512, nb=384, pixel=1.2,
           src_iso=600.0, src_det=1200.0)
METRIC = "ray-voxel intersections/s (forward + adjoint)"
UNIT = "intersections/s"


def workload_name(c=CFG):
    return (f"cone-beam fwd+adjoint {c['n']}^3 @{c['voxel']}mm, {c['ellipsoids']} ellipsoids, {c['nv']} views, "
            f"{c['na']}x{c['nb']} @{c['pixel']}mm, SID {c['src_iso']:.0f} / SDD {c['src_det']:.0f} mm")


def config_dict(extra=None):
    d = {"workload": workload_name(), "volume": [CFG["n"]] * 3, "views": CFG["nv"],
         "detector": [CFG["na"], CFG["nb"]], "l2": "flushed between timed steps (256 MiB write)",
         "parallelism": "independent scan per GPU"}
    if extra:
        d.update(extra)
    return d


def angles():
    return np.linspace(0, 2 * np.pi, CFG["nv"], endpoint=False).astype(np.float32)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic():
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(n_gpus):
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        rank, local = dist.get_rank(), int(os.environ.get("LOCAL_RANK", "0"))
    else:
        rank, local = 0, 0
    torch.cuda.set_device(local)
    return rank, ws, local


def max_over_ranks(x, ws):
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    import torch
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()


# ---------------- CPU baseline (the reference, compiled for the host) ----------------

def cpu_sample(views_per_step, steps, warmup=0, seed=2):
    """Times the reference's own forward + backprojection (oracle/_ref, or the
    oracle restatement when the reference build is absent) on a subset of
    views of the workload, all host threads.  Returns (I/s, kind, cores, sample)."""
    import oracle
    import nefct_b200 as nb
    import torch
    kind = "reference" if oracle.have_ref() else "port"
    n = CFG["n"]
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(CFG["ellipsoids"], seed),
                               device="cuda" if torch.cuda.is_available() else None)
    vol = vol.permute(2, 1, 0).contiguous().cpu().numpy()
    g = oracle.grid((n, n, n), (0, 0, 0), (n * CFG["voxel"],) * 3)
    ang = angles()
    a = (CFG["src_iso"], CFG["src_det"], CFG["na"], CFG["pixel"], 0.5, CFG["nb"], CFG["pixel"], 0.5)
    tot_i, tot_t = 0, 0.0
    for s in range(warmup + steps):
        idx = [(s * views_per_step + k) * 37 % CFG["nv"] for k in range(views_per_step)]
        sub = ang[idx]
        _, cnt = oracle.cb_forward(g, vol, sub, *a)        # exact count of the sample
        t0 = time.perf_counter()
        if kind == "reference":
            sino = oracle.ref_cb_forward(g, vol, sub, *a)
            oracle.ref_cb_backward(g, sino, sub, *a)
        else:
            sino, _ = oracle.cb_forward(g, vol, sub, *a, use_cosf=True)
            oracle.cb_backward(g, sino, sub, *a, use_cosf=True)
        dt = time.perf_counter() - t0
        if s >= warmup:
            tot_i += 2 * cnt
            tot_t += dt
    cores = os.cpu_count() or 1
    sample = (f"{views_per_step} views per step ({steps} steps) of the workload: reference siddon_3d "
              f"project_flat + backproject_flat device code compiled as host C++ (-O3, OpenMP)")
    return tot_i / tot_t, kind, cores, sample


def run_reference(args):
    """--impl reference: the reference's CPU path on the host cores."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    views = 2
    v, kind, cores, sample = cpu_sample(views, args.steps, args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict({"ranks_running": 1 if ws > 1 else 1}),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------- GPU arm ----------------

def run_gpu(args):
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops

    rank, ws, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    n = CFG["n"]
    geom = nb.ConeBeam((n, n, n), angles(), CFG["src_iso"], CFG["src_det"], CFG["na"], CFG["pixel"], CFG["nb"],
                       CFG["pixel"], size=(n * CFG["voxel"],) * 3)
    vol = nb.ellipsoid_phantom(n, nb.random_ellipsoids(CFG["ellipsoids"], CFG["seed"] + rank), device=dev)
    vol = vol.permute(2, 1, 0).contiguous()
    inter = ops.cb_count_intersections(geom, 0, device=dev)
    rays = CFG["nv"] * CFG["na"] * CFG["nb"]
    sino = torch.empty(geom.sino_shape, device=dev)
    back = torch.empty(geom.vol_shape, device=dev)
    gen = torch.Generator(device=dev).manual_seed(35 + rank)
    grad = torch.rand(geom.sino_shape, device=dev, generator=gen) + 0.5     # dense incoming gradient
    flush = torch.empty(256 * 2 ** 20 // 4, device=dev)

    def step():
        ops.cb_forward(vol, geom, 0, out=sino)
        ops.cb_backward(grad, geom, 0, out=back)

    from nefct_b200 import autotune
    if args.rows:
        autotune.apply(args.rows, args.order, args.walk)               # fixed launch shape (profiling)
        tuned = {"rows": args.rows, "order": args.order, "walk": args.walk, "ms": None}
    else:
        tuned = autotune.tune_cone_beam(geom, 0, dev, use_cache=False)  # untimed launch-shape choice
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(ws)
    with ClockSampler(local) as clk:
        wall0 = time.perf_counter()
        for e0, e1, e2 in ev:
            flush.fill_(1.0)                                   # L2 flush, outside the timed events
            e0.record()
            ops.cb_forward(vol, geom, 0, out=sino)
            e1.record()
            ops.cb_backward(grad, geom, 0, out=back)
            e2.record()
        barrier(ws)
        wall = time.perf_counter() - wall0
    t_fwd = sum(a.elapsed_time(b) for a, b, _ in ev) / 1e3
    t_bwd = sum(b.elapsed_time(c) for _, b, c in ev) / 1e3
    t_step = max_over_ranks(t_fwd + t_bwd, ws)
    value = ws * args.steps * 2 * inter / t_step

    # e2e through the public op API with pinned host buffers: every step
    # copies its volume host->device, runs forward + adjoint and copies the
    # adjoint volume device->host.  The copies run on their own streams with
    # double buffers, so step i's upload overlaps step i-1's kernels and its
    # download overlaps step i+1's (how a pipelined caller drives the API);
    # every copy lies inside the timed region.
    h_in = torch.empty(geom.vol_shape, pin_memory=True)
    h_in.copy_(vol.cpu())
    h_out = [torch.empty(geom.vol_shape, pin_memory=True) for _ in range(2)]
    d_in = [torch.empty_like(vol) for _ in range(2)]
    d_back = [torch.empty_like(vol) for _ in range(2)]
    ks = torch.cuda.current_stream()
    hs, ds = torch.cuda.Stream(), torch.cuda.Stream()

    def e2e_steps(n, start):
        ev_up = [torch.cuda.Event() for _ in range(2)]
        ev_k = [torch.cuda.Event() for _ in range(2)]
        ev_down = [torch.cuda.Event() for _ in range(2)]
        hs.wait_event(start)
        for i in range(n):
            b = i % 2
            if i >= 2:
                hs.wait_event(ev_k[b])            # step i-2's kernels are done with d_in[b]
            with torch.cuda.stream(hs):
                d_in[b].copy_(h_in, non_blocking=True)
            ev_up[b].record(hs)
            ks.wait_event(ev_up[b])
            if i >= 2:
                ks.wait_event(ev_down[b])         # step i-2's download has read d_back[b]
            ops.cb_forward(d_in[b], geom, 0, out=sino)
            ops.cb_backward(grad, geom, 0, out=d_back[b])
            ev_k[b].record(ks)
            ds.wait_event(ev_k[b])
            with torch.cuda.stream(ds):
                h_out[b].copy_(d_back[b], non_blocking=True)
            ev_down[b].record(ds)
        for ev in ev_down:
            ks.wait_event(ev)

    w0 = torch.cuda.Event()
    w0.record(ks)
    e2e_steps(max(2, args.warmup), w0)
    torch.cuda.synchronize()
    barrier(ws)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ks)
    e2e_steps(args.steps, e0)
    e1.record(ks)
    barrier(ws)
    t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3, ws)
    e2e = ws * args.steps * 2 * inter / t_e2e
    vbytes = int(vol.numel() * 4)

    # roofline of the dominant op (forward or adjoint) on its algorithmic bytes
    peak, peak_kind = load_peaks()
    fwd_s, bwd_s = t_fwd / args.steps, t_bwd / args.steps
    walk = tuned["walk"]
    if bwd_s >= fwd_s:
        dom = "cb_colwarp_kernel<transpose>" if walk & 2 else "cb_backward_kernel"
        dom_t, alg = bwd_s, 8 * inter + 4 * rays
    else:
        dom = "cb_colwarp_kernel<forward>" if walk & 1 else "cb_forward_kernel"
        dom_t, alg = fwd_s, 4 * inter + 4 * rays
    achieved = alg / dom_t / 1e9
    traffic = load_traffic().get(dom)

    extras = {"intersections_per_direction": inter, "rays": rays,
              "forward_ms": 1e3 * fwd_s, "adjoint_ms": 1e3 * bwd_s,
              "forward_intersections_per_s": inter / fwd_s, "adjoint_intersections_per_s": inter / bwd_s,
              "wall_s_timed_loop": wall, "launch_shape": {"rows_per_cta": tuned["rows"],
                                                          "grid_order": "row-band outermost" if tuned["order"] == 0
                                                          else "view outermost",
                                                          "walk": {"forward": "column warps" if tuned["walk"] & 1
                                                                   else "thread per ray",
                                                                   "adjoint": "column warps" if tuned["walk"] & 2
                                                                   else "thread per ray"},
                                                          "autotune_ms": tuned["ms"]}}

    # FDK of this scanner (256^3, 360 views): line-integral projections of the
    # phantom, cosine weight + ramp filter + weighted voxel-driven backprojection
    from nefct_b200 import recon
    fdk = {}
    lines = ops.cb_forward(vol, geom, nb._lib.LINE_INTEGRAL)
    for win in ("ram-lak", "shepp-logan"):
        recon.fdk(lines, geom, win)
        ef = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ef[0].record()
        filt = ops.fdk_filter(lines, geom, win)
        ef[1].record()
        rec = ops.fdk_backproject(filt, geom)
        ef[2].record()
        torch.cuda.synchronize()
        t_f, t_b = ef[0].elapsed_time(ef[1]) / 1e3, ef[1].elapsed_time(ef[2]) / 1e3
        c = slice(n // 4, 3 * n // 4)
        err = float((rec[c, c, c] - vol[c, c, c]).norm() / vol[c, c, c].norm())
        fdk[win] = {"filter_ms": 1e3 * t_f, "backproject_ms": 1e3 * t_b,
                    "voxels_per_s": n ** 3 / (t_f + t_b), "voxel_views_per_s": n ** 3 * CFG["nv"] / t_b,
                    "central_rel_error_vs_phantom": err}
    # the reference's voxel-driven backprojection (pixel_3d: the FDK body
    # without its distance weight) built for the host, on a 2-view sample
    # scaled to the scan, beside the GPU backprojection of all views
    if rank == 0 and ws == 1 and not args.no_cpu:
        import oracle
        if oracle.have_ref():
            hs = filt[:2].cpu().numpy()
            side = n * CFG["voxel"]
            t0 = time.perf_counter()
            oracle.ref_pixel_backproject(hs, angles()[:2], (n, n, n), (-side / 2,) * 3, (side,) * 3,
                                         CFG["src_iso"], CFG["src_det"], CFG["na"], CFG["pixel"], 0.0,
                                         CFG["nb"], CFG["pixel"], 0.0)
            t_host = (time.perf_counter() - t0) * CFG["nv"] / 2
            fdk["reference_host_build"] = {"cores": os.cpu_count(), "sample": "2 views, scaled to the scan",
                                           "pixel_backproject_ms": 1e3 * t_host,
                                           "speedup_of_fdk_backproject": t_host / t_b}
    # short scan 180 deg + fan with Parker weights (views spaced like the full scan)
    fan = 2 * np.degrees(np.arctan(CFG["na"] * CFG["pixel"] / 2 / CFG["src_det"]))
    step = 360.0 / CFG["nv"]
    nss = int(np.ceil((180 + fan) / step)) + 1
    gss = nb.ConeBeam((n, n, n), np.deg2rad(np.arange(nss) * step - fan / 2), CFG["src_iso"], CFG["src_det"],
                      CFG["na"], CFG["pixel"], CFG["nb"], CFG["pixel"], size=(n * CFG["voxel"],) * 3)
    lss = ops.cb_forward(vol, gss, nb._lib.LINE_INTEGRAL)
    best = None
    for d in (1, -1):
        rec = recon.fdk(lss, gss, "ram-lak", d)
        c = slice(n // 4, 3 * n // 4)
        err = float((rec[c, c, c] - vol[c, c, c]).norm() / vol[c, c, c].norm())
        best = (err, d) if best is None or err < best[0] else best
    fdk["short_scan_parker"] = {"views": nss, "dir": best[1], "central_rel_error_vs_phantom": best[0]}
    del lines, filt, rec, lss
    extras["fdk"] = fdk

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        v, kind, cores, sample = cpu_sample(2, 3)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_step / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid phantom)",
                "config": config_dict(),
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "peak_source": peak_kind,
                             "algorithmic_bytes": alg, "traffic": traffic},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": vbytes, "d2h_bytes_per_step": vbytes},
                "gpu_launches": 4 * args.steps,
                "clocks": clk.summary(), "extras": extras}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------- batched uneven problems (64 problems, edges 64..384) ----------------

def uneven_geoms(n_problems=64, seed=4, scale=1.0, view_scale=1.0):
    """Seeded uneven problems: edge log-uniform in [64, 384] (times scale),
    views U{60..720} (times view_scale, at least 4), detector rows/cols
    U{128..1024} (times scale), source-axis
    U[400, 700] mm, source-detector = source-axis x U[1.5, 2.0], 1 mm voxels,
    square pixels sized so the detector width covers the volume."""
    import nefct_b200 as nb
    rng = np.random.default_rng(seed)
    geoms = []
    for _ in range(n_problems):
        n = int(round(np.exp(rng.uniform(np.log(64), np.log(384))) * scale))
        nv = max(4, int(round(int(rng.integers(60, 721)) * view_scale)))
        rows, cols = (int(round(v * scale)) for v in rng.integers(128, 1025, 2))
        si = float(rng.uniform(400, 700))
        sd = si * float(rng.uniform(1.5, 2.0))
        pixel = (sd / si) * n * 1.0 / cols
        ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
        geoms.append(nb.ConeBeam((n, n, n), ang, si, sd, cols, pixel, rows, pixel, size=(float(n),) * 3))
    return geoms


def run_batched(args):
    """Batched fwd+adjoint iterations/s of the uneven problems vs the plain
    per-problem drop-in path (numpy in/out per call, like the reference's
    operators) and vs sequential per-problem device calls."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops
    from nefct_b200.batch import BatchProjector
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    geoms = uneven_geoms(args.problems, 4, args.scale, args.view_scale)
    gen = torch.Generator(device=dev).manual_seed(4)
    vols = [torch.rand(g.vol_shape, device=dev, generator=gen) for g in geoms]
    bp = BatchProjector(geoms, vols)            # grads = the forward outputs (loss = |Ax|^2 / 2)
    inter = sum(ops.cb_count_intersections(g, 0, dev) for g in geoms)
    graph = bp.capture()
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    t_batch = e0.elapsed_time(e1) / 1e3 / args.steps

    # sequential per-problem device calls (the same kernels, one problem at a time)
    for g, v, s_, b in zip(geoms, vols, bp.sinos, bp.backs):      # warm the allocator's workspaces
        ops.cb_forward(v, g, 0, out=s_)
        ops.cb_backward(s_, g, 0, out=b)
    torch.cuda.synchronize()
    e0.record()
    for g, v, s_, b in zip(geoms, vols, bp.sinos, bp.backs):
        ops.cb_forward(v, g, 0, out=s_)
        ops.cb_backward(s_, g, 0, out=b)
    e1.record()
    torch.cuda.synchronize()
    t_seq = e0.elapsed_time(e1) / 1e3

    # plain drop-in path: numpy volume in, Project3D, BackProject3D, numpy out
    sc = [nb.ScannerConfig3D("flat", g.src_det, g.src_iso, nb.DetectorDirectAConfig(g.na, g.na * g.da),
                             nb.DetectorDirectBConfig(g.nb, g.nb * g.db)) for g in geoms]
    host = [v.permute(2, 1, 0).cpu().numpy() for v in vols]
    t0 = time.perf_counter()
    for g, c, h in zip(geoms, sc, host):
        img = nb.Image3D(h, [0, 0, 0], list(g.size))
        proj = nb.Project3D(c, g.angles, None)(img)
        nb.BackProject3D(c, list(g.shape), 1.0, "transpose")(proj)
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    line = {"metric": "batched fwd+adjoint iterations/s (64 uneven cone-beam problems)", "value": 1.0 / t_batch,
            "unit": "iterations/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_batch, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded uniform random volumes)",
            "config": {"workload": f"{args.problems} problems, edge log-U[64,384]x{args.scale}, "
                                   f"views U[60,720]x{args.view_scale}, "
                                   f"detector U[128,1024]^2 x{args.scale}, seed 4",
                       "voxels": int(sum(np.prod(g.shape) for g in geoms)),
                       "rays": int(sum(g.nv * g.na * g.nb for g in geoms)), "tiles": bp.tiles},
            "extras": {"strategy": bp.strategy, "strategy_step_ms": bp.timings,
                       "intersections_per_iteration": 2 * inter,
                       "batched_intersections_per_s": 2 * inter / t_batch,
                       "sequential_device_s": t_seq, "plain_dropin_s": t_plain,
                       "speedup_vs_plain_dropin": t_plain / t_batch,
                       "speedup_vs_sequential_device": t_seq / t_batch}}
    print(json.dumps(line), flush=True)


# ---------------- differentiable projector at 512^3, 720 views ----------------

def run_diff512(args):
    """512^3 phantom (50 ellipsoids, seed 3), 720 views, 1024x768 at 1 mm,
    source-axis 700 / source-detector 1400 mm, b = A x + 1 % noise (seed 33):
    forward + adjoint intersections/s through autograd, and 20 SIRT
    iterations."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops, recon
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, nv = int(512 * args.scale), int(720 * args.scale)
    na, nbr = int(1024 * args.scale), int(768 * args.scale)
    g = nb.ConeBeam((n, n, n), np.linspace(0, 2 * np.pi, nv, endpoint=False), 700.0, 1400.0, na, 1.0, nbr, 1.0,
                    size=(float(n),) * 3)
    x_true = nb.ellipsoid_phantom(n, nb.random_ellipsoids(50, 3), device=dev).permute(2, 1, 0).contiguous()
    flags = nb._lib.LINE_INTEGRAL
    b = ops.cb_forward(x_true, g, flags)
    gen = torch.Generator(device=dev).manual_seed(33)
    b += 0.01 * float(b.max()) * torch.randn(b.shape, device=dev, generator=gen)
    inter = ops.cb_count_intersections(g, flags, dev)
    x = torch.zeros_like(x_true, requires_grad=True)

    def fb():
        loss = ((nb.project(x, g, flags) - b) ** 2).sum()
        loss.backward()
        return loss
    for _ in range(args.warmup):
        fb()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fb()
    e1.record()
    torch.cuda.synchronize()
    t_fb = e0.elapsed_time(e1) / 1e3 / args.steps
    # 20 SIRT iterations
    e0.record()
    rec = recon.sirt(b, g, 20, flags)
    e1.record()
    torch.cuda.synchronize()
    t_sirt = e0.elapsed_time(e1) / 1e3
    err = float((rec - x_true).norm() / x_true.norm())
    line = {"metric": "ray-voxel intersections/s (autograd forward + adjoint, 512^3 differentiable projector)",
            "value": 2 * inter / t_fb, "unit": "intersections/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_fb, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid phantom + 1 % noise)",
            "config": {"workload": f"{n}^3 @1mm, 50 ellipsoids, {nv} views, {na}x{nbr} @1mm, SID 700 / SDD 1400 mm"},
            "extras": {"intersections_per_direction": inter, "sirt_20_iterations_s": t_sirt,
                       "sirt_rel_error_vs_phantom": err}}
    print(json.dumps(line), flush=True)


# ---------------- motion-compensated 4D through the warp (10 phases x 72 views) ----------------

def run_motion4d(args):
    """256^3 reference volume, 10 phases x 72 views, 512x384, per-phase
    displacement fields (4 seeded sinusoids, <= 5 voxels): warp then project,
    gradients w.r.t. the volume and every field (autograd)."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops, recon
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = 256
    phases, per = 10, 72
    ang = np.linspace(0, 2 * np.pi, phases * per, endpoint=False)
    geoms = [nb.ConeBeam((n, n, n), ang[p::phases], 600.0, 1200.0, 512, 1.2, 384, 1.2, size=(float(n),) * 3)
             for p in range(phases)]
    ref = nb.ellipsoid_phantom(n, nb.random_ellipsoids(30, 5), device=dev).permute(2, 1, 0).contiguous()
    rng = np.random.default_rng(5)
    fields = [recon.sinusoid_field(ref.shape, 5.0, rng, device=dev) for _ in range(phases)]
    targets = [ops.cb_forward(ops.warp_forward(ref, *m), g) for m, g in zip(fields, geoms)]
    inter = sum(ops.cb_count_intersections(g, 0, dev) for g in geoms)
    x = ref.clone().mul_(0.9).requires_grad_()
    ms = [[c.clone().requires_grad_() for c in m] for m in fields]

    def fb():
        sinos = recon.motion_project(x, ms, geoms)
        loss = sum(((s_ - t) ** 2).sum() for s_, t in zip(sinos, targets))
        loss.backward()
    for _ in range(args.warmup):
        fb()
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fb()
    e1.record()
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    line = {"metric": "ray-voxel intersections/s (4D warp + forward + adjoint with image and field gradients)",
            "value": 2 * inter / t, "unit": "intersections/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom and sinusoid fields)",
            "config": {"workload": f"{n}^3, {phases} phases x {per} views, 512x384 @1.2mm, fields 3x{n}^3 per phase"},
            "extras": {"intersections_per_direction": inter, "voxels_warped_per_step": phases * n ** 3,
                       "peak_allocated_bytes": peak}}
    print(json.dumps(line), flush=True)


# ---------------- per-row timings of the other operators on this path ----------------

def run_rows(args):
    """Device time of each operator beside the headline pair, on workloads of
    the bench's sizes, with the reference's host build timed on a sample where
    it has the operator: the LOR pair (16 Mi random PET-like lines through
    256^3), the reference backprojection (Q8 off), the deterministic and the
    exact-mode transposes and the exact-mode forward (36 views of the bench
    scanner), the warp family at 256^3, and the distance-driven FDK
    backprojection (72 views of the bench scanner in voxel units)."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import _lib, ops
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    gen = torch.Generator(device=dev).manual_seed(9)
    n = CFG["n"]

    def timed(fn, reps=None):
        reps = reps or max(1, args.steps)
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    rows = {}
    vol = torch.rand((n, n, n), device=dev, generator=gen)
    # LOR pair: end points on a 300 mm ring (random angles, z in +-100 mm)
    nl = 16 * 2 ** 20
    rng = np.random.default_rng(9)
    phi1, phi2 = rng.uniform(0, 2 * np.pi, nl), rng.uniform(0, 2 * np.pi, nl)
    lors = np.stack([300 * np.cos(phi1), 300 * np.sin(phi1), rng.uniform(-100, 100, nl),
                     300 * np.cos(phi2), 300 * np.sin(phi2), rng.uniform(-100, 100, nl)]).astype(np.float32)
    d_lors = torch.from_numpy(lors).to(dev)
    vals = torch.rand(nl, device=dev, generator=gen)
    t_lf0 = timed(lambda: ops.lor_forward(d_lors, vol, (n, n, n)))
    t_lb0 = timed(lambda: ops.lor_backward(d_lors, vals, (n, n, n)))
    t_ord = timed(lambda: ops.lor_order(d_lors, (n, n, n)), reps=2)
    order = ops.lor_order(d_lors, (n, n, n))
    t_lf = timed(lambda: ops.lor_forward(d_lors, vol, (n, n, n), order=order))
    t_lb = timed(lambda: ops.lor_backward(d_lors, vals, (n, n, n), order=order))
    rows["lor_pair"] = {"lors": nl, "grid": [n] * 3, "forward_ms": 1e3 * t_lf, "backward_ms": 1e3 * t_lb,
                        "forward_lors_per_s": nl / t_lf, "backward_lors_per_s": nl / t_lb,
                        "walk_order": "ordered (lor_order, computed once per list)", "order_ms": 1e3 * t_ord,
                        "list_order_forward_ms": 1e3 * t_lf0, "list_order_backward_ms": 1e3 * t_lb0}
    # reference backprojection / deterministic / exact on 36 views of the bench scanner
    ang = angles()[::10]
    g = nb.ConeBeam((n, n, n), ang, CFG["src_iso"], CFG["src_det"], CFG["na"], CFG["pixel"], CFG["nb"],
                    CFG["pixel"], size=(n * CFG["voxel"],) * 3)
    y = torch.rand(g.sino_shape, device=dev, generator=gen)
    back = torch.empty_like(vol)
    i_fwd = ops.cb_count_intersections(g, 0, dev)
    i_ref = ops.cb_count_intersections(g, _lib.REF_BACKPROJECT, dev)
    t_atomic = timed(lambda: ops.cb_backward(y, g, 0, out=back))
    t_refbp = timed(lambda: ops.cb_backward(y, g, _lib.REF_BACKPROJECT, out=back))
    t_det = timed(lambda: ops.cb_backward(y, g, _lib.DETERMINISTIC, out=back))
    sino = torch.empty(g.sino_shape, device=dev)
    t_exf = timed(lambda: ops.cb_forward(vol, g, _lib.EXACT, out=sino))
    t_exb = timed(lambda: ops.cb_backward(y, g, _lib.EXACT, out=back))
    rows["cone_beam_36_views"] = {
        "intersections_forward_walk": i_fwd, "intersections_reference_backprojection": i_ref,
        "transpose_ms": 1e3 * t_atomic, "reference_backprojection_ms": 1e3 * t_refbp,
        "reference_backprojection_intersections_per_s": i_ref / t_refbp,
        "deterministic_transpose_ms": 1e3 * t_det, "deterministic_over_atomic": t_det / t_atomic,
        "exact_mode_forward_ms": 1e3 * t_exf, "exact_mode_transpose_ms": 1e3 * t_exb}
    # warp family at 256^3 (fields up to 5 voxels)
    from nefct_b200 import recon
    m = recon.sinusoid_field(vol.shape, 5.0, np.random.default_rng(5), device=dev)
    gout = torch.rand_like(vol)
    t_wf = timed(lambda: ops.warp_forward(vol, *m))
    t_wa = timed(lambda: ops.warp_adjoint(gout, *m))
    t_wg = timed(lambda: ops.warp_grad_dvf(vol, *m, gout))
    t_wi = timed(lambda: ops.warp_invert(*m), reps=2)
    nvox = n ** 3
    rows["warp_256cube"] = {"forward_ms": 1e3 * t_wf, "forward_gbs_of_48B_per_voxel": 48 * nvox / t_wf / 1e9,
                            "adjoint_ms": 1e3 * t_wa, "dvf_gradient_ms": 1e3 * t_wg,
                            "invert_30_passes_ms": 1e3 * t_wi}
    # distance-driven FDK backprojection: the bench scanner in voxel units, 72 views
    ang72 = angles()[::5]
    proj = torch.rand((ang72.size, CFG["nb"], CFG["na"]), device=dev, generator=gen)
    px = CFG["pixel"] / CFG["voxel"]
    sad, sid = CFG["src_iso"] / CFG["voxel"], CFG["src_det"] / CFG["voxel"]
    t_dd = timed(lambda: ops.dd_backproject(proj, (n, n, n), ang72, sad, sid, px, px), reps=2)
    rows["distance_driven_72_views"] = {"ms": 1e3 * t_dd, "bins_per_s": proj.numel() / t_dd}
    # the reference's host build on samples of the same operators
    if not args.no_cpu:
        import oracle
        if oracle.have_ref():
            og = oracle.grid((n, n, n), (0, 0, 0), (float(n),) * 3)
            hv = vol.cpu().numpy()
            k = 2 ** 17
            t0 = time.perf_counter()
            oracle.ref_lor_forward(og, hv, np.ascontiguousarray(lors[:, :k]))
            t_cpu_lor = time.perf_counter() - t0
            mh = [c.cpu().numpy() for c in m]
            t0 = time.perf_counter()
            oracle.ref_deform(hv, *mh)
            t_cpu_warp = time.perf_counter() - t0
            ph = proj[:2].cpu().numpy()
            t0 = time.perf_counter()
            oracle.ref_dd_backproject(ph, ang72[:2], (n, n, n), sid, sad, CFG["na"], px, 0.0, CFG["nb"], px, 0.0)
            t_cpu_dd = (time.perf_counter() - t0) * ang72.size / 2
            rows["reference_host_build"] = {
                "cores": os.cpu_count(), "lor_forward_lors_per_s": k / t_cpu_lor,
                "lor_forward_speedup": (nl / t_lf) / (k / t_cpu_lor),
                "warp_forward_ms": 1e3 * t_cpu_warp, "warp_forward_speedup": t_cpu_warp / t_wf,
                "distance_driven_72_views_ms_from_2_view_sample": 1e3 * t_cpu_dd,
                "distance_driven_speedup": t_cpu_dd / t_dd}
    line = {"metric": "LOR forward + backward lines/s (16 Mi lines, 256^3); other operators in extras",
            "value": nl / (t_lf + t_lb), "unit": "lines/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * (t_lf + t_lb), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded uniform volumes, lines, sinograms and fields)",
            "config": {"workload": "per-operator timings beside the 256^3 / 360-view pair"}, "extras": rows}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--views", type=int, default=360, help="views of the scan (360 = the workload; fewer only for profiling)")
    ap.add_argument("--rows", type=int, default=0, help="fix the detector rows per CTA instead of autotuning")
    ap.add_argument("--order", type=int, default=1, help="with --rows: 0 row bands outermost, 1 views outermost")
    ap.add_argument("--walk", type=int, default=3,
                    help="with --rows: column warps for the forward (bit 0) / adjoint (bit 1), else thread per ray")
    ap.add_argument("--workload", default="fdk-scanner",
                    choices=["fdk-scanner", "batched", "diff512", "motion4d", "rows"],
                    help="batched: the 64 uneven problems (its own JSON line)")
    ap.add_argument("--problems", type=int, default=64)
    ap.add_argument("--scale", type=float, default=1.0, help="batched: scale of volume edges and detector sizes")
    ap.add_argument("--view-scale", type=float, default=1.0, help="batched: scale of the view counts")
    args = ap.parse_args()
    CFG["nv"] = args.views
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "diff512":
        run_diff512(args)
    elif args.workload == "motion4d":
        run_motion4d(args)
    elif args.workload == "rows":
        run_rows(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
