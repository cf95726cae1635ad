"""Benchmark: cone-beam forward projection + exact adjoint on one B200.

Headline workload (the differentiable-projector scan, the largest that runs
on one GPU): 512^3 float32 volume of 1 mm voxels holding 50 seeded
ellipsoids, 720 views over 360 deg, flat detector 1024 x 768 at 1 mm,
source-axis 700 mm, source-detector 1400 mm.  One step = forward projection
(reference slab-split weights) of the volume plus the exact transpose applied
to a dense incoming gradient sinogram (what one autograd forward+backward of
the projector does; a dense gradient has no zero rays for the adjoint to
skip).  ``--workload fdk-scanner`` runs the same step on the FDK scanner
(256^3 at 1 mm, 30 ellipsoids, 360 views, 512 x 384 at 1.2 mm, 600 / 1200 mm).

Metric: ray-voxel intersections per second, forward + adjoint (I
intersections each, I counted exactly by the count kernel).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1: launched by torchrun, one rank per GPU; every rank runs its own scan
(independent seeded phantom), no collective on the data path ("weak").
Rank 0 prints one JSON line.

--impl reference: the reference's own projector code (siddon_3d forward and
backprojection device routines compiled for the host, oracle/_ref) on a
sample of the same scan's views, on every host core; same metric and
config.
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

SCANS = {
    "diff-projector": dict(n=512, voxel=1.0, ellipsoids=50, seed=3, nv=720, na=1024, nb=768, pixel=1.0,
                           src_iso=700.0, src_det=1400.0, tune_every=6),
    "fdk-scanner": dict(n=256, voxel=1.0, ellipsoids=30, seed=2, nv=360, na=512, nb=384, pixel=1.2,
                        src_iso=600.0, src_det=1200.0, tune_every=1),
}
METRIC = "ray-voxel intersections/s (forward + adjoint)"
UNIT = "intersections/s"
CPU_VIEWS_PER_STEP = 2        # views of the reference's host build per sampled step


def workload_name(c):
    return (f"cone-beam fwd+adjoint {c['n']}^3 @{c['voxel']}mm, {c['ellipsoids']} ellipsoids (seed {c['seed']}), "
            f"{c['nv']} views, {c['na']}x{c['nb']} @{c['pixel']}mm, SID {c['src_iso']:.0f} / SDD "
            f"{c['src_det']:.0f} mm")


def config_dict(c):
    """The config both arms print (identical dicts)."""
    return {"workload": workload_name(c), "volume": [c["n"]] * 3, "views": c["nv"],
            "detector": [c["na"], c["nb"]],
            "l2": "inputs larger than L2; 256 MiB L2 flush between timed steps" if c["n"] >= 512
            else "256 MiB L2 flush between timed steps",
            "parallelism": "independent scan per GPU"}


def angles(c):
    return np.linspace(0, 2 * np.pi, c["nv"], endpoint=False).astype(np.float32)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(workload):
    """Per-launch DRAM bytes of each kernel of a workload, from the committed
    ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(workload, {})
    return {}


def load_issue(workload):
    """Warp instructions per view of each kernel of a workload, from the
    committed ncu summary (profiles/issue.json)."""
    p = os.path.join(ROOT, "profiles", "issue.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(workload, {})
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


def dist_setup():
    import torch
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0")) if ws > 1 else 0
    torch.cuda.set_device(local)                     # before the group: its communicator binds this GPU
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        rank = dist.get_rank()
    else:
        rank = 0
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


# ---------------- the reference's host build on sampled views ----------------

def phantom_xfast(c, device=None):
    """The scan's phantom as a [z][y][x] float32 array (torch on ``device``)."""
    import nefct_b200 as nb
    vol = nb.ellipsoid_phantom(c["n"], nb.random_ellipsoids(c["ellipsoids"], c["seed"]), device=device)
    return vol.permute(2, 1, 0).contiguous()


def sample_views(c, step, pairs=8):
    """Views of sampled step `step`: CPU_VIEWS_PER_STEP views spread over the
    scan, cycling through `pairs` fixed sets (so their exact intersection
    counts are computed once)."""
    s = step % pairs
    return [((s * CPU_VIEWS_PER_STEP + k) * 97 + 13 * s) % c["nv"] for k in range(CPU_VIEWS_PER_STEP)]


class HostReference:
    """The reference's forward (ProjectFlatKernel) and backprojection
    (BackProjectFlatKernel, atomic adds) built for the host (oracle/_ref; the
    oracle restatement if the build is absent), over (view, row) pairs on
    every host thread.  Intersections are counted exactly by the oracle's
    walk, once per view set."""

    def __init__(self, c, vol_np):
        import oracle
        self.o = oracle
        self.c = c
        self.kind = "reference" if oracle.have_ref() else "port"
        n = c["n"]
        self.g = oracle.grid((n, n, n), (0, 0, 0), (n * c["voxel"],) * 3)
        self.vol = vol_np
        self.ang = angles(c)
        self.args = (c["src_iso"], c["src_det"], c["na"], c["pixel"], 0.5, c["nb"], c["pixel"], 0.5)
        self.counts = {}

    def threads(self):
        return self.o.ref_threads() if self.kind == "reference" else (os.cpu_count() or 1)

    def count(self, idx):
        key = tuple(idx)
        if key not in self.counts:
            _, cnt = self.o.cb_forward(self.g, self.vol, self.ang[idx], *self.args)
            self.counts[key] = cnt
        return self.counts[key]

    def step(self, idx):
        """(seconds, forward sinogram, backprojection) of the views idx."""
        sub = self.ang[idx]
        t0 = time.perf_counter()
        if self.kind == "reference":
            sino = self.o.ref_cb_forward(self.g, self.vol, sub, *self.args)
            back = self.o.ref_cb_backward(self.g, sino, sub, *self.args, atomic=True)
        else:
            sino, _ = self.o.cb_forward(self.g, self.vol, sub, *self.args, use_cosf=True)
            back = self.o.cb_backward(self.g, sino, sub, *self.args, use_cosf=True)
        return time.perf_counter() - t0, sino, back

    def sample(self):
        return (f"{CPU_VIEWS_PER_STEP} views per step of the workload, cycling through 8 fixed view sets: the "
                f"reference's siddon_3d ProjectFlatKernel + BackProjectFlatKernel device code compiled as host C++ "
                f"(-O3 -march=x86-64-v3, OpenMP over (view, detector row), atomic adds for the backprojection)")


def run_reference(args):
    """--impl reference: the reference's CPU path on the host cores."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    c = SCANS[args.workload]
    c["nv"] = args.views or c["nv"]
    ref = HostReference(c, phantom_xfast(c).numpy())
    times, inter = [], []
    for s in range(args.warmup + args.steps):
        idx = sample_views(c, s)
        cnt = ref.count(idx)
        dt, _, _ = ref.step(idx)
        if s >= args.warmup:
            times.append(dt)
            inter.append(2 * cnt)
    v = sum(inter) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid phantom)", "config": config_dict(c),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": ref.threads(), "kind": ref.kind,
                             "sample": ref.sample()},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------- ceilings of the walks ----------------

def measure_ceilings(dev):
    """L2 read bandwidth and L2 reduction rate of this GPU (nefct_probe_*),
    over 32 MiB buffers (L2-resident), best of 3 after a warm-up."""
    import ctypes as C
    import torch
    from nefct_b200 import _lib
    lib = _lib.load()
    n = 8 << 20                                   # 32 MiB of floats
    buf = torch.ones(n, device=dev)
    sink = torch.empty(int(lib.nefct_probe_sink_floats(8)), device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    out = {}
    for name, reps, call in (
            ("l2_read", 200, lambda r: _lib.call("nefct_probe_l2_read", buf.data_ptr(), n, r, 8, sink.data_ptr(), s)),
            ("l2_red", 20, lambda r: _lib.call("nefct_probe_l2_red", buf.data_ptr(), n, r, 8, s))):
        call(2)
        best = None
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            call(reps)
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1) / 1e3
            best = t if best is None else min(best, t)
        out[name] = (reps * n, best)
    nr, tr = out["l2_read"]
    nd, td = out["l2_red"]
    del buf, sink
    return {"l2_read_gbs": 4 * nr / tr / 1e9, "l2_reductions_per_s": nd / td,
            "how": "nefct_probe_l2_read (16-byte ld.global.cg) and nefct_probe_l2_red (coalesced "
                   "red.global.add.f32) over 32 MiB, 8 x 148 CTAs of 256 threads, best of 3"}


# ---------------- GPU arm ----------------

def run_gpu(args):
    import torch
    import nefct_b200 as nb
    from nefct_b200 import _lib, autotune, ops

    c = SCANS[args.workload]
    c["nv"] = args.views or c["nv"]
    legs = set(args.legs.split(","))
    rank, ws, local = dist_setup()
    dev = torch.device("cuda", local)
    n = c["n"]
    ang = angles(c)
    geom = nb.ConeBeam((n, n, n), ang, c["src_iso"], c["src_det"], c["na"], c["pixel"], c["nb"], c["pixel"],
                       size=(n * c["voxel"],) * 3)
    cr = dict(c, seed=c["seed"] + rank)
    vol = phantom_xfast(cr, device=dev)
    inter = ops.cb_count_intersections(geom, 0, device=dev)
    rays = c["nv"] * c["na"] * c["nb"]
    vbytes, sbytes = 4 * n ** 3, 4 * rays
    sino = torch.empty(geom.sino_shape, device=dev)
    back = torch.empty(geom.vol_shape, device=dev)
    gen = torch.Generator(device=dev).manual_seed(35 + rank)
    grad = torch.rand(geom.sino_shape, device=dev, generator=gen) + 0.5     # dense incoming gradient
    flush = torch.empty(256 * 2 ** 20 // 4, device=dev)

    ceil = measure_ceilings(dev)

    if args.rows:
        autotune.apply(args.rows, args.order, args.walk)               # fixed launch shape (profiling)
        tuned = {"rows": args.rows, "order": args.order, "walk": args.walk, "ms": None, "views": None}
    else:
        # untimed launch-shape choice on every tune_every-th view of the scan
        sub = geom.subset(np.arange(0, c["nv"], c["tune_every"]))
        tuned = dict(autotune.tune_cone_beam(sub, 0, dev, use_cache=False), views=sub.nv)
    for _ in range(args.warmup):
        ops.cb_forward(vol, geom, 0, out=sino)
        ops.cb_backward(grad, geom, 0, out=back)
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
    t_bwd = sum(b.elapsed_time(e) for _, b, e in ev) / 1e3
    t_step = max_over_ranks(t_fwd + t_bwd, ws)
    value = ws * args.steps * 2 * inter / t_step
    del flush

    # e2e through the public op API with pinned host buffers, the traffic of
    # the drop-in pair (Project3D: volume in, sinogram out; BackProject3D:
    # sinogram in, volume out): every step uploads its volume and its
    # incoming gradient sinogram, runs forward + adjoint, and downloads the
    # forward sinogram and the adjoint volume.  Copies run on their own
    # streams with double-buffered device tensors, so step i's uploads
    # overlap step i-1's kernels and its downloads overlap step i+1's; every
    # copy lies inside the timed region.
    e2e = None
    if "e2e" in legs:
        h_vol = torch.empty(geom.vol_shape, pin_memory=True)
        h_vol.copy_(vol.cpu())
        h_grad = torch.empty(geom.sino_shape, pin_memory=True)
        h_grad.copy_(grad.cpu())
        h_sino = [torch.empty(geom.sino_shape, pin_memory=True) for _ in range(2)]
        h_back = [torch.empty(geom.vol_shape, pin_memory=True) for _ in range(2)]
        d_vol = [torch.empty_like(vol) for _ in range(2)]
        d_grad = [torch.empty_like(grad) for _ in range(2)]
        d_sino = [torch.empty_like(sino) for _ in range(2)]
        d_back = [torch.empty_like(back) for _ in range(2)]
        ks = torch.cuda.current_stream()
        hs, ds = torch.cuda.Stream(), torch.cuda.Stream()

        def e2e_steps(count, start):
            ev_up = [torch.cuda.Event() for _ in range(2)]
            ev_f = [torch.cuda.Event() for _ in range(2)]
            ev_k = [torch.cuda.Event() for _ in range(2)]
            ev_dn = [torch.cuda.Event() for _ in range(2)]
            hs.wait_event(start)
            for i in range(count):
                b = i % 2
                if i >= 2:
                    hs.wait_event(ev_k[b])        # step i-2's kernels are done with d_vol[b], d_grad[b]
                with torch.cuda.stream(hs):
                    d_vol[b].copy_(h_vol, non_blocking=True)
                    d_grad[b].copy_(h_grad, non_blocking=True)
                ev_up[b].record(hs)
                ks.wait_event(ev_up[b])
                if i >= 2:
                    ks.wait_event(ev_dn[b])       # step i-2's downloads have read d_sino[b], d_back[b]
                ops.cb_forward(d_vol[b], geom, 0, out=d_sino[b])
                ev_f[b].record(ks)
                ops.cb_backward(d_grad[b], geom, 0, out=d_back[b])
                ev_k[b].record(ks)
                ds.wait_event(ev_f[b])
                with torch.cuda.stream(ds):
                    h_sino[b].copy_(d_sino[b], non_blocking=True)
                ds.wait_event(ev_k[b])
                with torch.cuda.stream(ds):
                    h_back[b].copy_(d_back[b], non_blocking=True)
                ev_dn[b].record(ds)
            for e in ev_dn:
                ks.wait_event(e)

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
        e2e = {"value": ws * args.steps * 2 * inter / t_e2e, "unit": UNIT, "h2d_bytes_per_step": vbytes + sbytes,
               "d2h_bytes_per_step": sbytes + vbytes, "ms_per_step": 1e3 * t_e2e / args.steps}
        del h_vol, h_grad, h_sino, h_back, d_vol, d_grad, d_sino, d_back
        torch.cuda.empty_cache()

    # rooflines of both kernels against the ceilings measured above: the
    # HBM copy bandwidth (compulsory bytes), the L2 read bandwidth (forward
    # gathers) and the L2 reduction rate (transpose)
    peak, peak_kind = load_peaks()
    fwd_s, bwd_s = t_fwd / args.steps, t_bwd / args.steps
    walk = tuned["walk"]
    names = {"fwd": "cb_colwarp_rows_kernel<forward>" if walk & 1 else "cb_forward_kernel",
             "bwd": "cb_colwarp_kernel<transpose>" if walk & 2 else "cb_backward_kernel"}
    traffic = load_traffic(args.workload)
    issue = load_issue(args.workload)
    clk_sum = clk.summary()
    sm_hz = 1e6 * (clk_sum.get("sm_mhz") or clk_sum.get("sm_max_mhz") or 1965.0)
    n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
    roof = {}
    for d, t, alg, comp in (("fwd", fwd_s, 4 * inter + 4 * rays, vbytes + sbytes),
                            ("bwd", bwd_s, 8 * inter + 4 * rays, 2 * vbytes + sbytes)):
        t_hbm = comp / (peak * 1e9)
        t_l2 = (4 * inter / (ceil["l2_read_gbs"] * 1e9)) if d == "fwd" else inter / ceil["l2_reductions_per_s"]
        tr = traffic.get(names[d])
        roof[d] = {"kernel": names[d], "ms": 1e3 * t, "algorithmic_bytes": alg, "compulsory_bytes": comp,
                   "traffic": tr, "traffic_gbs": tr / t / 1e9 if tr else None,
                   "t_hbm_ms": 1e3 * t_hbm, "t_l2_ms": 1e3 * t_l2,
                   "binding": "l2_read" if d == "fwd" and t_l2 >= t_hbm else
                              "l2_reductions" if t_l2 >= t_hbm else "hbm",
                   "frac_binding": max(t_hbm, t_l2) / t}
        per_view = issue.get(names[d])
        if per_view:
            # one warp instruction per cycle on each of the 4 schedulers of every SM
            inst = per_view * geom.nv
            t_issue = inst / (4 * n_sm * sm_hz)
            roof[d]["issue_ceiling"] = {"warp_instructions": inst, "ms": 1e3 * t_issue, "frac": t_issue / t,
                                        "sm_mhz": sm_hz / 1e6}
    dom = "bwd" if bwd_s >= fwd_s else "fwd"
    rd = roof[dom]
    achieved = rd["algorithmic_bytes"] / (rd["ms"] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": rd["kernel"], "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "algorithmic_bytes": rd["algorithmic_bytes"],
                "traffic": rd["traffic"],
                "traffic_frac_of_hbm": rd["traffic_gbs"] / peak if rd["traffic_gbs"] else None,
                "binding_ceiling": rd["binding"], "frac_of_binding_ceiling": rd["frac_binding"],
                "ceilings": ceil, "per_kernel": roof}

    extras = {"intersections_per_direction": inter, "rays": rays,
              "forward_ms": 1e3 * fwd_s, "adjoint_ms": 1e3 * bwd_s,
              "forward_intersections_per_s": inter / fwd_s, "adjoint_intersections_per_s": inter / bwd_s,
              "wall_s_timed_loop": wall,
              "launch_shape": {"rows_per_cta": tuned["rows"],
                               "grid_order": "row-band outermost" if tuned["order"] == 0 else "view outermost",
                               "walk": {"forward": "column warps" if walk & 1 else "thread per ray",
                                        "adjoint": "column warps" if walk & 2 else "thread per ray"},
                               "tuned_on_views": tuned.get("views"), "autotune_ms": tuned["ms"]}}

    # parity and CPU baseline: the reference's host build on sampled views
    # of this scan, element-wise against the GPU kernels on the same views
    cpu = None
    if rank == 0 and ws == 1 and "parity" in legs:
        cpu, extras["parity"] = parity_and_baseline(c, geom, vol, dev)

    if "extras" in legs and rank == 0 and ws == 1:
        extras.update(other_scans(c, dev, with_cpu="parity" in legs))

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_step / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid phantom)",
                "config": config_dict(c), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": 4 * args.steps, "clocks": clk.summary(), "extras": extras}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def parity_and_baseline(c, geom, vol, dev):
    """Times the reference's host build on CPU_VIEWS_PER_STEP-view samples
    (3 steps) and compares its forward sinograms and backprojections with the
    GPU's for the same views (rel-L2, max-abs / max); states the GPU
    forward's error against the oracle's FP64 walk on the first sample."""
    import torch
    from nefct_b200 import _lib, ops
    import oracle
    ref = HostReference(c, vol.cpu().numpy())
    tot_i, tot_t = 0, 0.0
    worst = {"forward_rel_l2": 0.0, "forward_max_abs_over_max": 0.0, "backprojection_rel_l2": 0.0,
             "backprojection_max_abs_over_max": 0.0}

    def err(a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b)), float(np.abs(a - b).max() / np.abs(b).max())

    views = []
    for s in range(3):
        idx = sample_views(c, s)
        views += idx
        cnt = ref.count(idx)
        dt, r_sino, r_back = ref.step(idx)
        tot_i += 2 * cnt
        tot_t += dt
        sub = geom.subset(idx)
        g_sino = ops.cb_forward(vol, sub, 0).cpu().numpy()
        g_back = ops.cb_backward(torch.from_numpy(r_sino).to(dev), sub, _lib.REF_BACKPROJECT).cpu().numpy()
        for key, (a, b) in (("forward", (g_sino, r_sino)), ("backprojection", (g_back, r_back))):
            rl, ma = err(a, b)
            worst[f"{key}_rel_l2"] = max(worst[f"{key}_rel_l2"], rl)
            worst[f"{key}_max_abs_over_max"] = max(worst[f"{key}_max_abs_over_max"], ma)
        if s == 0:
            f64, _ = oracle.cb_forward(ref.g, ref.vol, ref.ang[idx], *ref.args, f64=True)
            worst["forward_rel_l2_vs_fp64_oracle"], _ = err(g_sino, f64)
            worst["reference_forward_rel_l2_vs_fp64_oracle"], _ = err(r_sino, f64)
    worst.update({"views": views, "against": ref.kind, "bar": "rel-L2 <= 1e-5, max-abs <= 1e-4 x max",
                  "backprojection": "reference backprojection (no 1/L^2) of the reference's own sinogram"})
    cpu = {"value": tot_i / tot_t, "unit": UNIT, "cores": ref.threads(), "kind": ref.kind,
           "sample": ref.sample().replace("per step", "per step (3 steps)")}
    return cpu, worst


def other_scans(c, dev, with_cpu=False):
    """Extras beside the headline: the fwd+adjoint pair on the other scan,
    and FDK (Ram-Lak, Shepp-Logan, Parker short scan) of the FDK scanner."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops, recon
    out = {}
    f = SCANS["fdk-scanner"]
    n = f["n"]
    geom = nb.ConeBeam((n, n, n), angles(f), f["src_iso"], f["src_det"], f["na"], f["pixel"], f["nb"], f["pixel"],
                       size=(n * f["voxel"],) * 3)
    vol = phantom_xfast(f, device=dev)
    if c is not f:
        inter = ops.cb_count_intersections(geom, 0, device=dev)
        y = torch.rand(geom.sino_shape, device=dev, generator=torch.Generator(device=dev).manual_seed(36)) + 0.5
        sino, back = torch.empty(geom.sino_shape, device=dev), torch.empty(geom.vol_shape, device=dev)
        for _ in range(2):
            ops.cb_forward(vol, geom, 0, out=sino)
            ops.cb_backward(y, geom, 0, out=back)
        ef = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        reps = 5
        ts = [0.0, 0.0]
        for _ in range(reps):
            ef[0].record()
            ops.cb_forward(vol, geom, 0, out=sino)
            ef[1].record()
            ops.cb_backward(y, geom, 0, out=back)
            ef[2].record()
            torch.cuda.synchronize()
            ts[0] += ef[0].elapsed_time(ef[1]) / 1e3 / reps
            ts[1] += ef[1].elapsed_time(ef[2]) / 1e3 / reps
        out["fdk_scanner_fwd_adjoint"] = {"workload": workload_name(f), "forward_ms": 1e3 * ts[0],
                                          "adjoint_ms": 1e3 * ts[1],
                                          "intersections_per_s": 2 * inter / (ts[0] + ts[1])}
        del y, sino, back
    fdk = {}
    lines = ops.cb_forward(vol, geom, nb._lib.LINE_INTEGRAL)
    c3 = slice(n // 4, 3 * n // 4)
    filt_rl = None
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
        e = float((rec[c3, c3, c3] - vol[c3, c3, c3]).norm() / vol[c3, c3, c3].norm())
        if filt_rl is None:
            filt_rl = filt
        fdk[win] = {"filter_ms": 1e3 * t_f, "backproject_ms": 1e3 * t_b,
                    "voxels_per_s": n ** 3 / (t_f + t_b), "voxel_views_per_s": n ** 3 * f["nv"] / t_b,
                    "central_rel_error_vs_phantom": e}
    # short scan 180 deg + fan with Parker weights in the direction the
    # geometry gives (views spaced like the full scan)
    fan = 2 * np.degrees(np.arctan(f["na"] * f["pixel"] / 2 / f["src_det"]))
    step = 360.0 / f["nv"]
    nss = int(np.ceil((180 + fan) / step)) + 1
    gss = nb.ConeBeam((n, n, n), np.deg2rad(np.arange(nss) * step - fan / 2), f["src_iso"], f["src_det"],
                      f["na"], f["pixel"], f["nb"], f["pixel"], size=(n * f["voxel"],) * 3)
    lss = ops.cb_forward(vol, gss, nb._lib.LINE_INTEGRAL)
    d = ops.parker_direction(gss)
    rec = recon.fdk(lss, gss, "ram-lak", d)
    e = float((rec[c3, c3, c3] - vol[c3, c3, c3]).norm() / vol[c3, c3, c3].norm())
    fdk["short_scan_parker"] = {"views": nss, "dir": d, "central_rel_error_vs_phantom": e}
    fdk["workload"] = workload_name(f)
    if with_cpu:
        # the reference's voxel-driven backprojection (pixel_3d: the FDK body
        # without its distance weight) built for the host, on a 2-view
        # sample scaled to the scan, beside the GPU backprojection
        import oracle
        if oracle.have_ref():
            hs = filt_rl[:2].cpu().numpy()
            side = n * f["voxel"]
            t0 = time.perf_counter()
            oracle.ref_pixel_backproject(hs, angles(f)[:2], (n, n, n), (-side / 2,) * 3, (side,) * 3,
                                         f["src_iso"], f["src_det"], f["na"], f["pixel"], 0.0, f["nb"], f["pixel"],
                                         0.0)
            t_host = (time.perf_counter() - t0) * f["nv"] / 2
            t_b = fdk["ram-lak"]["backproject_ms"] / 1e3
            fdk["reference_host_build"] = {"cores": oracle.ref_threads(), "sample": "2 views, scaled to the scan",
                                           "pixel_backproject_ms": 1e3 * t_host,
                                           "speedup_of_fdk_backproject": t_host / t_b}
    out["fdk"] = fdk
    del lines, filt, filt_rl, rec, lss, vol
    torch.cuda.empty_cache()
    return out


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


def small_geoms(n_problems=96, seed=44):
    """Many small uneven problems (a minibatch of small reconstructions):
    edge log-uniform in [16, 64], views U{8..64}, detector rows/cols
    U{24..128}, the same scanner distribution as uneven_geoms."""
    import nefct_b200 as nb
    rng = np.random.default_rng(seed)
    geoms = []
    for _ in range(n_problems):
        n = int(round(np.exp(rng.uniform(np.log(16), np.log(64)))))
        nv = int(rng.integers(8, 65))
        rows, cols = (int(v) for v in rng.integers(24, 129, 2))
        si = float(rng.uniform(400, 700))
        sd = si * float(rng.uniform(1.5, 2.0))
        pixel = (sd / si) * n * 1.0 / cols
        ang = np.linspace(0, 2 * np.pi, nv, endpoint=False).astype(np.float32)
        geoms.append(nb.ConeBeam((n, n, n), ang, si, sd, cols, pixel, rows, pixel, size=(float(n),) * 3))
    return geoms


def run_batched(args):
    """Batched fwd+adjoint iterations/s of uneven problems: the batch plan
    replayed as a CUDA graph, and one autograd iteration through
    batch_project (loss sum_i ||A_i x_i||^2 / 2, backward = one batched
    transpose), against sequential per-problem device calls (plain and
    through autograd) and the plain per-problem drop-in path (numpy in/out
    per call, like the reference's operators; warmed up first)."""
    import torch
    import nefct_b200 as nb
    from nefct_b200 import ops
    from nefct_b200.batch import BatchProjector, batch_project
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    if args.regime == "small":
        geoms = small_geoms(args.problems if args.problems else 96)
        workload = (f"{len(geoms)} small problems, edge log-U[16,64], views U[8,64], detector U[24,128]^2, "
                    f"seed 44")
    else:
        geoms = uneven_geoms(args.problems if args.problems else 64, 4, args.scale, args.view_scale)
        workload = (f"{len(geoms)} problems, edge log-U[64,384]x{args.scale}, views U[60,720]x{args.view_scale}, "
                    f"detector U[128,1024]^2 x{args.scale}, seed 4")
    gen = torch.Generator(device=dev).manual_seed(4)
    vols = [torch.rand(g.vol_shape, device=dev, generator=gen) for g in geoms]
    # grads = the forward outputs (loss = |Ax|^2 / 2); tile shape autotuned for the small regime
    bp = BatchProjector(geoms, vols, tune_rows=args.regime == "small")
    inter = sum(ops.cb_count_intersections(g, 0, dev) for g in geoms)

    def timed(fn, reps):
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

    graph = bp.capture()
    t_batch = timed(graph.replay, args.steps)
    strategies = {}
    for name in ("persistent", "per-problem"):
        bp.set_strategy(name)
        g2 = bp.capture()
        strategies[name] = 1e3 * timed(g2.replay, args.steps)
        del g2
    best = min(strategies, key=strategies.get)
    bp.set_strategy(best)

    # one autograd iteration through the batched Function (a plan of the same tile shape)
    from nefct_b200 import autotune
    xs = [v.clone().requires_grad_() for v in vols]
    saved = autotune.current()
    if bp.tuned_rows:
        autotune.apply(bp.tuned_rows["rows"], saved["order"])
    grads_bp = BatchProjector(geoms, [v.detach().clone() for v in vols],
                              grads=[torch.empty(g.sino_shape, device=dev) for g in geoms], strategy=best)
    autotune.apply(saved["rows"], saved["order"])

    def autograd_batched():
        for x in xs:
            x.grad = None
        sinos = batch_project(grads_bp, xs)
        (sum((s * s).sum() for s in sinos) / 2).backward()
    t_autograd = timed(autograd_batched, args.steps)

    # sequential per-problem device calls (the same kernels, one problem at a time)
    sinos = [torch.empty(g.sino_shape, device=dev) for g in geoms]
    backs = [torch.empty(g.vol_shape, device=dev) for g in geoms]

    def sequential():
        for g, v, s_, b in zip(geoms, vols, sinos, backs):
            ops.cb_forward(v, g, 0, out=s_)
            ops.cb_backward(s_, g, 0, out=b)
    t_seq = timed(sequential, max(1, args.steps // 2))

    def sequential_autograd():
        for g, x in zip(geoms, xs):
            x.grad = None
            s_ = nb.project(x, g)
            ((s_ * s_).sum() / 2).backward()
    t_seq_ag = timed(sequential_autograd, max(1, args.steps // 2))

    # plain drop-in path: numpy volume in, Project3D, BackProject3D, numpy out
    sc = [nb.ScannerConfig3D("flat", g.src_det, g.src_iso, nb.DetectorDirectAConfig(g.na, g.na * g.da),
                             nb.DetectorDirectBConfig(g.nb, g.nb * g.db)) for g in geoms]
    host = [v.permute(2, 1, 0).cpu().numpy() for v in vols]

    def plain(idx):
        for i in idx:
            g = geoms[i]
            img = nb.Image3D(host[i], [0, 0, 0], list(g.size))
            proj = nb.Project3D(sc[i], g.angles, None)(img)
            nb.BackProject3D(sc[i], list(g.shape), 1.0, "transpose")(proj)
        torch.cuda.synchronize()
    plain(range(min(4, len(geoms))))                 # warm-up (first calls, allocator growth)
    t0 = time.perf_counter()
    plain(range(len(geoms)))
    t_plain = time.perf_counter() - t0
    line = {"metric": "batched autograd fwd+adjoint iterations/s (uneven cone-beam problems)",
            "value": 1.0 / t_autograd, "unit": "iterations/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_autograd, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform random volumes)",
            "config": {"workload": workload, "voxels": int(sum(np.prod(g.shape) for g in geoms)),
                       "rays": int(sum(g.nv * g.na * g.nb for g in geoms)), "tiles": bp.tiles},
            "extras": {"strategy": best, "graph_replay_ms_by_strategy": strategies,
                       "tile_shape_tuning": bp.tuned_rows,
                       "intersections_per_iteration": 2 * inter,
                       "batched_graph_replay_ms": 1e3 * t_batch,
                       "batched_autograd_ms": 1e3 * t_autograd,
                       "batched_autograd_intersections_per_s": 2 * inter / t_autograd,
                       "sequential_device_ms": 1e3 * t_seq, "sequential_device_autograd_ms": 1e3 * t_seq_ag,
                       "plain_dropin_ms": 1e3 * t_plain,
                       "speedup_vs_plain_dropin": t_plain / t_autograd,
                       "speedup_vs_sequential_device": t_seq / t_autograd,
                       "speedup_vs_sequential_device_autograd": t_seq_ag / t_autograd,
                       "graph_replay_speedup_vs_sequential_device": t_seq / t_batch}}
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
    CFG = SCANS["fdk-scanner"]
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
    ang = angles(CFG)[::10]
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
    ang72 = angles(CFG)[::5]
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
                "cores": oracle.ref_threads(), "lor_forward_lors_per_s": k / t_cpu_lor,
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
    ap.add_argument("--workload", default="diff-projector",
                    choices=["diff-projector", "fdk-scanner", "batched", "diff512", "motion4d", "rows"],
                    help="diff-projector: the headline scan (512^3, 720 views); fdk-scanner: the same step on the "
                         "256^3 / 360-view scanner; the others print their own JSON lines")
    ap.add_argument("--legs", default="e2e,parity,extras",
                    help="parts of the scan workloads besides the timed loop: e2e (host copies), parity (reference "
                         "host build on sampled views, CPU baseline), extras (the other scan, FDK)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the reference host-build legs")
    ap.add_argument("--views", type=int, default=0, help="views of the scan (0 = the workload's; fewer only for "
                                                         "profiling)")
    ap.add_argument("--rows", type=int, default=0, help="fix the detector rows per CTA instead of autotuning")
    ap.add_argument("--order", type=int, default=0, help="with --rows: 0 row bands outermost, 1 views outermost")
    ap.add_argument("--walk", type=int, default=3,
                    help="with --rows: column warps for the forward (bit 0) / adjoint (bit 1), else thread per ray")
    ap.add_argument("--problems", type=int, default=0, help="batched: problem count (0 = the regime's)")
    ap.add_argument("--regime", default="uneven", choices=["uneven", "small"],
                    help="batched: the 64 uneven problems (edges 64..384) or 96 small ones (edges 16..64)")
    ap.add_argument("--scale", type=float, default=1.0, help="batched: scale of volume edges and detector sizes")
    ap.add_argument("--view-scale", type=float, default=1.0, help="batched: scale of the view counts")
    args = ap.parse_args()
    if args.no_cpu:
        args.legs = ",".join(x for x in args.legs.split(",") if x != "parity")
    if args.impl == "reference":
        if args.workload not in SCANS:
            print(json.dumps({"impl": "reference", "unavailable": f"no reference arm for workload {args.workload}"}))
            return
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
