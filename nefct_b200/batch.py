"""Batched uneven cone-beam problems: one persistent launch per direction,
optionally replayed as a CUDA graph (include/nefct_b200.h, nefct_cb_batch_*).

    bp = BatchProjector(geoms, vols)          # plans, allocates, binds
    bp.step()                                 # forward of all, then transpose of all
    g = bp.capture()                          # CUDA graph of one step; g.replay()
    sinos = bp.project(vols)                  # autograd: backward runs the batched transpose

Per problem i: ``sinos[i] = A_i vols[i]`` and ``backs[i] = A_i^T grads[i]``
(``grads`` defaults to ``sinos``).  Forward outputs are bitwise equal to
``ops.cb_forward`` of each problem (same per-ray code).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib, ops

__all__ = ["BatchProjector", "batch_project"]


def _direct(t: torch.Tensor | None, like: torch.Tensor) -> bool:
    """True when t can be read by the plan in place of its bound tensor."""
    return (t is not None and t.is_contiguous() and t.dtype == torch.float32 and t.device == like.device
            and t.shape == like.shape)


class _BatchProject(torch.autograd.Function):
    """Forward: the plan's batched forward of every problem; backward: the
    plan's batched exact transpose of the incoming gradients.  Inputs are
    read in place (the plan is pointed at them for the one launch, then back
    at its own tensors) when they are contiguous float32 tensors of the
    plan's shapes, else copied into the bound tensors; the returned sinograms
    are the plan's bound output tensors (no copy), valid until the plan's
    next forward."""

    @staticmethod
    def forward(ctx, bp, *vols):
        use = [v if _direct(v, dst) else None for v, dst in zip(vols, bp.vols)]
        for v, u, dst in zip(vols, use, bp.vols):
            if u is None and v.data_ptr() != dst.data_ptr():
                dst.copy_(v)
        rebound = any(u is not None and u.data_ptr() != dst.data_ptr() for u, dst in zip(use, bp.vols))
        if rebound:
            bp._set_buffers(vols=use)
        try:
            bp.forward()
        finally:
            if rebound:
                bp._set_buffers(vols=bp.vols)
        ctx.bp = bp
        return tuple(bp.sinos)

    @staticmethod
    def backward(ctx, *grads):
        bp = ctx.bp
        use = [g if _direct(g, dst) else None for g, dst in zip(grads, bp.grads)]
        for g, u, dst in zip(grads, use, bp.grads):
            if u is not None:
                continue
            if g is None:
                dst.zero_()
            elif g.data_ptr() != dst.data_ptr():
                dst.copy_(g)
        rebound = any(u is not None and u.data_ptr() != dst.data_ptr() for u, dst in zip(use, bp.grads))
        if rebound:
            bp._set_buffers(grads=use)
        try:
            bp.backward()
        finally:
            if rebound:
                bp._set_buffers(grads=bp.grads)
        return (None, *bp.backs)


def batch_project(bp: "BatchProjector", vols: list) -> tuple:
    """Differentiable batched forward projection of vols (one per problem of
    the plan); d(loss)/d(vols[i]) = A_i^T d(loss)/d(sinos[i]), computed by
    one batched transpose."""
    if len(vols) != len(bp.vols):
        raise _lib.NefctError(_lib.ERR_INVALID, f"{len(vols)} volumes for a plan of {len(bp.vols)} problems")
    for v, g in zip(vols, bp.geoms):
        if tuple(v.shape) != g.vol_shape or v.dtype != torch.float32 or v.device != bp.device:
            raise _lib.NefctError(_lib.ERR_INVALID, "volumes must match the plan (float32 [nz, ny, nx], its device)")
    return _BatchProject.apply(bp, *vols)


class BatchProjector:
    def __init__(self, geoms: list[ops.ConeBeam], vols: list[torch.Tensor], sinos=None, grads=None, backs=None,
                 flags: int = 0, strategy: str = "auto", tune_rows: bool = False):
        if len(geoms) != len(vols) or not geoms:
            raise ValueError("need one volume per geometry")
        dev = vols[0].device
        self.geoms = list(geoms)
        self.vols = [v.contiguous() for v in vols]
        for g, v in zip(self.geoms, self.vols):
            if v.dtype != torch.float32 or tuple(v.shape) != g.vol_shape or v.device != dev:
                raise _lib.NefctError(_lib.ERR_INVALID, "volumes must be float32 [nz, ny, nx] on one device")
        self.sinos = sinos or [torch.empty(g.sino_shape, device=dev) for g in geoms]
        self.grads = grads or self.sinos
        self.backs = backs or [torch.empty(g.vol_shape, device=dev) for g in geoms]
        self.flags = flags
        self.device = dev
        self.tuned_rows = None
        if tune_rows:
            self.tuned_rows = self._tune_rows(strategy)
            strategy = self.tuned_rows["strategy"]
        n = len(geoms)
        probs = (_lib.CBProblem * n)()
        self._structs = []
        for i, g in enumerate(self.geoms):
            probs[i].geom = g.struct()
            probs[i].vol = self.vols[i].data_ptr()
            probs[i].sino = self.sinos[i].data_ptr()
            probs[i].grad = self.grads[i].data_ptr()
            probs[i].back = self.backs[i].data_ptr()
        lib = _lib.load()
        plan = C.c_void_p()
        nbytes = C.c_size_t()
        try:
            _lib.check(lib.nefct_cb_batch_plan(probs, n, flags, C.byref(plan), C.byref(nbytes)))
        finally:
            if self.tuned_rows is not None:          # the plan has fixed its rows: restore the caller's
                from . import autotune
                autotune.apply(self.tuned_rows["saved_rows"], self.tuned_rows["saved_order"])
        self._plan = plan
        self.workspace = torch.empty(nbytes.value, dtype=torch.uint8, device=dev)
        with torch.cuda.device(dev):
            _lib.check(lib.nefct_cb_batch_bind(plan, self.workspace.data_ptr(), nbytes.value,
                                               torch.cuda.current_stream(dev).cuda_stream))
        self.tiles = int(lib.nefct_cb_batch_tiles(plan))
        self.timings = {}
        if strategy == "auto":
            strategy = self._pick()
        self.set_strategy(strategy)

    def _tune_rows(self, strategy: str) -> dict:
        """Autotunes the plan's tile shape: times one step of a plan with 2,
        4 and 8 rows (columns, for column warps) per CTA under each strategy
        and applies the fastest rows setting (NEFCT_TUNE_CB_ROWS) for the
        plan to fix; the caller's setting is restored once it has."""
        from . import autotune
        saved = autotune.current()
        times = {}
        try:
            for rows in (2, 4, 8):
                autotune.apply(rows, saved["order"])
                trial = BatchProjector(self.geoms, self.vols, sinos=self.sinos, grads=self.grads, backs=self.backs,
                                       flags=self.flags, strategy=strategy)
                for name, ms in (trial.timings or {trial.strategy: None}).items():
                    if ms is None:
                        trial.step()
                        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        e0.record()
                        trial.step()
                        e1.record()
                        e1.synchronize()
                        ms = e0.elapsed_time(e1)
                    times[f"{rows}/{name}"] = ms
                del trial
            best = min(times, key=times.get)
            rows, strat = best.split("/")
            autotune.apply(int(rows), saved["order"])
            return {"rows": int(rows), "strategy": strat, "ms": times, "saved_rows": saved["rows"],
                    "saved_order": saved["order"]}
        except Exception:
            autotune.apply(saved["rows"], saved["order"])
            raise

    def set_strategy(self, strategy: str) -> None:
        code = {"persistent": _lib.BATCH_PERSISTENT, "per-problem": _lib.BATCH_PER_PROBLEM}[strategy]
        _lib.check(_lib.load().nefct_cb_batch_set_strategy(self._plan, code))
        self.strategy = strategy

    def _pick(self) -> str:
        """Times one step with each strategy (after a warm-up) and returns the faster."""
        for name in ("persistent", "per-problem"):
            self.set_strategy(name)
            self.step()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            self.step()
            e1.record()
            e1.synchronize()
            self.timings[name] = e0.elapsed_time(e1)
        return min(self.timings, key=self.timings.get)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _set_buffers(self, vols=None, grads=None):
        """Points the plan's problems at other volumes / gradient sinograms
        (lists in problem order; None entries keep the current buffer) until
        the next call (nefct_cb_batch_set_buffers; host-only)."""
        def arr(ts):
            if ts is None:
                return None
            return (C.c_void_p * len(ts))(*[None if t is None else t.data_ptr() for t in ts])
        _lib.check(_lib.load().nefct_cb_batch_set_buffers(self._plan, arr(vols), None, arr(grads), None))

    def forward(self):
        _lib.check(_lib.load().nefct_cb_batch_forward(self._plan, self._stream()))
        return self.sinos

    def backward(self):
        _lib.check(_lib.load().nefct_cb_batch_backward(self._plan, self._stream()))
        return self.backs

    def step(self):
        self.forward()
        self.backward()

    def project(self, vols: list) -> tuple:
        """batch_project(self, vols): differentiable batched forward."""
        return batch_project(self, vols)

    def capture(self) -> torch.cuda.CUDAGraph:
        """CUDA graph of one step (forward of all problems, then transpose of all)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.step()                      # warm-up outside the capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step()
        return g

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib.load().nefct_cb_batch_destroy(plan)
            except Exception:
                pass
            self._plan = None
