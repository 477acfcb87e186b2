"""Batched execution: many TlmSolver handles advanced by one launch per step.

A ``Batch`` drives solvers that were set up as usual. Members of one storage
mode share each step's kernel launch; windows of ``steps_per_launch`` steps
are replayed as CUDA graphs; members join and leave between windows; each
runs to its own ``totalSteps``. Results are read from the member solvers and
are bitwise those of the same solver stepped alone.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib
from ._lib import check


@dataclass
class BatchTuning:
    kernel_variant: int = 0
    steps_per_launch: int = 64
    blocks_per_sm: int = 0
    use_graphs: bool = True
    overlap: bool = False
    ms_per_step: float = 0.0

    def to_c(self):
        return _lib.BatchTuningC(int(self.kernel_variant), int(self.steps_per_launch),
                                 int(self.blocks_per_sm), 1 if self.use_graphs else 0,
                                 1 if self.overlap else 0, float(self.ms_per_step))

    @classmethod
    def from_c(cls, c):
        return cls(c.kernel_variant, c.steps_per_launch, c.blocks_per_sm, bool(c.use_graphs),
                   bool(c.overlap), c.ms_per_step)


class Batch:
    def __init__(self, device: int = 0, variant: str | None = None):
        self._L = _lib.load(variant)
        h = C.c_void_p()
        st = self._L.tlm_batch_create(C.byref(h), device)
        if st != _lib.TLM_OK:
            raise _lib.TlmError(st, self._L.tlm_last_error(None).decode())
        self._b = h
        self._members = []

    def _c(self, status):
        return check(self._L, None, status)

    def attach(self, solver):
        self._c(self._L.tlm_batch_attach(self._b, solver._h))
        self._members.append(solver)

    def detach(self, solver):
        self._c(self._L.tlm_batch_detach(self._b, solver._h))
        self._members.remove(solver)

    def size(self):
        return self._L.tlm_batch_size(self._b)

    def active(self):
        return self._L.tlm_batch_active(self._b)

    def step(self, n: int):
        self._c(self._L.tlm_batch_step(self._b, int(n)))

    def run(self):
        self._c(self._L.tlm_batch_run(self._b))

    def launch_window(self) -> int:
        """Queue one window without waiting; returns its length in steps (0
        when no member is active). Call sync() before attaching, detaching
        or reading members."""
        n = C.c_int(0)
        self._c(self._L.tlm_batch_launch_window(self._b, C.byref(n)))
        return n.value

    def sync(self):
        self._c(self._L.tlm_batch_sync(self._b))

    def solve(self, workloads, build, collect, chunk: int = 32):
        """Solve every workload through this batch and return collect(solver,
        workload) for each, in order. While the device runs a window for the
        attached members, the host sets up (build(w), then prepares the
        solver's tables) the next `chunk` workloads, which join at the next
        window; a member that reaches its last step is collected, detached
        and closed at once, so its device memory serves the next ones."""
        pending = list(enumerate(workloads))
        running = {}
        out = [None] * len(pending)
        while pending or running:
            launched = self.launch_window() if running else 0
            fresh = []
            for k, w in pending[:chunk]:
                s = build(w)
                s.stepAsync(0)  # builds the source/monitor and tile tables now, on the host
                fresh.append((k, w, s))
            pending = pending[chunk:]
            if launched:
                self.sync()
            for k, w, s in fresh:
                self.attach(s)
                running[k] = (w, s)
            for k, (w, s) in list(running.items()):
                if s.currentStep() >= s.totalSteps():
                    out[k] = collect(s, w)
                    self.detach(s)
                    s.close()
                    del running[k]
        return out

    def set_tuning(self, t: BatchTuning):
        c = t.to_c()
        self._c(self._L.tlm_batch_set_tuning(self._b, C.byref(c)))

    def get_tuning(self) -> BatchTuning:
        c = _lib.BatchTuningC()
        self._c(self._L.tlm_batch_get_tuning(self._b, C.byref(c)))
        return BatchTuning.from_c(c)

    def autotune(self, trial_windows: int = 2) -> BatchTuning:
        c = _lib.BatchTuningC()
        self._c(self._L.tlm_batch_autotune(self._b, int(trial_windows), C.byref(c)))
        return BatchTuning.from_c(c)

    def stream(self):
        s = C.c_void_p()
        self._c(self._L.tlm_batch_get_stream(self._b, C.byref(s)))
        return s.value

    def close(self):
        b = getattr(self, "_b", None)
        if b is not None and b.value:
            self._L.tlm_batch_destroy(b)
        self._b = None
        self._members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
