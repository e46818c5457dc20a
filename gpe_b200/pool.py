"""Batched solves and serving over the gpe_pool_* C ABI.

A Pool owns an HBM budget.  Solves are submitted with their initial state
and step count, join the running batch at the next step() (continuous
batching), advance together -- one persistent launch per Runge-Kutta stage
per (precision, scheme) class -- and are retired into poll() with their
final state when they reach their step count.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .solver import RunParams


@dataclass
class PoolResult:
    tag: int
    status: int
    steps: int
    rejected: int
    t: float
    im_t: float
    dt: complex
    norm: float
    submit_s: float
    start_s: float
    finish_s: float
    psi: np.ndarray

    @property
    def latency_s(self) -> float:
        return self.finish_s - self.submit_s


class Pool:
    def __init__(self, budget_bytes: int):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.gpe_pool_create(int(budget_bytes), C.byref(h))
        if rc != L.GPE_OK:
            raise L.GpeError(rc, "gpe_pool_create failed")
        self.h = h
        self._out: dict[int, np.ndarray] = {}
        self._keep: dict[int, np.ndarray] = {}

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gpe_pool_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, rc):
        msg = self.lib.gpe_pool_last_error(self.h)
        return L.GpeError(rc, msg.decode() if msg else "")

    @staticmethod
    def solve_bytes(params: RunParams) -> int:
        lib = L.load()
        cp = params.to_c()
        return int(lib.gpe_pool_solve_bytes(C.byref(cp)))

    def free_bytes(self) -> int:
        return int(self.lib.gpe_pool_free_bytes(self.h))

    def submit(self, params: RunParams, psi0: np.ndarray, nsteps: int, tag: int,
               out: np.ndarray | None = None) -> bool:
        """Admit a solve; False when it does not fit in the free budget.  The
        final state is written to `out` (default: a new array); a reused
        buffer from gpe_b200._lib.pinned_empty makes the copy back a DMA."""
        dt = np.complex64 if params.storage == "c64" else np.complex128
        code = L.GPE_C64 if params.storage == "c64" else L.GPE_C128
        psi = np.ascontiguousarray(psi0, dtype=dt)
        if psi.shape != (params.nz, params.ny, params.nx):
            raise ValueError("psi0 must have shape (nz, ny, nx)")
        if out is None:
            out = np.empty_like(psi)
        elif out.shape != psi.shape or out.dtype != psi.dtype or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous array of psi0's shape and dtype")
        cp = params.to_c()
        rc = self.lib.gpe_pool_submit(self.h, C.byref(cp), psi.ctypes.data, code, int(nsteps), int(tag),
                                      out.ctypes.data)
        if rc == L.GPE_ERR_NOMEM_BUDGET:
            return False
        if rc != L.GPE_OK:
            raise self._err(rc)
        self._out[int(tag)] = out
        return True

    def submit_ic(self, params: RunParams, spec, nsteps: int, tag: int, out: np.ndarray | None = None) -> bool:
        """Admit a solve whose initial state is generated on the device."""
        dt = np.complex64 if params.storage == "c64" else np.complex128
        shape = (params.nz, params.ny, params.nx)
        if out is None:
            out = np.empty(shape, dtype=dt)
        elif out.shape != shape or out.dtype != np.dtype(dt) or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous (nz, ny, nx) array of the storage dtype")
        cp = params.to_c()
        rc = self.lib.gpe_pool_submit_ic(self.h, C.byref(cp), C.byref(spec), int(nsteps), int(tag),
                                         out.ctypes.data)
        if rc == L.GPE_ERR_NOMEM_BUDGET:
            return False
        if rc != L.GPE_OK:
            raise self._err(rc)
        self._out[int(tag)] = out
        return True

    def step(self, max_steps: int) -> int:
        n = C.c_int32()
        rc = self.lib.gpe_pool_step(self.h, int(max_steps), C.byref(n))
        if rc != L.GPE_OK:
            raise self._err(rc)
        return n.value

    def poll(self) -> list[PoolResult]:
        out = []
        buf = (L.GpeResult * 64)()
        while True:
            n = C.c_int32()
            self.lib.gpe_pool_poll(self.h, buf, 64, C.byref(n))
            for q in range(n.value):
                r = buf[q]
                out.append(PoolResult(int(r.tag), r.status, r.steps, r.rejected, r.t, r.im_t,
                                      complex(r.dt_re, r.dt_im), r.norm, r.submit_s, r.start_s, r.finish_s,
                                      self._out.pop(int(r.tag))))
            if n.value < 64:
                return out

    def run_all(self, max_steps: int = 1 << 30) -> list[PoolResult]:
        """Step until every admitted solve has finished; return all results."""
        res = []
        while True:
            active = self.step(max_steps)
            res.extend(self.poll())
            if active == 0:
                return res
