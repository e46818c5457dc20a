"""z-slab decomposition of one solve (the gpe_create_slab family of the C
ABI): the reference's MPI domain decomposition (src/variables.f90:203-375)
along z, with an NCCL transport for one process per GPU and an in-process
hub whose slabs are driven by one host thread each."""
from __future__ import annotations

import ctypes as C
import threading

import numpy as np

from . import _lib as L
from .solver import RunParams, Solver


def partition(nz: int, nranks: int, rank: int) -> tuple[int, int]:
    """(k0, nzl) of slab `rank`: the first nz % nranks slabs get one plane more."""
    lib = L.load()
    k0, nzl = C.c_int32(), C.c_int32()
    rc = lib.gpe_slab_partition(int(nz), int(nranks), int(rank), C.byref(k0), C.byref(nzl))
    if rc != L.GPE_OK:
        raise ValueError("bad slab partition arguments")
    return k0.value, nzl.value


def nccl_unique_id() -> bytes:
    """The 128-byte NCCL id rank 0 creates and sends to every rank."""
    lib = L.load()
    buf = C.create_string_buffer(128)
    rc = lib.gpe_slab_nccl_id(buf)
    if rc != L.GPE_OK:
        raise L.GpeError(rc, (lib.gpe_last_error(None) or b"").decode())
    return buf.raw


class SlabHub:
    """The in-process transport: n slabs on the current device, one host
    thread per slab, one shared stream."""

    def __init__(self, nslabs: int):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.gpe_slab_hub_create(int(nslabs), C.byref(h))
        if rc != L.GPE_OK:
            raise L.GpeError(rc, (self.lib.gpe_last_error(None) or b"").decode())
        self.h = h
        self.n = nslabs

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gpe_slab_hub_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_threaded(params: RunParams, nslabs: int, body) -> list:
    """Run body(solver) for each slab of a hub on its own thread; returns the
    bodies' results in rank order.  Each slab is destroyed (collectively)
    after its body returns; the first exception is re-raised."""
    hub = SlabHub(nslabs)
    out: list = [None] * nslabs
    errs: list = []

    def work(r: int) -> None:
        s = None
        try:
            s = Solver(params, rank=r, nranks=nslabs, hub=hub)
            out[r] = body(s)
        except BaseException as e:  # noqa: BLE001 - reported to the caller
            errs.append(e)
        finally:
            if s is not None:
                s.close()

    ts = [threading.Thread(target=work, args=(r,)) for r in range(nslabs)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    hub.close()
    if errs:
        raise errs[0]
    return out


def step_decomposed(params: RunParams, psi: np.ndarray, nslabs: int, nsteps: int, want_norm: bool = True):
    """One solve split into nslabs z-slabs of a hub: (final psi, norm)."""

    def body(s: Solver):
        s.set_state(psi[s.k0:s.k0 + s.nzl])
        info = s.solver(nsteps, want_norm=want_norm)
        return s.get_state(), info.norm, (s.t, s.im_t, s.dt, s.p)

    res = run_threaded(params, nslabs, body)
    return np.concatenate([r[0] for r in res], axis=0), res[0][1], res[0][2]
