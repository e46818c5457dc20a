"""Python host interface of the B200 stepper, mirroring the reference's
solver interface (anthonyyoud/gpe):

    call solver(psi%old, psi%new)   -> Solver.solver(nsteps)      (src/solve.f90:25)
    call get_norm(psi, norm)        -> Solver.get_norm()          (src/variables.f90:554)
    call energy(psi, E)             -> Solver.energy()            (src/variables.f90:580)
    call renormalise(psi, norm)     -> Solver.renormalise(norm)   (src/variables.f90:715)
    call get_grid()                 -> Solver.grid()              (src/ic.f90:32)

The globals of src/parameters.f90 (t, im_t, dt, p) live on the Solver and
are advanced by solver() exactly as the reference's routines advance them.
Arrays are numpy complex128/complex64 of shape (nz, ny, nx) in C order,
which is the reference's psi(0:nx-1,0:ny-1,0:nz-1) memory layout.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib as L


@dataclass
class RunParams:
    """run.in / parameters.in quantities the stepper needs
    (src/parameters.f90:24-56, src/parameters.in:22-30)."""
    nx: int = 64
    ny: int = 64
    nz: int = 64
    xr: float = 16.0
    yr: float = 16.0
    zr: float = 16.0
    tau: float = 0.01
    scheme: str = "rk4"
    eqn_to_solve: int = 4
    bcs: int = 2
    order: int = 2
    real_time: bool = True
    Urhs: float = 0.0
    diss_amp: float = 0.0
    scal: float = 1.0
    g: float = 1.0
    mu: float = 1.0
    nn: float = 1.0
    omx: float = 0.0
    omy: float = 0.0
    omz: float = 0.0
    gamma: float = 0.0
    storage: str = "c128"      # "c128" | "c64"
    compute: str = "auto"      # stencil compute type for c64 storage: "auto" | "f32" | "f64"
    tile_zc: int = 0           # z planes per CTA work item (0 = library default; set by the autotuner)
    eps: float = 0.0
    safety: float = 0.0
    dt_decrease: float = 0.0
    dt_increase: float = 0.0

    def to_c(self) -> L.GpeParams:
        if self.scheme not in L.SCHEMES:
            raise ValueError("ERROR: Unrecognised time stepping scheme.")
        p = L.GpeParams()
        p.nx, p.ny, p.nz = self.nx, self.ny, self.nz
        p.scheme = L.SCHEMES[self.scheme]
        p.eqn, p.bcs, p.order = self.eqn_to_solve, self.bcs, self.order
        p.real_time = 1 if self.real_time else 0
        p.storage = {"c128": L.GPE_C128, "c64": L.GPE_C64}[self.storage]
        p.compute = {"auto": L.GPE_COMPUTE_AUTO, "f32": L.GPE_COMPUTE_F32, "f64": L.GPE_COMPUTE_F64}[self.compute]
        p.tile_zc = int(self.tile_zc)
        for f in ("xr", "yr", "zr", "tau", "Urhs", "diss_amp", "scal", "g", "mu", "nn", "omx", "omy",
                  "omz", "gamma", "eps", "safety", "dt_decrease", "dt_increase"):
            setattr(p, f, float(getattr(self, f)))
        return p

    def replace(self, **kw) -> "RunParams":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return RunParams(**d)


def _check(lib, h, rc: int) -> None:
    if rc != L.GPE_OK:
        msg = lib.gpe_last_error(h)
        raise L.GpeError(rc, msg.decode() if msg else "")


class Solver:
    """One device-resident solve."""

    def __init__(self, params: RunParams, rank: int | None = None, nranks: int = 1, nccl_id: bytes | None = None,
                 hub=None):
        """The whole grid, or with rank/nranks z-slab `rank` of a decomposed
        solve over NCCL (nccl_id from gpe_b200.slab.nccl_unique_id) or an
        in-process gpe_b200.slab.SlabHub."""
        self.lib = L.load()
        self.params = params
        self._cp = params.to_c()
        h = C.c_void_p()
        if rank is None:
            rc = self.lib.gpe_create(C.byref(self._cp), C.byref(h))
        else:
            idb = C.create_string_buffer(bytes(nccl_id), 128) if nccl_id is not None else None
            rc = self.lib.gpe_create_slab(C.byref(self._cp), int(rank), int(nranks), idb,
                                          hub.h if hub is not None else None, C.byref(h))
        _check(self.lib, None, rc)
        self.h = h
        k0, nzl = C.c_int32(), C.c_int32()
        self.lib.gpe_slab_extent(self.h, C.byref(k0), C.byref(nzl))
        self.k0, self.nzl = k0.value, nzl.value
        # src/gpe.f90:78-82
        self.t = 0.0
        self.im_t = 0.0
        self.dt = complex(params.tau, 0.0) if params.real_time else complex(0.0, -params.tau)
        self.p = 0
        self.last = L.GpeStepInfo()

    # -- lifetime -----------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.gpe_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state --------------------------------------------------------------
    @property
    def shape(self) -> tuple[int, int, int]:
        """(nz, ny, nx) of the state this handle holds (its own slab's nz)."""
        return (self.nzl, self.params.ny, self.params.nx)

    def set_state(self, psi: np.ndarray) -> None:
        psi = np.asarray(psi)
        if psi.shape != self.shape:
            raise ValueError(f"psi must have shape (nz, ny, nx) = {self.shape}")
        if psi.dtype == np.complex64:
            arr, dt = np.ascontiguousarray(psi), L.GPE_C64
        else:
            arr, dt = np.ascontiguousarray(psi, dtype=np.complex128), L.GPE_C128
        _check(self.lib, self.h, self.lib.gpe_set_state(self.h, arr.ctypes.data, dt))

    def get_state(self, dtype=np.complex128, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=dtype)
        code = L.GPE_C64 if out.dtype == np.complex64 else L.GPE_C128
        _check(self.lib, self.h, self.lib.gpe_get_state(self.h, out.ctypes.data, code))
        return out

    def snapshot_begin(self, dtype=np.complex128) -> None:
        """Start an asynchronous copy of the current state to host memory."""
        code = L.GPE_C64 if np.dtype(dtype) == np.complex64 else L.GPE_C128
        _check(self.lib, self.h, self.lib.gpe_snapshot_begin(self.h, code))
        self._snap_dtype = np.dtype(dtype)

    def snapshot_wait(self) -> np.ndarray:
        """The state captured by the last snapshot_begin (a copy)."""
        ptr, n = C.c_void_p(), C.c_size_t()
        _check(self.lib, self.h, self.lib.gpe_snapshot_wait(self.h, C.byref(ptr), C.byref(n)))
        buf = (C.c_char * n.value).from_address(ptr.value)
        return np.frombuffer(buf, dtype=self._snap_dtype).reshape(self.shape).copy()

    def set_state_async(self, psi: np.ndarray) -> None:
        """gpe_set_state_async: psi must be page-locked (gpe_b200._lib.pinned_empty),
        C-contiguous, and left untouched until sync()."""
        if psi.shape != self.shape or not psi.flags.c_contiguous:
            raise ValueError(f"psi must be a C-contiguous array of shape {self.shape}")
        code = L.GPE_C64 if psi.dtype == np.complex64 else L.GPE_C128
        _check(self.lib, self.h, self.lib.gpe_set_state_async(self.h, psi.ctypes.data, code))

    def get_state_async(self, out: np.ndarray) -> None:
        """gpe_get_state_async into a page-locked array; valid after sync()."""
        if out.shape != self.shape or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous array of shape {self.shape}")
        code = L.GPE_C64 if out.dtype == np.complex64 else L.GPE_C128
        _check(self.lib, self.h, self.lib.gpe_get_state_async(self.h, out.ctypes.data, code))

    def wait_copies(self) -> None:
        _check(self.lib, self.h, self.lib.gpe_wait_copies(self.h))

    def set_ic(self, spec) -> None:
        """Generate the initial state on the device (see ic.device_spec)."""
        _check(self.lib, self.h, self.lib.gpe_set_ic(self.h, C.byref(spec)))

    def multiply_ic(self, spec, modulus: bool = False) -> None:
        """psi <- psi * IC, or |psi| * IC with modulus (imprint_vortex_line,
        src/variables.f90:1166-1180), on the device."""
        _check(self.lib, self.h, self.lib.gpe_multiply_ic(self.h, C.byref(spec), 1 if modulus else 0))

    # -- stepping -----------------------------------------------------------
    def solver(self, nsteps: int = 1, want_norm: bool = False, want_energy: bool = False,
               wait: bool = True) -> L.GpeStepInfo:
        """nsteps calls of the reference's solver() with its time update."""
        io = L.GpeStepInfo()
        io.t, io.im_t = self.t, self.im_t
        io.dt_re, io.dt_im = self.dt.real, self.dt.imag
        io.p = self.p
        io.want_norm = 1 if want_norm else 0
        io.want_energy = 1 if want_energy else 0
        fn = self.lib.gpe_step if wait else self.lib.gpe_step_async
        _check(self.lib, self.h, fn(self.h, int(nsteps), C.byref(io)))
        self.t, self.im_t = io.t, io.im_t
        self.dt = complex(io.dt_re, io.dt_im)
        self.p = io.p
        self.last = io
        return io

    step = solver

    def sync(self) -> None:
        _check(self.lib, self.h, self.lib.gpe_sync(self.h))

    # -- diagnostics --------------------------------------------------------
    def get_norm(self) -> float:
        v = C.c_double()
        _check(self.lib, self.h, self.lib.gpe_norm(self.h, C.byref(v)))
        return v.value

    def energy(self) -> float:
        v = C.c_double()
        _check(self.lib, self.h, self.lib.gpe_energy(self.h, C.byref(v)))
        return v.value

    def condensed(self, spectrum: bool = False):
        """condensed_particles (src/io.f90:304-395) of the current state on the
        device: a dict with the mass.dat quantities and, with spectrum=True,
        eta/nharm (7 shells) and F (kk = 1..nx/2) of src/io.f90:668-714."""
        info = L.GpeCondensedInfo()
        if spectrum:
            eta = np.zeros(L.GPE_SPECTRUM_SHELLS)
            nharm = np.zeros(L.GPE_SPECTRUM_SHELLS, dtype=np.int32)
            F = np.zeros(self.params.nx // 2)
            rc = self.lib.gpe_condensed(self.h, C.byref(info), eta.ctypes.data, nharm.ctypes.data, F.ctypes.data,
                                        len(F))
        else:
            rc = self.lib.gpe_condensed(self.h, C.byref(info), None, None, None, 0)
        _check(self.lib, self.h, rc)
        out = {n: getattr(info, n) for n, _ in L.GpeCondensedInfo._fields_}
        if spectrum:
            out.update(eta=eta, nharm=nharm, F=F)
        return out

    def filtered(self, filter_kc: float, m: float = 1.0, dtype=np.complex128) -> np.ndarray:
        """filtered_surface's low-passed field (src/io.f90:524-571), (nz, ny, nx)."""
        p = self.params
        out = np.empty((p.nz, p.ny, p.nx), dtype=dtype)
        code = L.GPE_C128 if out.dtype == np.complex128 else L.GPE_C64
        _check(self.lib, self.h, self.lib.gpe_filtered(self.h, float(m), float(filter_kc), out.ctypes.data, code))
        return out

    def renormalise(self, norm: float) -> None:
        _check(self.lib, self.h, self.lib.gpe_renormalise(self.h, float(norm)))

    def grid(self):
        p = self.params
        x, y, z = np.empty(p.nx), np.empty(p.ny), np.empty(p.nz)
        d = np.empty(3)
        self.lib.gpe_get_grid(self.h, x.ctypes.data, y.ctypes.data, z.ctypes.data, d.ctypes.data)
        return x, y, z, d

    def stream(self) -> int:
        s = C.c_void_p()
        self.lib.gpe_get_stream(self.h, C.byref(s))
        return s.value or 0


def state_bytes(params: RunParams) -> int:
    lib = L.load()
    cp = params.to_c()
    return int(lib.gpe_state_bytes(C.byref(cp)))
