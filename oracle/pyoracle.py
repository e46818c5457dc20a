"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product never imports it.
Parity of the oracle is unpinned by reference artefacts (the reference ships
no tests or golden vectors and its Fortran cannot be built here); it is pinned
by analytic known-answer tests (tests/test_oracle_kat.py).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"

SCHEMES = {"euler": 0, "rk2": 1, "rk4": 2, "rk45": 3}


class OrParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("xr", C.c_double), ("yr", C.c_double), ("zr", C.c_double),
        ("scheme", C.c_int), ("eqn", C.c_int), ("bcs", C.c_int), ("order", C.c_int),
        ("real_time", C.c_int), ("tau", C.c_double),
        ("Urhs", C.c_double), ("diss_amp", C.c_double), ("scal", C.c_double), ("g", C.c_double),
        ("mu", C.c_double), ("nn", C.c_double), ("omx", C.c_double), ("omy", C.c_double),
        ("omz", C.c_double), ("gamma", C.c_double),
    ]


class OrClock(C.Structure):
    _fields_ = [("t", C.c_double), ("im_t", C.c_double), ("dt_re", C.c_double), ("dt_im", C.c_double),
                ("p", C.c_int64), ("errmax", C.c_double), ("rejected", C.c_int64)]


class OrRing(C.Structure):
    _fields_ = [("plane", C.c_char * 3), ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
                ("r0", C.c_double), ("amp", C.c_double), ("mm", C.c_int), ("r1", C.c_double),
                ("kk", C.c_int), ("dir", C.c_double)]


class OrLine(C.Structure):
    _fields_ = [("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("amp1", C.c_double),
                ("amp2", C.c_double), ("ll", C.c_double), ("sgn", C.c_double), ("dir", C.c_char),
                ("imprint_phase", C.c_int)]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    lib = C.CDLL(str(LIB_PATH))
    P, D, I64 = C.c_void_p, C.c_double, C.c_int64
    sig = {
        "or_create": (P, [C.POINTER(OrParams)]),
        "or_destroy": (None, [P]),
        "or_set_threads": (None, [C.c_int]),
        "or_get_threads": (C.c_int, []),
        "or_set_faithful_cost": (None, [P, C.c_int]),
        "or_get_grid": (None, [P, P, P, P, P]),
        "or_laplacian": (None, [P, P, P]),
        "or_deriv_x": (None, [P, P, P]),
        "or_get_rhs": (None, [P, P, P]),
        "or_solver": (None, [P, P, C.POINTER(OrClock)]),
        "or_run": (None, [P, P, C.POINTER(OrClock), I64]),
        "or_get_norm": (D, [P, P]),
        "or_energy": (D, [P, P]),
        "or_renormalise": (None, [P, P, D]),
        "or_get_rr": (None, [P, P, I64]),
        "or_vortex_ring": (C.c_int, [P, C.POINTER(OrRing), P]),
        "or_vortex_line": (C.c_int, [P, C.POINTER(OrLine), P]),
        "or_vortex_line_pade": (C.c_int, [P, C.POINTER(OrLine), P]),
        "or_fermi": (None, [P, P]),
        "or_vtrap": (None, [P, P]),
        "or_pade_pulse_ring": (C.c_int, [P, C.c_int, D, D, D, D, P]),
        "or_vortex_pair": (None, [P, P]),
        "or_sphere": (None, [P, P]),
        "or_sphere2": (None, [P, P]),
        "or_wall": (None, [P, P]),
        "or_cmul": (None, [P, P, P, I64]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def set_threads(n: int) -> None:
    load().or_set_threads(int(n))


class Oracle:
    """One oracle context: same parameter names as the product's RunParams."""

    def __init__(self, rp):
        self.lib = load()
        p = OrParams()
        p.nx, p.ny, p.nz = rp.nx, rp.ny, rp.nz
        p.xr, p.yr, p.zr = rp.xr, rp.yr, rp.zr
        p.scheme = SCHEMES[rp.scheme]
        p.eqn, p.bcs, p.order = rp.eqn_to_solve, rp.bcs, rp.order
        p.real_time = 1 if rp.real_time else 0
        p.tau = rp.tau
        for f in ("Urhs", "diss_amp", "scal", "g", "mu", "nn", "omx", "omy", "omz", "gamma"):
            setattr(p, f, float(getattr(rp, f)))
        self.rp = rp
        self.ctx = self.lib.or_create(C.byref(p))
        if not self.ctx:
            raise ValueError("oracle rejected the parameters")
        self.shape = (rp.nz, rp.ny, rp.nx)
        self.clock = OrClock()
        self.clock.dt_re, self.clock.dt_im = (rp.tau, 0.0) if rp.real_time else (0.0, -rp.tau)

    def __del__(self):
        try:
            if self.ctx:
                self.lib.or_destroy(self.ctx)
        except Exception:
            pass

    def _c(self, a):
        a = np.ascontiguousarray(a, dtype=np.complex128)
        assert a.shape == self.shape
        return a

    def faithful_cost(self, on: bool = True) -> None:
        self.lib.or_set_faithful_cost(self.ctx, 1 if on else 0)

    def grid(self):
        x, y, z = np.empty(self.rp.nx), np.empty(self.rp.ny), np.empty(self.rp.nz)
        d = np.empty(3)
        self.lib.or_get_grid(self.ctx, x.ctypes.data, y.ctypes.data, z.ctypes.data, d.ctypes.data)
        return x, y, z, d

    def laplacian(self, psi):
        psi = self._c(psi)
        out = np.empty_like(psi)
        self.lib.or_laplacian(self.ctx, psi.ctypes.data, out.ctypes.data)
        return out

    def deriv_x(self, psi):
        psi = self._c(psi)
        out = np.empty_like(psi)
        self.lib.or_deriv_x(self.ctx, psi.ctypes.data, out.ctypes.data)
        return out

    def get_rhs(self, psi):
        psi = self._c(psi)
        out = np.empty_like(psi)
        self.lib.or_get_rhs(self.ctx, psi.ctypes.data, out.ctypes.data)
        return out

    def run(self, psi, nsteps: int):
        """Advance psi (copied) by nsteps solver() calls; returns the new psi."""
        psi = self._c(psi).copy()
        self.lib.or_run(self.ctx, psi.ctypes.data, C.byref(self.clock), int(nsteps))
        return psi

    def get_norm(self, psi) -> float:
        psi = self._c(psi)
        return self.lib.or_get_norm(self.ctx, psi.ctypes.data)

    def energy(self, psi) -> float:
        psi = self._c(psi)
        return self.lib.or_energy(self.ctx, psi.ctypes.data)

    def renormalise(self, psi, norm: float):
        psi = self._c(psi).copy()
        self.lib.or_renormalise(self.ctx, psi.ctypes.data, float(norm))
        return psi

    def vortex_ring(self, plane="xy", x0=0.0, y0=0.0, z0=0.0, r0=4.0, amp=0.0, mm=0, r1=0.0, kk=0, dir=1.0):
        vr = OrRing(plane.encode(), x0, y0, z0, r0, amp, mm, r1, kk, dir)
        out = np.empty(self.shape, np.complex128)
        if self.lib.or_vortex_ring(self.ctx, C.byref(vr), out.ctypes.data):
            raise ValueError("ERROR: Unrecognised vortex ring plane.")
        return out

    def vortex_line(self, x0=0.0, y0=0.0, z0=0.0, amp1=0.0, amp2=0.0, ll=0.0, sgn=1.0, dir="z",
                    imprint_phase=False, pade=False):
        vl = OrLine(x0, y0, z0, amp1, amp2, ll, sgn, dir.encode(), 1 if imprint_phase else 0)
        out = np.empty(self.shape, np.complex128)
        fn = self.lib.or_vortex_line_pade if pade else self.lib.or_vortex_line
        if fn(self.ctx, C.byref(vl), out.ctypes.data):
            raise ValueError("ERROR: vortex line disturbance wavelength is zero, but amplitude is non-zero.")
        return out

    def fermi(self):
        out = np.empty(self.shape, np.complex128)
        self.lib.or_fermi(self.ctx, out.ctypes.data)
        return out

    def pade_pulse_ring(self, pulse_or_ring="pulse", x0=0.0, y0=0.0, z0=0.0, r0=0.0):
        if pulse_or_ring not in ("pulse", "ring"):
            raise ValueError("pulse_or_ring must be 'pulse' or 'ring'")
        out = np.empty(self.shape, np.complex128)
        self.lib.or_pade_pulse_ring(self.ctx, 1 if pulse_or_ring == "pulse" else 0, float(x0), float(y0), float(z0),
                                    float(r0), out.ctypes.data)
        return out

    def _fill(self, fn):
        out = np.empty(self.shape, np.complex128)
        fn(self.ctx, out.ctypes.data)
        return out

    def vortex_pair(self):
        return self._fill(self.lib.or_vortex_pair)

    def sphere(self):
        return self._fill(self.lib.or_sphere)

    def sphere2(self):
        return self._fill(self.lib.or_sphere2)

    def wall(self):
        return self._fill(self.lib.or_wall)

    def vtrap(self):
        out = np.empty(self.shape, np.float64)
        self.lib.or_vtrap(self.ctx, out.ctypes.data)
        return out

    @staticmethod
    def get_rr(r):
        lib = load()
        r = np.ascontiguousarray(r, dtype=np.float64)
        out = np.empty_like(r)
        lib.or_get_rr(r.ctypes.data, out.ctypes.data, r.size)
        return out
