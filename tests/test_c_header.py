"""include/gpe_cuda.h is a self-contained plain-C header: a strict C99
program that includes only it compiles without warnings, links against
libgpe_cuda.so and calls a host-only entry point (no GPU needed)."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

from gpe_b200 import _lib as L
from gpe_b200.pool import Pool
from gpe_b200.solver import RunParams

INCLUDE = Path(__file__).resolve().parents[1] / "include"
LIB = Path(L.LIB_PATH)

PROG = r"""
#include "gpe_cuda.h"
#include <stdio.h>
#include <string.h>
int main(void) {
  gpe_params p;
  memset(&p, 0, sizeof(p));
  p.nx = 32; p.ny = 24; p.nz = 16; p.scheme = GPE_RK4; p.eqn = 4; p.bcs = 2; p.order = 4;
  p.real_time = 1; p.storage = GPE_C128; p.xr = 7.75; p.yr = 5.75; p.zr = 3.75; p.tau = 0.01;
  p.g = 1.0; p.mu = 1.0;
  printf("%lld\n", (long long)gpe_pool_solve_bytes(&p));
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_plain_c99(tmp_path):
    src = tmp_path / "t.c"
    exe = tmp_path / "t"
    src.write_text(PROG)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", str(INCLUDE), str(src),
                         "-o", str(exe), "-L", str(LIB.parent), "-lgpe_cuda", f"-Wl,-rpath,{LIB.parent}"],
                        capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert run.returncode == 0, run.stderr
    rp = RunParams(nx=32, ny=24, nz=16, xr=7.75, yr=5.75, zr=3.75, tau=0.01, scheme="rk4", eqn_to_solve=4, bcs=2,
                   order=4, g=1.0, mu=1.0)
    assert int(run.stdout.strip()) == Pool.solve_bytes(rp) > 0
