"""The reference program with its stepper switched to the B200 drop-in.

adapter/_build/Vortex-Transport-b200 is the reference's own main.cpp and
sources with the rk4 / forward_euler call sites redirected to vt_rk4_dropin /
vt_forward_euler_dropin (vortex-transport_b200/adapter). It must write the
same per-element output files as the unmodified reference program
(oracle/_ref/Vortex-Transport), whose text has 6 decimals. Both programs are
built where the reference sources are available and travel with the repo.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

DROPIN = os.path.join(ROOT, "vortex-transport_b200", "adapter", "_build", "Vortex-Transport-b200")
REFPROG = os.path.join(ROOT, "oracle", "_ref", "Vortex-Transport")

INPUT = """p={p}
domain_x=10.0 //cm
domain_y=10.0 //cm
num_element_in_x={nx}
num_element_in_y={ny}
perturb_grid=0
integration_order={io}
simulation_time={T}
number_time_steps={n}
write_every_steps={w}
U_initialization_type={init}
stepping_method={method}
"""


def run(binary, workdir, text):
    os.makedirs(workdir, exist_ok=True)
    with open(os.path.join(workdir, "input"), "w") as f:
        f.write(text)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    r = subprocess.run([binary, "input"], cwd=workdir, capture_output=True, text=True, env=env,
                       timeout=600)
    return r


def read_step(workdir, step):
    files = sorted(glob.glob(os.path.join(workdir, "output", f"step_{step}", "element_*.txt")),
                   key=lambda p: int(p.rsplit("_", 1)[1][:-4]))
    return np.stack([np.loadtxt(f, skiprows=1) for f in files])


@pytest.mark.skipif(not (os.path.exists(DROPIN) and os.path.exists(REFPROG)),
                    reason="drop-in and reference programs are built only where the reference sources are")
@pytest.mark.parametrize("p,io,nx,ny,method,init", [(3, 10, 8, 8, 1, 0), (2, 6, 12, 6, 0, 0),
                                                    (3, 6, 8, 8, 1, 1)])
def test_dropin_program_writes_the_reference_output(tmp_path, p, io, nx, ny, method, init):
    text = INPUT.format(p=p, io=io, nx=nx, ny=ny, T=0.2, n=40, w=20, method=method, init=init)
    a = run(REFPROG, str(tmp_path / "ref"), text)
    b = run(DROPIN, str(tmp_path / "b200"), text)
    assert a.returncode == 0, a.stderr[-2000:]
    assert b.returncode == 0, b.stderr[-2000:]
    for step in (0, 20, 40):
        ra, rb = read_step(str(tmp_path / "ref"), step), read_step(str(tmp_path / "b200"), step)
        assert ra.shape == rb.shape and ra.shape[0] == 2 * nx * ny
        # the files print 6 decimals: equal up to one unit in the last place
        np.testing.assert_allclose(rb, ra, rtol=0, atol=1.01e-6)
