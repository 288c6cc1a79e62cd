"""The drop-in Fortran modules (fortran/) built with gfortran and run through the same
calls as the reference's test program: E at every particle must equal the Python API's
FP64 step (deposit with refit, space_charge_3d, interpolate_field) to round-off.  Skipped
where no Fortran compiler is installed."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import openspacecharge_b200 as osc
from openspacecharge_b200.bunch import gendist

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fortran_shim_matches_python_api(ctx, tmp_path):
    fc = shutil.which(os.environ.get("FC", "gfortran"))
    if not fc:
        pytest.skip("no Fortran compiler on this machine")
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "fortran"), f"FC={fc}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    x, y, z = gendist(50000, sigma=(0.5e-3, 0.5e-3, 2e-3), seed=71)
    fin, fout = tmp_path / "p.bin", tmp_path / "E.bin"
    with open(fin, "wb") as f:
        np.array([len(x)], dtype=np.int64).tofile(f)
        for a in (x, y, z):
            a.astype(np.float64).tofile(f)
    r = subprocess.run([os.path.join(ROOT, "fortran", "_build", "demo_shim"), str(fin), str(fout)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    Ef = np.fromfile(fout, dtype=np.float64).reshape(-1, 3)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=(24, 24, 32), gamma=9.784756683727565)
    Ep, _ = osc.space_charge_step(ctx, m, x, y, z, total_charge=1e-9, resize_mesh=True, precision=osc.PREC_FP64)
    assert np.abs(Ef - Ep).max() <= 1e-12 * np.abs(Ep).max()
