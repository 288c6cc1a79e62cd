"""Line-out and plane files of the reference's test program (write_lines / write_plane,
code/test_opensc.f90:237-295).  The CPU tests pin the Fortran 1PE14.7 formatting; the GPU
test checks the files' points and fields against the oracle's interpolate_field."""
import os

import numpy as np
import pytest

import openspacecharge_b200 as osc

# Fortran 1PE14.7: d.dddddddE+xx right-justified in 14 columns; the E is dropped for
# three-digit exponents
CASES = [
    (1.0, " 1.0000000E+00"),
    (-2.5e-7, "-2.5000000E-07"),
    (0.0, " 0.0000000E+00"),
    (123456789.0, " 1.2345679E+08"),
    (-9.99999996e99, "-1.0000000+100"),
    (1e-100, " 1.0000000-100"),
    (3.14159265358979, " 3.1415927E+00"),
    (6.02214076e23, " 6.0221408E+23"),
]


@pytest.mark.parametrize("v,s", CASES)
def test_format_1pe14_7(v, s):
    out = osc.format_1pe14_7(v)
    assert out == s and len(out) == 14


@pytest.mark.gpu
def test_lineouts_and_plane_match_oracle(ctx, oracle, tmp_path):
    from openspacecharge_b200.bunch import gendist
    x, y, z = gendist(100000, sigma=(1e-3, 1e-3, 1e-3), seed=61)
    n = (20, 24, 30)
    m = osc.Mesh3D(nlo=(1, 1, 1), nhi=n, gamma=9.784756683727565)
    osc.deposit_particles(ctx, x, y, z, m, total_charge=1e-9)
    osc.space_charge_3d(ctx, m, calc_bfield=True, precision=osc.PREC_FP64)
    xc, yc, zc = float(x.mean()), float(y.mean()), float(z.mean())
    osc.write_lines(ctx, m, xc, yc, zc, tmp_path)
    osc.write_plane(ctx, m, tmp_path)
    om = oracle.make_mesh((1, 1, 1), n, (1, 1, 1), m.min, m.max, m.delta, m.gamma)
    for ax, name in enumerate(("x_lineout.dat", "y_lineout.dat", "z_lineout.dat")):
        lines = open(os.path.join(tmp_path, name)).read().splitlines()
        assert len(lines) == n[ax] - 1
        assert all(len(l) == 90 for l in lines)  # 6 x (14 + 1)
        a = np.array([[float(v) for v in l.split()] for l in lines])
        i = np.arange(1, n[ax])
        pts = [np.full(n[ax] - 1, c) for c in (xc, yc, zc)]
        pts[ax] = (i - 1) * m.delta[ax] + m.min[ax]
        E0, _, _ = oracle.interpolate_field(om, m.efield, *pts)
        for c in range(3):
            assert np.allclose(a[:, c], pts[c], rtol=1e-7, atol=0)
            assert np.allclose(a[:, 3 + c], E0[:, c], rtol=1e-7, atol=1e-7 * np.abs(E0).max())
    a = np.loadtxt(os.path.join(tmp_path, "x_z_Ex_Ez_By.dat"))
    assert a.shape == ((n[0] - 1) * (n[2] - 1), 5)
    xs = np.tile((np.arange(1, n[0]) - 1) * m.delta[0] + m.min[0], n[2] - 1)
    zs = np.repeat((np.arange(1, n[2]) - 1) * m.delta[2] + m.min[2], n[0] - 1)
    E0, B0, _ = oracle.interpolate_field(om, m.efield, xs, np.zeros_like(xs), zs, bfield=m.bfield)
    assert np.allclose(a[:, 0], xs, rtol=1e-15) and np.allclose(a[:, 1], zs, rtol=1e-15)
    for col, ref in ((2, E0[:, 0]), (3, E0[:, 2]), (4, B0[:, 1])):
        assert np.abs(a[:, col] - ref).max() <= 1e-13 * np.abs(ref).max()
