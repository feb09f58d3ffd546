"""The reference's file formats and diagnostics (ek_io.cu; host arrays, no
GPU): each against a numpy restatement of the reference's host code, cited
per test, and the restart file's text against its printf format."""
import numpy as np


def fields(nx=12, ny=9, seed=0):
    rng = np.random.default_rng(seed)
    f = {k: rng.normal(scale=s, size=(ny, nx)) for k, s in
         (("ux", 1e-3), ("uy", 1e-4), ("rho", 1e-2), ("cp", 0.5), ("psi", 1.0), ("ex", 1e-2), ("ey", 1e-2), ("cn", 0.5))}
    f["rho"] += 1.0
    f["cp"] += 2.0
    f["cn"] += 2.0
    return f


def test_restart_text_and_round_trip(tmp_path):
    """save_data_end (LBM.cu:1272-1312) writes nx*ny lines of nine %10.6f
    columns, y-major; read_data (LBM.cu:1350-1392) reads them back."""
    from ekpnp import io
    f = fields()
    path = tmp_path / "data_end.dat"
    io.write_restart(path, 12.5, f)
    lines = path.read_text().splitlines()
    assert len(lines) == 12 * 9
    y, x = 3, 7
    want = "%10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f %10.6f" % (
        12.5, f["ux"][y, x], f["uy"][y, x], f["rho"][y, x], f["cp"][y, x], f["psi"][y, x], f["ex"][y, x],
        f["ey"][y, x], f["cn"][y, x])
    assert lines[y * 12 + x] == want
    t, g = io.read_restart(path, 12, 9)
    assert t == 12.5
    for k in f:
        assert np.abs(g[k] - f[k]).max() <= 5e-7 + 1e-15, k   # six decimals


def test_current_and_umax():
    """current (LBM.cu:1394-1417): wall rows of c+ extrapolated linearly, then
    K dy sum_x c+ Ey on the top row; record_umax (LBM.cu:1419-1451): top row
    of u_y extrapolated, max of u_y from 0."""
    from ekpnp import io
    f = fields()
    c = f["cp"].copy()
    c[-1] = 2 * c[-2] - c[-3]
    want = (c[-1] * f["ey"][-1]).sum() * 0.07 * 0.5
    assert abs(io.current(f["cp"], f["ey"], 0.07, 0.5) - want) <= 1e-15 * abs(want)
    uy = f["uy"].copy()
    uy[-1] = 2 * uy[-2] - uy[-3]
    assert io.umax(f["uy"]) == max(0.0, uy.max())
    assert io.umax(-np.abs(f["uy"]) - 1.0) == 0.0


def test_tecplot_zone(tmp_path):
    """save_data_tecplot (LBM.cu:1100-1270): header once, a ZONE line and
    nx*ny rows of 14 columns per call; derived columns against numpy."""
    from ekpnp import io
    nx, ny, dx, dy = 10, 11, 1.0, 0.5
    f = fields(nx, ny, seed=1)
    path = tmp_path / "data.dat"
    io.write_tecplot(path, 3.0, f, dx, dy, first=True)
    io.write_tecplot(path, 4.0, f, dx, dy, first=False)
    text = path.read_text().splitlines()
    assert text[0].startswith('VARIABLES="x","y","u","v","p"') and text.count("") == 2
    assert text[2] == 'ZONE T="t=3", F=POINT, I = 10, J = 11'
    assert text[3 + nx * ny + 1] == 'ZONE T="t=4", F=POINT, I = 10, J = 11'
    rows = np.array([[float(v) for v in line.split()] for line in text[3:3 + nx * ny]]).reshape(ny, nx, 14)
    # vorticity: central differences, periodic in x, interior rows, then extrapolated walls, / 0.25
    vor = np.zeros((ny, nx))
    vor[1:-1] = ((np.roll(f["uy"], -1, 1) - np.roll(f["uy"], 1, 1)) / dx / 2)[1:-1] - \
        ((f["ux"][2:] - f["ux"][:-2]) / dy / 2)
    vor[0] = 2 * vor[1] - vor[2]
    vor[-1] = 2 * vor[-2] - vor[-3]
    assert np.abs(rows[:, :, 9] - vor / 0.25).max() < 1e-11
    # curl of the force: (dc/dx Ey - dc/dy Ex) / 1e5 with the same stencils
    rdx = np.zeros((ny, nx))
    rdy = np.zeros((ny, nx))
    rdx[1:-1] = ((np.roll(f["cp"], -1, 1) - np.roll(f["cp"], 1, 1)) / dx / 2)[1:-1]
    rdy[1:-1] = (f["cp"][2:] - f["cp"][:-2]) / dy / 2
    for a in (rdx, rdy):
        a[0] = 2 * a[1] - a[2]
        a[-1] = 2 * a[-2] - a[-3]
    curl = (rdx * f["ey"] - rdy * f["ex"]) / 1e5
    assert np.abs(rows[:, :, 10] - curl).max() < 1e-11
    assert np.abs(rows[:, :, 12] - 1000 * curl).max() < 1e-9
    # x, y columns and the extrapolated u at the walls
    assert rows[0, 3, 0] == 3 * dx and rows[4, 0, 1] == 4 * dy
    assert abs(rows[0, 2, 2] - (2 * f["ux"][1, 2] - f["ux"][2, 2])) < 1e-11


def test_dmd_snapshot(tmp_path):
    """save_data_dmd (LBM.cu:1314-1348): c+ with the top row extrapolated, one
    "%10.6f " line per node."""
    from ekpnp import io
    f = fields()
    path = tmp_path / "dmd.dat"
    io.write_dmd(path, f["cp"])
    io.write_dmd(path, f["cp"], append=True)
    lines = path.read_text().splitlines()
    assert len(lines) == 2 * 12 * 9
    c = f["cp"].copy()
    c[-1] = 2 * c[-2] - c[-3]
    assert lines[8 * 12 + 5] == "%10.6f " % c[8, 5]
