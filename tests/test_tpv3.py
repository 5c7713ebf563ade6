"""SCEC TPV3 (spontaneous slip-weakening rupture on a planar fault in a
homogeneous whole space) against the boundary-integral solution the
reference ships (data/TPV3-BI-*.npy, fixture tests/golden/tpv3_bi.npz):
the setup of scripts/TPV3-sim.py at dx = 100 m (a quarter of the problem
between mirror planes through the hypocentre) and the comparison of
scripts/TPV3-plot.py: slip, slip rate and shear traction at the mode II
station P1 (7.5 km along strike) and the mode III station P2 (6 km along
dip) over 1-11 s, and the rupture-time field of the fault quarter (BI
grid of 0.1 km cells, interpolated to the fault nodes)."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
DX = 100.0
DT = DX / 12500.0
WINDOW = (1.0, 11.0)


def tpv3_prm(dx=DX):
    """TPV3 as the benchmark defines it, on the whole fault: 30 x 15 km
    frictional region (mus 0.677, mud 0.525, Dc 0.4 m) in a locked plane,
    sigma_n = -120 MPa, tau_0 = 70 MPa, a 3 km nucleation square of 81.6 MPa
    (its edge and corner nodes the averages with 70 MPa: 75.8, 72.9, as
    scripts/TPV3-sim.py sets them), viscosity 0.02 within 3 km of the fault
    and 0.2 beyond, PML all round.  The shipped script runs a quarter of
    this between mirror planes through the hypocentre; those planes are the
    last node row and column of its fault plane, which fault-plane input
    ops never reach (they are clipped to the cell range of the plane,
    sord/input_output.f90:150-160), so there the prestress stays zero.
    Stations are written with node-exact '=>' ops (a '.>' probe of a fault
    field at a node position reads half a cell away for the same reason)."""
    dt = dx / 12500.0
    hx, hy, hz = int(16500.0 / dx), int(9000.0 / dx), int(6000.0 / dx)
    npml = 10
    nx, ny, nz = 2 * hx + 1 + 2 * npml, 2 * hy + 1 + 2 * npml, 2 * hz + 2 + 2 * npml
    jh, kh, lh = hx + npml, hy + npml, hz + npml     # hypocentre node (0-based); fault between lh, lh + 1
    nt = int(12.0 / dt + 1.5)
    fx, fy, fz = int(15000.0 / dx + 0.5), int(7500.0 / dx + 0.5), int(3000.0 / dx + 0.5)
    n0, n1 = int(1500.0 / dx + 0.5) - 1, int(1500.0 / dx + 0.5)   # inside / edge of the nucleation square
    rj = lambda n: [jh - n, jh + n + 1]
    rk = lambda n: [kh - n, kh + n + 1]
    prm = {
        'shape': [nx, ny, nz, nt], 'delta': [dx, dx, dx, dt], 'npml': npml,
        'faultnormal': '+z', 'hypocenter': [float(jh), float(kh), lh + 0.5], 'hourglass': [1.0, 2.0],
        'bc1': ['pml', 'pml', 'pml'], 'bc2': ['pml', 'pml', 'pml'],
        'rho': [2670.0], 'vp': [6000.0], 'vs': [3464.0],
        'dc': [0.4], 'mud': [0.525], 'tn': [-120.0e6],
        'mus': [10000.0, ([rj(fx), rk(fy)], '=', 0.677)],
        'gam': [0.2, ([rj(fx), rk(fy), [lh - fz, lh + fz + 2]], '=', 0.02)],
        'ts': [70.0e6, ([rj(n1), rk(n1)], '=', 72.9e6), ([rj(n0), rk(n1)], '=', 75.8e6),
               ([rj(n1), rk(n0)], '=', 75.8e6), ([rj(n0), rk(n0)], '=', 81.6e6)],
        'trup': [([rj(fx), rk(fy), -1], '=>', 'trup.bin')],
        'x': [([rj(fx), rk(fy), lh], '=>', 'x.bin')],
        'y': [([rj(fx), rk(fy), lh], '=>', 'y.bin')],
    }
    p1 = (jh + int(7500.0 / dx + 0.5), kh)   # mode II station: 7.5 km along strike
    p2 = (jh, kh + int(6000.0 / dx + 0.5))   # mode III station: 6 km along dip
    for f in ('sux', 'svx', 'tsx'):
        prm[f] = [([p1[0], p1[1], []], '=>', 'P1-%s.bin' % f),
                  ([p2[0], p2[1], []], '=>', 'P2-%s.bin' % f)]
    return prm, (jh, kh)


def bi():
    return np.load(os.path.join(HERE, 'golden', 'tpv3_bi.npz'))


def station_misfits(path, z, dt):
    """Relative L2 misfit over the window of slip, slip rate and shear
    traction (MPa) at P1 and P2, BI interpolated to the solver's times."""
    nt = os.path.getsize(os.path.join(path, 'P1-sux.bin')) // 4
    t = np.arange(nt) * dt
    w = (t >= WINDOW[0]) & (t <= WINDOW[1])
    out = {}
    for sta in ('P1', 'P2'):
        for f, key, scale in (('sux', 'slip', 1.0), ('svx', 'sv', 1.0), ('tsx', 'ts', 1e-6)):
            s = np.fromfile(os.path.join(path, '%s-%s.bin' % (sta, f)), '<f4').astype(np.float64) * scale
            b = np.interp(t[w], z['t'].astype(np.float64), z['%s_%s' % (sta.lower(), key)].astype(np.float64))
            out['%s-%s' % (sta, key)] = float(np.linalg.norm(s[w] - b) / np.linalg.norm(b))
    return out


def rupture_time_rms(path, z, hypo_xy):
    """RMS difference (s) of the rupture time over the frictional region;
    BI cell-centred grid of 0.1 km centred on the hypocentre."""
    from scipy.interpolate import RegularGridInterpolator
    tr = np.fromfile(os.path.join(path, 'trup.bin'), '<f4').astype(np.float64)
    x = np.fromfile(os.path.join(path, 'x.bin'), '<f4').astype(np.float64)
    y = np.fromfile(os.path.join(path, 'y.bin'), '<f4').astype(np.float64)
    x, y = (x - hypo_xy[0]) * 1e-3, (y - hypo_xy[1]) * 1e-3
    tb = z['trup'].astype(np.float64)
    nx, ny = tb.shape
    gx = np.arange(nx) * 0.1 - 0.5 * (nx - 1) * 0.1
    gy = np.arange(ny) * 0.1 - 0.5 * (ny - 1) * 0.1
    inside = (np.abs(x) <= gx[-1]) & (np.abs(y) <= gy[-1]) & (tr < 1e8)
    f = RegularGridInterpolator((gx, gy), tb)
    b = f(np.stack([x[inside], y[inside]], -1))
    return float(np.sqrt(np.mean((tr[inside] - b) ** 2))), int(inside.sum())


def test_bi_fixture():
    z = bi()
    assert z['t'].size == 1351 and z['trup'].shape == (300, 150)
    # the BI rupture starts inside the 3 km nucleation square at the centre
    c = np.unravel_index(z['trup'].argmin(), z['trup'].shape)
    assert abs(c[0] - 149.5) <= 15 and abs(c[1] - 74.5) <= 15
    assert 2.5 < z['p1_slip'].max() < 3.5 and 60 < z['p1_ts'].min() < 75


@pytest.mark.gpu
@pytest.mark.parametrize('arithmetic', ['reference', 'fast'])
def test_tpv3_against_boundary_integral(arithmetic, tmp_path, gpu_lib):
    import sordcases as sc
    d = str(tmp_path)
    prm, (jh, kh) = tpv3_prm()
    sc.stage(prm, d)
    sc.run_gpu(d, arithmetic=arithmetic)
    z = bi()
    mis = station_misfits(d, z, prm['delta'][3])
    rms, n = rupture_time_rms(d, z, (jh * DX, kh * DX))
    print('TPV3 %s: %s; rupture time RMS %.4f s over %d nodes' % (
        arithmetic, ', '.join('%s %.4f' % kv for kv in sorted(mis.items())), rms, n))
    # measured (both arithmetics): slip 0.017 / 0.024, traction 0.014 /
    # 0.018, slip rate 0.34 / 0.50 (P1 / P2; the sharp slip-rate pulse at
    # 100 m), rupture time RMS 0.055 s over 44551 nodes
    assert n > 40000
    bound = {'slip': 0.04, 'ts': 0.03, 'sv': 0.6}
    assert all(v < bound[k.split('-')[1]] for k, v in mis.items()), mis
    assert rms < 0.08
