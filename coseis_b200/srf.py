"""Graves Standard Rupture Format (SRF) and the SORD finite-source files.

Same functions as the reference's cst/srf.py (read, write, write_sord) and
the geometry they use from cst/coord.py (euler_rotation, slip_vectors,
potency_tensor, rotation).  ``write_sord`` writes the ``source-*.bin`` files
that the solver's finite source reads (sord/kinematic_source.f90:10-62):
with ``path='source-'`` and ``nsource`` set to the returned count, a staged
run picks them up.

Defects of cst/srf.py that are fixed here:

* cst/srf.py:256-257 opens ``w23.bin`` for the W22 component, so W22 was
  overwritten by W23 and ``w22.bin`` never written; here it goes to
  ``w22.bin``.
* cst/srf.py:279-296 reuses ``n`` for the source count and for each
  source's sample count, so the second and third slip components' loops
  ran over the wrong number of sources; here each loop runs over all
  sources.
* cst/srf.py:105 reshapes to the plane grid whenever the header has one
  PLANE, and raises KeyError when the file has no PLANE block; here files
  without PLANE keep flat arrays.
* cst/srf.py:130-194 (write) and :209-276 (write_sord) index the per-point
  arrays as read returns them; for a one-plane file those are the reshaped
  plane grids, so write fails and write_sord orders nt, dt, t0, xi and W
  by the grid while the histories follow the file order.  Here both take
  the points in file order.
"""
import math

import numpy as np

REARTH = 6370000.0  # Earth radius of cst/coord.py:7 (m)


def euler_rotation(phi=0.0, theta=0.0, psi=0.0):
    """Rotation matrix of Z-X-Z Euler angles in degrees (cst/coord.py:165-187);
    angles may be arrays, the matrix is then indexed [row, column, ...]."""
    a, b, c = (np.radians(np.asarray(x, dtype=np.float64)) for x in (phi, theta, psi))
    a, b, c = np.broadcast_arrays(a, b, c)
    z, o = np.zeros_like(a), np.ones_like(a)

    def rz(t):
        ct, st = np.cos(t), np.sin(t)
        return np.array([[ct, st, z], [-st, ct, z], [z, z, o]])

    cb, sb = np.cos(b), np.sin(b)
    B = np.array([[o, z, z], [z, cb, sb], [z, -sb, cb]])
    return np.einsum('ij...,jk...->ik...', np.einsum('ij...,jk...->ik...', rz(c), B), rz(a))


def slip_vectors(strike, dip, rake):
    """Rows of the rotation from (east, north, up) to fault-local (slip 1,
    slip 2, normal) coordinates for strike, dip and rake in degrees, dip to
    the right of strike (cst/coord.py:190-202)."""
    return euler_rotation(90.0 - np.asarray(strike, dtype=np.float64), dip, rake)


def potency_tensor(normal, slip):
    """Symmetric potency tensor of a unit normal and a slip vector as volume
    components (W11, W22, W33) and shear components (W23, W31, W12)
    (cst/coord.py:336-351)."""
    n, s = normal, slip
    v = [n[0] * s[0], n[1] * s[1], n[2] * s[2]]
    w = [0.5 * (n[1] * s[2] + n[2] * s[1]), 0.5 * (n[2] * s[0] + n[0] * s[2]), 0.5 * (n[0] * s[1] + n[1] * s[0])]
    return [v, w]


def rotation(lon, lat, projection, eps=100.0):
    """(matrix, theta): the rotation taking geographic vector components to
    the projected system and the clockwise angle to add to a strike
    (cst/coord.py:205-230), by finite differences of `projection` over
    `eps` metres."""
    lon = np.asarray(lon, dtype=np.float64)
    lat = np.asarray(lat, dtype=np.float64)
    dlon = eps * 180.0 / (math.pi * REARTH) * np.cos(math.pi / 180.0 * lat)
    dlat = eps * 180.0 / (math.pi * REARTH)
    lo = np.array([[lon - dlon, lon], [lon + dlon, lon]])
    la = np.array([[lat, lat - dlat], [lat, lat + dlat]])
    x, y = projection(lo, la)
    x = x[1] - x[0]
    y = y[1] - y[0]
    s = 1.0 / np.sqrt(x * x + y * y)
    mat = np.array([s * x, s * y])
    theta = 180.0 / math.pi * np.arctan2(mat[0], mat[1])
    theta = 0.5 * theta.sum(0) - 45.0
    return mat, theta


_KM, _CM, _CM2 = 1000, 0.01, 0.0001  # SRF units to SI
_TO_KM, _TO_CM, _TO_CM2 = 0.001, 100, 10000  # and back


def read(fh):
    """(meta, data) of an SRF file (cst/srf.py:13-127): meta holds the
    header and summary scalars, data NumPy arrays per point source (SI
    units; slip-rate samples concatenated in sv1, sv2, sv3)."""
    lines = (ln for ln in fh)
    name = getattr(fh, 'name', 'SRF')
    meta = {'version': next(lines).split()[0]}
    s = next(lines).split()
    if s[0] == 'PLANE':
        plane = []
        for _ in range(int(s[1])):
            t = next(lines).split() + next(lines).split()
            if len(t) != 11:
                raise Exception('error reading %s' % name)
            j, k = int(t[2]), int(t[3])
            x, y = float(t[4]) * _KM, float(t[5]) * _KM
            plane.append({
                'shape': [j, k], 'length': [x, y], 'area': x * y, 'delta': [x / j, y / k],
                'topcenter': [float(t[0]), float(t[1]), float(t[8])],
                'strike': float(t[6]), 'dip': float(t[7]),
                'hypocenter': [float(t[9]) * _KM, float(t[10]) * _KM],
            })
        meta['plane'] = plane
        s = next(lines).split()
    if s[0] != 'POINTS':
        raise Exception('error reading %s' % name)
    meta['nsource'] = n = int(s[1])
    keys_i = ('nt1', 'nt2', 'nt3')
    keys_f = ('lon', 'lat', 'dep', 'stk', 'dip', 'rake', 'area', 't0', 'dt', 'slip1', 'slip2', 'slip3')
    data = {k: np.empty(n, 'i') for k in keys_i}
    data.update({k: np.empty(n, 'f') for k in keys_f})
    sv = ([], [], [])
    for i in range(n):
        t = next(lines).split() + next(lines).split()
        if len(t) != 15:
            raise Exception('error reading %s %s' % (name, i))
        data['lon'][i], data['lat'][i] = float(t[0]), float(t[1])
        data['dep'][i] = float(t[2]) * _KM
        data['stk'][i], data['dip'][i], data['rake'][i] = float(t[3]), float(t[4]), float(t[8])
        data['area'][i] = float(t[5]) * _CM2
        data['t0'][i], data['dt'][i] = float(t[6]), float(t[7])
        for c in range(3):
            data['slip%d' % (c + 1)][i] = float(t[9 + 2 * c]) * _CM
            data['nt%d' % (c + 1)][i] = int(t[10 + 2 * c])
        counts = [int(data['nt%d' % (c + 1)][i]) for c in range(3)]
        vals = []
        while len(vals) < sum(counts):
            vals += next(lines).split()
        if len(vals) != sum(counts):
            raise Exception('error reading %s %s' % (name, i))
        o = 0
        for c in range(3):
            sv[c].extend(float(v) * _CM for v in vals[o:o + counts[c]])
            o += counts[c]
    for c in range(3):
        data['sv%d' % (c + 1)] = np.array(sv[c], 'f')
    if len(meta.get('plane', [])) == 1:
        shp = meta['plane'][0]['shape']
        for k in keys_f + keys_i:
            data[k] = data[k].reshape(shp[::-1]).T
    nz = [(data['nt%d' % c] > 0).sum() for c in (1, 2, 3)]
    meta['nsource_nonzero'] = int(sum(nz))
    i = int(np.argmin(data['t0']))
    meta['hypocenter'] = [float(data['lon'].flat[i]), float(data['lat'].flat[i]), float(data['dep'].flat[i])]
    meta['area'] = a = float(data['area'].sum(dtype='d'))
    meta['potency'] = p = float(np.sqrt(sum((data['area'] * data['slip%d' % c]).sum(dtype='d') ** 2
                                            for c in (1, 2, 3))))
    meta['displacement'] = p / a
    return meta, data


def write(fh, srf):
    """Write (meta, data) as SRF text (cst/srf.py:130-194)."""
    meta, data = srf
    fh.write('%s\n' % meta['version'])
    for i, seg in enumerate(meta.get('plane', [])):
        fh.write('PLANE %s\n%s %s %s %s %s %s\n%s %s %s %s %s\n' % (
            i + 1, seg['topcenter'][0], seg['topcenter'][1], seg['shape'][0], seg['shape'][1],
            seg['length'][0] * _TO_KM, seg['length'][1] * _TO_KM, seg['strike'], seg['dip'],
            seg['topcenter'][2], seg['hypocenter'][0] * _TO_KM, seg['hypocenter'][1] * _TO_KM))
    n = meta['nsource']
    fh.write('POINTS %s\n' % n)
    flat = {k: np.asarray(v).T.ravel() if np.ndim(v) > 1 else np.asarray(v) for k, v in data.items()}
    o = [0, 0, 0]
    for i in range(n):
        fh.write('%s %s %s %s %s %s %s %s\n%s %s %s %s %s %s %s\n' % (
            flat['lon'][i], flat['lat'][i], flat['dep'][i] * _TO_KM, flat['stk'][i], flat['dip'][i],
            flat['area'][i] * _TO_CM2, flat['t0'][i], flat['dt'][i], flat['rake'][i],
            flat['slip1'][i] * _TO_CM, flat['nt1'][i], flat['slip2'][i] * _TO_CM, flat['nt2'][i],
            flat['slip3'][i] * _TO_CM, flat['nt3'][i]))
        parts = []
        for c in range(3):
            m = int(flat['nt%d' % (c + 1)][i])
            parts.append(np.asarray(data['sv%d' % (c + 1)][o[c]:o[c] + m]) * _TO_CM)
            o[c] += m
        s = np.concatenate(parts)
        k = s.size // 6 * 6
        np.savetxt(fh, s[:k].reshape([-1, 6]), '%13.5e', '')
        np.savetxt(fh, s[k:].reshape([1, -1]), '%13.5e', '')


def write_sord(path, srf, delta=(1, 1, 1), proj=None, dbytes=4):
    """Write the SORD finite-source files ``path + name`` (nt, dt, t0,
    xi1-3, w11 w22 w33 w23 w31 w12, history) of the potency tensor sources
    of an SRF rupture (cst/srf.py:197-299): one source per point and
    non-zero slip component, positions in grid units (x / delta), slip
    histories as the running sum of slip rate times dt.  Returns the number
    of sources (the run's ``nsource``)."""
    meta, data = srf
    d = {k: np.asarray(v).T.ravel() if np.ndim(v) > 1 else np.asarray(v) for k, v in data.items()
         if not k.startswith('sv')}
    it = 'i%d' % dbytes
    ft = 'f%d' % dbytes
    sel = [d['nt%d' % c] > 0 for c in (1, 2, 3)]
    with open(path + 'nt.bin', 'wb') as f:
        for c, s in zip((1, 2, 3), sel):
            d['nt%d' % c][s].astype(it).tofile(f)
    for name in ('dt', 't0'):
        with open(path + name + '.bin', 'wb') as f:
            for s in sel:
                d[name][s].astype(ft).tofile(f)
    x = d['lon'].astype(np.float64)
    y = d['lat'].astype(np.float64)
    z = d['dep'].astype(np.float64)
    rot = 0.0
    if proj:
        rot = rotation(x, y, proj)[1]
        x, y = proj(x, y)
    xi = (np.asarray(x) / delta[0], np.asarray(y) / delta[1], z / delta[2])
    for c in range(3):
        with open(path + 'xi%d.bin' % (c + 1), 'wb') as f:
            for s in sel:
                xi[c][s].astype(ft).tofile(f)
    R = slip_vectors(d['stk'] + rot, d['dip'], d['rake'])
    s1, s2, nrm = R[0], R[1], R[2]
    area = d['area'].astype(np.float64)
    pot = [potency_tensor(nrm, s1), potency_tensor(nrm, s2), potency_tensor(nrm, nrm)]
    names = (('w11', 0, 0), ('w22', 0, 1), ('w33', 0, 2), ('w23', 1, 0), ('w31', 1, 1), ('w12', 1, 2))
    for name, a, b in names:
        with open(path + name + '.bin', 'wb') as f:
            for p, s in zip(pot, sel):
                (area * p[a][b])[s].astype(ft).tofile(f)
    with open(path + 'history.bin', 'wb') as f:
        for c in (1, 2, 3):
            nt = d['nt%d' % c]
            sv = np.asarray(data['sv%d' % c])
            o = 0
            for i in range(nt.size):
                m = int(nt[i])
                (sv[o:o + m].cumsum() * d['dt'][i]).astype(ft).tofile(f)
                o += m
    return int(sum(s.sum() for s in sel))
