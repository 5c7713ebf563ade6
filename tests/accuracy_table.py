"""Accuracy of the CUDA solver on the benchmark configurations (a script,
not a pytest module: the FP64 oracle runs take minutes).

For each configuration the FP32 oracle, the FP64 oracle and the CUDA solver
in reference order and in fast arithmetic run the same staged problem; the
script reports, per output family (velocity, displacement, slip, slip
rate), the relative L2 error against the FP64 oracle of the CUDA solver in
both arithmetics and of the FP32 oracle, whether the reference-order run is
bit-identical to the FP32 oracle, and the largest rupture-time difference
in time steps:

  explosion   61^3 nodes, 200 steps (its stated size)
  wave        the wave226 generator at 128 x 128 x 64 nodes, all 1000 steps
  rupture     the planar-fault problem (20 x 10 km region, 3 km patch) at
              dx 100 m: 200 x 100 x 100 nodes, 750 steps (6 s)
  ensemble    rupture-ensemble scenarios 0-4, 600 steps each

    python tests/accuracy_table.py [--out accuracy.json] [--only name ...]
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import bench  # noqa: E402
import sordcases as sc  # noqa: E402
from test_fast_arithmetic import floor_of, load, rel_l2  # noqa: E402

FAMILIES = (('velocity', ('snap-v', 'rec', 'vol-v', 'r0', 'r1', 'r2', 'r3', 'r4', 'r5', 'r6')),
            ('displacement', ('vol-u',)), ('slip', ('sum', 'sl.', 'su')), ('slip rate', ('svm', 'sv', 'psv')))


def family(f):
    for name, pre in FAMILIES:
        if f.startswith(pre):
            return name
    return None


def measure(name, prm, files, exes, work):
    t0 = time.time()
    dirs = {t: os.path.join(work, name, t) for t in ('o32', 'o64', 'ref', 'fast')}
    for t, d in dirs.items():
        bench.stage_files(prm, files, d, realsize=8 if t == 'o64' else 4)
    thr = os.cpu_count() or 1
    for t, exe in (('o32', exes['f32']), ('o64', exes['f64'])):
        r = subprocess.run([exe, '--threads', str(thr)], cwd=dirs[t], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stderr[-2000:])
    sc.run_gpu(dirs['ref'], arithmetic='reference')
    sc.run_gpu(dirs['fast'], arithmetic='fast')
    same = sc.compare(dirs['o32'], dirs['ref'])
    skip = ('stats-e', 'stats-moment', 'stats-mw')
    exact = all(e for f, (r, e) in same.items() if not f.startswith(skip))
    fam = {}
    trup = None
    dt = prm['delta'][3]
    for f in sc.outputs(dirs['fast']):
        if f.startswith('stats-'):
            continue
        b = load(dirs['o64'], f, '<f8')
        if f in ('trup.bin', 'tarr.bin'):
            worst = 0.0
            for t in ('fast', 'ref', 'o32'):
                a = load(dirs[t], f, '<f4')
                m = (b < 1e8) | (a < 1e8)
                if m.any():
                    worst = max(worst, float(np.abs(a[m] - b[m]).max() / dt))
            trup = max(trup or 0.0, worst)
            continue
        k = family(f)
        if k is None:
            continue
        fl = floor_of(dirs['o64'], f, '<f8')
        e = [rel_l2(load(dirs[t], f, '<f4'), b, fl) for t in ('fast', 'ref', 'o32')]
        old = fam.get(k, [0.0, 0.0, 0.0])
        fam[k] = [max(x, y) for x, y in zip(old, e)]
    shutil.rmtree(os.path.join(work, name), ignore_errors=True)
    return {'families': {k: {'fast_vs_fp64': v[0], 'reference_order_vs_fp64': v[1], 'fp32_oracle_vs_fp64': v[2]}
                         for k, v in fam.items()},
            'reference_order_bit_identical_to_fp32_oracle': bool(exact),
            'rupture_time_max_diff_steps': trup, 'seconds': round(time.time() - t0, 1)}


def with_peak_rate(p):
    """Add the peak slip rate over the run (psv) to a rupture's outputs.  The
    final slip rate (svm) of an arrested rupture is zero up to rounding, so
    its error is measured against the size of the peak slip rate (the floor
    of the 'sv' family), and psv itself is reported."""
    p = dict(p)
    p['psv'] = [([[], [], -1], '=>', 'psv.bin')]
    return p


def configs():
    out = []
    p = bench.explosion_prm()
    p['ux'] = [([[], [], [], -1], '=>', 'vol-ux.bin')]
    p['vz'].append(([[], [], [], -1], '=>', 'vol-vz.bin'))
    out.append(('explosion', '61^3 x 200 steps', p, {}))

    def wave(work):
        shape = (128, 128, 64)
        inp = os.path.join(work, 'wave_inputs')
        bench.make_inputs(shape, inp, use_torch=False)
        p = bench.wave_prm(shape, 1000)
        p['ux'] = [([[], [], [], -1], '=>', 'vol-ux.bin')]
        p['vz'].append(([[], [], [], -1], '=>', 'vol-vz.bin'))
        files = {f: np.fromfile(os.path.join(inp, f), '<f4') for f in ('rho.bin', 'vp.bin', 'vs.bin', 'z.bin')}
        return p, files
    out.append(('wave', '128x128x64 x 1000 steps (wave226 generator)', wave, None))
    p, files = bench.rupture3_prm(nt=750, shape=(200, 100, 100), dx=100.0, dt=0.008)
    out.append(('rupture', '200x100x100 x 750 steps at dx 100 m', with_peak_rate(p), files))
    for i in range(5):
        p, files = bench.rupture_scenario(i)
        out.append(('ensemble%d' % i, 'scenario %d: %dx%dx%d x %d steps' % ((i,) + tuple(p['shape'])),
                    with_peak_rate(p), files))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--out', default='accuracy.json')
    ap.add_argument('--only', nargs='*')
    args = ap.parse_args()
    from oracle import build as ob
    exes = ob.build()
    work = tempfile.mkdtemp(prefix='sord_acc_')
    res = {}
    try:
        for name, desc, p, files in configs():
            if args.only and name not in args.only:
                continue
            if callable(p):
                p, files = p(work)
            r = measure(name, p, files, exes, work)
            r['config'] = desc
            res[name] = r
            print(name, json.dumps(r), flush=True)
            json.dump(res, open(args.out, 'w'), indent=1)
    finally:
        shutil.rmtree(work, ignore_errors=True)


if __name__ == '__main__':
    main()
