"""Signal processing helpers for SORD inputs and outputs, as cst/dsp.py.

``time_function`` evaluates the source time functions of the solver
(sord/utilities.f90:223-281) on arrays, in double precision;
``brune2gauss`` swaps a Brune pulse for a Gaussian by convolution;
``filter`` applies Butterworth (scipy.signal) or Hann-window filters.
"""
import math

import numpy as np


def time_function(pulse, t, tau=1.0):
    """Samples of time function `pulse` at times `t` with characteristic
    time `tau` (cst/dsp.py:26-82)."""
    t = np.asarray(t, dtype=np.float64)
    f = np.zeros_like(t)
    if pulse == 'const':
        f[...] = 1.0
    elif pulse == 'delta':
        i = int(abs(t).argmin())
        f.flat[i] = 1.0 / (t.flat[i + 1] - t.flat[i])
    elif pulse in ('step', 'integral_delta'):
        f[t > 0.0] = 1.0
        i = int(abs(t).argmin())
        if t.flat[i] == 0.0:
            f.flat[i] = 0.5
    elif pulse == 'brune':
        a = 1.0 / tau
        m = t > 0.0
        f[m] = np.exp(-a * t[m]) * a * a * t[m]
    elif pulse == 'integral_brune':
        a = 1.0 / tau
        m = t > 0.0
        f[m] = 1.0 - np.exp(-a * t[m]) * (a * t[m] + 1.0)
    elif pulse == 'hann':
        a = 1.0 / tau
        b = math.pi * tau
        m = (-b < t) & (t < b)
        f[m] = 0.5 / math.pi * a * (1.0 + np.cos(a * t[m]))
    elif pulse == 'integral_hann':
        a = 1.0 / tau
        b = math.pi * tau
        f[t > 0.0] = 1.0
        m = (-b < t) & (t < b)
        f[m] = 0.5 + 0.5 / math.pi * (a * t[m] + np.sin(a * t[m]))
    elif pulse in ('gaussian', 'integral_ricker1'):
        a = 0.5 / (tau * tau)
        f = np.exp(-a * t * t) * math.sqrt(a / math.pi)
    elif pulse in ('ricker1', 'integral_ricker2'):
        a = 0.5 / (tau * tau)
        f = np.exp(-a * t * t) * (math.sqrt(a / math.pi) * 2.0 * a) * -t
    elif pulse == 'ricker2':
        a = 0.5 / (tau * tau)
        f = np.exp(-a * t * t) * (math.sqrt(a / math.pi) * 4.0 * a) * (a * t * t - 0.5)
    else:
        raise Exception('invalid time func: ' + pulse)
    return f


def brune2gauss(x, dt, tau, sigma=None, mode='same'):
    """Deconvolve a Brune pulse of characteristic time `tau` from the time
    series `x` (sample interval `dt`, last axis) and put a Gaussian of
    spread `sigma` (default sqrt(2) tau) in its place (cst/dsp.py:85-104)."""
    x = np.asarray(x)
    if sigma is None:
        sigma = math.sqrt(2.0) * tau
    s = 1.0 / (sigma * sigma)
    n = int(6.0 * sigma / dt)
    t = np.arange(-n, n + 1) * dt
    G = 1.0 - 2.0 * s * tau * t - s * tau * tau * (1.0 - s * t * t)
    b = dt * G * math.sqrt(0.5 / math.pi * s) * np.exp(-0.5 * s * t * t)
    return np.apply_along_axis(np.convolve, -1, x, b, mode)


def filter(x, dt, fcorner, btype='lowpass', order=2, repeat=0, mode='same'):
    """Butterworth ('lowpass', 'highpass', 'bandpass', 'bandstop'; `order`
    poles) or Hann-window ('hann') filter of `x` along its last axis
    (cst/dsp.py:107-142).  repeat: 0 one pass, 1 two passes, -1 two passes
    forward and backward (zero phase)."""
    if not fcorner:
        return x
    if btype == 'hann':
        n = int(0.5 / (fcorner * dt))
        if n > 0:
            w = 2.0 * math.pi * dt * fcorner
            b = (1.0 + np.cos(np.arange(-n, n + 1) * w)) * dt * fcorner
            x = np.apply_along_axis(np.convolve, -1, x, b, mode)
            if repeat:
                x = np.apply_along_axis(np.convolve, -1, x, b, mode)
        return x
    import scipy.signal
    if isinstance(fcorner, (list, tuple)):
        wn = (2.0 * dt * fcorner[0], 2.0 * dt * fcorner[1])
    else:
        wn = 2.0 * dt * fcorner
    b, a = scipy.signal.butter(order, wn, btype)
    x = scipy.signal.lfilter(b, a, x)
    if repeat < 0:
        x = scipy.signal.lfilter(b, a, x[..., ::-1])[..., ::-1]
    elif repeat:
        x = scipy.signal.lfilter(b, a, x)
    return x
