"""CPU restatement of the reference's tune estimates.

TEST INFRASTRUCTURE ONLY (the checker of tests/).

* birkhoff_tune: src/dynamic_indicator.cpp:81-131
* fft_tune: compute_fft + interpolation + A, src/dynamic_indicator.cpp:32-61,
  134-196 (numpy's FFT in place of FFTW: spectra agree to rounding, so FFT
  tunes are compared with a tolerance)
* tune_vec: birkhoff_tune_vec / fft_tune_vec windows, :198-330
* all_tunes orbit handling (mean removal), src/henon.cu:2969-3078
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def birkhoff_tune(q, p) -> float:
    theta = np.arctan2(np.asarray(p, float), np.asarray(q, float))
    d = theta[1:] - theta[:-1]
    d = np.where(d < 0.0, d + 2.0 * math.pi, d)
    w = O.birkhoff_weights(len(d))
    s = 0.0
    for wi, di in zip(w, d):  # left-to-right sum, as the reference
        s += wi * di
    return 1 - s / (2 * math.pi)


def _a(a, b, c):
    return (-(a + b * c) * (a - b) + b * math.sqrt(c ** 2 * (a + b) ** 2 -
                                                  2 * a * b * (2 * c ** 2 - c - 1))) / \
        (a ** 2 + b ** 2 + 2 * a * b * c)


def interpolation(data) -> float:
    index = int(np.argmax(data))
    N = float(len(data))
    if index == 0:
        return 1.0
    if index == len(data) - 1:
        return 0.0
    if data[index - 1] > data[index + 1]:
        i1, i2 = index - 1, index
        index = index - 1
    else:
        i1, i2 = index, index + 1
    value = (index / N) + (1.0 / (2.0 * math.pi)) * math.asin(
        _a(data[i1], data[i2], math.cos(2.0 * math.pi / N)) * math.sin(2.0 * math.pi / N))
    return abs(1.0 - value)


def fft_tune(q, p) -> float:
    q = np.asarray(q, float)
    p = np.asarray(p, float)
    n = len(q)
    h = 2 * np.sin(math.pi * np.arange(n) / n) ** 2
    spec = np.fft.fft(q * h + 1j * (p * h))
    return interpolation(np.abs(spec))


def tune_vec(x, px, y, py, frm, to, method: str):
    """Windows [from, to] (inclusive samples) then the full orbit; NaN for a
    window holding a NaN.  Full orbit: Birkhoff all samples, FFT samples
    1..end."""
    out = []
    for f, t in zip(frm, to):
        sub = [np.asarray(a[f:t + 1], float) for a in (x, px, y, py)]
        if any(np.isnan(s).any() for s in sub):
            out += [math.nan, math.nan]
            continue
        fn = birkhoff_tune if method == "birkhoff" else fft_tune
        out += [fn(sub[0], sub[1]), fn(sub[2], sub[3])]
    if method == "birkhoff":
        out += [birkhoff_tune(x, px), birkhoff_tune(y, py)]
    elif any(np.isnan(np.asarray(a, float)).any() for a in (x, px, y, py)):
        out += [math.nan, math.nan]
    else:
        out += [fft_tune(x[1:], px[1:]), fft_tune(y[1:], py[1:])]
    return out


def orbit(x0, px0, y0, py0, tabs, n_turns, mu, barrier=10.0, kick_module=math.nan, seed=0,
          inverse=False, steps0=None):
    """Samples 0..n_turns of every particle: arrays [n_turns + 1][n].  With
    kick_module, the reproducible kicks of (seed, particle index, table
    index); with inverse, backward turns from steps0 (the particles' steps)."""
    n = len(np.atleast_1d(x0))
    cur = [np.array(np.atleast_1d(a), dtype=float) for a in (x0, px0, y0, py0)]
    steps = np.zeros(n, np.uint32) if steps0 is None else np.array(steps0, dtype=np.uint32)
    out = np.empty((4, n_turns + 1, n))
    for c in range(4):
        out[c, 0] = cur[c]
    for k in range(n_turns):
        if math.isnan(kick_module):
            x, px, y, py, steps = O.track(*cur, steps, tabs, 1, mu, barrier, inverse=inverse)
        else:
            x, px, y, py, steps = O.track_kicked(*cur, steps, tabs, 1, mu, barrier, kick_module,
                                                 seed, inverse=inverse)
        cur = [x, px, y, py]
        for c in range(4):
            out[c, k + 1] = cur[c]
    return out


def remove_mean(samples):
    """v - mean(v) over the samples axis (std::accumulate order)."""
    out = np.empty_like(samples)
    for c in range(samples.shape[0]):
        for i in range(samples.shape[2]):
            col = samples[c, :, i]
            s = 0.0
            for v in col:
                s += v
            out[c, :, i] = col - s / len(col)
    return out
