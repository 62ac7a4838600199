"""CPU restatement of the tangent-map containers and indicator constructs.

TEST INFRASTRUCTURE ONLY (the checker of tests/ and smoke()).

numpy elementwise arithmetic on float64 arrays is one IEEE-754 operation per
ufunc call, so every expression below, written in the reference's order,
reproduces the reference's products and sums bit for bit.  The
transcendentals (log, log10, arctan2) come from numpy and may differ from
CUDA's in the last unit in the last place; comparisons that involve them use
a relative tolerance.  Each function cites the reference code it restates
(carlidel/henon_map_cpp).
"""
from __future__ import annotations

import numpy as np

from . import oracle as O


def tangent_matrix(x, y, sx, cx, sy, cy, mu):
    """tangent_matrix, src/henon.cu:175-196; returns (n, 4, 4)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = x.size
    m = np.zeros((n, 4, 4))
    mu3xx = ((mu * 3) * x) * x
    mu3yy = ((mu * 3) * y) * y
    a = (2 * x + mu3xx) - mu3yy
    b = (-2 * y) - ((mu * 6) * x) * y
    d = ((-2 * x) - mu3xx) + mu3yy
    m[:, 0, 0] = cx + sx * a
    m[:, 0, 1] = sx
    m[:, 0, 2] = sx * b
    m[:, 1, 0] = -sx + cx * a
    m[:, 1, 1] = cx
    m[:, 1, 2] = cx * b
    m[:, 2, 0] = sy * b
    m[:, 2, 2] = cy + sy * d
    m[:, 2, 3] = sy
    m[:, 3, 0] = cy * b
    m[:, 3, 2] = -sy + cy * d
    m[:, 3, 3] = cy
    return m


def matmul(a, b):
    """a @ b per particle, each sum from 0.0 in k order (:279-288)."""
    out = np.empty_like(b)
    for i in range(4):
        for j in range(4):
            s = np.zeros(a.shape[0])
            for k in range(4):
                s = s + a[:, i, k] * b[:, k, j]
            out[:, i, j] = s
    return out


def matvec(m, v):
    """v <- M v, rows from 0.0 (matrix_vector_multiply, :316-338)."""
    out = np.empty_like(v)
    for i in range(4):
        s = np.zeros(v.shape[0])
        for j in range(4):
            s = s + m[:, i, j] * v[:, j]
        out[:, i] = s
    return out


def norm(a):
    """sqrt of the sum of squares from 0.0 in index order."""
    flat = a.reshape(a.shape[0], -1)
    s = np.zeros(a.shape[0])
    for k in range(flat.shape[1]):
        s = s + flat[:, k] * flat[:, k]
    return np.sqrt(s)


class ConstructLoop:
    """The per-turn reference loop over the constructs:

        M_old <- M; track 1; M <- DF(x; table[g]) M; megno.add(M, M_old);
        megno_b.add(M, M_old); v <- DF v; lyap.add(v); v <- v/|v|; tune.add(p)

    on n particles, with the map from the C oracle (bit-exact)."""

    def __init__(self, x, px, y, py, tables, mu, barrier, v0, lyap_windows, megno_windows,
                 tune_windows):
        self.x, self.px, self.y, self.py = (np.array(a, dtype=np.float64) for a in (x, px, y, py))
        n = self.x.size
        self.steps = np.zeros(n, np.uint32)
        self.tables = tuple(np.asarray(t) for t in tables)
        self.mu, self.barrier = mu, barrier
        self.g = 0
        self.M = np.tile(np.eye(4), (n, 1, 1))
        self.v = np.array(np.broadcast_to(np.asarray(v0, dtype=np.float64), (n, 4)))
        self.m_l1 = np.zeros(n)
        self.m_l2 = np.zeros(n)
        self.m_l3 = np.zeros(n)
        self.m_idx = 1
        self.mb_T = list(megno_windows)
        self.mb_w = [O.birkhoff_weights(t) for t in self.mb_T]
        self.mb_l1 = np.zeros(n)
        self.mb_l2 = np.zeros((len(self.mb_T), n))
        self.mb_idx = 1
        self.ly_len = list(lyap_windows)
        self.ly_w = [O.birkhoff_weights(t) for t in self.ly_len]
        self.ly_raw = np.zeros((len(self.ly_len), n))
        self.ly_b = np.zeros((len(self.ly_len), n))
        self.ly_idx = 0
        self.tu_T = list(tune_windows)
        self.tu_w = [O.birkhoff_weights(t) for t in self.tu_T]
        self.t1x = np.zeros((len(self.tu_T), n))
        self.t1y = np.zeros_like(self.t1x)
        self.t2x = np.zeros_like(self.t1x)
        self.t2y = np.zeros_like(self.t1x)
        self.tu_idx = 1
        # tune_birkhoff_construct::first_add (:2533-2546)
        self.store_x = np.arctan2(self.px, self.x)
        self.store_y = np.arctan2(self.py, self.y)
        self.megno_history = []

    def turn(self):
        sx, cx, sy, cy = self.tables
        x, px, y, py, s = O.track(self.x, self.px, self.y, self.py, self.steps, self.tables, 1,
                                  self.mu, self.barrier)
        # track() advances only the steps of live particles; the tables are
        # indexed by each particle's own steps, so run it from copies.
        self.x, self.px, self.y, self.py, self.steps = x, px, y, py, s
        self.g += 1
        g = self.g
        df = tangent_matrix(self.x, self.y, sx[g], cx[g], sy[g], cy[g], self.mu)
        # MEGNO (kernel_megno :2253-2284, kernel_megno_birkhoff :2366-2402)
        old = norm(self.M)
        self.M = matmul(df, self.M)
        new = norm(self.M)
        lr = np.log10(new / old)
        di = float(self.m_idx)
        self.m_l1 = self.m_l1 + lr * di
        self.m_l2 = self.m_l2 + (1.0 / di) * self.m_l1
        self.m_l3 = (1.0 / di) * self.m_l2
        self.megno_history.append(self.m_l3.copy())
        self.m_idx += 1
        di = float(self.mb_idx)
        self.mb_l1 = self.mb_l1 + lr * di
        for j, T in enumerate(self.mb_T):
            if self.mb_idx <= T:
                self.mb_l2[j] = self.mb_l2[j] + (self.mb_l1 * self.mb_w[j][self.mb_idx - 1]) / di
        self.mb_idx += 1
        # Lyapunov (matrix_vector_multiply, kernel_lyap_birk :2083-2098,
        # normalize_vectors :341-359)
        self.v = matvec(df, self.v)
        nv = norm(self.v)
        lv = np.log(nv)
        for j, L in enumerate(self.ly_len):
            if self.ly_idx < L:
                self.ly_raw[j] = self.ly_raw[j] + lv / float(L)
                self.ly_b[j] = self.ly_b[j] + lv * self.ly_w[j][self.ly_idx]
        self.ly_idx += 1
        self.v = self.v / nv[:, None]
        # Birkhoff tunes (kernel_tune_birkhoff :2548-2584)
        ax = np.arctan2(self.px, self.x)
        ay = np.arctan2(self.py, self.y)
        dx = ax - self.store_x
        dy = ay - self.store_y
        dx = np.where(dx > 0, dx, dx + 2 * np.pi)
        dy = np.where(dy > 0, dy, dy + 2 * np.pi)
        self.store_x, self.store_y = ax, ay
        for j, T in enumerate(self.tu_T):
            if self.tu_idx < T:
                w = self.tu_w[j][self.tu_idx]
                self.t1x[j] = self.t1x[j] + dx * w
                self.t1y[j] = self.t1y[j] + dy * w
            elif self.tu_idx < 2 * T:
                w = self.tu_w[j][self.tu_idx - T]
                self.t2x[j] = self.t2x[j] + dx * w
                self.t2y[j] = self.t2y[j] + dy * w
        self.tu_idx += 1

    def run(self, n_turns: int):
        for _ in range(n_turns):
            self.turn()
        return self
