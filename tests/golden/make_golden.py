"""Generates the golden fixtures of tests/golden/ by running the reference
itself (carlidel/henon_map_cpp built from its own sources by
oracle/build_ref.sh, CPU path) on seeded inputs.

    python tests/golden/make_golden.py

The fixtures are small .npz files; the tests compare both the oracle and
the CUDA library against them, so the oracle is pinned to the reference and
the GPU path to both.  Needs oracle/_ref/ (built where the reference sources
are present); the fixtures themselves travel without it.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import oracle as O  # noqa: E402

TUNES = (0.168, 0.201)
NAN = float("nan")

# (name, grid extent, grid side, epsilon, mu, turns)
TRACK_CASES = [
    ("c1_like", 0.5, 24, 0.0, 0.0, 3000),
    ("eps16_mu02", 0.6, 24, 16.0, 0.2, 3000),
    ("eps64_mu02", 0.6, 24, 64.0, 0.2, 3000),
    ("eps1_mu0", 0.6, 24, 1.0, 0.0, 3000),
    ("eps32_mum05", 0.45, 20, 32.0, -0.5, 2500),
]


def grid(extent: float, side: int):
    v = np.linspace(0.0, extent, side)
    xx, yy = np.meshgrid(v, v)
    x = xx.ravel()
    y = yy.ravel()
    return x, np.zeros_like(x), y, np.zeros_like(y)


def ref_track(R, x, px, y, py, n_turns, eps, mu, barrier=10.0, chunks=None):
    t = R.henon_tracker(n_turns, TUNES[0], TUNES[1], "sps", NAN, eps, 0)
    p = R.particles_4d(x, px, y, py)
    for n in (chunks or [n_turns]):
        t.track(p, n, mu, barrier)
    return [np.asarray(p.get_x()), np.asarray(p.get_px()), np.asarray(p.get_y()),
            np.asarray(p.get_py()), np.asarray(p.get_steps()).astype(np.uint32)]


def main() -> None:
    R = O.reference_module("fmad_off")
    if R is None:
        raise SystemExit("oracle/_ref/fmad_off is missing: run oracle/build_ref.sh first")
    for name, ext, side, eps, mu, nt in TRACK_CASES:
        x, px, y, py = grid(ext, side)
        rx, rpx, ry, rpy, rs = ref_track(R, x, px, y, py, nt, eps, mu)
        np.savez_compressed(HERE / f"ref_track_{name}.npz", x0=x, px0=px, y0=y, py0=py,
                            x=rx, px=rpx, y=ry, py=rpy, steps=rs,
                            epsilon=eps, mu=mu, n_turns=nt, tunes=np.array(TUNES))
        print(name, "survivors", int(np.sum(rs == nt)), "/", rs.size)

    # Forward then inverse (reversibility; henon.cu:510-528).
    rng = np.random.default_rng(7)
    x = rng.uniform(0, 0.3, 200)
    y = rng.uniform(0, 0.3, 200)
    px = rng.normal(0, 0.01, 200)
    py = rng.normal(0, 0.01, 200)
    t = R.henon_tracker(1000, TUNES[0], TUNES[1], "sps", NAN, 64.0, 0)
    p = R.particles_4d(x, px, y, py)
    t.track(p, 1000, 0.1, 10.0)
    fwd = [np.asarray(p.get_x()), np.asarray(p.get_px()), np.asarray(p.get_y()),
           np.asarray(p.get_py()), np.asarray(p.get_steps()).astype(np.uint32)]
    t.track(p, 1000, 0.1, 10.0, NAN, True)
    back = [np.asarray(p.get_x()), np.asarray(p.get_px()), np.asarray(p.get_y()),
            np.asarray(p.get_py()), np.asarray(p.get_steps()).astype(np.uint32)]
    np.savez_compressed(HERE / "ref_reverse.npz", x0=x, px0=px, y0=y, py0=py,
                        fx=fwd[0], fpx=fwd[1], fy=fwd[2], fpy=fwd[3], fsteps=fwd[4],
                        bx=back[0], bpx=back[1], by=back[2], bpy=back[3], bsteps=back[4],
                        epsilon=64.0, mu=0.1, n_turns=1000, tunes=np.array(TUNES))

    # Modulation tables and Birkhoff weights.
    np.savez_compressed(
        HERE / "ref_modulation.npz",
        sps_x_eps16=np.asarray(R.sps_modulation(TUNES[0], 16.0, 0, 4000)),
        sps_y_eps64_off=np.asarray(R.sps_modulation(TUNES[1], 64.0, 12345, 12345 + 3000)),
        basic_x=np.asarray(R.basic_modulation(0.31, 0.01, 0.5, 0, 2000)),
        bw10=np.asarray(R.birkhoff_weights(10)),
        bw1000=np.asarray(R.birkhoff_weights(1000)),
    )
    meta = {"generator": "tests/golden/make_golden.py",
            "reference": "carlidel/henon_map_cpp built by oracle/build_ref.sh (fmad_off)",
            "cases": [c[0] for c in TRACK_CASES]}
    (HERE / "ref_fixtures.json").write_text(json.dumps(meta, indent=1) + "\n")


if __name__ == "__main__":
    main()
