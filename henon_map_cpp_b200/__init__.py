"""henon_map_cpp_b200 -- B200-native drop-in for henon_map_cpp's Python API.

    import henon_map_cpp_b200 as hm      # instead of: import henon_map_cpp as hm

The classes, method names, argument order and defaults are those of the
reference facade (henon_map_cpp/__init__.py), including its Python-side
defaults (for example track(..., barrier=10.0)).  Under them sit the
pybind11 module `henon_map_engine` (C++) and the C ABI of libhenon_b200.so
(include/henon_b200.h), whose kernels are written for sm_100a.

This package is the GPU path only: `force_CPU=True` and machines without a
CUDA device raise instead of falling back to a CPU implementation.
Additions over the reference are keyword-only or new methods:
`henon_tracker.set_arith("exact" | "fast")` and
`henon_tracker.track_indicators(...)` (the fused per-turn indicator loop).
"""
from __future__ import annotations

import numpy as np

try:
    from . import henon_map_engine as _E
    _IMPORT_ERROR = None
except ImportError as _e:  # library not built: every class raises on use
    _E = None
    _IMPORT_ERROR = _e

__all__ = ["gpu_available", "birkhoff_weights", "particles", "matrix_4d_vector", "vector_4d",
           "lyapunov_birkhoff_construct", "lyapunov_birkhoff_construct_multi",
           "megno_construct", "megno_birkhoff_construct", "tune_birkhoff_construct",
           "henon_tracker", "storage", "storage_gpu"]


def _engine():
    if _E is None:
        raise ImportError("henon_map_cpp_b200's compiled engine is missing; build it with "
                          f"`python -m henon_map_cpp_b200.build` ({_IMPORT_ERROR})")
    return _E


def _need_gpu(force_cpu: bool) -> None:
    if force_cpu:
        raise NotImplementedError("henon_map_cpp_b200 is the GPU path; the reference's CPU "
                                  "classes are not provided (force_CPU=True)")
    if not gpu_available():
        raise RuntimeError("henon_map_cpp_b200 needs a CUDA device; none is visible")


def gpu_available() -> bool:
    return _E is not None and bool(_E.is_cuda_device_available())


def birkhoff_weights(n):
    return np.asarray(_engine().birkhoff_weights(n))


class particles:
    def __init__(self, x_0, px_0, y_0, py_0, force_CPU=False):
        if not (isinstance(x_0, np.ndarray) and isinstance(px_0, np.ndarray)
                and isinstance(y_0, np.ndarray) and isinstance(py_0, np.ndarray)):
            raise TypeError("Arguments must be numpy arrays.")
        if not (x_0.ndim == 1 and px_0.ndim == 1 and y_0.ndim == 1 and py_0.ndim == 1):
            raise TypeError("Arguments must be 1D arrays.")
        if not (x_0.shape == px_0.shape == y_0.shape == py_0.shape):
            raise ValueError("Arguments must be of the same shape.")
        _need_gpu(force_CPU)
        self.particles = _engine().particles_4d_gpu(x_0, px_0, y_0, py_0)

    def reset(self):
        self.particles.reset()

    @property
    def kick_seed(self):
        """Key of the reproducible random kicks of henon_tracker.track
        (kick_module not NaN): the kick of a particle at a turn is a
        function of (kick_seed, particle index, turn)."""
        return self.particles.kick_seed

    @kick_seed.setter
    def kick_seed(self, seed):
        self.particles.kick_seed = int(seed)

    def add_ghost(self, module, displacement_kind):
        self.particles.add_ghost(module, displacement_kind)

    def renormalize(self, module):
        self.particles.renormalize(module)

    def get_displacement_module(self):
        return np.asarray(self.particles.get_displacement_module())

    def get_displacement_direction(self):
        return np.asarray(self.particles.get_displacement_direction())

    def get_x(self):
        return self.particles.get_x()

    def get_px(self):
        return np.asarray(self.particles.get_px())

    def get_y(self):
        return np.asarray(self.particles.get_y())

    def get_py(self):
        return np.asarray(self.particles.get_py())

    def get_steps(self):
        return np.asarray(self.particles.get_steps())

    def get_radius(self):
        return np.asarray(self.particles.get_radius())

    def get_radius_mean(self):
        return np.asarray(self.particles.get_radius_mean())

    def get_radius_std(self):
        return np.asarray(self.particles.get_radius_std())

    def get_action(self):
        return np.asarray(self.particles.get_action())

    def get_action_mean(self):
        return np.asarray(self.particles.get_action_mean())

    def get_action_std(self):
        return np.asarray(self.particles.get_action_std())

    def get_action_x(self):
        return np.asarray(self.particles.get_action_x())

    def get_action_x_mean(self):
        return np.asarray(self.particles.get_action_x_mean())

    def get_action_x_std(self):
        return np.asarray(self.particles.get_action_x_std())

    def get_action_y(self):
        return np.asarray(self.particles.get_action_y())

    def get_action_y_mean(self):
        return np.asarray(self.particles.get_action_y_mean())

    def get_action_y_std(self):
        return np.asarray(self.particles.get_action_y_std())

    def get_angle_x(self):
        return np.asarray(self.particles.get_angles_x())

    def get_angle_x_mean(self):
        return np.asarray(self.particles.get_angles_x_mean())

    def get_angle_x_std(self):
        return np.asarray(self.particles.get_angles_x_std())

    def get_angle_y(self):
        return np.asarray(self.particles.get_angles_y())

    def get_angle_y_mean(self):
        return np.asarray(self.particles.get_angles_y_mean())

    def get_angle_y_std(self):
        return np.asarray(self.particles.get_angles_y_std())


class matrix_4d_vector:
    def __init__(self, N, force_cpu=False):
        _need_gpu(force_cpu)
        print("Using GPU")
        self.GPU = True
        self.matrix = _engine().matrix_4d_vector_gpu(N)

    def reset(self):
        self.matrix.reset()

    def multiply(self, matrices):
        # The reference offers this on its CPU class only.
        raise NotImplementedError("multiply(matrices) exists on the reference's CPU class only")

    def structured_multiply(self, tracker, particles, mu, reverse=False):
        # The reference's GPU class has no reverse form (henon_map_cpp
        # __init__.py:155-160); neither has this one.
        self.matrix.structured_multiply(tracker.tracker, particles.particles, mu)

    def set_with_tracker(self, tracker, particles, mu, reverse=False):
        self.matrix.set_with_tracker(tracker.tracker, particles.particles, mu)

    def explicit_copy(self, other_matrix):
        self.matrix.explicit_copy(other_matrix.matrix)

    def get_matrix(self):
        return np.asarray(self.matrix.get_matrix())

    def get_vector(self, vector):
        return np.asarray(self.matrix.get_vector(np.asarray(vector, dtype=np.float64)))


class vector_4d:
    def __init__(self, initial_vector):
        assert gpu_available()
        self.vector = _engine().vector_4d_gpu(np.asarray(initial_vector, dtype=np.float64))

    def set_vectors(self, vector):
        self.vector.set_vectors(np.asarray(vector, dtype=np.float64))

    def multiply(self, matrix: matrix_4d_vector):
        self.vector.multiply(matrix.matrix)

    def normalize(self):
        self.vector.normalize()

    def get_vectors(self):
        return np.asarray(self.vector.get_vectors())


class lyapunov_birkhoff_construct:
    def __init__(self, n, n_weights):
        assert gpu_available()
        self.construct = _engine().lyapunov_birkhoff_construct(n, n_weights)

    def reset(self):
        self.construct.reset()

    def change_weights(self, n_weights):
        self.construct.change_weights(n_weights)

    def add(self, vectors):
        self.construct.add(vectors.vector)

    def get_weights(self):
        return np.asarray(self.construct.get_weights())

    def get_values_raw(self):
        return np.asarray(self.construct.get_values_raw())

    def get_values_b(self):
        return np.asarray(self.construct.get_values_b())


class lyapunov_birkhoff_construct_multi:
    def __init__(self, n, n_weights):
        assert gpu_available()
        self.construct = _engine().lyapunov_birkhoff_construct_multi(n, list(n_weights))

    def reset(self):
        self.construct.reset()

    def add(self, vectors):
        self.construct.add(vectors.vector)

    def get_values_raw(self):
        return np.asarray(self.construct.get_values_raw())

    def get_values_b(self):
        return np.asarray(self.construct.get_values_b())


class megno_construct:
    def __init__(self, n):
        assert gpu_available()
        self.construct = _engine().megno_construct(n)

    def reset(self):
        self.construct.reset()

    def add(self, matrix_a: matrix_4d_vector, matrix_b: matrix_4d_vector):
        self.construct.add(matrix_a.matrix, matrix_b.matrix)

    def get_values(self):
        return np.asarray(self.construct.get_values())


class megno_birkhoff_construct:
    def __init__(self, n, n_weights):
        assert gpu_available()
        self.construct = _engine().megno_birkhoff_construct(n, list(n_weights))

    def reset(self):
        self.construct.reset()

    def add(self, matrix_a: matrix_4d_vector, matrix_b: matrix_4d_vector):
        self.construct.add(matrix_a.matrix, matrix_b.matrix)

    def get_values(self):
        return np.asarray(self.construct.get_values())


class tune_birkhoff_construct:
    def __init__(self, n, n_weights):
        assert gpu_available()
        self.construct = _engine().tune_birkhoff_construct(n, list(n_weights))
        self.first_called = False

    def reset(self):
        self.construct.reset()

    def first_add(self, particles):
        self.construct.first_add(particles.particles)
        self.first_called = True

    def add(self, particles):
        if not self.first_called:
            raise ValueError("First call add_first")
        self.construct.add(particles.particles)

    def get_tune1_x(self):
        return self.construct.get_tune1_x()

    def get_tune1_y(self):
        return self.construct.get_tune1_y()

    def get_tune2_x(self):
        return self.construct.get_tune2_x()

    def get_tune2_y(self):
        return self.construct.get_tune2_y()


class henon_tracker:
    def __init__(self, N, omega_x, omega_y, modulation_kind, omega_0=np.nan, epsilon=0.0,
                 offset=0, force_CPU=False):
        _need_gpu(force_CPU)
        print("creating gpu tracker")
        self.tracker = _engine().henon_tracker_gpu(N, omega_x, omega_y, modulation_kind,
                                                   omega_0, epsilon, offset)

    def compute_a_modulation(self, n_turns, omega_x, omega_y, epsilon=0.0,
                             modulation_kind="sps", omega_0=np.nan, offset=0):
        self.tracker.compute_a_modulation(n_turns, omega_x, omega_y, modulation_kind, omega_0,
                                          epsilon, offset)

    def track(self, particles, n_turns, mu, barrier=10.0, kick_module=np.nan, inverse=False):
        self.tracker.track(particles.particles, n_turns, mu, barrier, kick_module, inverse)

    def megno(self, particles, n_turns, mu, barrier=10.0, kick_module=np.nan, inverse=False,
              turn_samples=np.array([]), n_threads=-1):
        """MEGNO at turn_samples (default: n_turns), shape (n, samples).

        Computed on the GPU with the megno_construct definition (Frobenius
        norm of the tangent map of the orbit); the reference's CPU routine
        uses the matrix trace instead and returns NaN in practice."""
        return np.asarray(self.tracker.megno(particles.particles, n_turns, mu, barrier,
                                             kick_module, inverse,
                                             [int(s) for s in np.asarray(turn_samples).ravel()],
                                             n_threads))

    def tune_birkhoff(self, particles, n_turns, mu, barrier=10.0, kick_module=np.nan,
                      inverse=False, from_idx=np.array([]), to_idx=np.array([])):
        import pandas as pd

        result = np.asarray(self.tracker.birkhoff_tunes(
            particles.particles, n_turns, mu, barrier, kick_module, inverse,
            [int(v) for v in np.asarray(from_idx).ravel()],
            [int(v) for v in np.asarray(to_idx).ravel()]))
        pd_result = pd.DataFrame(columns=["from", "to", "tune_x", "tune_y"])
        for i in range(len(from_idx)):
            pd_result.loc[i] = [from_idx[i], to_idx[i], result[:, i * 2], result[:, i * 2 + 1]]
        pd_result.loc[len(from_idx)] = [0, n_turns, result[:, -2], result[:, -1]]
        return pd_result

    def tune_all(self, particles, n_turns, mu, barrier=10.0, kick_module=np.nan, inverse=False,
                 from_idx=np.array([]), to_idx=np.array([])):
        import pandas as pd

        result_birkhoff, result_fft = (np.asarray(r) for r in self.tracker.all_tunes(
            particles.particles, n_turns, mu, barrier, kick_module, inverse,
            [int(v) for v in np.asarray(from_idx).ravel()],
            [int(v) for v in np.asarray(to_idx).ravel()]))
        pd_result = pd.DataFrame(columns=["from", "to", "tune_x_birkhoff", "tune_y_birkhoff",
                                          "tune_x_fft", "tune_y_fft"])
        for i in range(len(from_idx)):
            pd_result.loc[i] = [from_idx[i], to_idx[i], result_birkhoff[:, i * 2],
                                result_birkhoff[:, i * 2 + 1], result_fft[:, i * 2],
                                result_fft[:, i * 2 + 1]]
        pd_result.loc[len(from_idx)] = [0, n_turns, result_birkhoff[:, -2], result_birkhoff[:, -1],
                                        result_fft[:, -2], result_fft[:, -1]]
        return pd_result

    def get_tangent_matrix(self, particles, mu, reverse=False):
        return self.tracker.get_tangent_matrix(particles.particles, mu, reverse)

    def track_ghost_lyapunov(self, particles, n_steps, every, mu, module, barrier=10.0):
        """The displacement Lyapunov loop of the reference's notebooks,

            for _ in range(n_steps):
                tracker.track(particles, every, mu, barrier)
                lyap += np.log(particles.get_displacement_module() / module)
                particles.renormalize(module)

        in fused GPU launches; returns lyap (n_particles x n_ghosts) and
        leaves the particles as that loop does."""
        return np.asarray(self.tracker.track_ghost_lyapunov(particles.particles, int(n_steps),
                                                            int(every), mu, barrier, module))

    # ---- additions ---------------------------------------------------------------
    def set_arith(self, mode: str) -> None:
        """'exact' (default; bit-identical to the reference CPU path) or
        'fast' (fused multiply-adds)."""
        self.tracker.set_arith(mode)

    def track_indicators(self, particles, n_turns, mu, barrier=10.0, *, matrix=None,
                         matrix_old=None, megno=None, megno_birkhoff=None, vectors=None,
                         lyapunov=None, tune=None, megno_sample_turns=()):
        """n_turns iterations of the per-turn construct loop in fused launches:

            matrix_old <- matrix; track(p, 1); matrix.structured_multiply;
            megno.add(matrix, matrix_old); megno_birkhoff.add(matrix, matrix_old);
            J = DF; vectors.multiply(J); lyapunov.add(vectors); vectors.normalize();
            tune.add(p)

        Each argument is one of this package's objects (or None).  Returns the
        MEGNO values recorded when megno's add counter hits each of
        megno_sample_turns, shape (len(megno_sample_turns), n)."""
        def inner(obj, attr):
            return getattr(obj, attr) if obj is not None else None
        if tune is not None and not tune.first_called:
            raise ValueError("First call add_first")
        return np.asarray(self.tracker.track_indicators(
            particles.particles, n_turns, mu, barrier,
            matrix=inner(matrix, "matrix"), matrix_old=inner(matrix_old, "matrix"),
            megno=inner(megno, "construct"), megno_birkhoff=inner(megno_birkhoff, "construct"),
            vectors=inner(vectors, "vector"), lyapunov=inner(lyapunov, "construct"),
            tune=inner(tune, "construct"),
            megno_sample_turns=[int(s) for s in megno_sample_turns]))


class storage:
    """Turn-by-turn snapshots kept on the host (storage_4d); the tune
    estimates run on the GPU (hm_orbit_tunes)."""

    def __init__(self, N):
        self.N = N
        self._x, self._px, self._y, self._py = [], [], [], []

    def store(self, particles):
        p = particles.particles
        self._x.append(np.asarray(p.get_x())[:self.N])
        self._px.append(np.asarray(p.get_px())[:self.N])
        self._y.append(np.asarray(p.get_y())[:self.N])
        self._py.append(np.asarray(p.get_py())[:self.N])

    def _tunes(self, from_idx, to_idx, method):
        return np.asarray(_engine().orbit_tunes(
            np.asarray(self._x), np.asarray(self._px), np.asarray(self._y),
            np.asarray(self._py), [int(v) for v in from_idx], [int(v) for v in to_idx], method))

    def _frame(self, result, from_idx, to_idx, max_value):
        import pandas as pd

        pd_result = pd.DataFrame(columns=["from", "to", "tune_x", "tune_y"])
        for i in range(len(from_idx)):
            pd_result.loc[i] = [from_idx[i], to_idx[i], result[:, i * 2], result[:, i * 2 + 1]]
        pd_result.loc[len(from_idx)] = [0, max_value, result[:, -2], result[:, -1]]
        return pd_result

    def tune_fft(self, from_idx, to_idx, max_value):
        return self._frame(self._tunes(from_idx, to_idx, 1), from_idx, to_idx, max_value)

    def tune_birkhoff(self, from_idx, to_idx, max_value):
        return self._frame(self._tunes(from_idx, to_idx, 0), from_idx, to_idx, max_value)

    def get_x(self):
        return np.asarray(self._x).T

    def get_px(self):
        return np.asarray(self._px).T

    def get_y(self):
        return np.asarray(self._y).T

    def get_py(self):
        return np.asarray(self._py).T


class storage_gpu:
    def __init__(self, N, batch_size):
        self.storage = _engine().storage_4d_gpu(N, batch_size)

    def store(self, particles):
        self.storage.store(particles.particles)

    def reset(self):
        self.storage.reset()

    def get_x(self):
        return np.asarray(self.storage.get_x())

    def get_px(self):
        return np.asarray(self.storage.get_px())

    def get_y(self):
        return np.asarray(self.storage.get_y())

    def get_py(self):
        return np.asarray(self.storage.get_py())
