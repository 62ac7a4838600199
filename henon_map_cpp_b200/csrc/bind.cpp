// pybind11 module `henon_map_engine`: the reference's Python-facing engine
// (src/bind.cpp:224-577) re-exposed over the C ABI of libhenon_b200.so.
//
// Class names, method names, argument names and defaults follow the
// reference's GPU classes (particles_4d_gpu, henon_tracker_gpu,
// matrix_4d_vector_gpu, vector_4d_gpu, the constructs, storage_4d_gpu).
// Long calls release the GIL; Ctrl-C stops them between turn chunks.
#include <pybind11/eval.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <cmath>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "henon_b200.h"

namespace py = pybind11;

namespace {

// Raises the Python exception that matches a non-OK status.  Budget and
// modulation errors are RuntimeError with the reference's messages.
void check(hm_status s) {
    if (s == HM_OK) return;
    const std::string msg = hm_last_error();
    switch (s) {
        case HM_ERR_INVALID_ARG: throw py::value_error(msg);
        case HM_ERR_NOT_SUPPORTED: throw std::domain_error(msg);
        case HM_ERR_OOM: throw std::bad_alloc();
        case HM_ERR_CANCELLED:
            if (PyErr_Occurred()) throw py::error_already_set();
            PyErr_SetNone(PyExc_KeyboardInterrupt);
            throw py::error_already_set();
        default: throw std::runtime_error(msg);
    }
}

// Cancel callback: runs between chunks with the GIL released by the caller.
int check_signals(void *) {
    py::gil_scoped_acquire gil;
    return PyErr_CheckSignals() != 0 ? 1 : 0;
}

template <class T>
py::array_t<T> array1(size_t n) {
    return py::array_t<T>(std::vector<py::ssize_t>{py::ssize_t(n)});
}

py::array_t<double> array2(size_t a, size_t b) {
    return py::array_t<double>(std::vector<py::ssize_t>{py::ssize_t(a), py::ssize_t(b)});
}

std::vector<double> as_vec(const py::array_t<double, py::array::c_style | py::array::forcecast> &a) {
    return std::vector<double>(a.data(), a.data() + a.size());
}

double nan_mean(const double *v, size_t n) {
    double sum = 0.0;
    size_t count = 0;
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(v[i])) {
            sum += v[i];
            ++count;
        }
    return count ? sum / count : std::numeric_limits<double>::quiet_NaN();
}

double nan_std(const double *v, size_t n) {
    const double mean = nan_mean(v, n);
    double sum = 0.0;
    size_t count = 0;
    for (size_t i = 0; i < n; ++i)
        if (!std::isnan(v[i])) {
            sum += (v[i] - mean) * (v[i] - mean);
            ++count;
        }
    return count ? std::sqrt(sum / count) : std::numeric_limits<double>::quiet_NaN();
}

// ---- particles_4d_gpu --------------------------------------------------------------

struct Particles {
    hm_particles *h = nullptr;
    Particles(const std::vector<double> &x, const std::vector<double> &px,
              const std::vector<double> &y, const std::vector<double> &py) {
        if (px.size() != x.size() || y.size() != x.size() || py.size() != x.size())
            throw py::value_error("x, px, y, py must have the same length");
        check(hm_particles_create(x.data(), px.data(), y.data(), py.data(), x.size(), &h));
    }
    ~Particles() { hm_particles_destroy(h); }
    Particles(const Particles &) = delete;
    Particles &operator=(const Particles &) = delete;

    size_t n_total() const {
        size_t n = 0;
        check(hm_particles_size(h, &n, nullptr, nullptr));
        return n;
    }
    template <class T>
    py::array_t<T> field(hm_field f) const {
        auto out = array1<T>(n_total());
        check(hm_particles_get(h, f, out.mutable_data()));
        return out;
    }
    py::array_t<double> observable(hm_observable k) const {
        auto out = array1<double>(n_total());
        check(hm_particles_observable(h, k, out.mutable_data()));
        return out;
    }
    double mean(hm_observable k) const {
        auto a = observable(k);
        return nan_mean(a.data(), size_t(a.size()));
    }
    double stdev(hm_observable k) const {
        auto a = observable(k);
        return nan_std(a.data(), size_t(a.size()));
    }
    size_t n_particles() const {
        size_t n = 0;
        check(hm_particles_size(h, nullptr, &n, nullptr));
        return n;
    }
    size_t n_ghosts() const {
        size_t n = 0;
        check(hm_particles_size(h, nullptr, nullptr, &n));
        return n;
    }
    uint32_t global_steps() const {
        uint32_t g = 0;
        check(hm_particles_global_steps(h, &g));
        return g;
    }
};

// ---- henon_tracker_gpu -------------------------------------------------------------

struct Tracker {
    hm_tracker *h = nullptr;
    Tracker(unsigned n, double wx, double wy, const std::string &kind, double w0, double eps,
            unsigned offset) {
        check(hm_tracker_create(n, wx, wy, kind.c_str(), w0, eps, offset, &h));
    }
    ~Tracker() { hm_tracker_destroy(h); }
    Tracker(const Tracker &) = delete;
    Tracker &operator=(const Tracker &) = delete;
};

struct Matrices {
    hm_matrices *h = nullptr;
    size_t n = 0;
    explicit Matrices(size_t n_) : n(n_) { check(hm_matrices_create(n, &h)); }
    ~Matrices() { hm_matrices_destroy(h); }
    Matrices(const Matrices &) = delete;
    Matrices &operator=(const Matrices &) = delete;
};

struct Vectors {
    hm_vectors *h = nullptr;
    size_t n = 0;
    explicit Vectors(const std::vector<std::vector<double>> &rv) : n(rv.size()) {
        std::vector<double> flat(4 * n);
        for (size_t i = 0; i < n; ++i) {
            if (rv[i].size() != 4) throw py::value_error("vectors must have 4 components");
            for (int k = 0; k < 4; ++k) flat[4 * i + k] = rv[i][k];
        }
        check(hm_vectors_create(flat.data(), n, &h));
    }
    ~Vectors() { hm_vectors_destroy(h); }
    Vectors(const Vectors &) = delete;
    Vectors &operator=(const Vectors &) = delete;
};

struct Lyapunov {
    hm_lyapunov *h = nullptr;
    size_t n = 0;
    std::vector<uint64_t> lengths;
    Lyapunov(size_t n_, std::vector<uint64_t> w) : n(n_), lengths(std::move(w)) {
        check(hm_lyapunov_create(n, lengths.data(), lengths.size(), &h));
    }
    ~Lyapunov() { hm_lyapunov_destroy(h); }
    Lyapunov(const Lyapunov &) = delete;
    Lyapunov &operator=(const Lyapunov &) = delete;
    py::array_t<double> values(int birkhoff) const {
        auto out = array2(lengths.size(), n);
        check(hm_lyapunov_get(h, birkhoff, out.mutable_data()));
        return out;
    }
    py::array_t<double> weights(size_t w) const {
        auto out = array1<double>(lengths.at(w));
        check(hm_lyapunov_get_weights(h, w, out.mutable_data()));
        return out;
    }
};

// Several windows (lyapunov_birkhoff_construct_multi); a subclass so that the
// fused call takes either form.
struct LyapunovMulti : Lyapunov {
    using Lyapunov::Lyapunov;
};

struct Megno {
    hm_megno *h = nullptr;
    size_t n = 0;
    explicit Megno(size_t n_) : n(n_) { check(hm_megno_create(n, &h)); }
    ~Megno() { hm_megno_destroy(h); }
    Megno(const Megno &) = delete;
    Megno &operator=(const Megno &) = delete;
};

struct MegnoBirkhoff {
    hm_megno_birkhoff *h = nullptr;
    size_t n = 0;
    std::vector<uint64_t> T;
    MegnoBirkhoff(size_t n_, std::vector<uint64_t> t) : n(n_), T(std::move(t)) {
        check(hm_megno_birkhoff_create(n, T.data(), T.size(), &h));
    }
    ~MegnoBirkhoff() { hm_megno_birkhoff_destroy(h); }
    MegnoBirkhoff(const MegnoBirkhoff &) = delete;
    MegnoBirkhoff &operator=(const MegnoBirkhoff &) = delete;
};

struct TuneBirkhoff {
    hm_tune_birkhoff *h = nullptr;
    size_t n = 0;
    std::vector<uint64_t> T;
    TuneBirkhoff(size_t n_, std::vector<uint64_t> t) : n(n_), T(std::move(t)) {
        check(hm_tune_birkhoff_create(n, T.data(), T.size(), &h));
    }
    ~TuneBirkhoff() { hm_tune_birkhoff_destroy(h); }
    TuneBirkhoff(const TuneBirkhoff &) = delete;
    TuneBirkhoff &operator=(const TuneBirkhoff &) = delete;
    py::array_t<double> get(int which) const {
        auto out = array2(T.size(), n);
        check(hm_tune_birkhoff_get(h, which, out.mutable_data()));
        return out;
    }
};

struct Storage {
    hm_storage *h = nullptr;
    size_t n = 0, batch = 0;
    Storage(size_t n_, size_t b) : n(n_), batch(b) { check(hm_storage_create(n, batch, &h)); }
    ~Storage() { hm_storage_destroy(h); }
    Storage(const Storage &) = delete;
    Storage &operator=(const Storage &) = delete;
    py::array_t<double> get(hm_field f) const {
        auto out = array2(batch, n);
        check(hm_storage_get(h, f, out.mutable_data()));
        return out;
    }
};

}  // namespace

PYBIND11_MODULE(henon_map_engine, m) {
    m.doc() = "Henon map engine (B200-native): particles, tracker, tangent map, indicators";
    check(hm_set_cancel_callback(&check_signals, nullptr));

    m.def("is_cuda_device_available", []() { return hm_device_count() > 0; });
    m.def("version", []() { return hm_version(); });

    m.def("sps_modulation", [](double tune, double epsilon, int start, int end) {
        auto out = array1<double>(end > start ? size_t(end - start) : 0);
        check(hm_sps_modulation(tune, epsilon, start, end, out.mutable_data()));
        return out;
    }, py::arg("tune"), py::arg("epsilon"), py::arg("start"), py::arg("end"));
    m.def("basic_modulation", [](double tune, double omega, double epsilon, int start, int end) {
        auto out = array1<double>(end > start ? size_t(end - start) : 0);
        check(hm_basic_modulation(tune, omega, epsilon, start, end, out.mutable_data()));
        return out;
    }, py::arg("tune"), py::arg("omega"), py::arg("epsilon"), py::arg("start"), py::arg("end"));
    m.def("gaussian_modulation", [](double tune, double sigma, int start, int end) {
        const uint32_t n = end > start ? uint32_t(end - start) : 0;
        auto out = array1<double>(n);
        std::vector<double> other(n);
        check(hm_modulation("gaussian", n, tune, tune, NAN, sigma, uint32_t(start), out.mutable_data(),
                            other.data()));
        return out;
    }, py::arg("tune"), py::arg("sigma"), py::arg("start"), py::arg("end"));
    m.def("uniform_modulation", [](double from, double to, int start, int end) {
        const uint32_t n = end > start ? uint32_t(end - start) : 0;
        auto out = array1<double>(n);
        std::vector<double> other(n);
        check(hm_modulation("uniform", n, from, from, NAN, to, uint32_t(start), out.mutable_data(),
                            other.data()));
        return out;
    }, py::arg("from"), py::arg("to"), py::arg("start"), py::arg("end"));
    m.def("orbit_tunes", [](py::array_t<double, py::array::c_style | py::array::forcecast> x,
                            py::array_t<double, py::array::c_style | py::array::forcecast> px,
                            py::array_t<double, py::array::c_style | py::array::forcecast> y,
                            py::array_t<double, py::array::c_style | py::array::forcecast> py_,
                            std::vector<uint32_t> from, std::vector<uint32_t> to, int method) {
        // Tunes of host orbits [samples][particles]: windows + full orbit.
        if (x.ndim() != 2 || px.ndim() != 2 || y.ndim() != 2 || py_.ndim() != 2)
            throw py::value_error("orbits must be 2D [samples][particles]");
        const size_t S = size_t(x.shape(0)), n = size_t(x.shape(1));
        if (from.size() != to.size())
            throw std::runtime_error("compute_tune: from and to must be of the same size");
        auto out = array2(n, 2 * (from.size() + 1));
        check(hm_orbit_tunes_host(x.data(), px.data(), y.data(), py_.data(), n, S, from.data(),
                                  to.data(), from.size(), method, out.mutable_data()));
        return out;
    }, py::arg("x"), py::arg("px"), py::arg("y"), py::arg("py"), py::arg("from_idx"),
       py::arg("to_idx"), py::arg("method"));
    // get_tunes (src/dynamic_indicator.cpp:333-362, bound at src/bind.cpp:241):
    // (FFT tune, Birkhoff tune) of one plane's orbit over all its samples,
    // i.e. the window [0, n-1] of the windowed tunes; NaN when the orbit
    // holds a NaN.
    m.def("get_tunes", [](std::vector<double> x, std::vector<double> px) {
        if (x.size() != px.size())
            throw std::runtime_error("get_tunes: x and px must be of the same size");
        if (x.size() < 2) throw py::value_error("get_tunes: need at least two samples");
        const uint32_t from = 0u, to = uint32_t(x.size() - 1);
        double fft[4], birk[4];
        check(hm_orbit_tunes_host(x.data(), px.data(), x.data(), px.data(), 1, x.size(), &from, &to,
                                  1, 1, fft));
        check(hm_orbit_tunes_host(x.data(), px.data(), x.data(), px.data(), 1, x.size(), &from, &to,
                                  1, 0, birk));
        return std::array<double, 2>{fft[0], birk[0]};
    }, py::arg("x"), py::arg("px"));
    // The reference's CPU classes (particles_4d, henon_tracker,
    // matrix_4d_vector, storage_4d; src/bind.cpp:243-557) exist here by name,
    // so that code importing them -- the reference's own Python package
    // among it -- keeps working.  This build is the GPU path: constructing
    // one raises, as the facade's force_CPU does; use the _gpu classes.
    py::exec(R"(
class _CpuClassNotProvided:
    _name = ''
    def __init__(self, *args, **kwargs):
        raise NotImplementedError(
            self._name + ': the CPU classes are not provided by this build; '
            'use ' + self._name + '_gpu (bit-identical results on the GPU)')
class particles_4d(_CpuClassNotProvided):
    _name = 'particles_4d'
class henon_tracker(_CpuClassNotProvided):
    _name = 'henon_tracker'
class matrix_4d_vector(_CpuClassNotProvided):
    _name = 'matrix_4d_vector'
class storage_4d(_CpuClassNotProvided):
    _name = 'storage_4d'
)", m.attr("__dict__"));
    m.def("birkhoff_weights", [](unsigned n) {
        auto out = array1<double>(n);
        check(hm_birkhoff_weights(n, out.mutable_data()));
        return out;
    }, py::arg("n_weights"));

    // ---- particles_4d_gpu ----------------------------------------------------------
    py::class_<Particles>(m, "particles_4d_gpu")
        .def(py::init<const std::vector<double> &, const std::vector<double> &,
                      const std::vector<double> &, const std::vector<double> &>(),
             py::arg("x"), py::arg("px"), py::arg("y"), py::arg("py"))
        .def("reset", [](Particles &p) { check(hm_particles_reset(p.h)); })
        // Key of the reproducible random kicks of track(kick_module=...);
        // no counterpart in the reference, whose kicks are clock()-seeded.
        .def_property(
            "kick_seed",
            [](const Particles &p) {
                uint64_t v = 0;
                check(hm_particles_get_kick_seed(p.h, &v));
                return v;
            },
            [](Particles &p, uint64_t v) { check(hm_particles_set_kick_seed(p.h, v)); })
        .def("add_ghost", [](Particles &p, double module, const std::string &dir) {
            check(hm_particles_add_ghost(p.h, module, dir.c_str()));
        }, py::arg("displacement_module"), py::arg("direction"))
        .def("renormalize", [](Particles &p, double module) {
            check(hm_particles_renormalize(p.h, module));
        }, py::arg("module_target"))
        .def("get_displacement_module", [](const Particles &p) {
            auto out = array2(p.n_particles(), p.n_ghosts());
            check(hm_particles_displacement_module(p.h, out.mutable_data()));
            return out;
        })
        .def("get_displacement_direction", [](const Particles &p) {
            const size_t nb = p.n_particles(), ng = p.n_ghosts();
            py::array_t<double> out(std::vector<py::ssize_t>{4, py::ssize_t(nb), py::ssize_t(ng)});
            check(hm_particles_displacement_direction(p.h, out.mutable_data()));
            return out;
        })
        .def("get_x", [](const Particles &p) { return p.field<double>(HM_FIELD_X); })
        .def("get_px", [](const Particles &p) { return p.field<double>(HM_FIELD_PX); })
        .def("get_y", [](const Particles &p) { return p.field<double>(HM_FIELD_Y); })
        .def("get_py", [](const Particles &p) { return p.field<double>(HM_FIELD_PY); })
        .def("get_steps", [](const Particles &p) { return p.field<uint32_t>(HM_FIELD_STEPS); })
        .def("get_valid", [](const Particles &p) { return p.field<uint8_t>(HM_FIELD_VALID); })
        .def("get_ghost", [](const Particles &p) { return p.field<uint8_t>(HM_FIELD_GHOST); })
        .def("get_idx", [](const Particles &p) { return p.field<uint64_t>(HM_FIELD_IDX); })
        .def("get_idx_base", [](const Particles &p) { return p.field<uint64_t>(HM_FIELD_IDX_BASE); })
        .def("get_radius", [](const Particles &p) { return p.observable(HM_OBS_RADIUS); })
        .def("get_radius_mean", [](const Particles &p) { return p.mean(HM_OBS_RADIUS); })
        .def("get_radius_std", [](const Particles &p) { return p.stdev(HM_OBS_RADIUS); })
        .def("get_action", [](const Particles &p) { return p.observable(HM_OBS_ACTION); })
        .def("get_action_mean", [](const Particles &p) { return p.mean(HM_OBS_ACTION); })
        .def("get_action_std", [](const Particles &p) { return p.stdev(HM_OBS_ACTION); })
        .def("get_action_x", [](const Particles &p) { return p.observable(HM_OBS_ACTION_X); })
        .def("get_action_x_mean", [](const Particles &p) { return p.mean(HM_OBS_ACTION_X); })
        .def("get_action_x_std", [](const Particles &p) { return p.stdev(HM_OBS_ACTION_X); })
        .def("get_action_y", [](const Particles &p) { return p.observable(HM_OBS_ACTION_Y); })
        .def("get_action_y_mean", [](const Particles &p) { return p.mean(HM_OBS_ACTION_Y); })
        .def("get_action_y_std", [](const Particles &p) { return p.stdev(HM_OBS_ACTION_Y); })
        .def("get_angles_x", [](const Particles &p) { return p.observable(HM_OBS_ANGLE_X); })
        .def("get_angles_x_mean", [](const Particles &p) { return p.mean(HM_OBS_ANGLE_X); })
        .def("get_angles_x_std", [](const Particles &p) { return p.stdev(HM_OBS_ANGLE_X); })
        .def("get_angles_y", [](const Particles &p) { return p.observable(HM_OBS_ANGLE_Y); })
        .def("get_angles_y_mean", [](const Particles &p) { return p.mean(HM_OBS_ANGLE_Y); })
        .def("get_angles_y_std", [](const Particles &p) { return p.stdev(HM_OBS_ANGLE_Y); })
        .def("get_n_particles", &Particles::n_particles)
        .def("get_n_ghosts_per_particle", &Particles::n_ghosts)
        .def("get_global_steps", &Particles::global_steps);

    // ---- henon_tracker_gpu ---------------------------------------------------------
    py::class_<Tracker>(m, "henon_tracker_gpu")
        .def(py::init<unsigned, double, double, const std::string &, double, double, unsigned>(),
             py::arg("N"), py::arg("omega_x"), py::arg("omega_y"),
             py::arg("modulation_kind") = "sps", py::arg("omega_0") = NAN,
             py::arg("epsilon") = 0.0, py::arg("offset") = 0)
        .def("compute_a_modulation", [](Tracker &t, unsigned n, double wx, double wy,
                                        const std::string &kind, double w0, double eps,
                                        unsigned offset) {
            check(hm_tracker_compute_a_modulation(t.h, n, wx, wy, kind.c_str(), w0, eps, offset));
        }, py::arg("N"), py::arg("omega_x"), py::arg("omega_y"), py::arg("modulation_kind"),
           py::arg("omega_0"), py::arg("epsilon"), py::arg("offset"))
        .def("track", [](Tracker &t, Particles &p, unsigned n_turns, double mu, double barrier,
                         double kick_module, bool inverse) {
            hm_status s;
            {
                py::gil_scoped_release nogil;
                s = hm_track(t.h, p.h, n_turns, mu, barrier, kick_module, inverse ? 1 : 0);
            }
            check(s);
        }, "Track particles", py::arg("particles"), py::arg("n_turns"), py::arg("mu"),
           py::arg("barrier") = 100.0, py::arg("kick_module") = NAN, py::arg("inverse") = false)
        .def("track_ghost_lyapunov", [](Tracker &t, Particles &p, unsigned n_steps,
                                        unsigned every, double mu, double barrier,
                                        double module) {
            auto out = array2(p.n_particles(), p.n_ghosts());
            hm_status s;
            double *dst = out.mutable_data();
            {
                py::gil_scoped_release nogil;
                s = hm_track_ghost_lyapunov(t.h, p.h, n_steps, every, mu, barrier, module, dst);
            }
            check(s);
            return out;
        }, "n_steps x (track `every` turns; sum log(displacement / module); renormalize) "
           "in fused launches",
           py::arg("particles"), py::arg("n_steps"), py::arg("every"), py::arg("mu"),
           py::arg("barrier"), py::arg("module"))
        .def("get_tangent_matrix", [](const Tracker &t, const Particles &p, double mu,
                                      bool reverse) {
            const size_t n = p.n_total();
            py::array_t<double> out(std::vector<py::ssize_t>{py::ssize_t(n), 4, 4});
            check(hm_tracker_tangent_matrices(t.h, p.h, mu, reverse ? 1 : 0, out.mutable_data()));
            return out;
        }, py::arg("particles"), py::arg("mu"), py::arg("reverse"))
        .def("set_arith", [](Tracker &t, const std::string &mode) {
            if (mode != "exact" && mode != "fast")
                throw py::value_error("arithmetic must be 'exact' or 'fast'");
            check(hm_tracker_set_arith(t.h, mode == "fast" ? HM_ARITH_FAST : HM_ARITH_EXACT));
        }, py::arg("mode"))
        .def("get_arith", [](const Tracker &t) {
            hm_arith a;
            check(hm_tracker_get_arith(t.h, &a));
            return std::string(a == HM_ARITH_FAST ? "fast" : "exact");
        })
        .def("allowed_steps", [](const Tracker &t) {
            uint64_t n = 0;
            check(hm_tracker_allowed_steps(t.h, &n));
            return n;
        })
        .def("birkhoff_tunes", [](Tracker &t, Particles &p, unsigned n_turns, double mu,
                                  double barrier, double kick, bool inverse,
                                  std::vector<uint32_t> from, std::vector<uint32_t> to) {
            // henon_tracker::birkhoff_tunes (src/henon.cu:2890-2967): the
            // window [0, n_turns] is appended to the caller's, then the full
            // orbit; result [n][2 (W + 2)].
            if (from.size() != to.size())
                throw std::runtime_error("compute_tune: from and to must be of the same size");
            from.push_back(0);
            to.push_back(n_turns);
            auto out = array2(p.n_total(), 2 * (from.size() + 1));
            hm_status s;
            {
                py::gil_scoped_release nogil;
                s = hm_tracker_orbit_tunes(t.h, p.h, n_turns, mu, barrier, kick, inverse ? 1 : 0,
                                           from.data(), to.data(), from.size(), 0,
                                           out.mutable_data(), nullptr);
            }
            check(s);
            return out;
        }, py::arg("particles"), py::arg("n_turns"), py::arg("mu"), py::arg("barrier") = 100.0,
           py::arg("kick_module") = NAN, py::arg("inverse") = false,
           py::arg("from_idx") = std::vector<uint32_t>(), py::arg("to_idx") = std::vector<uint32_t>())
        .def("all_tunes", [](Tracker &t, Particles &p, unsigned n_turns, double mu,
                             double barrier, double kick, bool inverse, std::vector<uint32_t> from,
                             std::vector<uint32_t> to) {
            // henon_tracker::all_tunes (src/henon.cu:2969-3078): orbit mean
            // removed, Birkhoff and FFT tunes; ([n][2(W+2)], [n][2(W+2)]).
            if (from.size() != to.size())
                throw std::runtime_error("compute_tune: from and to must be of the same size");
            from.push_back(0);
            to.push_back(n_turns);
            auto b = array2(p.n_total(), 2 * (from.size() + 1));
            auto f = array2(p.n_total(), 2 * (from.size() + 1));
            hm_status s;
            {
                py::gil_scoped_release nogil;
                s = hm_tracker_orbit_tunes(t.h, p.h, n_turns, mu, barrier, kick, inverse ? 1 : 0,
                                           from.data(), to.data(), from.size(), 1,
                                           b.mutable_data(), f.mutable_data());
            }
            check(s);
            return py::make_tuple(b, f);
        }, py::arg("particles"), py::arg("n_turns"), py::arg("mu"), py::arg("barrier") = 100.0,
           py::arg("kick_module") = NAN, py::arg("inverse") = false,
           py::arg("from_idx") = std::vector<uint32_t>(), py::arg("to_idx") = std::vector<uint32_t>())
        .def("megno", [](Tracker &t, Particles &p, unsigned n_turns, double mu, double barrier,
                         double kick, bool inverse, std::vector<uint64_t> samples, int) {
            // Whole-orbit MEGNO (henon_tracker::megno, src/henon.cu:2755-2887)
            // with the GPU construct's definition (Frobenius norm of the
            // tangent map, src/henon.cu:2253-2284) and the tangent map of each
            // turn; values at the turn counts in turn_samples: [n][samples].
            if (samples.empty()) samples.push_back(n_turns);
            auto out = array2(p.n_total(), samples.size());
            double *o = out.mutable_data();
            hm_status st;
            {
                py::gil_scoped_release nogil;
                st = hm_tracker_megno(t.h, p.h, n_turns, mu, barrier, kick, inverse ? 1 : 0,
                                      samples.data(), samples.size(), o);
            }
            check(st);
            return out;
        }, py::arg("particles"), py::arg("n_turns"), py::arg("mu"), py::arg("barrier") = 100.0,
           py::arg("kick_module") = NAN, py::arg("inverse") = false,
           py::arg("turn_samples") = std::vector<uint64_t>(), py::arg("n_threads") = -1)
        .def("track_indicators", [](Tracker &t, Particles &p, unsigned n_turns, double mu,
                                    double barrier, Matrices *matrix, Matrices *matrix_old,
                                    Megno *megno, MegnoBirkhoff *megno_b, Vectors *vectors,
                                    Lyapunov *lyap, TuneBirkhoff *tune,
                                    std::vector<uint64_t> samples) {
            hm_indicator_set s{};
            s.matrix = matrix ? matrix->h : nullptr;
            s.matrix_old = matrix_old ? matrix_old->h : nullptr;
            s.megno = megno ? megno->h : nullptr;
            s.megno_birkhoff = megno_b ? megno_b->h : nullptr;
            s.vectors = vectors ? vectors->h : nullptr;
            s.lyapunov = lyap ? lyap->h : nullptr;
            s.tune = tune ? tune->h : nullptr;
            py::array_t<double> snap = array2(samples.size(), p.n_total());
            if (!samples.empty()) {
                std::fill(snap.mutable_data(), snap.mutable_data() + snap.size(),
                          std::numeric_limits<double>::quiet_NaN());
                s.megno_sample_turns = samples.data();
                s.n_megno_samples = samples.size();
                s.megno_samples_out = snap.mutable_data();
            }
            hm_status st;
            {
                py::gil_scoped_release nogil;
                st = hm_track_indicators(t.h, p.h, n_turns, mu, barrier, &s);
            }
            check(st);
            return snap;
        }, "Fused tracking + tangent map + indicators (the per-turn construct loop)",
           py::arg("particles"), py::arg("n_turns"), py::arg("mu"), py::arg("barrier") = 100.0,
           py::arg("matrix") = nullptr, py::arg("matrix_old") = nullptr,
           py::arg("megno") = nullptr, py::arg("megno_birkhoff") = nullptr,
           py::arg("vectors") = nullptr, py::arg("lyapunov") = nullptr,
           py::arg("tune") = nullptr, py::arg("megno_sample_turns") = std::vector<uint64_t>());

    // ---- matrix_4d_vector_gpu / vector_4d_gpu ------------------------------------
    py::class_<Matrices>(m, "matrix_4d_vector_gpu")
        .def(py::init<size_t>())
        .def("reset", [](Matrices &M) { check(hm_matrices_reset(M.h)); })
        .def("structured_multiply", [](Matrices &M, const Tracker &t, const Particles &p,
                                       double mu) {
            check(hm_matrices_structured_multiply(M.h, t.h, p.h, mu));
        }, py::arg("tracker"), py::arg("particles"), py::arg("mu"))
        .def("set_with_tracker", [](Matrices &M, const Tracker &t, const Particles &p, double mu) {
            check(hm_matrices_set_with_tracker(M.h, t.h, p.h, mu));
        }, py::arg("tracker"), py::arg("particles"), py::arg("mu"))
        .def("explicit_copy", [](Matrices &M, const Matrices &o) { check(hm_matrices_copy(M.h, o.h)); },
             py::arg("other"))
        .def("get_matrix", [](const Matrices &M) {
            py::array_t<double> out(std::vector<py::ssize_t>{py::ssize_t(M.n), 4, 4});
            check(hm_matrices_get(M.h, out.mutable_data()));
            return out;
        })
        .def("get_vector", [](const Matrices &M,
                              py::array_t<double, py::array::c_style | py::array::forcecast> rv) {
            if (size_t(rv.size()) != 4 * M.n) throw py::value_error("need one 4-vector per matrix");
            auto out = array2(M.n, 4);
            check(hm_matrices_get_vector(M.h, rv.data(), out.mutable_data()));
            return out;
        }, py::arg("vector"));

    py::class_<Vectors>(m, "vector_4d_gpu")
        .def(py::init<const std::vector<std::vector<double>> &>())
        .def("set_vectors", [](Vectors &v, py::array_t<double, py::array::c_style |
                                                                 py::array::forcecast> a) {
            if (a.size() == 4 && a.ndim() == 1) {
                check(hm_vectors_set(v.h, a.data(), 1));
            } else {
                if (size_t(a.size()) != 4 * v.n) throw py::value_error("need n x 4 vectors");
                check(hm_vectors_set(v.h, a.data(), 0));
            }
        }, py::arg("vectors"))
        .def("multiply", [](Vectors &v, const Matrices &M) { check(hm_vectors_multiply(v.h, M.h)); },
             py::arg("matrix"))
        .def("normalize", [](Vectors &v) { check(hm_vectors_normalize(v.h)); })
        .def("get_vectors", [](const Vectors &v) {
            auto out = array2(v.n, 4);
            check(hm_vectors_get(v.h, out.mutable_data()));
            return out;
        });

    // ---- constructs ----------------------------------------------------------------
    py::class_<Lyapunov>(m, "lyapunov_birkhoff_construct")
        .def(py::init([](size_t n, uint64_t w) { return new Lyapunov(n, {w}); }))
        .def("reset", [](Lyapunov &l) { check(hm_lyapunov_reset(l.h)); })
        .def("change_weights", [](Lyapunov &l, uint64_t w) {
            check(hm_lyapunov_change_weights(l.h, w));
            l.lengths = {w};
        }, py::arg("n_weights"))
        .def("add", [](Lyapunov &l, const Vectors &v) { check(hm_lyapunov_add(l.h, v.h)); },
             py::arg("vectors"))
        .def("get_weights", [](const Lyapunov &l) { return l.weights(0); })
        .def("get_values_raw", [](const Lyapunov &l) {
            auto a = l.values(0);
            return py::array_t<double>(std::vector<py::ssize_t>{py::ssize_t(l.n)}, a.data());
        })
        .def("get_values_b", [](const Lyapunov &l) {
            auto a = l.values(1);
            return py::array_t<double>(std::vector<py::ssize_t>{py::ssize_t(l.n)}, a.data());
        });

    py::class_<LyapunovMulti, Lyapunov>(m, "lyapunov_birkhoff_construct_multi")
        .def(py::init([](size_t n, std::vector<uint64_t> w) { return new LyapunovMulti(n, w); }))
        .def("get_weights", [](const LyapunovMulti &l) {
            std::vector<py::array_t<double>> out;
            for (size_t w = 0; w < l.lengths.size(); ++w) out.push_back(l.weights(w));
            return out;
        })
        .def("get_values_raw", [](const LyapunovMulti &l) { return l.values(0); })
        .def("get_values_b", [](const LyapunovMulti &l) { return l.values(1); });

    py::class_<Megno>(m, "megno_construct")
        .def(py::init<size_t>())
        .def("reset", [](Megno &g) { check(hm_megno_reset(g.h)); })
        .def("add", [](Megno &g, const Matrices &a, const Matrices &b) {
            check(hm_megno_add(g.h, a.h, b.h));
        }, py::arg("matrix_a"), py::arg("matrix_b"))
        .def("get_values", [](const Megno &g) {
            auto out = array1<double>(g.n);
            check(hm_megno_get(g.h, out.mutable_data()));
            return out;
        });

    py::class_<MegnoBirkhoff>(m, "megno_birkhoff_construct")
        .def(py::init<size_t, std::vector<uint64_t>>())
        .def("reset", [](MegnoBirkhoff &g) { check(hm_megno_birkhoff_reset(g.h)); })
        .def("add", [](MegnoBirkhoff &g, const Matrices &a, const Matrices &b) {
            check(hm_megno_birkhoff_add(g.h, a.h, b.h));
        }, py::arg("matrix_a"), py::arg("matrix_b"))
        .def("get_values", [](const MegnoBirkhoff &g) {
            auto out = array2(g.T.size(), g.n);
            check(hm_megno_birkhoff_get(g.h, out.mutable_data()));
            return out;
        });

    py::class_<TuneBirkhoff>(m, "tune_birkhoff_construct")
        .def(py::init<size_t, std::vector<uint64_t>>())
        .def("reset", [](TuneBirkhoff &t) { check(hm_tune_birkhoff_reset(t.h)); })
        .def("first_add", [](TuneBirkhoff &t, const Particles &p) {
            check(hm_tune_birkhoff_first_add(t.h, p.h));
        }, py::arg("particles"))
        .def("add", [](TuneBirkhoff &t, const Particles &p) { check(hm_tune_birkhoff_add(t.h, p.h)); },
             py::arg("particles"))
        .def("get_tune1_x", [](const TuneBirkhoff &t) { return t.get(0); })
        .def("get_tune1_y", [](const TuneBirkhoff &t) { return t.get(1); })
        .def("get_tune2_x", [](const TuneBirkhoff &t) { return t.get(2); })
        .def("get_tune2_y", [](const TuneBirkhoff &t) { return t.get(3); });

    py::class_<Storage>(m, "storage_4d_gpu")
        .def(py::init<size_t, size_t>())
        .def("store", [](Storage &s, const Particles &p) { check(hm_storage_store(s.h, p.h)); },
             py::arg("particles"))
        .def("reset", [](Storage &s) { check(hm_storage_reset(s.h)); })
        .def("get_x", [](const Storage &s) { return s.get(HM_FIELD_X); })
        .def("get_px", [](const Storage &s) { return s.get(HM_FIELD_PX); })
        .def("get_y", [](const Storage &s) { return s.get(HM_FIELD_Y); })
        .def("get_py", [](const Storage &s) { return s.get(HM_FIELD_PY); })
        .def("tune_birkhoff", [](const Storage &s, std::vector<uint32_t> from, std::vector<uint32_t> to) {
            if (from.size() != to.size())
                throw std::runtime_error("compute_tune: from and to must be of the same size");
            auto out = array2(s.n, 2 * (from.size() + 1));
            check(hm_storage_tunes(s.h, from.data(), to.data(), from.size(), 0, out.mutable_data()));
            return out;
        }, py::arg("from_idx"), py::arg("to_idx"))
        .def("tune_fft", [](const Storage &s, std::vector<uint32_t> from, std::vector<uint32_t> to) {
            if (from.size() != to.size())
                throw std::runtime_error("compute_tune: from and to must be of the same size");
            auto out = array2(s.n, 2 * (from.size() + 1));
            check(hm_storage_tunes(s.h, from.data(), to.data(), from.size(), 1, out.mutable_data()));
            return out;
        }, py::arg("from_idx"), py::arg("to_idx"));
}
