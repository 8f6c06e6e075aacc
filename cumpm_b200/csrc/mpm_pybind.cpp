// Python module `_cuMPM`: the reference module's classes (Dipole_Solver,
// Near_Field, PrecisionMode, FieldCalcMode; dipole_solver_bindings.cpp:68-178,
// near_field_bindings.cpp:8-25, electric_field_bindings.cpp:14-25) bound on
// top of the C ABI in include/cumpm_b200.h.  Status codes map to ValueError
// (invalid argument) or RuntimeError.
#include <pybind11/complex.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <array>
#include <complex>
#include <string>
#include <vector>

#include "../../include/cumpm_b200.h"

namespace py = pybind11;
using cd = std::complex<double>;

namespace {

enum class PrecisionMode { AUTO = MPM_PREC_AUTO, MIXED = MPM_PREC_MIXED, DOUBLE = MPM_PREC_DOUBLE };
enum class FieldCalcMode { SOLVER_AX = MPM_MODE_SOLVER_AX, INTERACTION_FIELD = MPM_MODE_INTERACTION };

void check(int st) {
    if (st == MPM_OK) return;
    const std::string msg = mpm_last_error();
    if (st == MPM_ERR_INVALID) throw py::value_error(msg);
    throw std::runtime_error(msg);
}

class PyDipoleSolver {
public:
    PyDipoleSolver(const std::vector<double>& box, const std::vector<std::vector<cd>>& eps, const std::vector<double>& radius,
                   double eps_m, double xi, double tol, bool quiet, const std::string& guess_type,
                   const std::string& solver_type, const std::string& field_type,
                   const std::vector<std::vector<cd>>& E0, bool solve_quads, const std::vector<int>& quad_idxs,
                   PrecisionMode precision) {
        if (box.size() < 3) throw py::value_error("box must have length 3");
        const int W = int(eps.size());
        if (W == 0) throw std::runtime_error("eps_p is empty.");
        const int cols = int(eps[0].size());
        for (const auto& row : eps)
            if (int(row.size()) != cols) throw py::value_error("eps_p rows must have equal length");
        std::vector<cd> flat;
        for (const auto& row : eps) flat.insert(flat.end(), row.begin(), row.end());
        std::vector<int> sizes;
        std::vector<cd> e0;
        for (const auto& v : E0) {
            sizes.push_back(int(v.size()));
            e0.insert(e0.end(), v.begin(), v.end());
        }
        check(mpm_solver_create(&s_, box.data(), reinterpret_cast<const double*>(flat.data()), W, cols,
                                radius.empty() ? nullptr : radius.data(), int(radius.size()), eps_m, xi, tol,
                                quiet, guess_type.c_str(), solver_type.c_str(), field_type.c_str(),
                                e0.empty() ? nullptr : reinterpret_cast<const double*>(e0.data()),
                                sizes.empty() ? nullptr : sizes.data(), int(sizes.size()), solve_quads,
                                quad_idxs.empty() ? nullptr : quad_idxs.data(), int(quad_idxs.size()),
                                int(precision)));
    }
    ~PyDipoleSolver() { mpm_solver_destroy(s_); }

    // coordinates as float64 arrays (lists and other sequences are converted)
    using darr = py::array_t<double, py::array::c_style | py::array::forcecast>;
    void compute(const darr& x, const darr& y, const darr& z) {
        if (x.ndim() != 1 || y.ndim() != 1 || z.ndim() != 1 || x.size() != y.size() || x.size() != z.size())
            throw py::value_error("Input coordinate vectors must have the exact same size.");
        const double *px = x.data(), *py_ = y.data(), *pz = z.data();
        const int n = int(x.size());
        int st;
        {
            py::gil_scoped_release nogil;
            st = mpm_solver_compute(s_, px, py_, pz, n);
        }
        check(st);
    }
    std::array<int64_t, 5> dims() const {
        std::array<int64_t, 5> d{};
        check(mpm_solver_dims(s_, d.data()));
        return d;
    }
    py::array_t<cd> eff(bool physical) const {
        auto d = dims();
        py::array_t<cd> a({d[1], d[3], int64_t(3)});
        check(mpm_solver_get_eff_polarizability(s_, physical, reinterpret_cast<double*>(a.mutable_data()), a.size()));
        return a;
    }
    py::array_t<cd> dipoles(bool physical) const {
        auto d = dims();
        py::array_t<cd> a({d[0], d[1], d[2], d[3], int64_t(3)});
        check(mpm_solver_get_dipoles(s_, physical, reinterpret_cast<double*>(a.mutable_data()), a.size()));
        return a;
    }
    py::array_t<cd> quadrupoles(bool physical) const {
        auto d = dims();
        py::array_t<cd> a({d[0], d[1], d[4], d[3], int64_t(5)});
        check(mpm_solver_get_quadrupoles(s_, physical, reinterpret_cast<double*>(a.mutable_data()), a.size()));
        return a;
    }
    bool jacobi() const {
        int e = 0;
        check(mpm_solver_get_jacobi(s_, &e));
        return e != 0;
    }
    void set_jacobi(bool on) { check(mpm_solver_set_jacobi(s_, on)); }
    void set_options(int restart, int maxiter, bool batch_all, bool refine, double inner_tol, bool real_fp32) {
        check(mpm_solver_set_options(s_, restart, maxiter, batch_all, refine, inner_tol, real_fp32));
    }
    py::dict autotune(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z) {
        if (x.size() != y.size() || x.size() != z.size())
            throw py::value_error("Input coordinate vectors must have the exact same size.");
        mpm_field_tuning t{};
        mpm_tune_report r{};
        int st;
        {
            py::gil_scoped_release nogil;
            st = mpm_solver_autotune(s_, x.data(), y.data(), z.data(), int(x.size()), &t, &r);
        }
        check(st);
        py::dict d;
        d["xi"] = t.xi;
        d["grid"] = py::make_tuple(t.grid[0], t.grid[1], t.grid[2]);
        d["support"] = t.support;
        d["tile"] = py::make_tuple(t.tile[0], t.tile[1]);
        d["apply_ms"] = r.apply_ms;
        d["apply_ms_rule"] = r.apply_ms_rule;
        d["error"] = r.error;
        d["error_rule"] = r.error_rule;
        d["error_bound"] = r.error_bound;
        d["candidates"] = r.candidates;
        d["accepted"] = r.accepted;
        return d;
    }
    void set_tuning(double xi, const std::array<int, 3>& grid, int support, const std::array<int, 2>& tile) {
        mpm_field_tuning t{};
        t.xi = xi;
        for (int d = 0; d < 3; ++d) t.grid[d] = grid[d];
        t.support = support;
        t.tile[0] = tile[0];
        t.tile[1] = tile[1];
        check(mpm_solver_set_tuning(s_, &t));
    }
    std::vector<int> iterations() const {
        size_t n = 0;
        check(mpm_solver_iterations(s_, nullptr, 0, &n));
        std::vector<int> v(n);
        check(mpm_solver_iterations(s_, v.data(), n, &n));
        return v;
    }

private:
    mpm_solver* s_ = nullptr;
};

class PyNearField {
public:
    PyNearField(const std::vector<double>& box, const std::vector<cd>& E0, const std::vector<double>& radius, double xi,
                double errortol, const std::string& field_type) {
        if (box.size() != 3) throw py::value_error("Near_Field box must have length 3.");
        if (E0.size() != 3) throw py::value_error("Near_Field E0 must have length 3.");
        check(mpm_near_create(&n_, box.data(), reinterpret_cast<const double*>(E0.data()),
                              radius.empty() ? nullptr : radius.data(), int(radius.size()), xi, errortol,
                              field_type.c_str()));
    }
    ~PyNearField() { mpm_near_destroy(n_); }
    void set_dipoles(const std::vector<cd>& dip) {
        check(mpm_near_set_dipoles(n_, reinterpret_cast<const double*>(dip.data()), int(dip.size())));
    }
    void set_dipole_positions(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z) {
        if (x.size() != y.size() || x.size() != z.size())
            throw py::value_error("Dipole coordinates x, y, z must have the same size.");
        check(mpm_near_set_dipole_positions(n_, x.data(), y.data(), z.data(), int(x.size())));
        npos_ = x.size();
    }
    void set_field_points(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z) {
        if (x.size() != y.size() || x.size() != z.size())
            throw py::value_error("Field point coordinates x, y, z must have the same size.");
        check(mpm_near_set_field_points(n_, x.data(), y.data(), z.data(), int(x.size())));
        nfp_ = x.size();
    }
    std::vector<double> calculate() {
        std::vector<double> out(nfp_);
        int st;
        {
            py::gil_scoped_release nogil;
            st = mpm_near_calculate(n_, out.data(), int(out.size()));
        }
        check(st);
        return out;
    }

private:
    mpm_near* n_ = nullptr;
    size_t npos_ = 0, nfp_ = 0;
};

}  // namespace

PYBIND11_MODULE(_cuMPM, m) {
    m.doc() = "B200-native Mutual Polarization Method solve (cumpm_b200)";
    py::enum_<PrecisionMode>(m, "PrecisionMode")
        .value("AUTO", PrecisionMode::AUTO)
        .value("MIXED", PrecisionMode::MIXED)
        .value("DOUBLE", PrecisionMode::DOUBLE)
        .value("FP32", PrecisionMode::MIXED)
        .value("FP64", PrecisionMode::DOUBLE);
    py::enum_<FieldCalcMode>(m, "FieldCalcMode")
        .value("SOLVER_AX", FieldCalcMode::SOLVER_AX)
        .value("INTERACTION_FIELD", FieldCalcMode::INTERACTION_FIELD);

    using VV = std::vector<std::vector<cd>>;
    auto cls = py::class_<PyDipoleSolver>(m, "Dipole_Solver");
    cls.def(py::init<const std::vector<double>&, const VV&, const std::vector<double>&, double, double, double, bool,
                     const std::string&, const std::string&, const std::string&, const VV&, bool,
                     const std::vector<int>&, PrecisionMode>(),
            py::arg("box"), py::arg("eps_p"), py::arg("radius") = std::vector<double>{}, py::arg("eps_m") = 1.0,
            py::arg("xi") = 0.5, py::arg("tol") = 1e-3, py::arg("quiet") = false, py::arg("guess_type") = "derivative",
            py::arg("solver_type") = "gmres", py::arg("field_type") = "auto", py::arg("E0") = VV{},
            py::arg("solve_quadrupoles") = false, py::arg("quad_idxs") = std::vector<int>{},
            py::arg("precision") = PrecisionMode::AUTO);
    cls.def(py::init([](const std::vector<double>& box, const std::vector<cd>& eps1, const std::vector<double>& radius,
                        double eps_m, double xi, double tol, bool quiet, const std::string& gt, const std::string& st,
                        const std::string& ft, const VV& E0, bool sq, const std::vector<int>& qi, PrecisionMode p) {
                VV e(eps1.size());
                for (size_t w = 0; w < eps1.size(); ++w) e[w] = {eps1[w]};
                return new PyDipoleSolver(box, e, radius, eps_m, xi, tol, quiet, gt, st, ft, E0, sq, qi, p);
            }),
            py::arg("box"), py::arg("eps_p_1d"), py::arg("radius") = std::vector<double>{}, py::arg("eps_m") = 1.0,
            py::arg("xi") = 0.5, py::arg("tol") = 1e-3, py::arg("quiet") = false, py::arg("guess_type") = "derivative",
            py::arg("solver_type") = "gmres", py::arg("field_type") = "auto", py::arg("E0") = VV{},
            py::arg("solve_quadrupoles") = false, py::arg("quad_idxs") = std::vector<int>{},
            py::arg("precision") = PrecisionMode::AUTO);
    cls.def(py::init([](const std::vector<double>& box, cd eps, const std::vector<double>& radius, double eps_m,
                        double xi, double tol, bool quiet, const std::string& gt, const std::string& st,
                        const std::string& ft, const VV& E0, bool sq, const std::vector<int>& qi, PrecisionMode p) {
                return new PyDipoleSolver(box, VV{{eps}}, radius, eps_m, xi, tol, quiet, gt, st, ft, E0, sq, qi, p);
            }),
            py::arg("box"), py::arg("eps_p_scalar"), py::arg("radius") = std::vector<double>{}, py::arg("eps_m") = 1.0,
            py::arg("xi") = 0.5, py::arg("tol") = 1e-3, py::arg("quiet") = false, py::arg("guess_type") = "derivative",
            py::arg("solver_type") = "gmres", py::arg("field_type") = "auto", py::arg("E0") = VV{},
            py::arg("solve_quadrupoles") = false, py::arg("quad_idxs") = std::vector<int>{},
            py::arg("precision") = PrecisionMode::AUTO);
    cls.def("compute", &PyDipoleSolver::compute, py::arg("x_part"), py::arg("y_part"), py::arg("z_part"))
        .def("get_eff_polarizability", &PyDipoleSolver::eff, py::arg("physical") = true)
        .def("get_dipoles", &PyDipoleSolver::dipoles, py::arg("physical") = true)
        .def("get_quadrupoles", &PyDipoleSolver::quadrupoles, py::arg("physical") = true)
        .def("get_num_frames", [](const PyDipoleSolver& s) { return s.dims()[0]; })
        .def("get_num_particles", [](const PyDipoleSolver& s) { return s.dims()[2]; })
        .def("get_num_quads", [](const PyDipoleSolver& s) { return s.dims()[4]; })
        .def("get_num_wavevectors", [](const PyDipoleSolver& s) { return s.dims()[1]; })
        .def("get_num_incident_polarizations", [](const PyDipoleSolver& s) { return s.dims()[3]; })
        .def("isUsingJacobiPrecond", &PyDipoleSolver::jacobi)
        .def("setUseJacobiPrecond", &PyDipoleSolver::set_jacobi)
        .def("set_solver_options", &PyDipoleSolver::set_options, py::arg("restart") = 50, py::arg("maxiter") = 1000,
             py::arg("batch_all") = false, py::arg("refine") = false, py::arg("inner_tol") = 1e-4,
             py::arg("real_fp32") = false)
        .def("get_iterations", &PyDipoleSolver::iterations)
        .def("autotune", &PyDipoleSolver::autotune)
        .def("set_tuning", &PyDipoleSolver::set_tuning, py::arg("xi"), py::arg("grid") = std::array<int, 3>{0, 0, 0},
             py::arg("support") = 0, py::arg("tile") = std::array<int, 2>{0, 0});

    py::class_<PyNearField>(m, "Near_Field")
        .def(py::init<const std::vector<double>&, const std::vector<cd>&, const std::vector<double>&, double, double,
                      const std::string&>(),
             py::arg("box"), py::arg("E0"), py::arg("radius") = std::vector<double>{}, py::arg("xi") = 0.5,
             py::arg("errortol") = 1e-3, py::arg("field_type") = "auto")
        .def("set_dipoles", &PyNearField::set_dipoles, py::arg("dip"))
        .def("set_dipole_positions", &PyNearField::set_dipole_positions, py::arg("x"), py::arg("y"), py::arg("z"))
        .def("set_field_points", &PyNearField::set_field_points, py::arg("x"), py::arg("y"), py::arg("z"))
        .def("calculate", &PyNearField::calculate);
}
