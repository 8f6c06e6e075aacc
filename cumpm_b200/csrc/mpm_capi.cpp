// extern "C" entry points (include/cumpm_b200.h).  Exceptions never cross
// the boundary: each call maps them to a status code and a thread-local
// message.
#include "../../include/cumpm_b200.h"

#include <complex>
#include <cmath>
#include <cstring>
#include <string>

#include "mpm_field.h"
#include "mpm_fft.h"
#include "mpm_krylov.h"
#include "mpm_solver.h"
#include "mpm_tune.h"

#include "mpm_capi_internal.h"
#include "mpm_poly.cuh"

struct mpm_solver { mpm::DipoleSolver* impl; };
struct mpm_near { mpm::NearField* impl; };

namespace {

thread_local std::string g_last_error;

template <typename F>
int guard(F&& f) {
    try {
        f();
        return MPM_OK;
    } catch (const std::invalid_argument& e) {
        g_last_error = e.what();
        return MPM_ERR_INVALID;
    } catch (const mpm::CudaError& e) {
        g_last_error = e.what();
        return MPM_ERR_CUDA;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return MPM_ERR_RUNTIME;
    } catch (...) {
        g_last_error = "unknown error";
        return MPM_ERR_RUNTIME;
    }
}

using cd = std::complex<double>;

std::vector<cd> as_complex(const double* p, size_t n) {
    std::vector<cd> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = cd(p[2 * i], p[2 * i + 1]);
    return v;
}

void need(const void* p, const char* what) {
    if (!p) throw std::invalid_argument(std::string(what) + " must not be NULL");
}

void copy_out(const std::vector<cd>& v, double* out, size_t cap) {
    if (cap < v.size()) throw std::invalid_argument("output buffer too small");
    std::memcpy(out, v.data(), v.size() * sizeof(cd));
}

mpm::FieldSpec field_spec(int kind, int mode, const double box[3], double errortol, double xi, const double* radius,
                          int n_radius, int solve_quads, const int* quad_idxs, int n_quad_idxs) {
    mpm::FieldSpec fs;
    if (kind != MPM_FIELD_DIRECT && kind != MPM_FIELD_MONO && kind != MPM_FIELD_POLY)
        throw std::invalid_argument("unknown field kind");
    fs.kind = kind == MPM_FIELD_DIRECT ? mpm::FIELD_DIRECT : kind == MPM_FIELD_POLY ? mpm::FIELD_POLY : mpm::FIELD_MONO;
    if (fs.kind == mpm::FIELD_POLY && (!radius || n_radius < 1))
        throw std::invalid_argument("polydisperse field needs one radius per particle");
    fs.solver_ax = mode == MPM_MODE_SOLVER_AX;
    if (box) for (int d = 0; d < 3; ++d) fs.box[d] = box[d];
    if (fs.kind != mpm::FIELD_DIRECT) need(box, "box");
    fs.errortol = errortol;
    fs.xi = xi;
    if (radius) fs.radius.assign(radius, radius + n_radius);
    fs.quads = solve_quads != 0;
    if (quad_idxs) fs.quad_idxs.assign(quad_idxs, quad_idxs + n_quad_idxs);
    return fs;
}

mpm::FieldTuning from_c(const mpm_field_tuning& t) {
    mpm::FieldTuning r;
    if (!(t.xi > 0)) throw std::invalid_argument("tuning: xi must be > 0");
    r.xi = t.xi;
    for (int d = 0; d < 3; ++d) {
        if (t.grid[d] < 0 || (t.grid[d] > 0 && t.grid[d] < 8)) throw std::invalid_argument("tuning: grid sizes must be 0 or >= 8");
        r.grid[d] = t.grid[d];
    }
    if (t.support < 0) throw std::invalid_argument("tuning: support must be >= 0");
    r.support = t.support;
    for (int d = 0; d < 2; ++d) {
        if (t.tile[d] != 0 && t.tile[d] != 4 && t.tile[d] != 8 && t.tile[d] != 16)
            throw std::invalid_argument("tuning: tile sizes must be 0, 4, 8 or 16");
        r.tile[d] = t.tile[d];
    }
    if (r.tile[0] && r.tile[1] && r.tile[0] * r.tile[1] > 128)
        throw std::invalid_argument("tuning: a spread tile has at most 128 columns");
    return r;
}

void to_c(const mpm::FieldTuning& t, mpm_field_tuning* out) {
    std::memset(out, 0, sizeof(*out));
    out->xi = t.xi;
    for (int d = 0; d < 3; ++d) out->grid[d] = t.grid[d];
    out->support = t.support;
    out->tile[0] = t.tile[0];
    out->tile[1] = t.tile[1];
}

void to_c(const mpm::TuneReport& r, mpm_tune_report* out) {
    std::memset(out, 0, sizeof(*out));
    out->apply_ms = r.apply_ms;
    out->apply_ms_rule = r.apply_ms_rule;
    out->error = r.error;
    out->error_rule = r.error_rule;
    out->error_bound = r.error_bound;
    out->candidates = r.candidates;
    out->accepted = r.accepted;
}


}  // namespace

int mpm::capi_guard(const std::function<void()>& f) { return guard(f); }

extern "C" {

const char* mpm_last_error(void) { return g_last_error.c_str(); }
const char* mpm_version(void) { return "cumpm_b200 0.1"; }

int mpm_solver_create(mpm_solver** out, const double box[3], const double* eps, int n_freq, int eps_cols,
                      const double* radius, int n_radius, double eps_m, double xi, double tol, int quiet,
                      const char* guess_type, const char* solver_type, const char* field_type, const double* E0,
                      const int* E0_sizes, int n_E0, int solve_quads, const int* quad_idxs, int n_quad_idxs,
                      int precision) {
    return guard([&] {
        need(out, "out");
        need(box, "box");
        need(eps, "eps");
        if (n_freq <= 0 || eps_cols <= 0) throw std::invalid_argument("eps_p must have at least one value");
        std::vector<std::vector<cd>> e(n_freq);
        for (int w = 0; w < n_freq; ++w) e[w] = as_complex(eps + 2 * size_t(w) * eps_cols, eps_cols);
        std::vector<double> rad(radius, radius + (radius ? n_radius : 0));
        std::vector<std::vector<cd>> e0(n_E0);
        size_t off = 0;
        for (int k = 0; k < n_E0; ++k) {
            e0[k] = as_complex(E0 + 2 * off, E0_sizes[k]);
            off += E0_sizes[k];
        }
        std::vector<int> qi(quad_idxs, quad_idxs + (quad_idxs ? n_quad_idxs : 0));
        *out = new mpm_solver{new mpm::DipoleSolver(
            std::vector<double>(box, box + 3), std::move(e), std::move(rad), eps_m, xi, tol, quiet != 0,
            guess_type ? guess_type : "derivative", solver_type ? solver_type : "gmres",
            field_type ? field_type : "auto", std::move(e0), solve_quads != 0, std::move(qi), precision)};
    });
}

void mpm_solver_destroy(mpm_solver* s) {
    if (!s) return;
    delete s->impl;
    delete s;
}

int mpm_solver_compute(mpm_solver* s, const double* x, const double* y, const double* z, int n) {
    return guard([&] {
        need(s, "solver");
        if (n < 0) throw std::invalid_argument("negative particle count");
        std::vector<double> a(x, x + n), b(y, y + n), c(z, z + n);
        s->impl->compute(a, b, c);
    });
}

int mpm_solver_dims(const mpm_solver* s, int64_t dims[5]) {
    return guard([&] {
        need(s, "solver");
        dims[0] = int64_t(s->impl->num_frames());
        dims[1] = int64_t(s->impl->num_wavevectors());
        dims[2] = int64_t(s->impl->num_particles());
        dims[3] = int64_t(s->impl->num_polarizations());
        dims[4] = int64_t(s->impl->num_quads());
    });
}

int mpm_solver_get_dipoles(const mpm_solver* s, int physical, double* out, size_t n) {
    return guard([&] {
        need(s, "solver");
        need(out, "out");
        s->impl->get_dipoles_into(physical != 0, reinterpret_cast<cd*>(out), n);
    });
}
int mpm_solver_get_quadrupoles(const mpm_solver* s, int physical, double* out, size_t n) {
    return guard([&] { need(s, "solver"); copy_out(s->impl->get_quadrupoles(physical != 0), out, n); });
}
int mpm_solver_get_eff_polarizability(const mpm_solver* s, int physical, double* out, size_t n) {
    return guard([&] { need(s, "solver"); copy_out(s->impl->get_eff_polarizability(physical != 0), out, n); });
}
int mpm_solver_set_jacobi(mpm_solver* s, int enable) {
    return guard([&] { need(s, "solver"); s->impl->set_jacobi(enable != 0); });
}
int mpm_solver_get_jacobi(const mpm_solver* s, int* enable) {
    return guard([&] { need(s, "solver"); *enable = s->impl->jacobi() ? 1 : 0; });
}
int mpm_solver_set_options(mpm_solver* s, int restart, int maxiter, int batch_all, int refine, double inner_tol,
                           int real_fp32) {
    return guard([&] {
        need(s, "solver");
        if (restart < 1 || maxiter < 1 || !(inner_tol >= 0)) throw std::invalid_argument("invalid solver options");
        auto& o = s->impl->options();
        o.restart = restart;
        o.maxiter = maxiter;
        o.batch_all = batch_all != 0;
        o.refine = refine != 0;
        o.inner_tol = inner_tol;
        o.real_fp32 = real_fp32 != 0;
    });
}
int mpm_solver_set_tuning(mpm_solver* s, const mpm_field_tuning* tuning) {
    return guard([&] {
        need(s, "solver");
        need(tuning, "tuning");
        s->impl->set_tuning(from_c(*tuning));
    });
}
int mpm_solver_autotune(mpm_solver* s, const double* x, const double* y, const double* z, int n,
                        mpm_field_tuning* out, mpm_tune_report* report) {
    return guard([&] {
        need(s, "solver");
        need(x, "x");
        need(y, "y");
        need(z, "z");
        if (n <= 0) throw std::invalid_argument("autotune: empty coordinate set");
        mpm::TuneReport rep;
        const mpm::FieldTuning t = s->impl->autotune(std::vector<double>(x, x + n), std::vector<double>(y, y + n),
                                                     std::vector<double>(z, z + n), &rep);
        if (out) to_c(t, out);
        if (report) to_c(rep, report);
    });
}
int mpm_solver_iterations(const mpm_solver* s, int* out, size_t cap, size_t* n_out) {
    return guard([&] {
        need(s, "solver");
        const auto& v = s->impl->all_iterations();
        if (n_out) *n_out = v.size();
        if (out) std::memcpy(out, v.data(), sizeof(int) * std::min(cap, v.size()));
    });
}

int mpm_near_create(mpm_near** out, const double box[3], const double E0[6], const double* radius, int n_radius,
                    double xi, double errortol, const char* field_type) {
    return guard([&] {
        need(out, "out");
        need(box, "box");
        need(E0, "E0");
        *out = new mpm_near{new mpm::NearField(std::vector<double>(box, box + 3), as_complex(E0, 3),
                                               std::vector<double>(radius, radius + (radius ? n_radius : 0)), xi,
                                               errortol, field_type ? field_type : "auto")};
    });
}
void mpm_near_destroy(mpm_near* nf) {
    if (!nf) return;
    delete nf->impl;
    delete nf;
}
int mpm_near_set_dipoles(mpm_near* nf, const double* dip, int n) {
    return guard([&] { need(nf, "near field"); nf->impl->set_dipoles(as_complex(dip, n)); });
}
int mpm_near_set_dipole_positions(mpm_near* nf, const double* x, const double* y, const double* z, int n) {
    return guard([&] {
        need(nf, "near field");
        nf->impl->set_dipole_positions({x, x + n}, {y, y + n}, {z, z + n});
    });
}
int mpm_near_set_field_points(mpm_near* nf, const double* x, const double* y, const double* z, int n) {
    return guard([&] {
        need(nf, "near field");
        nf->impl->set_field_points({x, x + n}, {y, y + n}, {z, z + n});
    });
}
int mpm_near_calculate(mpm_near* nf, double* intensity, int n) {
    return guard([&] {
        need(nf, "near field");
        auto v = nf->impl->calculate();
        if (size_t(n) < v.size()) throw std::invalid_argument("output buffer too small");
        std::memcpy(intensity, v.data(), sizeof(double) * v.size());
    });
}


int mpm_field_create(mpm_field** out, int kind, int mode, const double box[3], double errortol, double xi,
                     const double* radius, int n_radius, int solve_quads, const int* quad_idxs, int n_quad_idxs) {
    return guard([&] {
        need(out, "out");
        const mpm::FieldSpec fs =
            field_spec(kind, mode, box, errortol, xi, radius, n_radius, solve_quads, quad_idxs, n_quad_idxs);
        auto* f = new mpm::Field(fs);
        *out = new mpm_field{f, nullptr};
    });
}
int mpm_field_create_tuned(mpm_field** out, int kind, int mode, const double box[3], double errortol,
                           const mpm_field_tuning* tuning, const double* radius, int n_radius, int solve_quads,
                           const int* quad_idxs, int n_quad_idxs) {
    return guard([&] {
        need(out, "out");
        need(tuning, "tuning");
        const mpm::FieldTuning t = from_c(*tuning);
        const mpm::FieldSpec fs = mpm::apply_tuning(
            field_spec(kind, mode, box, errortol, t.xi, radius, n_radius, solve_quads, quad_idxs, n_quad_idxs), t);
        auto* f = new mpm::Field(fs);
        *out = new mpm_field{f, nullptr};
    });
}
int mpm_field_autotune(int kind, const double box[3], double errortol, double xi, const double* radius, int n_radius,
                       int solve_quads, const int* quad_idxs, int n_quad_idxs, const double* x, const double* y,
                       const double* z, int n, int M, int recip_fp32, int real_fp32, mpm_field_tuning* out,
                       mpm_tune_report* report, void* stream) {
    return guard([&] {
        need(out, "out");
        need(x, "x");
        need(y, "y");
        need(z, "z");
        if (!(errortol > 0 && errortol < 1) || !(xi > 0)) throw std::invalid_argument("invalid Ewald parameters");
        const mpm::FieldSpec fs = field_spec(kind, MPM_MODE_SOLVER_AX, box, errortol, xi, radius, n_radius,
                                             solve_quads, quad_idxs, n_quad_idxs);
        mpm::TuneReport rep;
        const mpm::FieldTuning t = mpm::autotune(fs, x, y, z, n, M, recip_fp32 != 0, real_fp32 != 0,
                                                 static_cast<cudaStream_t>(stream), &rep);
        to_c(t, out);
        if (report) to_c(rep, report);
    });
}
int mpm_tune_xi_candidates(int kind, const double box[3], double errortol, double xi, const double* radius,
                           int n_radius, double* xi_out, int* grid_out, int* support_out, double* rc_out, int cap,
                           int* n_out) {
    return guard([&] {
        need(n_out, "n_out");
        if (!(errortol > 0 && errortol < 1) || !(xi > 0)) throw std::invalid_argument("invalid Ewald parameters");
        const mpm::FieldSpec fs =
            field_spec(kind, MPM_MODE_SOLVER_AX, box, errortol, xi, radius, n_radius, 0, nullptr, 0);
        const auto c = mpm::tune_xi_candidates(fs);
        *n_out = int(c.size());
        for (int i = 0; i < int(c.size()) && i < cap; ++i) {
            if (xi_out) xi_out[i] = c[i].xi;
            if (grid_out) for (int d = 0; d < 3; ++d) grid_out[3 * i + d] = c[i].grid[d];
            if (support_out) support_out[i] = c[i].support;
            if (rc_out) rc_out[i] = c[i].rc;
        }
    });
}
int mpm_tune_next_size(int n, int smooth23) {
    if (n < 1 || n > (1 << 24)) return -1;
    return smooth23 ? mpm::tune_next_smooth23(n) : mpm::tune_next_fast(n);
}
void mpm_field_destroy(mpm_field* f) {
    if (!f) return;
    delete f->solver;
    delete f->impl;
    delete f;
}
int mpm_field_set_positions(mpm_field* f, const double* x, const double* y, const double* z, int n, void* stream) {
    return guard([&] {
        need(f, "field");
        if (f->impl->spec().kind == mpm::FIELD_DIRECT && !f->impl->spec().radius.empty() &&
            int(f->impl->spec().radius.size()) != n && f->impl->spec().radius.size() != 1)
            throw std::invalid_argument("Direct field: radius size must match num_particles.");
        f->impl->set_positions(x, y, z, n, static_cast<cudaStream_t>(stream));
    });
}
int mpm_field_set_field_points(mpm_field* f, const double* x, const double* y, const double* z, int n,
                               void* stream) {
    return guard([&] {
        need(f, "field");
        f->impl->set_field_points(x, y, z, n, static_cast<cudaStream_t>(stream));
    });
}
int mpm_field_apply(mpm_field* f, const void* X, void* Y, int M, const void* sc, int jacobi, int recip_fp32,
                    int real_fp32, void* stream) {
    return guard([&] {
        need(f, "field");
        need(X, "X");
        need(Y, "Y");
        if (M < 1) throw std::invalid_argument("M must be >= 1");
        if (jacobi && !sc) throw std::invalid_argument("jacobi scaling needs self coefficients");
        f->impl->apply(static_cast<const double2*>(X), static_cast<double2*>(Y), M, static_cast<const double2*>(sc),
                       jacobi != 0, recip_fp32 != 0, real_fp32 != 0, static_cast<cudaStream_t>(stream));
    });
}
int mpm_field_apply_part(mpm_field* f, const void* X, void* Y, int M, const void* sc, int recip_fp32, int real_fp32,
                         int part, void* stream) {
    return guard([&] {
        need(f, "field");
        need(X, "X");
        need(Y, "Y");
        f->impl->apply_part(static_cast<const double2*>(X), static_cast<double2*>(Y), M,
                            static_cast<const double2*>(sc), recip_fp32 != 0, real_fp32 != 0, part,
                            static_cast<cudaStream_t>(stream));
    });
}
int mpm_field_set_bloch(mpm_field* f, double kx, double ky) {
    return guard([&] {
        need(f, "field");
        if (!std::isfinite(kx) || !std::isfinite(ky)) throw std::invalid_argument("Bloch wavevector must be finite");
        f->impl->set_bloch(kx, ky);
    });
}
int mpm_field_info_get(const mpm_field* f, mpm_field_info* info) {
    return guard([&] {
        need(f, "field");
        need(info, "info");
        const auto& F = *f->impl;
        const auto st = F.stats();
        const auto& g = F.geom();
        std::memset(info, 0, sizeof(*info));
        info->kind = F.spec().kind == mpm::FIELD_DIRECT ? MPM_FIELD_DIRECT
                     : F.spec().kind == mpm::FIELD_POLY ? MPM_FIELD_POLY : MPM_FIELD_MONO;
        info->mode = F.spec().solver_ax ? MPM_MODE_SOLVER_AX : MPM_MODE_INTERACTION;
        info->num_particles = F.num_particles();
        info->num_targets = F.num_targets();
        info->num_quads = F.num_quads();
        for (int d = 0; d < 3; ++d) {
            info->grid[d] = g.ng[d];
            info->h[d] = g.h[d];
            info->eta[d] = g.eta[d];
        }
        info->stencil = F.spec().kind == mpm::FIELD_POLY ? F.poly_geom().P : 2 * g.off + 1;
        if (F.spec().kind == mpm::FIELD_POLY)
            for (int d = 0; d < 3; ++d) info->eta[d] = F.poly_geom().eta;
        info->pruned = st.pruned;
        info->z_slots = st.z_slots;
        info->num_pairs = st.num_pairs;
        info->rc = g.rc;
        info->selfo = F.selfo();
        info->slab_fused = st.slab_fused;
        info->single_layer = st.single_layer;
    });
}

int mpm_batch_solve(mpm_field* f, const void* B, void* X, int M, const void* sc, const mpm_solve_options* opt,
                    mpm_solve_report* rep, void* stream) {
    return guard([&] {
        need(f, "field");
        need(opt, "options");
        need(sc, "self coefficients");
        if (!f->solver) f->solver = new mpm::BatchSolver();
        mpm::SolveOptions o;
        o.method = opt->method == MPM_METHOD_BICGSTAB ? mpm::SOLVER_BICGSTAB : mpm::SOLVER_GMRES;
        o.restart = opt->restart;
        o.maxiter = opt->maxiter;
        o.tol = opt->tol;
        o.jacobi = opt->jacobi != 0;
        o.recip_fp32 = opt->recip_fp32 != 0;
        o.real_fp32 = opt->real_fp32 != 0;
        o.refine = opt->refine != 0;
        o.inner_tol = opt->inner_tol;
        o.compact = opt->compact != 0;
        o.shifted = opt->shifted != 0;
        if (!(o.inner_tol >= 0.0)) throw std::invalid_argument("inner_tol must be >= 0");
        mpm::SolveStats st;
        f->solver->solve(*f->impl, static_cast<const double2*>(B), static_cast<double2*>(X), M,
                         static_cast<const double2*>(sc), o, st, static_cast<cudaStream_t>(stream));
        if (rep) {
            std::memset(rep, 0, sizeof(*rep));
            rep->matvecs = st.matvecs;
            rep->refine_steps = st.refine_steps;
            rep->column_matvecs = st.column_matvecs;
            rep->reorth_steps = st.reorth_steps;
            rep->shift_seeds = st.shift_seeds;
            rep->fp64_matvecs = st.fp64_matvecs;
            for (int m = 0; m < M; ++m) {
                rep->total_iterations += st.iters[m];
                rep->max_iterations = std::max(rep->max_iterations, st.iters[m]);
                rep->num_converged += st.converged[m];
            }
            rep->max_rel_resid = -1.0;
            for (double r : st.rel_resid) rep->max_rel_resid = std::max(rep->max_rel_resid, r);
        }
    });
}

int mpm_mono_tables(double xi, double* out, double* selfo, double* self_grad) {
    return guard([&] {
        need(out, "out");
        if (!(xi > 0)) throw std::invalid_argument("xi must be positive");
        const auto T = mpm::build_mono_tables(xi);
        std::memcpy(out, T.r.data(), sizeof(double) * mpm::kTableSize);
        for (int f = 0; f < mpm::T_COUNT; ++f)
            std::memcpy(out + size_t(f + 1) * mpm::kTableSize, T.f[f].data(), sizeof(double) * mpm::kTableSize);
        if (selfo) *selfo = T.selfo;
        if (self_grad) *self_grad = T.self_grad;
    });
}

int mpm_poly_quad_tables(double xi, double rc, double* out, size_t cap, int* n_nodes) {
    return guard([&] {
        if (!(xi > 0) || !(rc > 0)) throw std::invalid_argument("xi and rc must be positive");
        const double rc_val = rc < 1.001 ? 1.001 : rc;
        const int n = static_cast<int>(std::ceil((rc_val - 1.0) / mpm::kTableDr)) + 1;
        if (n_nodes) *n_nodes = n;
        if (!out) return;
        if (cap < size_t(mpm::PQ_COUNT + 1) * size_t(n))
            throw std::invalid_argument("out holds fewer than 8 x n_nodes doubles");
        const auto T = mpm::build_poly_quad_tables(xi, n);
        std::memcpy(out, T.r.data(), sizeof(double) * n);
        for (int f = 0; f < mpm::PQ_COUNT; ++f)
            std::memcpy(out + size_t(f + 1) * n, T.f[f].data(), sizeof(double) * n);
    });
}

int mpm_poly_quad_self(double xi, const double* radii, int n, double* out) {
    return guard([&] {
        if (!(xi > 0)) throw std::invalid_argument("xi must be positive");
        if (n < 0) throw std::invalid_argument("n must be non-negative");
        if (n == 0) return;
        need(radii, "radii");
        need(out, "out");
        for (int i = 0; i < n; ++i) {
            if (!(radii[i] > 0)) throw std::invalid_argument("radii must be positive");
            out[i] = mpm::poly_quad_self_value(radii[i], xi);
        }
    });
}

int mpm_ewald_geometry(const double box[3], double errortol, double xi, int grid[3], int* stencil, double* rc,
                       double h[3], double eta[3]) {
    return guard([&] {
        need(box, "box");
        if (!(errortol > 0 && errortol < 1) || !(xi > 0)) throw std::invalid_argument("invalid Ewald parameters");
        const auto g = mpm::make_ewald_geom(box, errortol, xi);
        for (int d = 0; d < 3; ++d) {
            if (grid) grid[d] = g.ng[d];
            if (h) h[d] = g.h[d];
            if (eta) eta[d] = g.eta[d];
        }
        if (stencil) *stencil = 2 * g.off + 1;
        if (rc) *rc = g.rc;
    });
}

int mpm_field_grad(mpm_field* f, const void* lam, const void* p, int M, void* gx, void* ga, void* stream) {
    return guard([&] {
        need(f, "field");
        need(lam, "lam");
        need(p, "p");
        need(gx, "gx");
        need(ga, "ga");
        f->impl->grad_bilinear(static_cast<const double2*>(lam), static_cast<const double2*>(p), M,
                               static_cast<double2*>(gx), static_cast<double2*>(ga),
                               static_cast<cudaStream_t>(stream));
    });
}

int mpm_line_fft(void* data, int fp64, int n, size_t es, int ncols, size_t os, int nouter, int mode,
                 const void* scale, int sz, int sb, int general, int* split, void* stream) {
    return guard([&] {
        need(data, "data");
        if (n < 1 || ncols < 1 || nouter < 1) throw std::invalid_argument("empty line transform");
        if (mode < 0 || mode > 2) throw std::invalid_argument("mode must be 0 (forward), 1 (inverse) or 2 (scaled)");
        if (mode == 2 && (!scale || sz < 1 || sb < 1)) throw std::invalid_argument("mode 2 needs scale, sz, sb");
        if (!mpm::AxisFFT::fits(n, true)) throw std::invalid_argument("line too long for the in-house transform");
        mpm::AxisFFT fft;
        fft.init(n);
        fft.set_force_general(general != 0);
        if (split) {
            const bool two = fft.path(ncols, mode) != 0;
            split[0] = two ? fft.split_r1() : 0;
            split[1] = two ? fft.split_r2() : 0;
        }
        const auto st = static_cast<cudaStream_t>(stream);
        if (fp64) {
            auto* d = static_cast<double2*>(data);
            if (mode == 2) fft.run_scaled<double>(d, es, ncols, os, nouter, static_cast<const double*>(scale), sz, sb, st);
            else fft.run<double>(d, es, ncols, os, nouter, mode == 1, st);
        } else {
            auto* d = static_cast<float2*>(data);
            if (mode == 2) fft.run_scaled<float>(d, es, ncols, os, nouter, static_cast<const float*>(scale), sz, sb, st);
            else fft.run<float>(d, es, ncols, os, nouter, mode == 1, st);
        }
        MPM_CUDA(cudaStreamSynchronize(st));
    });
}

int mpm_poly_geometry(const double box[3], double errortol, double xi, const double* radii, int n, int grid[3],
                      int* P, double* eta, double* rc, int* n_classes, int* cls) {
    return guard([&] {
        need(box, "box");
        need(radii, "radii");
        if (n < 1) throw std::invalid_argument("need at least one radius");
        if (!(errortol > 0 && errortol < 1) || !(xi > 0)) throw std::invalid_argument("invalid Ewald parameters");
        const auto g = mpm::make_poly_geom(box, errortol, xi, std::vector<double>(radii, radii + n));
        for (int d = 0; d < 3; ++d)
            if (grid) grid[d] = g.ng[d];
        if (P) *P = g.P;
        if (eta) *eta = g.eta;
        if (rc) *rc = g.rc;
        if (n_classes) *n_classes = int(g.unique.size());
        if (cls) std::copy(g.cls.begin(), g.cls.end(), cls);
    });
}

int mpm_poly_pair_functions(double a, double b, double xi, double rc, int lookup, const double* r, int n, double* fd1,
                            double* fd2, double* self_value) {
    return guard([&] {
        if (!(a > 0 && b >= a) || !(xi > 0)) throw std::invalid_argument("need 0 < a <= b and xi > 0");
        if (n > 0) {
            need(r, "r");
            need(fd1, "fd1");
            need(fd2, "fd2");
        }
        const double rc_val = rc < 1.001 ? 1.001 : rc;
        const int table_n = static_cast<int>(std::ceil((rc_val - 1.0) / 0.001)) + 1;
        for (int k = 0; k < n; ++k) {
            if (lookup) mpm::poly::table_lookup(r[k], a, b, xi, table_n, fd1[k], fd2[k]);
            else mpm::poly::pair_functions(r[k], a, b, xi, fd1[k], fd2[k]);
        }
        if (self_value) *self_value = mpm::poly::self_value(a, b, xi);
    });
}

}  // extern "C"

// ---- measurement hooks ----------------------------------------------------
#include "mpm_profile.h"

extern "C" {

int mpm_profile_enable(int on) {
    return guard([&] { mpm::Profiler::get().enable(on != 0); });
}
int mpm_profile_reset(void) {
    return guard([&] { mpm::Profiler::get().reset(); });
}
int mpm_profile_read(double* ms, long long* count, int n) {
    return guard([&] { mpm::Profiler::get().read(ms, count, n); });
}
long long mpm_kernel_launches(void) { return mpm::Profiler::get().launches(); }

}  // extern "C"
