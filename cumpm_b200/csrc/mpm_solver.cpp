// Host driver (see mpm_solver.h).  Reference semantics cited per function.
#include "mpm_solver.h"

#include <algorithm>
#include <cmath>
#include <iostream>
#include <stdexcept>

namespace mpm {

namespace {
constexpr double PI = 3.14159265358979323846;

bool all_equal(const std::vector<double>& r) {
    for (size_t i = 1; i < r.size(); ++i)
        if (r[i] != r[0]) return false;
    return true;
}
}  // namespace

// dipole_solver.cu:36-119 (three constructors collapse to one: eps_p is
// always [W][1 or N]; an empty E0 means the three unit polarisations)
DipoleSolver::DipoleSolver(std::vector<double> box, std::vector<std::vector<cdouble>> eps_p,
                           std::vector<double> radius, double eps_m, double xi, double tol, bool quiet,
                           std::string guess_type, std::string solver_type, std::string field_type,
                           std::vector<std::vector<cdouble>> E0, bool solve_quadrupoles, std::vector<int> quad_idxs,
                           int precision)
    : box_(std::move(box)), eps_p_(std::move(eps_p)), radius_(std::move(radius)), eps_m_(eps_m), xi_(xi), tol_(tol),
      quiet_(quiet), guess_type_(std::move(guess_type)), solver_type_(std::move(solver_type)),
      field_type_(std::move(field_type)), E0_(std::move(E0)), solve_quads_(solve_quadrupoles),
      quad_idxs_(std::move(quad_idxs)), precision_(precision) {
    if (E0_.empty()) E0_ = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
}

DipoleSolver::~DipoleSolver() {
    field_.reset();
    solver_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

void DipoleSolver::print(const std::string& msg) const {
    if (!quiet_) std::cout << std::string(indent_ * 2, ' ') << msg << std::endl;
}

// dipole_solver.cu:131-182
void DipoleSolver::set_dims(size_t n) {
    N_ = n;
    Nq_ = solve_quads_ ? (quad_idxs_.empty() ? N_ : quad_idxs_.size()) : 0;
    if (radius_.empty()) radius_.assign(N_, 1.0);
    else if (radius_.size() == 1) radius_.assign(N_, radius_[0]);
    else if (radius_.size() != N_)
        throw std::runtime_error("The number of particles is inconsistent with the number of radii provided.");
    if (field_type_ == "monodisperse" && !all_equal(radius_))
        throw std::runtime_error("field_type was set to 'monodisperse' but radii are not identical.");
    if (eps_p_.empty()) throw std::runtime_error("eps_p is empty.");
    for (auto& row : eps_p_) {
        if (row.size() == 1) row.assign(N_, row[0]);
        else if (row.size() != N_) throw std::runtime_error("The number of particles is inconsistent with eps_p provided.");
    }
    const size_t vs = N_ * 3 + Nq_ * 5;
    for (size_t d = 0; d < E0_.size(); ++d) {
        const size_t sz = E0_[d].size();
        if (sz != 3 && sz != N_ * 3 && sz != vs)
            throw std::runtime_error("Incident field E0[" + std::to_string(d) + "] has size " + std::to_string(sz) +
                                     ", but expected 3, " + std::to_string(N_ * 3) + ", or " + std::to_string(vs) + ".");
    }
}

// dipole_solver.cu:184-221
void DipoleSolver::nondimensionalize() {
    length_scale_ = *std::min_element(radius_.begin(), radius_.end());
    eps_scale_ = eps_m_;
    for (int d = 0; d < 3 && d < int(box_.size()); ++d) box_[d] /= length_scale_;
    for (auto& r : radius_) r /= length_scale_;
    eps_m_ /= eps_scale_;
    for (auto& row : eps_p_)
        for (auto& e : row) e /= eps_scale_;
    double s = 0.0;
    for (double r : radius_) s += std::pow(r, 3.0);
    const double V = box_.size() >= 3 ? box_[0] * box_[1] * box_[2] : 0.0;
    vol_frac_ = V == 0.0 ? 0.0 : (4.0 / 3.0) * PI * s / V;
}

// dipole_solver.cu:245-261
std::vector<cdouble> DipoleSolver::mean_field_guess(size_t w) const {
    const size_t K = E0_.size();
    std::vector<cdouble> g(N_ * K * 3 + Nq_ * K * 5, 0.0);
    // complex quotient a / b written out (std::complex division guards
    // against overflow and is several times slower; these values are O(1))
    auto quot = [](cdouble a, cdouble b) {
        const double d = std::norm(b);
        return cdouble((a.real() * b.real() + a.imag() * b.imag()) / d,
                       (a.imag() * b.real() - a.real() * b.imag()) / d);
    };
    for (size_t p = 0; p < N_; ++p) {
        const cdouble e = eps_p_[w][p];
        const cdouble beta = quot(e - 1.0, e + 2.0);
        const double r = radius_[p];
        const cdouble val = quot(4.0 * PI * r * r * r * beta, 1.0 - beta * vol_frac_);
        for (size_t d = 0; d < K; ++d) {
            const std::vector<cdouble>& ed = E0_[d];
            const cdouble* ev = ed.size() > 3 ? ed.data() + p * 3 : ed.data();
            cdouble* gp = g.data() + p * K * 3 + d * 3;
            for (int c = 0; c < 3; ++c) gp[c] = val * ev[c];
        }
    }
    return g;
}

// dipole_solver.cu:233-346 (previous / derivative extrapolation in
// X = (eps + 2)/(eps - 1))
std::vector<cdouble> DipoleSolver::guess(const std::vector<cdouble>& fd, const std::vector<cdouble>& fq,
                                         size_t w) const {
    const std::string& gt = guess_type_;
    const bool mean = gt == "mean_field" || gt == "mean-field";
    if (!mean && gt != "previous" && gt != "derivative")
        throw std::runtime_error("Guess type " + gt + " not supported.");
    if (mean || w < 1) return mean_field_guess(w);
    const size_t K = E0_.size();
    std::vector<cdouble> g(N_ * K * 3 + Nq_ * K * 5);
    if (gt == "previous" || w < 2) {
        std::copy(fd.begin() + (w - 1) * N_ * K * 3, fd.begin() + w * N_ * K * 3, g.begin());
        if (solve_quads_ && Nq_)
            std::copy(fq.begin() + (w - 1) * Nq_ * K * 5, fq.begin() + w * Nq_ * K * 5, g.begin() + N_ * K * 3);
        return g;
    }
    auto X = [](cdouble e) { return (e - 1.0 == 0.0) ? cdouble(0.0) : (e + 2.0) / (e - 1.0); };
    auto extrap = [&](size_t p, size_t width, const std::vector<cdouble>& src, size_t stride, size_t item,
                      size_t dst_off) {
        cdouble run = X(eps_p_[w - 1][p]) - X(eps_p_[w - 2][p]);
        cdouble nr = X(eps_p_[w][p]) - X(eps_p_[w - 1][p]);
        if (std::abs(run) < 1e-12) { run = 1.0; nr = 0.0; }
        for (size_t k = 0; k < width; ++k) {
            const cdouble a1 = src[(w - 1) * stride + item * width + k];
            const cdouble a2 = src[(w - 2) * stride + item * width + k];
            g[dst_off + item * width + k] = a1 + nr * (a1 - a2) / run;
        }
    };
    for (size_t p = 0; p < N_; ++p) extrap(p, K * 3, fd, N_ * K * 3, p, 0);
    if (solve_quads_ && Nq_)
        for (size_t q = 0; q < Nq_; ++q) extrap(quad_idxs_.empty() ? q : quad_idxs_[q], K * 5, fq, Nq_ * K * 5, q, N_ * K * 3);
    return g;
}

namespace {

inline int nblk_s(long long n, int b) { return int((n + b - 1) / b); }

// X[row][m] (row 3p + c, m = f K + k) of the all-frequency batch: frequency
// 0 from init (frame layout [p][k][c]) when given, the others the
// mean-field guess 4 pi a^3 beta / (1 - beta phi) E0_k, beta = (e-1)/(e+2)
// (the same quotients as DipoleSolver::mean_field_guess)
__global__ void k_batch_guess(double2* __restrict__ X, int M, int N, int K, const double2* __restrict__ eps,
                              const double* __restrict__ rad, double phi, const double2* __restrict__ E0,
                              const double2* __restrict__ init) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * 3 * M) return;
    const int m = int(t % M);
    const int row = int(t / M);
    const int p = row / 3, c = row % 3;
    const int f = m / K, k = m % K;
    if (f == 0 && init) {
        X[t] = init[(size_t(p) * K + k) * 3 + c];
        return;
    }
    const double2 e = eps[size_t(f) * N + p];
    auto quot = [](double2 a, double2 b) {
        const double d = b.x * b.x + b.y * b.y;
        return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
    };
    const double2 beta = quot(make_double2(e.x - 1.0, e.y), make_double2(e.x + 2.0, e.y));
    const double r3 = rad[p] * rad[p] * rad[p];
    const double2 num = make_double2(4.0 * kPi * r3 * beta.x, 4.0 * kPi * r3 * beta.y);
    const double2 den = make_double2(1.0 - beta.x * phi, -beta.y * phi);
    const double2 val = quot(num, den);
    const double2 ev = E0[size_t(k) * 3 + c];
    X[t] = make_double2(val.x * ev.x - val.y * ev.y, val.x * ev.y + val.y * ev.x);
}

// frame[f][p][k][c] = X[3p + c][f K + k]
__global__ void k_to_frame(const double2* __restrict__ X, int M, int N, int K, double2* __restrict__ frame) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)N * 3 * M) return;
    const int c = int(t % 3);
    const long long r = t / 3;
    const int k = int(r % K);
    const long long r2 = r / K;
    const int p = int(r2 % N);
    const int f = int(r2 / N);
    frame[t] = X[size_t(3 * p + c) * M + size_t(f) * K + k];
}

}  // namespace

bool DipoleSolver::device_batch_ok() const {
    if (!opt_.batch_all || (solve_quads_ && Nq_)) return false;
    for (const auto& e : E0_)
        if (e.size() != 3) return false;
    return true;
}

// The all-frequency batch with its guesses and results on the device: the
// same solve as solve_batch over every frequency, without the host loops
// over the [row][M] layout.
void DipoleSolver::solve_all_device(const std::vector<cdouble>& init, std::vector<cdouble>& frame_cap,
                                    std::vector<cdouble>& frame_dip) {
    const size_t K = E0_.size(), W = eps_p_.size();
    const size_t rows = N_ * 3;
    const int M = int(W * K);
    std::vector<size_t> freqs(W);
    for (size_t w = 0; w < W; ++w) freqs[w] = w;
    const size_t bytes = sizeof(double2) * rows * M;
    dB_.ensure(bytes);
    dX_.ensure(bytes);
    dSC_.ensure(sizeof(double2) * N_ * M);
    if (freqs != dev_freqs_) {
        // right-hand sides and self terms (dipole_solver.cu:452-460), once
        hB_.ensure(sizeof(cdouble) * rows * M);
        hSC_.ensure(sizeof(cdouble) * N_ * M);
        cdouble* hb = hB_.as<cdouble>();
        cdouble* hsc = hSC_.as<cdouble>();
        for (size_t p = 0; p < N_; ++p) {
            for (size_t f = 0; f < W; ++f) {
                cdouble diff = 1.0 - eps_p_[f][p];
                if (std::abs(diff) < 1e-12) diff = 1e-12;
                const cdouble sv = -3.0 / (4.0 * PI * diff) / std::pow(radius_[p], 3.0);
                for (size_t k = 0; k < K; ++k) hsc[p * M + f * K + k] = sv;
            }
            for (int c = 0; c < 3; ++c)
                for (size_t f = 0; f < W; ++f)
                    for (size_t k = 0; k < K; ++k) hb[(p * 3 + c) * M + f * K + k] = E0_[k][c];
        }
        MPM_CUDA(cudaMemcpyAsync(dB_.p, hb, bytes, cudaMemcpyHostToDevice, stream_));
        MPM_CUDA(cudaMemcpyAsync(dSC_.p, hsc, sizeof(double2) * N_ * M, cudaMemcpyHostToDevice, stream_));
        dev_freqs_ = freqs;
    }
    if (!dev_eps_) {
        std::vector<cdouble> e(W * N_), e0(K * 3);
        for (size_t w = 0; w < W; ++w)
            for (size_t p = 0; p < N_; ++p) e[w * N_ + p] = eps_p_[w][p];
        for (size_t k = 0; k < K; ++k)
            for (int c = 0; c < 3; ++c) e0[k * 3 + c] = E0_[k][c];
        dEps_.ensure(sizeof(double2) * W * N_);
        dRad_.ensure(sizeof(double) * N_);
        dE0_.ensure(sizeof(double2) * K * 3);
        MPM_CUDA(cudaMemcpy(dEps_.p, e.data(), sizeof(double2) * W * N_, cudaMemcpyHostToDevice));
        MPM_CUDA(cudaMemcpy(dRad_.p, radius_.data(), sizeof(double) * N_, cudaMemcpyHostToDevice));
        MPM_CUDA(cudaMemcpy(dE0_.p, e0.data(), sizeof(double2) * K * 3, cudaMemcpyHostToDevice));
        dev_eps_ = true;
    }
    dInit_.ensure(sizeof(double2) * N_ * K * 3);
    hX_.ensure(bytes);   // the init upload now, the frame's dipoles after the solve
    std::copy(init.begin(), init.begin() + N_ * K * 3, hX_.as<cdouble>());
    MPM_CUDA(cudaMemcpyAsync(dInit_.p, hX_.p, sizeof(double2) * N_ * K * 3, cudaMemcpyHostToDevice, stream_));
    const long long n = (long long)rows * M;
    k_batch_guess<<<nblk_s(n, 256), 256, 0, stream_>>>(dX_.as<double2>(), M, int(N_), int(K), dEps_.as<double2>(),
                                                        dRad_.as<double>(), vol_frac_, dE0_.as<double2>(),
                                                        dInit_.as<double2>());
    MPM_LAUNCH();
    SolveOptions so;
    so.method = solver_type_ == "bicgstab" ? SOLVER_BICGSTAB : SOLVER_GMRES;
    so.restart = opt_.restart;
    so.maxiter = opt_.maxiter;
    so.tol = tol_;
    so.jacobi = jacobi_;
    so.recip_fp32 = precision_ != PREC_DOUBLE;
    so.real_fp32 = opt_.real_fp32;
    so.refine = opt_.refine;
    so.inner_tol = opt_.inner_tol;
    solver_->solve(*field_, dB_.as<double2>(), dX_.as<double2>(), M, dSC_.as<double2>(), so, last_stats_, stream_);
    for (int v : last_stats_.iters) iters_.push_back(v);
    dFrame_.ensure(bytes);
    k_to_frame<<<nblk_s(n, 256), 256, 0, stream_>>>(dX_.as<double2>(), M, int(N_), int(K), dFrame_.as<double2>());
    MPM_LAUNCH();
    // into pinned memory at full link speed, then one copy into the frame
    // (frame_dip arrives empty: no zero fill first)
    // (hX_ last held the init upload, earlier on this stream)
    MPM_CUDA(cudaMemcpyAsync(hX_.p, dFrame_.p, bytes, cudaMemcpyDeviceToHost, stream_));
    MPM_CUDA(cudaStreamSynchronize(stream_));
    const cdouble* hf = hX_.as<cdouble>();
    frame_dip.assign(hf, hf + rows * M);
    // particle averages per (frequency, polarisation, component)
    for (size_t f = 0; f < W; ++f) {
        const cdouble* src = frame_dip.data() + f * N_ * K * 3;
        cdouble* cap = frame_cap.data() + f * K * 3;
        for (size_t p = 0; p < N_; ++p)
            for (size_t j = 0; j < K * 3; ++j) cap[j] += src[p * K * 3 + j];
        for (size_t j = 0; j < K * 3; ++j) cap[j] /= double(N_);
    }
}

// One batched device solve for the given frequencies (each with K
// polarisations); results scattered into the frame arrays
// (dipole_solver.cu:361-436 per polarisation, here all at once).
void DipoleSolver::solve_batch(const std::vector<size_t>& freqs, const std::vector<std::vector<cdouble>>& guesses,
                               std::vector<cdouble>& frame_cap, std::vector<cdouble>& frame_dip,
                               std::vector<cdouble>& frame_quad) {
    const size_t K = E0_.size();
    const size_t rows = N_ * 3 + Nq_ * 5;
    const int M = int(freqs.size() * K);
    hB_.ensure(sizeof(cdouble) * rows * M);
    hX_.ensure(sizeof(cdouble) * rows * M);
    hSC_.ensure(sizeof(cdouble) * N_ * M);
    cdouble* hb = hB_.as<cdouble>();
    cdouble* hx = hX_.as<cdouble>();
    cdouble* hsc = hSC_.as<cdouble>();
    const size_t F = freqs.size();
    // the right-hand sides and self terms of a batch depend only on its
    // frequencies: rebuilt (and copied to the device) when those change
    const bool rebuild = freqs != dev_freqs_;
    // rows outermost so that every host array is written contiguously
    // ([row][M] with m = f * K + k)
    for (size_t p = 0; p < N_; ++p) {
        if (rebuild) {
            cdouble* sp = hsc + p * M;
            for (size_t f = 0; f < F; ++f) {
                // self coefficients s = -3 / (4 pi (1 - eps) a^3) (dipole_solver.cu:452-460)
                cdouble diff = 1.0 - eps_p_[freqs[f]][p];
                if (std::abs(diff) < 1e-12) diff = 1e-12;
                const cdouble sv = -3.0 / (4.0 * PI * diff) / std::pow(radius_[p], 3.0);
                for (size_t k = 0; k < K; ++k) sp[f * K + k] = sv;
            }
        }
        for (int c = 0; c < 3; ++c) {
            const size_t row = p * 3 + c;
            cdouble* br = hb + row * M;
            cdouble* xr = hx + row * M;
            for (size_t k = 0; k < K; ++k) {
                const auto& e = E0_[k];
                const cdouble ev = e.size() == 3 ? e[c] : e[row];
                for (size_t f = 0; f < F; ++f) {
                    if (rebuild) br[f * K + k] = ev;
                    xr[f * K + k] = guesses[f][p * K * 3 + k * 3 + c];
                }
            }
        }
    }
    for (size_t q = 0; q < Nq_; ++q)
        for (int c = 0; c < 5; ++c) {
            const size_t row = N_ * 3 + q * 5 + c;
            cdouble* br = hb + row * M;
            cdouble* xr = hx + row * M;
            for (size_t k = 0; k < K; ++k) {
                const auto& e = E0_[k];
                const cdouble ev = (e.size() == rows) ? e[row] : cdouble(0.0);
                for (size_t f = 0; f < F; ++f) {
                    if (rebuild) br[f * K + k] = ev;
                    xr[f * K + k] = guesses[f][N_ * K * 3 + q * K * 5 + k * 5 + c];
                }
            }
        }
    const size_t bytes = sizeof(double2) * rows * M;
    dB_.ensure(bytes);
    dX_.ensure(bytes);
    dSC_.ensure(sizeof(double2) * N_ * M);
    if (rebuild) {
        MPM_CUDA(cudaMemcpyAsync(dB_.p, hb, bytes, cudaMemcpyHostToDevice, stream_));
        MPM_CUDA(cudaMemcpyAsync(dSC_.p, hsc, sizeof(double2) * N_ * M, cudaMemcpyHostToDevice, stream_));
    }
    MPM_CUDA(cudaMemcpyAsync(dX_.p, hx, bytes, cudaMemcpyHostToDevice, stream_));
    SolveOptions so;
    so.method = solver_type_ == "bicgstab" ? SOLVER_BICGSTAB : SOLVER_GMRES;
    so.restart = opt_.restart;
    so.maxiter = opt_.maxiter;
    so.tol = tol_;
    so.jacobi = jacobi_;
    so.recip_fp32 = precision_ != PREC_DOUBLE;
    so.real_fp32 = opt_.real_fp32;
    so.refine = opt_.refine;
    so.inner_tol = opt_.inner_tol;
    solver_->solve(*field_, dB_.as<double2>(), dX_.as<double2>(), M, dSC_.as<double2>(), so, last_stats_, stream_);
    for (int v : last_stats_.iters) iters_.push_back(v);
    MPM_CUDA(cudaMemcpyAsync(hx, dX_.p, bytes, cudaMemcpyDeviceToHost, stream_));
    MPM_CUDA(cudaStreamSynchronize(stream_));
    dev_freqs_ = freqs;
    std::vector<cdouble> avg(size_t(M) * 3, 0.0);
    for (size_t p = 0; p < N_; ++p)
        for (int c = 0; c < 3; ++c) {
            const cdouble* xr = hx + (p * 3 + c) * M;
            for (size_t f = 0; f < F; ++f) {
                cdouble* dst = frame_dip.data() + freqs[f] * N_ * K * 3 + p * K * 3 + c;
                for (size_t k = 0; k < K; ++k) {
                    const cdouble v = xr[f * K + k];
                    dst[k * 3] = v;
                    avg[(f * K + k) * 3 + c] += v;
                }
            }
        }
    for (size_t q = 0; q < Nq_; ++q)
        for (int c = 0; c < 5; ++c) {
            const cdouble* xr = hx + (N_ * 3 + q * 5 + c) * M;
            for (size_t f = 0; f < F; ++f)
                for (size_t k = 0; k < K; ++k)
                    frame_quad[freqs[f] * Nq_ * K * 5 + q * K * 5 + k * 5 + c] = xr[f * K + k];
        }
    for (size_t f = 0; f < F; ++f)
        for (size_t k = 0; k < K; ++k)
            for (int c = 0; c < 3; ++c)
                frame_cap[freqs[f] * K * 3 + k * 3 + c] = avg[(f * K + k) * 3 + c] / double(N_);
}

void DipoleSolver::setup(size_t n) {
    set_dims(n);
    nondimensionalize();
    if (!stream_) MPM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    solver_ = std::make_unique<BatchSolver>();
}

FieldSpec DipoleSolver::field_spec() const {
    FieldSpec fs;
    fs.solver_ax = true;
    fs.quads = solve_quads_;
    fs.quad_idxs = quad_idxs_;
    for (int d = 0; d < 3; ++d) fs.box[d] = box_[d];
    fs.errortol = tol_;
    fs.xi = xi_;
    if (field_type_ == "direct") {
        fs.kind = FIELD_DIRECT;
        fs.radius = radius_;
    } else {
        bool poly;
        if (field_type_ == "polydisperse") poly = true;
        else if (field_type_ == "monodisperse") poly = false;
        else if (field_type_ == "auto") poly = !all_equal(radius_);
        else throw std::runtime_error("Unknown field_type: " + field_type_);
        fs.kind = poly ? FIELD_POLY : FIELD_MONO;
        if (poly) fs.radius = radius_;
    }
    return fs;
}

std::vector<double> DipoleSolver::scaled(const std::vector<double>& v) const {
    std::vector<double> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i] / length_scale_;
    return out;
}

void DipoleSolver::set_tuning(const FieldTuning& t) {
    tuning_ = t;
    tuned_ = true;
    field_.reset();
}

FieldTuning DipoleSolver::autotune(const std::vector<double>& x, const std::vector<double>& y,
                                   const std::vector<double>& z, TuneReport* report) {
    if (x.size() != y.size() || x.size() != z.size())
        throw std::invalid_argument("Input coordinate vectors must have the exact same size.");
    const size_t n = x.size();
    if (n == 0) throw std::invalid_argument("autotune: empty coordinate set");
    if (N_ == 0) setup(n);
    else if (N_ != n) throw std::runtime_error("The number of particles has changed!");
    const int M = int(opt_.batch_all ? eps_p_.size() * E0_.size() : E0_.size());
    const std::vector<double> sx = scaled(x), sy = scaled(y), sz = scaled(z);
    const FieldTuning t = mpm::autotune(field_spec(), sx.data(), sy.data(), sz.data(), int(n), M,
                                        precision_ != PREC_DOUBLE, opt_.real_fp32, stream_, report);
    set_tuning(t);
    return t;
}

// dipole_solver.cu:495-607
void DipoleSolver::compute(const std::vector<double>& x, const std::vector<double>& y, const std::vector<double>& z) {
    if (x.size() != y.size() || x.size() != z.size())
        throw std::invalid_argument("Input coordinate vectors must have the exact same size.");
    const size_t n = x.size();
    if (n == 0) return;
    if (N_ == 0) setup(n);
    else if (N_ != n) throw std::runtime_error("The number of particles has changed!");
    if (!field_) field_ = std::make_unique<Field>(tuned_ ? apply_tuning(field_spec(), tuning_) : field_spec());
    num_frames_++;
    const std::vector<double> sx = scaled(x), sy = scaled(y), sz = scaled(z);
    field_->set_positions(sx.data(), sy.data(), sz.data(), int(N_), stream_);
    const size_t K = E0_.size(), W = eps_p_.size();
    std::vector<cdouble> init;
    if (num_frames_ == 1) {
        init = mean_field_guess(0);
    } else {
        // previous frame's first frequency (dipole_solver.cu:576-593)
        const size_t prev = num_frames_ - 2;
        init.assign(N_ * K * 3 + Nq_ * K * 5, 0.0);
        const std::vector<cdouble>& pd = dip_frames_[prev];
        std::copy(pd.begin(), pd.begin() + N_ * K * 3, init.begin());
        if (solve_quads_ && Nq_) {
            const std::vector<cdouble>& pq = quad_frames_[prev];
            std::copy(pq.begin(), pq.begin() + Nq_ * K * 5, init.begin() + N_ * K * 3);
        }
    }
    const bool dev_batch = device_batch_ok();
    std::vector<cdouble> frame_cap(W * K * 3, 0.0), frame_quad(W * Nq_ * K * 5, 0.0);
    std::vector<cdouble> frame_dip;   // the device batch fills it in one copy
    if (!dev_batch) frame_dip.assign(W * N_ * K * 3, 0.0);
    print("Wavenumber:");
    indent_++;
    if (dev_batch) {
        solve_all_device(init, frame_cap, frame_dip);
    } else if (opt_.batch_all) {
        std::vector<size_t> fr(W);
        std::vector<std::vector<cdouble>> gs(W);
        for (size_t w = 0; w < W; ++w) {
            fr[w] = w;
            gs[w] = w == 0 ? init : mean_field_guess(w);
        }
        solve_batch(fr, gs, frame_cap, frame_dip, frame_quad);
    } else {
        for (size_t w = 0; w < W; ++w) {
            print(std::to_string(w) + " of " + std::to_string(W));
            std::vector<cdouble> g = (w == 0) ? init : guess(frame_dip, frame_quad, w);
            solve_batch({w}, {g}, frame_cap, frame_dip, frame_quad);
        }
    }
    indent_--;
    avg_dips_.insert(avg_dips_.end(), frame_cap.begin(), frame_cap.end());
    dip_frames_.push_back(std::move(frame_dip));
    quad_frames_.push_back(solve_quads_ && Nq_ ? std::move(frame_quad) : std::vector<cdouble>());
}

// dipole_solver.cu:613-647
std::vector<cdouble> DipoleSolver::get_eff_polarizability(bool physical) const {
    const size_t K = E0_.size(), W = eps_p_.size();
    std::vector<cdouble> out(W * K * 3, 0.0);
    if (num_frames_ == 0) return out;
    const double f = physical ? eps_scale_ * std::pow(length_scale_, 3.0) : 1.0;
    for (size_t w = 0; w < W; ++w)
        for (size_t i = 0; i < K * 3; ++i) {
            cdouble s = 0.0;
            for (size_t fr = 0; fr < num_frames_; ++fr) s += avg_dips_[fr * W * K * 3 + w * K * 3 + i];
            out[w * K * 3 + i] = s / double(num_frames_) * f;
        }
    return out;
}

namespace {
// every frame's values, frames concatenated, times f
std::vector<cdouble> concat_frames(const std::vector<std::vector<cdouble>>& frames, double f) {
    size_t n = 0;
    for (const auto& fr : frames) n += fr.size();
    std::vector<cdouble> out;
    out.reserve(n);
    for (const auto& fr : frames)
        for (const cdouble& v : fr) out.push_back(v * f);
    return out;
}
}  // namespace

std::vector<cdouble> DipoleSolver::get_dipoles(bool physical) const {
    const double f = physical ? eps_scale_ * std::pow(length_scale_, 3.0) : 1.0;
    return concat_frames(dip_frames_, f);
}

size_t DipoleSolver::get_dipoles_into(bool physical, cdouble* out, size_t cap) const {
    size_t n = 0;
    for (const auto& fr : dip_frames_) n += fr.size();
    if (cap < n) throw std::invalid_argument("output buffer too small");
    const double f = physical ? eps_scale_ * std::pow(length_scale_, 3.0) : 1.0;
    for (const auto& fr : dip_frames_)
        for (const cdouble& v : fr) *out++ = v * f;
    return n;
}

std::vector<cdouble> DipoleSolver::get_quadrupoles(bool physical) const {
    const double f = physical ? eps_scale_ * std::pow(length_scale_, 4.0) : 1.0;
    return concat_frames(quad_frames_, f);
}

// ---------------------------------------------------------------- NearField

// near_field.cu:19-32
NearField::NearField(std::vector<double> box, std::vector<cdouble> E0, std::vector<double> radius, double xi,
                     double errortol, std::string field_type)
    : box_(std::move(box)), E0_(std::move(E0)), radius_(std::move(radius)), xi_(xi), errortol_(errortol),
      field_type_(std::move(field_type)) {
    if (box_.size() != 3) throw std::invalid_argument("Near_Field box must have length 3.");
    if (E0_.size() != 3) throw std::invalid_argument("Near_Field E0 must have length 3.");
}

NearField::~NearField() {
    field_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

void NearField::set_dipoles(const std::vector<cdouble>& dip) {
    if (dip.size() % 3 != 0) throw std::invalid_argument("Dipoles vector size must be a multiple of 3.");
    N_ = dip.size() / 3;
    dips_ = dip;
}

void NearField::set_dipole_positions(const std::vector<double>& x, const std::vector<double>& y,
                                     const std::vector<double>& z) {
    if (x.size() != y.size() || x.size() != z.size())
        throw std::invalid_argument("Dipole coordinates x, y, z must have the same size.");
    px_ = x; py_ = y; pz_ = z;
}

void NearField::set_field_points(const std::vector<double>& x, const std::vector<double>& y,
                                 const std::vector<double>& z) {
    if (x.size() != y.size() || x.size() != z.size())
        throw std::invalid_argument("Field point coordinates x, y, z must have the same size.");
    fx_ = x; fy_ = y; fz_ = z;
}

// near_field.cu:78-213: intensity |E + E0|^2 of the INTERACTION_FIELD
std::vector<double> NearField::calculate() {
    if (fx_.empty() || px_.empty() || dips_.empty())
        throw std::runtime_error("Near_Field: must set dipoles, dipole positions, and field points before calculation.");
    if (px_.size() != N_)
        throw std::runtime_error("Near_Field: dipole position size is inconsistent with dipole vector size.");
    if (!field_) {
        if (radius_.empty()) radius_.assign(N_, 1.0);
        else if (radius_.size() == 1) radius_.assign(N_, radius_[0]);
        else if (radius_.size() != N_)
            throw std::runtime_error("The number of particles is inconsistent with the number of radii provided.");
        length_scale_ = radius_[0];
        FieldSpec fs;
        fs.solver_ax = false;
        for (int d = 0; d < 3; ++d) fs.box[d] = box_[d] / length_scale_;
        fs.errortol = errortol_;
        fs.xi = xi_;
        std::vector<double> sr = radius_;
        for (auto& r : sr) r /= length_scale_;
        if (field_type_ == "direct") {
            fs.kind = FIELD_DIRECT;
            fs.radius = sr;
        } else {
            bool poly;
            if (field_type_ == "polydisperse") poly = true;
            else if (field_type_ == "monodisperse") poly = false;
            else if (field_type_ == "auto") poly = !all_equal(radius_);
            else throw std::runtime_error("Unknown field_type: " + field_type_);
            fs.kind = poly ? FIELD_POLY : FIELD_MONO;
            if (poly) fs.radius = sr;
        }
        if (!stream_) MPM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        field_ = std::make_unique<Field>(fs);
    }
    const size_t M = fx_.size();
    std::vector<double> x(N_), y(N_), z(N_), a(M), b(M), c(M);
    for (size_t i = 0; i < N_; ++i) { x[i] = px_[i] / length_scale_; y[i] = py_[i] / length_scale_; z[i] = pz_[i] / length_scale_; }
    for (size_t i = 0; i < M; ++i) { a[i] = fx_[i] / length_scale_; b[i] = fy_[i] / length_scale_; c[i] = fz_[i] / length_scale_; }
    field_->set_field_points(a.data(), b.data(), c.data(), int(M), stream_);
    field_->set_positions(x.data(), y.data(), z.data(), int(N_), stream_);
    dX_.ensure(sizeof(double2) * N_ * 3);
    dY_.ensure(sizeof(double2) * M * 3);
    MPM_CUDA(cudaMemcpyAsync(dX_.p, dips_.data(), sizeof(double2) * N_ * 3, cudaMemcpyHostToDevice, stream_));
    // the near field runs the reference's default (AUTO) precision: fp32 reciprocal / fp32 direct
    field_->apply(dX_.as<double2>(), dY_.as<double2>(), 1, nullptr, false, true, false, stream_);
    std::vector<cdouble> E(M * 3);
    MPM_CUDA(cudaMemcpyAsync(E.data(), dY_.p, sizeof(double2) * M * 3, cudaMemcpyDeviceToHost, stream_));
    MPM_CUDA(cudaStreamSynchronize(stream_));
    std::vector<double> out(M);
    for (size_t i = 0; i < M; ++i) {
        double s = 0.0;
        for (int k = 0; k < 3; ++k) s += std::norm(E[i * 3 + k] + E0_[k]);
        out[i] = s;
    }
    return out;
}

}  // namespace mpm
