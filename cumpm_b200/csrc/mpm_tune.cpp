// Autotuner of the spectral-Ewald field (see mpm_tune.h).
//
// Search, every candidate measured on the device:
//  1. xi in {0.7 .. 1.6} x the caller's xi, each with the rule's grid and
//     support (the rule config itself first: its error sets the bound);
//  2. for the two fastest accepted xi: the grid rounded up per axis to the
//     next size with prime factors 2, 3, 5, 7 and to the next 2^a 3^b;
//  3. for the fastest so far: the support trimmed by one and two points;
//  4. for the fastest so far (monodisperse): the spread tiles.
// A candidate's error is max over two test columns (a uniform x-polarised
// dipole set and a seeded random one) of |Y - Y_tight| / |Y_tight|, both
// operators in fp64; Y_tight comes from a field of tolerance errortol/1000
// (/100 or /10 where the kernels refuse the tighter one).
// Its time is the mean of repeated M-column applies in the caller's
// arithmetic, after two warm-up applies.
#include "mpm_tune.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>

namespace mpm {

namespace {

constexpr double kXiFactors[] = {1.0, 0.7, 0.8, 0.9, 1.12, 1.25, 1.4, 1.6};
constexpr int kMaxStencilPts = 31;   // 2 * off + 1 of the monodisperse kernels

bool factors_in(int n, const int* primes, int np) {
    if (n < 1) return false;
    for (int i = 0; i < np; ++i)
        while (n % primes[i] == 0) n /= primes[i];
    return n == 1;
}

double min_box(const FieldSpec& b) { return std::min(b.box[0], std::min(b.box[1], b.box[2])); }

// deterministic test columns [rows][2]: uniform x-polarised dipoles, then
// uniform random real and imaginary parts in [-1, 1] (64-bit LCG)
std::vector<double2> test_columns(int N, int rows) {
    std::vector<double2> X(size_t(rows) * 2);
    uint64_t st = 0x9E3779B97F4A7C15ull;
    auto uni = [&] {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return double(st >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    };
    for (int r = 0; r < rows; ++r) {
        X[size_t(r) * 2] = make_double2(r < 3 * N && r % 3 == 0 ? 1.0 : 0.0, 0.0);
        const double a = uni(), b = uni();
        X[size_t(r) * 2 + 1] = make_double2(a, b);
    }
    return X;
}

struct Bench {
    const FieldSpec& base;
    const double *x, *y, *z;
    int n, M;
    bool r32, re32;
    cudaStream_t s;
    int rows = 0;
    DevBuf Xt, Yt, Xm, Ym;
    std::vector<double2> yref;
    size_t mem_cap = 0;

    double err_of(Field& F) {
        F.apply(Xt.as<double2>(), Yt.as<double2>(), 2, nullptr, false, false, false, s);
        std::vector<double2> y(size_t(rows) * 2);
        MPM_CUDA(cudaMemcpyAsync(y.data(), Yt.p, sizeof(double2) * y.size(), cudaMemcpyDeviceToHost, s));
        MPM_CUDA(cudaStreamSynchronize(s));
        double worst = 0.0;
        for (int c = 0; c < 2; ++c) {
            double num = 0.0, den = 0.0;
            for (int r = 0; r < rows; ++r) {
                const double2 a = y[size_t(r) * 2 + c], b = yref[size_t(r) * 2 + c];
                num += (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y);
                den += b.x * b.x + b.y * b.y;
            }
            worst = std::max(worst, den > 0.0 ? std::sqrt(num / den) : std::sqrt(num));
        }
        return worst;
    }

    double time_of(Field& F) {
        auto once = [&] { F.apply(Xm.as<double2>(), Ym.as<double2>(), M, nullptr, false, r32, re32, s); };
        once();
        once();
        cudaEvent_t e0, e1;
        MPM_CUDA(cudaEventCreate(&e0));
        MPM_CUDA(cudaEventCreate(&e1));
        float ms = 0.f;
        MPM_CUDA(cudaEventRecord(e0, s));
        once();
        MPM_CUDA(cudaEventRecord(e1, s));
        MPM_CUDA(cudaEventSynchronize(e1));
        MPM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        const int reps = std::max(3, std::min(50, int(std::ceil(20.0 / std::max(1e-3, double(ms))))));
        MPM_CUDA(cudaEventRecord(e0, s));
        for (int k = 0; k < reps; ++k) once();
        MPM_CUDA(cudaEventRecord(e1, s));
        MPM_CUDA(cudaEventSynchronize(e1));
        MPM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return double(ms) / reps;
    }

    // builds the candidate's field; null if the geometry is rejected or its
    // grid for M columns would not fit in the memory budget
    std::unique_ptr<Field> make(const FieldSpec& spec) {
        std::unique_ptr<Field> F;
        try {
            F = std::make_unique<Field>(spec);
            F->set_positions(x, y, z, n, s);
        } catch (const std::invalid_argument&) {
            return nullptr;
        } catch (const std::runtime_error& e) {
            if (dynamic_cast<const CudaError*>(&e)) throw;
            return nullptr;
        }
        if (F->grid_bytes(M, !r32) + F->grid_bytes(2, true) > mem_cap) return nullptr;
        return F;
    }
};

struct Eval {
    FieldTuning t;
    double err = 0, ms = 0;
    bool ok = false;
};

}  // namespace

int tune_next_fast(int n) {
    static const int p[] = {2, 3, 5, 7};
    n = std::max(n, 1);
    while (!factors_in(n, p, 4)) ++n;
    return n;
}

int tune_next_smooth23(int n) {
    static const int p[] = {2, 3};
    n = std::max(n, 1);
    while (!factors_in(n, p, 2)) ++n;
    return n;
}

std::vector<XiCandidate> tune_xi_candidates(const FieldSpec& base) {
    std::vector<XiCandidate> out;
    if (base.kind == FIELD_DIRECT) return out;
    for (double f : kXiFactors) {
        const double xi = base.xi * f;
        XiCandidate c{};
        c.xi = xi;
        try {
            if (base.kind == FIELD_POLY) {
                const PolyGeom g = make_poly_geom(base.box, base.errortol, xi, base.radius, base.grid, base.support);
                for (int d = 0; d < 3; ++d) c.grid[d] = g.ng[d];
                c.support = g.P;
                c.rc = g.rc;
                if (g.P > 255) continue;
            } else {
                const EwaldGeom g = make_ewald_geom(base.box, base.errortol, xi, base.grid, base.support);
                for (int d = 0; d < 3; ++d) c.grid[d] = g.ng[d];
                c.support = g.P;
                c.rc = g.rc;
                if (2 * g.off + 1 > kMaxStencilPts) continue;
            }
        } catch (const std::exception&) {
            continue;   // cutoff beyond half the box
        }
        out.push_back(c);
    }
    return out;
}

std::vector<std::pair<int, int>> tune_tiles(int off) {
    // at most 8 bins of a tile's reach per axis (ceil((T + 2 off) / T) + 1)
    // and at most 128 columns per tile (the spread kernels' shared memory)
    std::vector<std::pair<int, int>> out;
    const int T[] = {8, 16, 4};
    for (int tx : T)
        for (int ty : T) {
            if (tx * ty > 128 || tx * ty < 32) continue;
            auto reach = [&](int t) { return (t + 2 * off + t - 1) / t + 1; };
            if (reach(tx) > 8 || reach(ty) > 8) continue;
            out.emplace_back(tx, ty);
        }
    return out;
}

FieldSpec apply_tuning(const FieldSpec& base, const FieldTuning& t) {
    FieldSpec s = base;
    if (t.xi > 0.0) s.xi = t.xi;
    for (int d = 0; d < 3; ++d) s.grid[d] = t.grid[d];
    s.support = t.support;
    s.tile[0] = t.tile[0];
    s.tile[1] = t.tile[1];
    return s;
}

FieldTuning autotune(const FieldSpec& base_in, const double* x, const double* y, const double* z, int n, int M,
                     bool r32, bool re32, cudaStream_t s, TuneReport* report) {
    if (n <= 0) throw std::invalid_argument("autotune: empty coordinate set");
    if (M < 1) throw std::invalid_argument("autotune: M must be >= 1");
    if (!base_in.solver_ax) throw std::invalid_argument("autotune: the field must be in SOLVER_AX mode");
    FieldSpec base = base_in;
    for (int d = 0; d < 3; ++d) base.grid[d] = 0;
    base.support = 0;
    base.tile[0] = base.tile[1] = 0;
    FieldTuning rule;
    rule.xi = base.xi;
    TuneReport rep;
    if (base.kind == FIELD_DIRECT) {
        if (report) *report = rep;
        return rule;
    }
    size_t free_b = 0, total_b = 0;
    MPM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    Bench B{base, x, y, z, n, M, r32, re32, s};
    B.mem_cap = free_b / 3;

    // tight field: tolerance / 1000 (/ 100, / 10 where the kernels' limits
    // refuse the tighter one), xi raised if its cutoff would pass half the
    // box
    std::unique_ptr<Field> Ft;
    for (double f : {1e-3, 1e-2, 1e-1}) {
        FieldSpec tight = base;
        tight.errortol = std::max(1e-14, base.errortol * f);
        const double rc_t = std::sqrt(-std::log(tight.errortol)) / tight.xi;
        if (rc_t > 0.49 * min_box(base)) tight.xi = std::sqrt(-std::log(tight.errortol)) / (0.49 * min_box(base));
        Ft = B.make(tight);
        if (Ft) break;
    }
    if (!Ft) throw std::runtime_error("autotune: no field tighter than the tolerance fits this geometry");
    B.rows = Ft->rows_in();
    const std::vector<double2> Xh = test_columns(n, B.rows);
    B.Xt.ensure(sizeof(double2) * Xh.size());
    B.Yt.ensure(sizeof(double2) * Xh.size());
    MPM_CUDA(cudaMemcpyAsync(B.Xt.p, Xh.data(), sizeof(double2) * Xh.size(), cudaMemcpyHostToDevice, s));
    {
        // the timing columns: the random test column repeated
        std::vector<double2> Xm(size_t(B.rows) * M);
        for (int r = 0; r < B.rows; ++r)
            for (int m = 0; m < M; ++m) Xm[size_t(r) * M + m] = Xh[size_t(r) * 2 + 1];
        B.Xm.ensure(sizeof(double2) * Xm.size());
        B.Ym.ensure(sizeof(double2) * Xm.size());
        MPM_CUDA(cudaMemcpyAsync(B.Xm.p, Xm.data(), sizeof(double2) * Xm.size(), cudaMemcpyHostToDevice, s));
        MPM_CUDA(cudaStreamSynchronize(s));
    }
    B.yref.resize(Xh.size());
    Ft->apply(B.Xt.as<double2>(), B.Yt.as<double2>(), 2, nullptr, false, false, false, s);
    MPM_CUDA(cudaMemcpyAsync(B.yref.data(), B.Yt.p, sizeof(double2) * Xh.size(), cudaMemcpyDeviceToHost, s));
    MPM_CUDA(cudaStreamSynchronize(s));
    Ft.reset();

    double bound = 0.0;
    auto eval = [&](const FieldTuning& t, bool timed) {
        Eval e;
        e.t = t;
        rep.candidates++;
        std::unique_ptr<Field> F = B.make(apply_tuning(base, t));
        if (!F) return e;
        e.err = B.err_of(*F);
        e.ok = !(e.err > bound);   // NaN fails
        if (e.ok && timed) e.ms = B.time_of(*F);
        if (e.ok) rep.accepted++;
        return e;
    };

    // 1. the rule, then xi
    bound = 1e300;
    Eval best = eval(rule, true);
    if (!best.ok) throw std::runtime_error("autotune: the rule configuration does not fit in device memory");
    rep.error_rule = best.err;
    rep.apply_ms_rule = best.ms;
    bound = std::max(base.errortol, best.err);
    std::vector<Eval> xs{best};
    for (const XiCandidate& c : tune_xi_candidates(base)) {
        if (c.xi == base.xi) continue;
        FieldTuning t;
        t.xi = c.xi;
        Eval e = eval(t, true);
        if (e.ok) xs.push_back(e);
    }
    std::sort(xs.begin(), xs.end(), [](const Eval& a, const Eval& b) { return a.ms < b.ms; });
    best = xs.front();

    // 2. grid sizes for the two fastest xi
    for (size_t i = 0; i < std::min<size_t>(2, xs.size()); ++i) {
        const FieldSpec sp = apply_tuning(base, xs[i].t);
        int g0[3];
        if (base.kind == FIELD_POLY) {
            const PolyGeom g = make_poly_geom(sp.box, sp.errortol, sp.xi, sp.radius);
            for (int d = 0; d < 3; ++d) g0[d] = g.ng[d];
        } else {
            const EwaldGeom g = make_ewald_geom(sp.box, sp.errortol, sp.xi);
            for (int d = 0; d < 3; ++d) g0[d] = g.ng[d];
        }
        for (int kind = 0; kind < 2; ++kind) {
            FieldTuning t = xs[i].t;
            bool differs = false;
            for (int d = 0; d < 3; ++d) {
                t.grid[d] = kind == 0 ? tune_next_fast(g0[d]) : tune_next_smooth23(g0[d]);
                differs |= t.grid[d] != g0[d];
            }
            if (!differs) continue;
            Eval e = eval(t, true);
            if (e.ok && e.ms < best.ms) best = e;
        }
    }

    // 3. support trimmed
    {
        const FieldSpec sp = apply_tuning(base, best.t);
        int P0;
        if (base.kind == FIELD_POLY) P0 = make_poly_geom(sp.box, sp.errortol, sp.xi, sp.radius, sp.grid).P;
        else P0 = make_ewald_geom(sp.box, sp.errortol, sp.xi, sp.grid).P;
        for (int dP = 1; dP <= 2; ++dP) {
            if (P0 - dP < 3) break;
            FieldTuning t = best.t;
            t.support = P0 - dP;
            Eval e = eval(t, true);
            if (!e.ok) break;
            if (e.ms < best.ms) best = e;
        }
    }

    // 4. spread tiles (monodisperse)
    if (base.kind == FIELD_MONO) {
        const FieldSpec sp = apply_tuning(base, best.t);
        const EwaldGeom g = make_ewald_geom(sp.box, sp.errortol, sp.xi, sp.grid, sp.support);
        for (const auto& tl : tune_tiles(g.off)) {
            if (tl.first == 8 && tl.second == 8) continue;
            FieldTuning t = best.t;
            t.tile[0] = tl.first;
            t.tile[1] = tl.second;
            Eval e = eval(t, true);
            if (e.ok && e.ms < best.ms) best = e;
        }
    }

    rep.apply_ms = best.ms;
    rep.error = best.err;
    rep.error_bound = bound;
    if (report) *report = rep;
    return best.t;
}

}  // namespace mpm
