// Real-space pair functions of the monodisperse spectral-Ewald split.
//
// Each function is tabulated on r = 0 (self value) and r = 1 + k*0.001,
// k = 0..8999, and looked up by linear interpolation, exactly as the
// reference does (monodisperse_ewald_electric_field.cu:92-542 builds the
// tables, :668-685 interpolates) so that pair couplings agree to rounding.
#pragma once
#include <vector>

namespace mpm {

enum TableId { T_FD1 = 0, T_FD2, T_FQ1, T_FQ2, T_FQ3, T_GQ1, T_GQ2, T_GQ3, T_GQ4, T_COUNT };

constexpr int kTableSteps = 9000;         // r = 1 .. 9.999
constexpr int kTableSize = kTableSteps + 1;  // plus the r = 0 entry
constexpr double kTableDr = 0.001;

struct MonoTables {
    std::vector<double> r;                 // kTableSize
    std::vector<double> f[T_COUNT];        // kTableSize each
    double selfo = 0.0;                    // r = 0 entry of the dipole tables
    double self_grad = 0.0;                // r = 0 entry of the gradient tables
};

MonoTables build_mono_tables(double xi);

// Radius-1 quadrupole tables of the polydisperse field
// (polydisperse_ewald_electric_field.cu:1690-2035): nodes r = 0 and
// r = 1 + k*0.001 up to the cutoff, as for its dipole tables.  fq1-fq3, gq1
// and gq4 are the monodisperse expressions; gq2 and gq3 are the polydisperse
// field's own.
enum PolyQuadTableId { PQ_FQ1 = 0, PQ_FQ2, PQ_FQ3, PQ_GQ1, PQ_GQ2, PQ_GQ3, PQ_GQ4, PQ_COUNT };

struct PolyQuadTables {
    std::vector<double> r;                 // n_nodes
    std::vector<double> f[PQ_COUNT];       // n_nodes each
    double self_grad = 0.0;                // r = 0 entry of the gradient tables
};

PolyQuadTables build_poly_quad_tables(double xi, int n_nodes);

// Quadrupole self value of a sphere of radius a (:1690-1706): the unit
// sphere's gradient self value at xi*a, over a^5.
double poly_quad_self_value(double a, double xi);

// Host copy of the device lookup (used by tests and host precalcs).
double table_lookup(double r, const double* r_table, const double* y, int n);

}  // namespace mpm
