// riemann.hpp -- the reference's Riemann-solver API (head/riemann.hpp:21-601)
// on the host, backed by libmhd_b200's FP64 solvers (bit-identical with the
// reference's).  The enum values are the ones the C ABI uses (MHD_HLL ...).
#pragma once

#include <cmath>

#include "physics.hpp"
#include "types.hpp"

enum class Direction { X, Y };
enum class RiemannSolver { HLL, HLLC, HLLD, FORCE };

// Slope limiter of the MUSCL-Hancock reconstruction.  The reference has only
// minmod; van Leer is this library's addition.
enum class Limiter { Minmod, VanLeer };

inline double normal_velocity(const Primitive& V, Direction d) { return d == Direction::X ? V.u : V.v; }
inline double normal_B(const Primitive& V, Direction d) { return d == Direction::X ? V.Bx : V.By; }
inline bool finite_number(double x) { return std::isfinite(x); }
inline bool primitive_is_physical(const Primitive& V) {
    return finite_number(V.rho) && finite_number(V.p) && V.rho > 0.0 && V.p > 0.0;
}

Conserved physical_flux(const Conserved& U, Direction dir);  // uses phys::ch_glm
Conserved hll_flux(const Conserved& UL, const Conserved& UR, Direction dir, double ch);
Conserved hllc_flux(const Conserved& UL, const Conserved& UR, Direction dir, double ch);
Conserved hlld_flux(const Conserved& UL, const Conserved& UR, Direction dir, double ch);
Conserved force_flux(const Conserved& UL, const Conserved& UR, Direction dir, double ch);
void apply_glm_flux(Conserved& F, const Conserved& UL, const Conserved& UR, Direction dir, double ch);
Conserved riemann_flux(const Conserved& UL, const Conserved& UR, Direction dir, RiemannSolver solver, double ch);
Conserved riemann_flux(const Conserved& UL, const Conserved& UR, Direction dir, RiemannSolver solver);
