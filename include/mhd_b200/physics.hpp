// physics.hpp -- the reference's GLM-MHD physics API (head/physics.hpp:21-217)
// on the host, backed by libmhd_b200's FP64 physics (the same functions the
// FP64 kernels run, bit-identical with the reference's CPU path).
#pragma once

#include "types.hpp"

namespace phys {

// Process-global physics scalars, as in the reference (head/physics.hpp:27-42).
// The GPU drop-in functions (gpu/solver_gpu.cuh) read gamma and ch_glm from
// here and write ch_glm back, like the reference's set_gpu_physics_* mirrors.
extern double gamma;   // adiabatic exponent, default 5/3
extern double ch_glm;  // GLM cleaning speed c_h, default 0
extern double cr_glm;  // c_r = c_p^2 / c_h, default 0.18

inline double get_gamma() { return gamma; }
inline double get_ch_glm() { return ch_glm; }

Primitive cons_to_prim(const Conserved& U);          // head/physics.hpp:69-78
Conserved prim_to_cons(const Primitive& V);          // head/physics.hpp:83-90
Conserved flux_x(const Conserved& U, double ch);     // head/physics.hpp:105-127
Conserved flux_y(const Conserved& U, double ch);     // head/physics.hpp:142-164
double fast_speed_x(const Primitive& V);             // head/physics.hpp:175-181
double fast_speed_y(const Primitive& V);             // head/physics.hpp:184-190
double sound_speed(const Primitive& V);              // head/physics.hpp:193-195
double max_signal_speed_x(const Primitive& V, double ch);  // head/physics.hpp:202-205
double max_signal_speed_y(const Primitive& V, double ch);  // head/physics.hpp:207-210
inline double pressure(const Conserved& U) { return cons_to_prim(U).p; }

}  // namespace phys
