// types.hpp -- the reference's state records (head/types.hpp:16-182), for code
// written against the reference's C++ API.  Same names, field order and
// element-wise operators; the kernels themselves use SoA planes (mhd_b200.h).
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define HD __host__ __device__
#else
#define HD
#endif

// U = (rho, rho u, rho v, rho w, Bx, By, Bz, E, psi)
struct Conserved {
    double rho, rhou, rhov, rhow, Bx, By, Bz, E, psi;
    HD Conserved() : rho(0), rhou(0), rhov(0), rhow(0), Bx(0), By(0), Bz(0), E(0), psi(0) {}
    HD Conserved(double r, double mu, double mv, double mw, double bx, double by, double bz, double e, double ps)
        : rho(r), rhou(mu), rhov(mv), rhow(mw), Bx(bx), By(by), Bz(bz), E(e), psi(ps) {}
    // hydrodynamic shorthand: B = 0, rhow = 0, psi = 0
    HD Conserved(double r, double mu, double mv, double e)
        : rho(r), rhou(mu), rhov(mv), rhow(0), Bx(0), By(0), Bz(0), E(e), psi(0) {}
};

// V = (rho, u, v, w, Bx, By, Bz, p, psi)
struct Primitive {
    double rho, u, v, w, Bx, By, Bz, p, psi;
    HD Primitive() : rho(0), u(0), v(0), w(0), Bx(0), By(0), Bz(0), p(0), psi(0) {}
    HD Primitive(double r, double u_, double v_, double w_, double bx, double by, double bz, double p_, double ps)
        : rho(r), u(u_), v(v_), w(w_), Bx(bx), By(by), Bz(bz), p(p_), psi(ps) {}
    HD Primitive(double r, double u_, double v_, double p_)
        : rho(r), u(u_), v(v_), w(0), Bx(0), By(0), Bz(0), p(p_), psi(0) {}
};

// Element-wise arithmetic over the nine fields (both records are nine
// consecutive doubles).  a / s multiplies by the reciprocal, as the reference
// does (head/types.hpp:104-106, 159-161).
#define MHD_STATE_OPS(T)                                                          \
    HD inline T operator+(const T& a, const T& b) {                               \
        T r;                                                                      \
        const double *x = &a.rho, *y = &b.rho;                                    \
        double* z = &r.rho;                                                       \
        for (int k = 0; k < 9; ++k) z[k] = x[k] + y[k];                           \
        return r;                                                                 \
    }                                                                             \
    HD inline T operator-(const T& a, const T& b) {                               \
        T r;                                                                      \
        const double *x = &a.rho, *y = &b.rho;                                    \
        double* z = &r.rho;                                                       \
        for (int k = 0; k < 9; ++k) z[k] = x[k] - y[k];                           \
        return r;                                                                 \
    }                                                                             \
    HD inline T operator*(double s, const T& a) {                                 \
        T r;                                                                      \
        const double* x = &a.rho;                                                 \
        double* z = &r.rho;                                                       \
        for (int k = 0; k < 9; ++k) z[k] = s * x[k];                              \
        return r;                                                                 \
    }                                                                             \
    HD inline T operator*(const T& a, double s) { return s * a; }                 \
    HD inline T operator/(const T& a, double s) { return (1.0 / s) * a; }         \
    HD inline T& operator+=(T& a, const T& b) { return a = a + b; }               \
    HD inline T& operator-=(T& a, const T& b) { return a = a - b; }               \
    HD inline T& operator*=(T& a, double s) { return a = s * a; }

MHD_STATE_OPS(Conserved)
MHD_STATE_OPS(Primitive)
#undef MHD_STATE_OPS
