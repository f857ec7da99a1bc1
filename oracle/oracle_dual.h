/*
 * oracle_dual.h -- forward-mode derivative numbers for the tangent build of
 * the CPU oracle (test infrastructure only).
 *
 * lbm_oracle.c computes in the type `real`.  The ordinary build makes it
 * double.  The tangent build (C++, -DORACLE_TANGENT) makes it `dual`: a value
 * and its derivative with respect to one seeded input (tau_y, nu, or one
 * disk's rho_p, x0 or y0).  Every operation does to the value exactly what
 * the double build does (same operations, same order, no contraction), and
 * carries the derivative by the chain rule, so a tangent run returns the
 * oracle's own results together with their exact derivatives: the
 * derivative of the reference's discrete time step, independent of the
 * hand-transposed adjoint kernels and free of finite-difference truncation.
 * Comparisons look at the value only, so a run takes the branches of the
 * ordinary run and differentiates the branch it takes.
 */
#ifndef ORACLE_DUAL_H
#define ORACLE_DUAL_H

#include <cmath>

struct dual {
    double v, d;
    dual() = default;  // trivial: calloc/memset give (0, 0)
    constexpr dual(double x) : v(x), d(0.0) {}
    constexpr dual(double x, double dx) : v(x), d(dx) {}
    explicit operator double() const { return v; }
    dual& operator+=(const dual& b) { d += b.d; v += b.v; return *this; }
    dual& operator-=(const dual& b) { d -= b.d; v -= b.v; return *this; }
    dual& operator*=(const dual& b) { *this = dual(v * b.v, d * b.v + v * b.d); return *this; }
    dual& operator/=(const dual& b) {
        const double q = v / b.v;
        *this = dual(q, (d - q * b.d) / b.v);
        return *this;
    }
};

inline dual operator+(const dual& a) { return a; }
inline dual operator-(const dual& a) { return dual(-a.v, -a.d); }
inline dual operator+(const dual& a, const dual& b) { return dual(a.v + b.v, a.d + b.d); }
inline dual operator-(const dual& a, const dual& b) { return dual(a.v - b.v, a.d - b.d); }
inline dual operator*(const dual& a, const dual& b) { return dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline dual operator/(const dual& a, const dual& b) {
    const double q = a.v / b.v;
    return dual(q, (a.d - q * b.d) / b.v);
}
inline dual operator+(const dual& a, double b) { return dual(a.v + b, a.d); }
inline dual operator+(double a, const dual& b) { return dual(a + b.v, b.d); }
inline dual operator-(const dual& a, double b) { return dual(a.v - b, a.d); }
inline dual operator-(double a, const dual& b) { return dual(a - b.v, -b.d); }
inline dual operator*(const dual& a, double b) { return dual(a.v * b, a.d * b); }
inline dual operator*(double a, const dual& b) { return dual(a * b.v, a * b.d); }
inline dual operator/(const dual& a, double b) { return dual(a.v / b, a.d / b); }
inline dual operator/(double a, const dual& b) {
    const double q = a / b.v;
    return dual(q, -q * b.d / b.v);
}

#define ORACLE_DUAL_CMP(op)                                                             \
    inline bool operator op(const dual& a, const dual& b) { return a.v op b.v; }          \
    inline bool operator op(const dual& a, double b) { return a.v op b; }                 \
    inline bool operator op(double a, const dual& b) { return a op b.v; }
ORACLE_DUAL_CMP(<)
ORACLE_DUAL_CMP(>)
ORACLE_DUAL_CMP(<=)
ORACLE_DUAL_CMP(>=)
ORACLE_DUAL_CMP(==)
ORACLE_DUAL_CMP(!=)
#undef ORACLE_DUAL_CMP

// d sqrt(x) = dx / (2 sqrt(x)); at x = 0 the derivative is taken as 0 (the
// callers use it only where x > 0 or where the result is discarded)
inline dual sqrt(const dual& a) {
    const double s = std::sqrt(a.v);
    return dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}
inline dual sin(const dual& a) { return dual(std::sin(a.v), std::cos(a.v) * a.d); }
inline dual cos(const dual& a) { return dual(std::cos(a.v), -std::sin(a.v) * a.d); }
inline dual exp(const dual& a) {
    const double e = std::exp(a.v);
    return dual(e, e * a.d);
}
inline dual fabs(const dual& a) { return a.v < 0.0 ? -a : a; }

typedef dual real;
#define RVAL(x) ((x).v)
#define RDER(x) ((x).d)

#endif
