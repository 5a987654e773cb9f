// ORACLE — test infrastructure only. Forward-mode dual numbers for the
// tangent-linear build of the oracle (liboracle_dual.so): every Real carries
// a value and a derivative along one input direction, so one run of the
// FP64 step gives the exact directional derivative of the step (with its
// discrete choices held at the value path's) to FP64 rounding. The adjoint
// tests compare the device gradient's inner product with a direction
// against this derivative, and with one run per input component they
// rebuild whole FP64 gradient vectors.
#pragma once
#include <cmath>
#include <limits>

namespace b3dual {

struct Dual {
    double v, d;
    Dual() : v(0.0), d(0.0) {}
    Dual(double x) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
    explicit operator double() const { return v; }
    explicit operator float() const { return (float)v; }
    explicit operator int() const { return (int)v; }
    Dual& operator+=(const Dual& o) {
        v += o.v;
        d += o.d;
        return *this;
    }
    Dual& operator-=(const Dual& o) {
        v -= o.v;
        d -= o.d;
        return *this;
    }
    Dual& operator*=(const Dual& o) {
        d = d * o.v + v * o.d;
        v *= o.v;
        return *this;
    }
    Dual& operator/=(const Dual& o) {
        const double q = v / o.v;
        d = (d - q * o.d) / o.v;
        v = q;
        return *this;
    }
};

inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
// comparisons follow the value path
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }

inline Dual sqrt(Dual a) {
    const double s = std::sqrt(a.v);
    return Dual(s, s > 0.0 ? a.d / (2.0 * s) : 0.0);
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual sin(Dual a) { return Dual(std::sin(a.v), a.d * std::cos(a.v)); }
inline Dual cos(Dual a) { return Dual(std::cos(a.v), -a.d * std::sin(a.v)); }

}  // namespace b3dual

namespace std {
template <>
class numeric_limits<b3dual::Dual> : public numeric_limits<double> {
public:
    static b3dual::Dual max() { return b3dual::Dual(numeric_limits<double>::max()); }
    static b3dual::Dual lowest() { return b3dual::Dual(numeric_limits<double>::lowest()); }
};
}  // namespace std
