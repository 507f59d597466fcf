// flopcount.h — host-side operation counting for the roofline numerator.
//
// Counted is a double that tallies every arithmetic operation applied to it
// (+ - * / and the elementary functions each count as one operation; a fused
// multiply-add is written as a multiply and an add, i.e. two). Instantiating
// the device templates of spacetime.cuh with T = Counted on the host gives the
// algorithmic operation count of the kernels' own right-hand side.
#pragma once

#include <cmath>

namespace sirius {

struct FlopCounter {
    static long long& n() {
        static thread_local long long count = 0;
        return count;
    }
};

struct Counted {
    double v = 0.0;
    Counted() = default;
    Counted(double x) : v(x) {}  // NOLINT: literals and parameters convert implicitly
    explicit operator double() const { return v; }
};

inline Counted tick(double v) {
    ++FlopCounter::n();
    return Counted(v);
}
inline Counted operator+(Counted a, Counted b) { return tick(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { return tick(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { return tick(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { return tick(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }  // sign flip: free
inline Counted& operator+=(Counted& a, Counted b) { a = a + b; return a; }
inline Counted& operator-=(Counted& a, Counted b) { a = a - b; return a; }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline Counted rcp_(Counted a) { return tick(1.0 / a.v); }
inline Counted sqrt_(Counted a) { return tick(std::sqrt(a.v)); }
inline Counted sqrtp_(Counted a) { return tick(std::sqrt(a.v)); }
inline Counted rsqrt_(Counted a) { return tick(1.0 / std::sqrt(a.v)); }
inline Counted exp_(Counted a) { return tick(std::exp(a.v)); }
inline Counted tanh_(Counted a) { return tick(std::tanh(a.v)); }
using ::cos;  // keep the float/double overloads visible next to the Counted ones
using ::sin;
inline Counted sin(Counted a) { return tick(std::sin(a.v)); }
inline Counted cos(Counted a) { return tick(std::cos(a.v)); }

}  // namespace sirius
