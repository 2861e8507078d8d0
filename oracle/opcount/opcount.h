// Operation-counting scalar for the oracle restatement (test infrastructure
// only; never linked into the product).
//
// `ocd` holds a double and counts every floating-point operation done on it:
// add/sub, mul, div, sqrt and each named transcendental.  opcount.cpp compiles
// the oracle restatement (src/oracle_3d.cpp) with `double` spelled as `ocd`,
// so running it on a ray counts the reference algorithm's own operations
// (the restatement is bit-identical to the reference and follows its
// operation order).  Constant expressions the compiler folds (literal
// arithmetic) are not counted; comparisons, negation, fabs, min/max and
// conversions are not floating-point work and are not counted either.
#pragma once
#include <cmath>
#include <istream>
#include <type_traits>

struct OpCounts {
    long long add = 0, mul = 0, div = 0, sqrt = 0;
    long long exp = 0, log = 0, pow = 0, trig = 0, cbrt = 0;
};

// Counts are kept per region: 0 for everything, 1 inside the absorption
// model (the oracle marks SB_alpha with ORC_REGION when built here), so the
// Sutherland-Bass share of a ray-step can be reported on its own.
inline int& op_region() {
    static int r = 0;
    return r;
}
inline OpCounts* op_count_table() {
    static OpCounts c[2];
    return c;
}
inline OpCounts& op_counts() { return op_count_table()[op_region()]; }

// Attributes the operations of the enclosing scope to region 1.
struct OpRegionScope {
    int saved;
    OpRegionScope() : saved(op_region()) { op_region() = 1; }
    ~OpRegionScope() { op_region() = saved; }
};
#define ORC_REGION_ABSORPTION OpRegionScope orc_region_scope_

struct ocd {
    double v;
    constexpr ocd() : v(0.0) {}
    template <class T, class = typename std::enable_if<std::is_arithmetic<T>::value>::type>
    constexpr ocd(T x) : v(static_cast<double>(x)) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return static_cast<int>(v); }
    explicit operator long long() const { return static_cast<long long>(v); }
    explicit operator bool() const { return v != 0.0; }
    ocd& operator+=(ocd o) { op_counts().add++; v += o.v; return *this; }
    ocd& operator-=(ocd o) { op_counts().add++; v -= o.v; return *this; }
    ocd& operator*=(ocd o) { op_counts().mul++; v *= o.v; return *this; }
    ocd& operator/=(ocd o);
};

inline ocd operator+(ocd a, ocd b) { op_counts().add++; return ocd(a.v + b.v); }
inline ocd operator-(ocd a, ocd b) { op_counts().add++; return ocd(a.v - b.v); }
inline ocd operator*(ocd a, ocd b) { op_counts().mul++; return ocd(a.v * b.v); }
// Division by an exact power of two is a multiply by its reciprocal (exact,
// and what an optimising compiler emits), so it counts as one.
inline bool pow2_divisor(double b) {
    int e;
    return b != 0.0 && std::isfinite(b) && std::fabs(std::frexp(b, &e)) == 0.5;
}
inline ocd operator/(ocd a, ocd b) {
    if (pow2_divisor(b.v)) op_counts().mul++;
    else op_counts().div++;
    return ocd(a.v / b.v);
}
inline ocd& ocd::operator/=(ocd o) { *this = *this / o; return *this; }
inline ocd operator-(ocd a) { return ocd(-a.v); }
inline ocd operator+(ocd a) { return a; }
inline bool operator<(ocd a, ocd b) { return a.v < b.v; }
inline bool operator>(ocd a, ocd b) { return a.v > b.v; }
inline bool operator<=(ocd a, ocd b) { return a.v <= b.v; }
inline bool operator>=(ocd a, ocd b) { return a.v >= b.v; }
inline bool operator==(ocd a, ocd b) { return a.v == b.v; }
inline bool operator!=(ocd a, ocd b) { return a.v != b.v; }
inline std::istream& operator>>(std::istream& in, ocd& x) { return in >> x.v; }

inline ocd sqrt(ocd a) { op_counts().sqrt++; return ocd(std::sqrt(a.v)); }
inline ocd exp(ocd a) { op_counts().exp++; return ocd(std::exp(a.v)); }
inline ocd log(ocd a) { op_counts().log++; return ocd(std::log(a.v)); }
inline ocd log10(ocd a) { op_counts().log++; return ocd(std::log10(a.v)); }
inline ocd cbrt(ocd a) { op_counts().cbrt++; return ocd(std::cbrt(a.v)); }
inline ocd sin(ocd a) { op_counts().trig++; return ocd(std::sin(a.v)); }
inline ocd cos(ocd a) { op_counts().trig++; return ocd(std::cos(a.v)); }
inline ocd tan(ocd a) { op_counts().trig++; return ocd(std::tan(a.v)); }
inline ocd asin(ocd a) { op_counts().trig++; return ocd(std::asin(a.v)); }
inline ocd acos(ocd a) { op_counts().trig++; return ocd(std::acos(a.v)); }
inline ocd atan(ocd a) { op_counts().trig++; return ocd(std::atan(a.v)); }
inline ocd atan2(ocd a, ocd b) { op_counts().trig++; return ocd(std::atan2(a.v, b.v)); }
// pow with a small integer exponent is what the reference writes for squares
// and cubes; the library evaluates it as that many multiplies, which is how it
// is counted.  Other exponents count as one transcendental.
inline ocd pow(ocd a, ocd b) {
    const double e = b.v;
    if (e == 2.0 || e == 3.0 || e == 4.0) {
        op_counts().mul += static_cast<long long>(e) - 1;
    } else {
        op_counts().pow++;
    }
    return ocd(std::pow(a.v, b.v));
}
inline ocd fabs(ocd a) { return ocd(std::fabs(a.v)); }
inline ocd floor(ocd a) { return ocd(std::floor(a.v)); }
inline ocd ceil(ocd a) { return ocd(std::ceil(a.v)); }
inline bool isfinite(ocd a) { return std::isfinite(a.v); }
inline bool isnan(ocd a) { return std::isnan(a.v); }
