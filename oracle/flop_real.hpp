// CPU ORACLE (test infrastructure): a floating-point type that counts its operations.
//
// oracle_flops.cpp compiles the oracle with `double` replaced by orc_flops::Real, so that a
// residual evaluation of the restated reference algorithm reports how many FP64 operations it
// performs: the algorithmic FLOP count of the path, independent of how the CUDA kernels
// arrange the work.  Each +, -, *, / and unary minus counts one; sqrt one; every other library
// function (pow, exp, log10, sin, cos) one call in its own counter; comparisons, fabs, min and
// max count nothing (they are not FP arithmetic on the FP64 pipe's FMA/ADD/MUL).  An addition
// or subtraction with an exact zero operand and a multiplication by an exact zero are counted
// apart as trivial (the reference adds a zero perturbation V to every coefficient of a plain
// residual and forms each volume flux against a unit normal).  The counts are kept per phase
// (g_phase: 0 volume and the rest, 1 interior face, 2 boundary face), so a caller can count
// each interior face once although the reference evaluates it from both sides.  A Real holds
// exactly one double, so arrays of doubles passed across the C interface read as arrays of Real.
#pragma once
#include <cmath>
#include <istream>
#include <limits>

namespace orc_flops {

struct Counters {
    unsigned long long add = 0, mul = 0, div = 0, sqrt = 0, fn = 0, triv = 0;
};
extern Counters g_counts[3];
extern int g_phase;
inline Counters& cur() { return g_counts[g_phase]; }
inline void count_add(double a, double b) {
    if (a == 0.0 || b == 0.0)
        ++cur().triv;
    else
        ++cur().add;
}
inline void count_mul(double a, double b) {
    if (a == 0.0 || b == 0.0)
        ++cur().triv;
    else
        ++cur().mul;
}

struct Real {
    double v;
    Real() = default;
    constexpr Real(double x) : v(x) {}  // NOLINT: implicit, as a double literal converts
    explicit constexpr operator double() const { return v; }
    explicit constexpr operator int() const { return (int)v; }
    Real& operator+=(Real o) { count_add(v, o.v); v += o.v; return *this; }
    Real& operator-=(Real o) { count_add(v, o.v); v -= o.v; return *this; }
    Real& operator*=(Real o) { count_mul(v, o.v); v *= o.v; return *this; }
    Real& operator/=(Real o) { ++cur().div; v /= o.v; return *this; }
    Real operator-() const { ++cur().add; return Real(-v); }
    Real operator+() const { return *this; }
};
static_assert(sizeof(Real) == sizeof(double), "Real must be layout-compatible with double");
inline std::istream& operator>>(std::istream& is, Real& a) { return is >> a.v; }

inline Real operator+(Real a, Real b) { count_add(a.v, b.v); return Real(a.v + b.v); }
inline Real operator-(Real a, Real b) { count_add(a.v, b.v); return Real(a.v - b.v); }
inline Real operator*(Real a, Real b) { count_mul(a.v, b.v); return Real(a.v * b.v); }
inline Real operator/(Real a, Real b) { ++cur().div; return Real(a.v / b.v); }
#define ORC_FLOPS_MIXED(op)                                             \
    inline Real operator op(Real a, double b) { return a op Real(b); }  \
    inline Real operator op(double a, Real b) { return Real(a) op b; }  \
    inline Real operator op(Real a, int b) { return a op Real(b); }     \
    inline Real operator op(int a, Real b) { return Real(a) op b; }
ORC_FLOPS_MIXED(+)
ORC_FLOPS_MIXED(-)
ORC_FLOPS_MIXED(*)
ORC_FLOPS_MIXED(/)
#undef ORC_FLOPS_MIXED
#define ORC_FLOPS_CMP(op)                                                       \
    inline bool operator op(Real a, Real b) { return a.v op b.v; }              \
    inline bool operator op(Real a, double b) { return a.v op b; }              \
    inline bool operator op(double a, Real b) { return a op b.v; }              \
    inline bool operator op(Real a, int b) { return a.v op (double)b; }         \
    inline bool operator op(int a, Real b) { return (double)a op b.v; }
ORC_FLOPS_CMP(<)
ORC_FLOPS_CMP(>)
ORC_FLOPS_CMP(<=)
ORC_FLOPS_CMP(>=)
ORC_FLOPS_CMP(==)
ORC_FLOPS_CMP(!=)
#undef ORC_FLOPS_CMP

}  // namespace orc_flops

// the library functions the oracle calls with std:: qualification
namespace std {
using orc_flops::Real;
inline Real sqrt(Real a) { ++orc_flops::cur().sqrt; return Real(std::sqrt(a.v)); }
inline Real fabs(Real a) { return Real(std::fabs(a.v)); }
inline Real abs(Real a) { return Real(std::fabs(a.v)); }
inline Real pow(Real a, Real b) { ++orc_flops::cur().fn; return Real(std::pow(a.v, b.v)); }
inline Real pow(Real a, double b) { ++orc_flops::cur().fn; return Real(std::pow(a.v, b)); }
inline Real pow(Real a, int b) { ++orc_flops::cur().fn; return Real(std::pow(a.v, b)); }
inline Real pow(double a, Real b) { ++orc_flops::cur().fn; return Real(std::pow(a, b.v)); }
inline Real exp(Real a) { ++orc_flops::cur().fn; return Real(std::exp(a.v)); }
inline Real log(Real a) { ++orc_flops::cur().fn; return Real(std::log(a.v)); }
inline Real log10(Real a) { ++orc_flops::cur().fn; return Real(std::log10(a.v)); }
inline Real sin(Real a) { ++orc_flops::cur().fn; return Real(std::sin(a.v)); }
inline Real cos(Real a) { ++orc_flops::cur().fn; return Real(std::cos(a.v)); }
inline Real atan(Real a) { ++orc_flops::cur().fn; return Real(std::atan(a.v)); }
inline Real tanh(Real a) { ++orc_flops::cur().fn; return Real(std::tanh(a.v)); }
inline Real floor(Real a) { return Real(std::floor(a.v)); }
inline Real ceil(Real a) { return Real(std::ceil(a.v)); }
inline bool isnan(Real a) { return std::isnan(a.v); }
inline bool isinf(Real a) { return std::isinf(a.v); }
inline bool isfinite(Real a) { return std::isfinite(a.v); }
inline const Real& max(const Real& a, const Real& b) { return a.v < b.v ? b : a; }
inline const Real& min(const Real& a, const Real& b) { return b.v < a.v ? b : a; }
inline Real max(Real a, double b) { return a.v < b ? Real(b) : a; }
inline Real max(double a, Real b) { return a < b.v ? b : Real(a); }
inline Real min(Real a, double b) { return b < a.v ? Real(b) : a; }
inline Real min(double a, Real b) { return b.v < a ? b : Real(a); }
inline string to_string(Real a) { return to_string(a.v); }
template <>
class numeric_limits<Real> : public numeric_limits<double> {
  public:
    static Real max() noexcept { return Real(numeric_limits<double>::max()); }
    static Real min() noexcept { return Real(numeric_limits<double>::min()); }
    static Real lowest() noexcept { return Real(numeric_limits<double>::lowest()); }
    static Real epsilon() noexcept { return Real(numeric_limits<double>::epsilon()); }
    static Real infinity() noexcept { return Real(numeric_limits<double>::infinity()); }
    static Real quiet_NaN() noexcept { return Real(numeric_limits<double>::quiet_NaN()); }
};
}  // namespace std
