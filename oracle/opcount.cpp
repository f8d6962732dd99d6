// opcount.cpp -- the oracle built with an arithmetic-operation counter.
//
// TEST / MEASUREMENT INFRASTRUCTURE ONLY (like nemo_oracle.cpp, which it compiles unchanged): it
// produces the algorithmic flop count per DOF-update that the roofline of the stage kernels is
// graded against.  Every FP64 value of the oracle becomes a `cdouble`, a one-double wrapper whose
// arithmetic is the same IEEE operation (the file is compiled with -ffp-contract=off, so results
// and therefore branches are bit-identical to the plain oracle) plus an increment of a counter:
//   + - * /        1 flop each (no FMA exists in the oracle: contraction is off)
//   sqrt           1 flop
//   log, exp       1 flop each (the oracle's own log/exp bodies are not counted operation by
//                  operation: a transcendental is one algorithmic operation)
//   comparisons, fabs, fmin/fmax, negation, conversions: 0 (not floating-point arithmetic).
// The C library's log and pow are used only for operator constants (the indicator threshold) and
// are not counted.  Counting is single-threaded: run the oracle with nthreads = 1.
//
// Layout: cdouble has the size, alignment and calling convention of double (one SSE-class member),
// so the oracle's extern "C" entry points keep their ABI and take the same numpy buffers.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

struct OpCounts {
    uint64_t add, mul, div, sqrt, log, exp;
};
static OpCounts g_ops = {0, 0, 0, 0, 0, 0};
static int g_ops_off = 0;   // > 0 inside the oracle's own log/exp bodies

struct cdouble {
    double v;
    cdouble() = default;
    constexpr cdouble(double x) : v(x) {}
    template <class T, class = std::enable_if_t<std::is_integral_v<T>>>
    constexpr cdouble(T x) : v((double)x) {}
    template <class T, class = std::enable_if_t<std::is_arithmetic_v<T>>>
    explicit constexpr operator T() const { return (T)v; }
    cdouble& operator+=(cdouble b);
    cdouble& operator-=(cdouble b);
    cdouble& operator*=(cdouble b);
    cdouble& operator/=(cdouble b);
};
static_assert(sizeof(cdouble) == sizeof(double) && alignof(cdouble) == alignof(double), "cdouble layout");

inline cdouble operator+(cdouble a, cdouble b) { if (!g_ops_off) g_ops.add++; return cdouble(a.v + b.v); }
inline cdouble operator-(cdouble a, cdouble b) { if (!g_ops_off) g_ops.add++; return cdouble(a.v - b.v); }
inline cdouble operator*(cdouble a, cdouble b) { if (!g_ops_off) g_ops.mul++; return cdouble(a.v * b.v); }
inline cdouble operator/(cdouble a, cdouble b) { if (!g_ops_off) g_ops.div++; return cdouble(a.v / b.v); }
inline cdouble operator-(cdouble a) { return cdouble(-a.v); }
inline cdouble operator+(cdouble a) { return a; }
inline cdouble& cdouble::operator+=(cdouble b) { return *this = *this + b; }
inline cdouble& cdouble::operator-=(cdouble b) { return *this = *this - b; }
inline cdouble& cdouble::operator*=(cdouble b) { return *this = *this * b; }
inline cdouble& cdouble::operator/=(cdouble b) { return *this = *this / b; }
inline bool operator<(cdouble a, cdouble b) { return a.v < b.v; }
inline bool operator>(cdouble a, cdouble b) { return a.v > b.v; }
inline bool operator<=(cdouble a, cdouble b) { return a.v <= b.v; }
inline bool operator>=(cdouble a, cdouble b) { return a.v >= b.v; }
inline bool operator==(cdouble a, cdouble b) { return a.v == b.v; }
inline bool operator!=(cdouble a, cdouble b) { return a.v != b.v; }

namespace std {
inline cdouble sqrt(cdouble x) { if (!g_ops_off) g_ops.sqrt++; return cdouble(std::sqrt(x.v)); }
inline cdouble fabs(cdouble x) { return cdouble(std::fabs(x.v)); }
inline cdouble fmin(cdouble a, cdouble b) { return cdouble(std::fmin(a.v, b.v)); }
inline cdouble fmax(cdouble a, cdouble b) { return cdouble(std::fmax(a.v, b.v)); }
inline cdouble min(cdouble a, cdouble b) { return (b < a) ? b : a; }
inline cdouble max(cdouble a, cdouble b) { return (a < b) ? b : a; }
inline cdouble nearbyint(cdouble x) { return cdouble(std::nearbyint(x.v)); }
inline cdouble cos(cdouble x) { return cdouble(std::cos(x.v)); }
inline cdouble atan(cdouble x) { return cdouble(std::atan(x.v)); }
inline cdouble log(cdouble x) { return cdouble(std::log(x.v)); }
inline cdouble pow(cdouble a, cdouble b) { return cdouble(std::pow(a.v, b.v)); }
inline bool isinf(cdouble x) { return std::isinf(x.v); }
}  // namespace std

// The oracle's own log/exp: one counted operation each, their bodies uncounted.
struct OpCountTranscendental {
    explicit OpCountTranscendental(uint64_t& c) { if (!g_ops_off) c++; ++g_ops_off; }
    ~OpCountTranscendental() { --g_ops_off; }
};
#define ORACLE_COUNT_LOG() OpCountTranscendental oracle_count_guard_(g_ops.log)
#define ORACLE_COUNT_EXP() OpCountTranscendental oracle_count_guard_(g_ops.exp)

#define double cdouble
#include "nemo_oracle.cpp"
#undef double

extern "C" {

void or_opcount_reset(void) { g_ops = OpCounts{0, 0, 0, 0, 0, 0}; }

// out[6] = additions/subtractions, multiplications, divisions, square roots, logs, exps
void or_opcount_read(uint64_t* out) {
    out[0] = g_ops.add;
    out[1] = g_ops.mul;
    out[2] = g_ops.div;
    out[3] = g_ops.sqrt;
    out[4] = g_ops.log;
    out[5] = g_ops.exp;
}

}  // extern "C"
