// opcount.cpp -- op-counting build of the oracle.
//
// TEST INFRASTRUCTURE ONLY (like liberi_oracle.c, which it compiles): the
// oracle's quartet arithmetic -- Rys roots and weights (Boys-moment rules of
// the rotated-axis classes, RYSDS + RYSGW of the Rys classes), vertical and
// horizontal recurrences, assembly, and DIRFCK digestion -- is compiled with
// a scalar type that counts floating-point operations: add, subtract,
// multiply and divide one each, exp, sqrt, acos and cos one each (no fused
// multiply-add is formed; negation, fabs and comparisons are free).  The
// counts per class, split into primitive-quartet and shell-quartet work,
// come back in oracle_counts.ops and give the per-class constants of the
// roofline numerator (oracle/make_flop_constants.py).
#include <cmath>
#include <cstdint>

namespace opc {
thread_local uint64_t g_ops = 0, g_mark = 0;

struct Counted {
    double v;
    Counted() : v(0.0) {}
    Counted(double x) : v(x) {}
    explicit operator double() const { return v; }
    Counted &operator+=(Counted o) { ++g_ops; v += o.v; return *this; }
    Counted &operator-=(Counted o) { ++g_ops; v -= o.v; return *this; }
    Counted &operator*=(Counted o) { ++g_ops; v *= o.v; return *this; }
    Counted &operator/=(Counted o) { ++g_ops; v /= o.v; return *this; }
};
inline Counted operator+(Counted a, Counted b) { ++g_ops; return Counted(a.v + b.v); }
inline Counted operator-(Counted a, Counted b) { ++g_ops; return Counted(a.v - b.v); }
inline Counted operator*(Counted a, Counted b) { ++g_ops; return Counted(a.v * b.v); }
inline Counted operator/(Counted a, Counted b) { ++g_ops; return Counted(a.v / b.v); }
inline Counted operator-(Counted a) { return Counted(-a.v); }
inline bool operator<(Counted a, Counted b) { return a.v < b.v; }
inline bool operator>(Counted a, Counted b) { return a.v > b.v; }
inline bool operator<=(Counted a, Counted b) { return a.v <= b.v; }
inline bool operator>=(Counted a, Counted b) { return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { return a.v != b.v; }
inline Counted exp(Counted a) { ++g_ops; return Counted(std::exp(a.v)); }
inline Counted expl(Counted a) { ++g_ops; return Counted(std::exp(a.v)); }
inline Counted sqrt(Counted a) { ++g_ops; return Counted(std::sqrt(a.v)); }
inline Counted sqrtl(Counted a) { ++g_ops; return Counted(std::sqrt(a.v)); }
inline Counted acosl(Counted a) { ++g_ops; return Counted(std::acos(a.v)); }
inline Counted cosl(Counted a) { ++g_ops; return Counted(std::cos(a.v)); }
inline Counted fabs(Counted a) { return Counted(std::fabs(a.v)); }
}  // namespace opc

#define ORACLE_REAL opc::Counted
#define ORACLE_REALL opc::Counted
#define ORACLE_OPS() (opc::g_ops)
#define ORACLE_MARK() (opc::g_mark = opc::g_ops)
#define ORACLE_MARKED() (opc::g_mark)

extern "C" {
#include "liberi_oracle.c"
}
