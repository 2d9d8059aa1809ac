// oracle_scalar.hpp - scalar types for the CPU oracle (test infrastructure only).
//
// The oracle's restatement of the reference hot path is a template over a
// scalar type S.  Three instantiations are used:
//   double     the FP64 oracle (parity baseline),
//   Dual<N>    forward-mode tangents, the dual-number gradient reference,
//   OpCount    counts the algorithmic operations of one formula iteration.
// Nothing outside tests/, the smoke check and bench.py's CPU baseline may use
// the oracle.
#pragma once
#include <cmath>
#include <cstdint>

namespace oracle {

// ---- value access ---------------------------------------------------------
inline double val(double x) { return x; }

// ---- forward-mode dual number with N tangents ------------------------------
template <int N>
struct Dual {
  double v;
  double d[N];
  Dual() : v(0.0) { for (int i = 0; i < N; i++) d[i] = 0.0; }
  Dual(double x) : v(x) { for (int i = 0; i < N; i++) d[i] = 0.0; }  // NOLINT implicit
  static Dual seed(double x, int k) { Dual r(x); if (k >= 0 && k < N) r.d[k] = 1.0; return r; }
};
template <int N> inline double val(const Dual<N> &x) { return x.v; }

#define DUAL_BINOP(OP, VEXPR, DEXPR)                                                 \
  template <int N> inline Dual<N> operator OP(const Dual<N> &a, const Dual<N> &b) {  \
    Dual<N> r; r.v = VEXPR; for (int i = 0; i < N; i++) r.d[i] = DEXPR; return r; }  \
  template <int N> inline Dual<N> operator OP(const Dual<N> &a, double bv) {          \
    Dual<N> b(bv); return a OP b; }                                                   \
  template <int N> inline Dual<N> operator OP(double av, const Dual<N> &b) {          \
    Dual<N> a(av); return a OP b; }
DUAL_BINOP(+, a.v + b.v, a.d[i] + b.d[i])
DUAL_BINOP(-, a.v - b.v, a.d[i] - b.d[i])
DUAL_BINOP(*, a.v * b.v, a.d[i] * b.v + a.v * b.d[i])
DUAL_BINOP(/, a.v / b.v, (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v))
#undef DUAL_BINOP
template <int N> inline Dual<N> operator-(const Dual<N> &a) {
  Dual<N> r; r.v = -a.v; for (int i = 0; i < N; i++) r.d[i] = -a.d[i]; return r; }
template <int N, class T> inline Dual<N> &operator+=(Dual<N> &a, const T &b) { a = a + b; return a; }
template <int N, class T> inline Dual<N> &operator-=(Dual<N> &a, const T &b) { a = a - b; return a; }
template <int N, class T> inline Dual<N> &operator*=(Dual<N> &a, const T &b) { a = a * b; return a; }
#define DUAL_CMP(OP)                                                                     \
  template <int N> inline bool operator OP(const Dual<N> &a, const Dual<N> &b) { return a.v OP b.v; } \
  template <int N> inline bool operator OP(const Dual<N> &a, double b) { return a.v OP b; }        \
  template <int N> inline bool operator OP(double a, const Dual<N> &b) { return a OP b.v; }
DUAL_CMP(<) DUAL_CMP(>) DUAL_CMP(<=) DUAL_CMP(>=) DUAL_CMP(==) DUAL_CMP(!=)
#undef DUAL_CMP

template <int N, class F>
inline Dual<N> dual_apply(const Dual<N> &a, double fv, double dfa) {
  Dual<N> r; r.v = fv; for (int i = 0; i < N; i++) r.d[i] = dfa * a.d[i]; return r; }
template <int N> inline Dual<N> sqrt(const Dual<N> &a) {
  double s = std::sqrt(a.v); return dual_apply<N, void>(a, s, s > 0 ? 0.5 / s : 0.0); }
template <int N> inline Dual<N> fabs(const Dual<N> &a) {
  return a.v < 0 ? -a : a; }
template <int N> inline Dual<N> sin(const Dual<N> &a) { return dual_apply<N, void>(a, std::sin(a.v), std::cos(a.v)); }
template <int N> inline Dual<N> cos(const Dual<N> &a) { return dual_apply<N, void>(a, std::cos(a.v), -std::sin(a.v)); }
template <int N> inline Dual<N> log(const Dual<N> &a) { return dual_apply<N, void>(a, std::log(a.v), 1.0 / a.v); }
template <int N> inline Dual<N> asin(const Dual<N> &a) {
  return dual_apply<N, void>(a, std::asin(a.v), 1.0 / std::sqrt(1.0 - a.v * a.v)); }
template <int N> inline Dual<N> acos(const Dual<N> &a) {
  return dual_apply<N, void>(a, std::acos(a.v), -1.0 / std::sqrt(1.0 - a.v * a.v)); }
template <int N> inline Dual<N> atan2(const Dual<N> &y, const Dual<N> &x) {
  Dual<N> r; r.v = std::atan2(y.v, x.v); double q = x.v * x.v + y.v * y.v;
  for (int i = 0; i < N; i++) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / q; return r; }
template <int N> inline Dual<N> pow(const Dual<N> &a, const Dual<N> &b) {
  // d(a^b) = b a^(b-1) da + a^b ln(a) db
  Dual<N> r; r.v = std::pow(a.v, b.v);
  double da = b.v * std::pow(a.v, b.v - 1.0);
  double db = a.v > 0 ? r.v * std::log(a.v) : 0.0;
  for (int i = 0; i < N; i++) r.d[i] = da * a.d[i] + db * b.d[i]; return r; }
template <int N> inline bool isfinite(const Dual<N> &a) { return std::isfinite(a.v); }

// ---- operation counter -------------------------------------------------------
// Counts operations as performed.  `essential` counts exclude operations with
// a structural-zero operand: a constant 0 (the unused 4-D component w when the
// initial w is 0, a zero Mandelbox offset) - work an implementation can skip
// without changing any result.  z0 marks such a value.
struct OpTally {
  uint64_t add = 0, mul = 0, div = 0, sqrt = 0, transc = 0, cmp = 0;
  uint64_t e_add = 0, e_mul = 0;  // essential adds / muls
};
extern thread_local OpTally g_tally;

struct OpCount {
  double v;
  bool z0;
  OpCount() : v(0.0), z0(true) {}
  OpCount(double x) : v(x), z0(x == 0.0) {}  // NOLINT implicit: constants
  static OpCount computed(double x) { OpCount r(x); r.z0 = false; return r; }
};
inline double val(const OpCount &x) { return x.v; }
inline OpCount add_op(OpCount a, OpCount b, double v) {
  g_tally.add++;
  if (a.z0 && b.z0) return OpCount(v);
  if (a.z0 || b.z0) { OpCount r = OpCount::computed(v); return r; }
  g_tally.e_add++;
  return OpCount::computed(v);
}
inline OpCount mul_op(OpCount a, OpCount b, double v) {
  g_tally.mul++;
  if (a.z0 || b.z0) return OpCount(v);  // structural zero result
  g_tally.e_mul++;
  return OpCount::computed(v);
}
inline OpCount operator+(OpCount a, OpCount b) { return add_op(a, b, a.v + b.v); }
inline OpCount operator-(OpCount a, OpCount b) { return add_op(a, b, a.v - b.v); }
inline OpCount operator*(OpCount a, OpCount b) { return mul_op(a, b, a.v * b.v); }
inline OpCount operator/(OpCount a, OpCount b) { g_tally.div++; return OpCount::computed(a.v / b.v); }
inline OpCount operator-(OpCount a) { OpCount r = a; r.v = -a.v; return r; }
inline OpCount operator+(OpCount a, double b) { return a + OpCount(b); }
inline OpCount operator-(OpCount a, double b) { return a - OpCount(b); }
inline OpCount operator*(OpCount a, double b) { return a * OpCount(b); }
inline OpCount operator/(OpCount a, double b) { return a / OpCount(b); }
inline OpCount operator+(double a, OpCount b) { return OpCount(a) + b; }
inline OpCount operator-(double a, OpCount b) { return OpCount(a) - b; }
inline OpCount operator*(double a, OpCount b) { return OpCount(a) * b; }
inline OpCount operator/(double a, OpCount b) { return OpCount(a) / b; }
template <class T> inline OpCount &operator+=(OpCount &a, const T &b) { a = a + b; return a; }
template <class T> inline OpCount &operator-=(OpCount &a, const T &b) { a = a - b; return a; }
template <class T> inline OpCount &operator*=(OpCount &a, const T &b) { a = a * b; return a; }
#define OPC_CMP(OP)                                                                          \
  inline bool operator OP(OpCount a, OpCount b) { g_tally.cmp++; return a.v OP b.v; }        \
  inline bool operator OP(OpCount a, double b) { g_tally.cmp++; return a.v OP b; }           \
  inline bool operator OP(double a, OpCount b) { g_tally.cmp++; return a OP b.v; }
OPC_CMP(<) OPC_CMP(>) OPC_CMP(<=) OPC_CMP(>=) OPC_CMP(==) OPC_CMP(!=)
#undef OPC_CMP
inline OpCount sqrt(OpCount a) { g_tally.sqrt++; return OpCount::computed(std::sqrt(a.v)); }
inline OpCount fabs(OpCount a) { OpCount r = a; r.v = std::fabs(a.v); return r; }
inline OpCount sin(OpCount a) { g_tally.transc++; return OpCount::computed(std::sin(a.v)); }
inline OpCount cos(OpCount a) { g_tally.transc++; return OpCount::computed(std::cos(a.v)); }
inline OpCount log(OpCount a) { g_tally.transc++; return OpCount::computed(std::log(a.v)); }
inline OpCount asin(OpCount a) { g_tally.transc++; return OpCount::computed(std::asin(a.v)); }
inline OpCount acos(OpCount a) { g_tally.transc++; return OpCount::computed(std::acos(a.v)); }
inline OpCount atan2(OpCount y, OpCount x) { g_tally.transc++; return OpCount::computed(std::atan2(y.v, x.v)); }
inline OpCount pow(OpCount a, OpCount b) { g_tally.transc++; return OpCount::computed(std::pow(a.v, b.v)); }
inline bool isfinite(OpCount a) { return std::isfinite(a.v); }

}  // namespace oracle
