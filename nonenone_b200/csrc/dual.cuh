// dual.cuh -- one-direction forward-mode dual numbers.
//
// The reference linearises the Natural residual with dense forward AD: every
// scalar carries its value and B derivatives (ad/include/ad/Evaluation.hpp,
// ad/include/ad/Math.hpp).  On the GPU each lane of a cell's group carries one
// direction instead -- value plus the derivative along one primary unknown --
// so a B-wide block column comes out of B lanes running the same code.  The
// value/derivative rules below follow the reference's, including its rounding
// choices (a Dual divided by a plain number multiplies by the reciprocal,
// Evaluation.hpp:462-470), so values and derivatives agree to rounding.
#pragma once

#include "eos.cuh"

namespace nz
{

struct Dual
{
    double v;   // value
    double d;   // derivative along the lane's direction

    NZ_BOTH Dual() : v(0.0), d(0.0) {}
    NZ_BOTH Dual(double value) : v(value), d(0.0) {}
    NZ_BOTH Dual(double value, double deriv) : v(value), d(deriv) {}
};

NZ_BOTH double val(double x) { return x; }
NZ_BOTH double val(const Dual &x) { return x.v; }
NZ_BOTH double der(double) { return 0.0; }
NZ_BOTH double der(const Dual &x) { return x.d; }
NZ_BOTH void clearDer(double &) {}
NZ_BOTH void clearDer(Dual &x) { x.d = 0.0; }
// A primary unknown: seeded with derivative 1 along the lane's direction.
template <class S>
NZ_BOTH S makeSeeded(double value);
template <>
NZ_BOTH double makeSeeded<double>(double value) { return value; }
template <>
NZ_BOTH Dual makeSeeded<Dual>(double value) { return Dual(value, 1.0); }

NZ_BOTH Dual operator-(const Dual &a) { return Dual(-a.v, -a.d); }
NZ_BOTH Dual operator+(const Dual &a, const Dual &b) { return Dual(a.v + b.v, a.d + b.d); }
NZ_BOTH Dual operator+(const Dual &a, double b) { return Dual(a.v + b, a.d); }
NZ_BOTH Dual operator+(double a, const Dual &b) { return Dual(b.v + a, b.d); }
NZ_BOTH Dual operator-(const Dual &a, const Dual &b) { return Dual(a.v - b.v, a.d - b.d); }
NZ_BOTH Dual operator-(const Dual &a, double b) { return Dual(a.v - b, a.d); }
NZ_BOTH Dual operator-(double a, const Dual &b) { return Dual(-b.v + a, -b.d); }
// product rule as Evaluation::operator*= (u' v + v' u)
NZ_BOTH Dual operator*(const Dual &a, const Dual &b) { return Dual(a.v * b.v, a.d * b.v + b.d * a.v); }
NZ_BOTH Dual operator*(const Dual &a, double b) { return Dual(a.v * b, a.d * b); }
NZ_BOTH Dual operator*(double a, const Dual &b) { return Dual(b.v * a, b.d * a); }
// quotient rule as Evaluation::operator/= ((v u' - u v') / v^2)
NZ_BOTH Dual operator/(const Dual &a, const Dual &b)
{
    return Dual(a.v / b.v, (b.v * a.d - a.v * b.d) / (b.v * b.v));
}
NZ_BOTH Dual operator/(const Dual &a, double b)
{
    const double r = 1.0 / b;
    return Dual(a.v * r, a.d * r);
}
NZ_BOTH Dual operator/(double a, const Dual &b)
{
    return Dual(a / b.v, (b.v * 0.0 - a * b.d) / (b.v * b.v));
}
NZ_BOTH Dual &operator+=(Dual &a, const Dual &b)
{
    a.v += b.v;
    a.d += b.d;
    return a;
}
NZ_BOTH Dual &operator+=(Dual &a, double b)
{
    a.v += b;
    return a;
}
NZ_BOTH Dual &operator-=(Dual &a, const Dual &b)
{
    a.v -= b.v;
    a.d -= b.d;
    return a;
}

// Plain-double overloads in this namespace, so templates over double / Dual
// find an exact match instead of converting a double to a Dual.
NZ_BOTH double sqrt(double x) { return ::sqrt(x); }
NZ_BOTH double exp(double x) { return ::exp(x); }
NZ_BOTH double log(double x) { return ::log(x); }
NZ_BOTH double pow(double x, double p) { return ::pow(x, p); }
NZ_BOTH double acos(double x) { return ::acos(x); }
NZ_BOTH double cos(double x) { return ::cos(x); }

// Math.hpp rules
NZ_BOTH Dual sqrt(const Dual &x)
{
    const double s = ::sqrt(x.v);
    return Dual(s, (0.5 / s) * x.d);
}
NZ_BOTH Dual exp(const Dual &x)
{
    const double e = ::exp(x.v);
    return Dual(e, e * x.d);
}
NZ_BOTH Dual log(const Dual &x) { return Dual(::log(x.v), (1.0 / x.v) * x.d); }
NZ_BOTH Dual pow(const Dual &x, double p)
{
    if (p == 0.0)
        return Dual(::pow(x.v, p), 0.0);
    return Dual(::pow(x.v, p), (p * ::pow(x.v, p - 1.0)) * x.d);
}
NZ_BOTH Dual acos(const Dual &x) { return Dual(::acos(x.v), (-1.0 / ::sqrt(1.0 - x.v * x.v)) * x.d); }
NZ_BOTH Dual cos(const Dual &x) { return Dual(::cos(x.v), (-::sin(x.v)) * x.d); }
NZ_BOTH Dual abs(const Dual &x) { return (x.v >= 0.0) ? x : -x; }
NZ_BOTH double abs(double x) { return ::fabs(x); }

// K-direction dual number: the value and the derivatives along K of the
// cell's primary unknowns, so one lane carries K columns of a Jacobian block
// and a cell needs ceil(B / K) lanes instead of B -- the value path, which
// each lane recomputes, runs B / K times fewer per cell.  Every derivative
// component follows exactly the one-direction rule of Dual above.
template <int K>
struct DualN
{
    double v;
    double d[K];

    NZ_BOTH DualN() : v(0.0)
    {
#pragma unroll
        for (int j = 0; j < K; ++j)
            d[j] = 0.0;
    }
    NZ_BOTH DualN(double value) : v(value)
    {
#pragma unroll
        for (int j = 0; j < K; ++j)
            d[j] = 0.0;
    }
};

template <int K>
NZ_BOTH double val(const DualN<K> &x) { return x.v; }
template <int K>
NZ_BOTH void clearDer(DualN<K> &x)
{
#pragma unroll
    for (int j = 0; j < K; ++j)
        x.d[j] = 0.0;
}

// A primary unknown of index `idx` for a lane whose directions start at
// `k` (k >= 0; a Dual lane has the one direction k): Seed<S>::at(value, idx, k).
template <class S>
struct Seed;
template <>
struct Seed<double>
{
    NZ_BOTH static double at(double value, int, int) { return value; }
};
template <>
struct Seed<Dual>
{
    NZ_BOTH static Dual at(double value, int idx, int k) { return idx == k ? Dual(value, 1.0) : Dual(value); }
};
template <int K>
struct Seed<DualN<K>>
{
    NZ_BOTH static DualN<K> at(double value, int idx, int k)
    {
        DualN<K> r(value);
#pragma unroll
        for (int j = 0; j < K; ++j)
            r.d[j] = idx == k + j ? 1.0 : 0.0;
        return r;
    }
};

#define NZ_DUALN_BINARY(OP, VALUE, DERIV)                                                \
    template <int K>                                                                     \
    NZ_BOTH DualN<K> operator OP(const DualN<K> &a, const DualN<K> &b)                   \
    {                                                                                    \
        DualN<K> r;                                                                      \
        r.v = VALUE;                                                                     \
        _Pragma("unroll") for (int j = 0; j < K; ++j) r.d[j] = DERIV;                    \
        return r;                                                                        \
    }
NZ_DUALN_BINARY(+, a.v + b.v, a.d[j] + b.d[j])
NZ_DUALN_BINARY(-, a.v - b.v, a.d[j] - b.d[j])
NZ_DUALN_BINARY(*, a.v * b.v, a.d[j] * b.v + b.d[j] * a.v)
NZ_DUALN_BINARY(/, a.v / b.v, (b.v * a.d[j] - a.v * b.d[j]) / (b.v * b.v))
#undef NZ_DUALN_BINARY

template <int K>
NZ_BOTH DualN<K> operator-(const DualN<K> &a)
{
    DualN<K> r;
    r.v = -a.v;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = -a.d[j];
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator+(const DualN<K> &a, double b)
{
    DualN<K> r = a;
    r.v = a.v + b;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator+(double a, const DualN<K> &b)
{
    DualN<K> r = b;
    r.v = b.v + a;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator-(const DualN<K> &a, double b)
{
    DualN<K> r = a;
    r.v = a.v - b;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator-(double a, const DualN<K> &b)
{
    DualN<K> r;
    r.v = -b.v + a;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = -b.d[j];
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator*(const DualN<K> &a, double b)
{
    DualN<K> r;
    r.v = a.v * b;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = a.d[j] * b;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator*(double a, const DualN<K> &b)
{
    DualN<K> r;
    r.v = b.v * a;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = b.d[j] * a;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator/(const DualN<K> &a, double b)
{
    const double q = 1.0 / b;
    DualN<K> r;
    r.v = a.v * q;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = a.d[j] * q;
    return r;
}
template <int K>
NZ_BOTH DualN<K> operator/(double a, const DualN<K> &b)
{
    DualN<K> r;
    r.v = a / b.v;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = (b.v * 0.0 - a * b.d[j]) / (b.v * b.v);
    return r;
}
template <int K>
NZ_BOTH DualN<K> &operator+=(DualN<K> &a, const DualN<K> &b)
{
    a.v += b.v;
#pragma unroll
    for (int j = 0; j < K; ++j)
        a.d[j] += b.d[j];
    return a;
}
template <int K>
NZ_BOTH DualN<K> &operator+=(DualN<K> &a, double b)
{
    a.v += b;
    return a;
}
template <int K>
NZ_BOTH DualN<K> &operator-=(DualN<K> &a, const DualN<K> &b)
{
    a.v -= b.v;
#pragma unroll
    for (int j = 0; j < K; ++j)
        a.d[j] -= b.d[j];
    return a;
}
// f(x) with f' given: the same scalar factor as Dual's rules, times each direction
template <int K>
NZ_BOTH DualN<K> chainN(double value, double factor, const DualN<K> &x)
{
    DualN<K> r;
    r.v = value;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = factor * x.d[j];
    return r;
}
template <int K>
NZ_BOTH DualN<K> sqrt(const DualN<K> &x)
{
    const double s = ::sqrt(x.v);
    return chainN(s, 0.5 / s, x);
}
template <int K>
NZ_BOTH DualN<K> exp(const DualN<K> &x)
{
    const double e = ::exp(x.v);
    DualN<K> r;
    r.v = e;
#pragma unroll
    for (int j = 0; j < K; ++j)
        r.d[j] = e * x.d[j];
    return r;
}
template <int K>
NZ_BOTH DualN<K> log(const DualN<K> &x) { return chainN(::log(x.v), 1.0 / x.v, x); }
template <int K>
NZ_BOTH DualN<K> pow(const DualN<K> &x, double p)
{
    if (p == 0.0)
        return DualN<K>(::pow(x.v, p));
    return chainN(::pow(x.v, p), p * ::pow(x.v, p - 1.0), x);
}
template <int K>
NZ_BOTH DualN<K> acos(const DualN<K> &x) { return chainN(::acos(x.v), -1.0 / ::sqrt(1.0 - x.v * x.v), x); }
template <int K>
NZ_BOTH DualN<K> cos(const DualN<K> &x) { return chainN(::cos(x.v), -::sin(x.v), x); }
template <int K>
NZ_BOTH DualN<K> abs(const DualN<K> &x) { return (x.v >= 0.0) ? x : -x; }

// Value-only scalar with the AD type's rounding.  The reference evaluates cell
// properties and local residuals in its AD type even when only values are
// used (the residual's cell cache), so value kernels use this type to round
// the same way: its only difference from double is that division by a plain
// number multiplies by the reciprocal.
struct Val
{
    double v;
    NZ_BOTH Val() : v(0.0) {}
    NZ_BOTH Val(double value) : v(value) {}
};

NZ_BOTH double val(const Val &x) { return x.v; }
NZ_BOTH double der(const Val &) { return 0.0; }
NZ_BOTH void clearDer(Val &) {}
template <>
NZ_BOTH Val makeSeeded<Val>(double value) { return Val(value); }
template <>
struct Seed<Val>
{
    NZ_BOTH static Val at(double value, int, int) { return Val(value); }
};

NZ_BOTH Val operator-(const Val &a) { return Val(-a.v); }
NZ_BOTH Val operator+(const Val &a, const Val &b) { return Val(a.v + b.v); }
NZ_BOTH Val operator+(const Val &a, double b) { return Val(a.v + b); }
NZ_BOTH Val operator+(double a, const Val &b) { return Val(b.v + a); }
NZ_BOTH Val operator-(const Val &a, const Val &b) { return Val(a.v - b.v); }
NZ_BOTH Val operator-(const Val &a, double b) { return Val(a.v - b); }
NZ_BOTH Val operator-(double a, const Val &b) { return Val(-b.v + a); }
NZ_BOTH Val operator*(const Val &a, const Val &b) { return Val(a.v * b.v); }
NZ_BOTH Val operator*(const Val &a, double b) { return Val(a.v * b); }
NZ_BOTH Val operator*(double a, const Val &b) { return Val(b.v * a); }
NZ_BOTH Val operator/(const Val &a, const Val &b) { return Val(a.v / b.v); }
NZ_BOTH Val operator/(const Val &a, double b) { return Val(a.v * (1.0 / b)); }
NZ_BOTH Val operator/(double a, const Val &b) { return Val(a / b.v); }
NZ_BOTH Val &operator+=(Val &a, const Val &b)
{
    a.v += b.v;
    return a;
}
NZ_BOTH Val &operator+=(Val &a, double b)
{
    a.v += b;
    return a;
}
NZ_BOTH Val &operator-=(Val &a, const Val &b)
{
    a.v -= b.v;
    return a;
}
NZ_BOTH Val sqrt(const Val &x) { return Val(::sqrt(x.v)); }
NZ_BOTH Val exp(const Val &x) { return Val(::exp(x.v)); }
NZ_BOTH Val log(const Val &x) { return Val(::log(x.v)); }
NZ_BOTH Val pow(const Val &x, double p) { return Val(::pow(x.v, p)); }
NZ_BOTH Val acos(const Val &x) { return Val(::acos(x.v)); }
NZ_BOTH Val cos(const Val &x) { return Val(::cos(x.v)); }
NZ_BOTH Val abs(const Val &x) { return (x.v >= 0.0) ? x : -x; }

} // namespace nz
