// ad_tape.hpp -- reverse-mode automatic differentiation by operator
// overloading (a Wengert list / tape).  TEST INFRASTRUCTURE ONLY.
//
// Every arithmetic operation on an adouble whose operands depend on an
// independent variable appends one entry to a global tape: the indices of its
// (at most two) operands and the partial derivatives with respect to them,
// evaluated in IEEE double at the operation.  A reverse sweep over the tape
// then propagates d(output)/d(entry) from the output back to the independent
// variables (the adjoint of the recorded computation).  Values are computed
// exactly as plain doubles would be, so the recorded forward is the double
// computation itself.  Comparisons look at values only (control flow is not
// differentiated).  Single-threaded.
#pragma once
#include <climits>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <vector>

namespace adt {

struct Entry {
    int32_t a, b;     // operand indices (0: a constant, never propagated)
    double da, db;    // partial derivatives
};

struct Tape {
    std::vector<Entry> e;
    Tape() { e.push_back({0, 0, 0.0, 0.0}); }   // index 0: the constant sink
    int64_t push(int64_t a, double da, int64_t b, double db)
    {
        if (e.size() >= (size_t)INT32_MAX) throw std::length_error("tape longer than 2^31 entries");
        e.push_back({(int32_t)a, (int32_t)b, da, db});
        return (int64_t)e.size() - 1;
    }
    void clear()
    {
        e.clear();
        e.push_back({0, 0, 0.0, 0.0});
    }
};

inline Tape &tape()
{
    static Tape t;
    return t;
}

struct adouble {
    double v;
    int64_t i;   // tape index; 0 = constant
    adouble() : v(0.0), i(0) {}
    adouble(double x) : v(x), i(0) {}
    adouble(int x) : v((double)x), i(0) {}
    adouble(long x) : v((double)x), i(0) {}
    adouble(long long x) : v((double)x), i(0) {}
    adouble(unsigned x) : v((double)x), i(0) {}
    explicit operator double() const { return v; }
    explicit operator int() const { return (int)v; }
    explicit operator long() const { return (long)v; }
    explicit operator long long() const { return (long long)v; }
    adouble &operator+=(const adouble &o);
    adouble &operator-=(const adouble &o);
    adouble &operator*=(const adouble &o);
    adouble &operator/=(const adouble &o);
};

// a new independent variable
inline adouble variable(double x)
{
    adouble r(x);
    r.i = tape().push(0, 0.0, 0, 0.0);
    return r;
}

inline adouble mk(double v, int64_t a, double da, int64_t b, double db)
{
    adouble r(v);
    if (a || b) r.i = tape().push(a, da, b, db);
    return r;
}

inline adouble operator+(const adouble &x, const adouble &y) { return mk(x.v + y.v, x.i, 1.0, y.i, 1.0); }
inline adouble operator-(const adouble &x, const adouble &y) { return mk(x.v - y.v, x.i, 1.0, y.i, -1.0); }
inline adouble operator*(const adouble &x, const adouble &y) { return mk(x.v * y.v, x.i, y.v, y.i, x.v); }
inline adouble operator/(const adouble &x, const adouble &y)
{
    const double q = x.v / y.v;
    return mk(q, x.i, 1.0 / y.v, y.i, -q / y.v);
}
inline adouble operator-(const adouble &x) { return mk(-x.v, x.i, -1.0, 0, 0.0); }
inline adouble operator+(const adouble &x) { return x; }
inline adouble &adouble::operator+=(const adouble &o) { return *this = *this + o; }
inline adouble &adouble::operator-=(const adouble &o) { return *this = *this - o; }
inline adouble &adouble::operator*=(const adouble &o) { return *this = *this * o; }
inline adouble &adouble::operator/=(const adouble &o) { return *this = *this / o; }

inline bool operator<(const adouble &x, const adouble &y) { return x.v < y.v; }
inline bool operator>(const adouble &x, const adouble &y) { return x.v > y.v; }
inline bool operator<=(const adouble &x, const adouble &y) { return x.v <= y.v; }
inline bool operator>=(const adouble &x, const adouble &y) { return x.v >= y.v; }
inline bool operator==(const adouble &x, const adouble &y) { return x.v == y.v; }
inline bool operator!=(const adouble &x, const adouble &y) { return x.v != y.v; }

inline adouble fabs(const adouble &x) { return mk(std::fabs(x.v), x.i, x.v < 0 ? -1.0 : 1.0, 0, 0.0); }
inline adouble sqrt(const adouble &x)
{
    const double s = std::sqrt(x.v);
    return mk(s, x.i, s > 0 ? 0.5 / s : 0.0, 0, 0.0);
}

// adjoints of every tape entry given d(output)/d(output) = 1
inline std::vector<double> reverse(const adouble &out)
{
    const auto &e = tape().e;
    std::vector<double> adj(e.size(), 0.0);
    if (!out.i) return adj;
    adj[out.i] = 1.0;
    for (int64_t k = (int64_t)e.size() - 1; k > 0; k--) {
        const double a = adj[k];
        if (a == 0.0) continue;
        const Entry &t = e[k];
        if (t.a) adj[t.a] += a * t.da;
        if (t.b) adj[t.b] += a * t.db;
    }
    return adj;
}

} // namespace adt
