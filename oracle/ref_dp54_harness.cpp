// ref_dp54_harness.cpp -- TEST INFRASTRUCTURE: drives the reference's own
// Dormand-Prince 5(4) integrator (the third overload of
// Tortoise::Algorithms::dormandPrince54, include/Generics/Algorithms/
// DormandPrince54.hpp:479-665, compiled from the reference tree where it lies;
// the header needs no Eigen or TBB) with callbacks for the right-hand side,
// enforceValue, the normalised error and the step vetoer.  The tests plug in
// the oracle's restated operators, so the same problem runs once through the
// reference's integrator and once through the oracle's restatement of it
// (dp54_core), and the two must take the same steps and give the same dense
// outputs.  Built by `make -C oracle ref` into oracle/_ref/ only when the
// reference tree is present; nothing in the product links it.
#include <stdint.h>

#include <algorithm>
#include <cassert>
#include <cmath>
#include <iostream>
#include <vector>

#include "Generics/Algorithms/DormandPrince54.hpp"

namespace {

// The state: elementwise +, - and scalar *, each operation rounded on its
// own (no fused multiply-adds: the harness is built with -ffp-contract=off),
// which is how the reference's containers evaluate the stage expressions.
struct Vec {
    std::vector<double> v;
};

Vec operator+(const Vec& a, const Vec& b) {
    Vec r{a.v};
    for (size_t i = 0; i < r.v.size(); ++i) r.v[i] = a.v[i] + b.v[i];
    return r;
}

Vec operator-(const Vec& a, const Vec& b) {
    Vec r{a.v};
    for (size_t i = 0; i < r.v.size(); ++i) r.v[i] = a.v[i] - b.v[i];
    return r;
}

Vec operator*(double s, const Vec& a) {
    Vec r{a.v};
    for (size_t i = 0; i < r.v.size(); ++i) r.v[i] = s * a.v[i];
    return r;
}

// The time container the integrator appends its dense outputs to.
struct Series {
    using ArgType = double;
    using ValType = Vec;
    std::vector<double> t;
    std::vector<Vec> y;
    bool empty() const { return t.empty(); }
    Vec& back() { return y.back(); }
    double argback() const { return t.back(); }
    void emplace_back(double tt, const Vec& yy) {
        t.push_back(tt);
        y.push_back(yy);
    }
};

}  // namespace

extern "C" {

typedef void (*ref_rhs_fn)(void* user, double t, const double* y, double* out);
typedef void (*ref_enforce_fn)(void* user, double t, double* y);
typedef double (*ref_norm_fn)(void* user, const double* err, const double* y);
typedef double (*ref_veto_fn)(void* user, const double* times, int n_times, double dense_step);

// Integrates y' = rhs(t, y) from (t0, y0) to tf with dense output every
// dense_step through the reference's dormandPrince54.  stats: attempts,
// accepted, rejected, right-hand sides.  Returns the number of dense outputs
// (all of them; at most max_dense are copied).
int64_t ref_dp54(int64_t n, const double* y0, double t0, double tf, double dense_step, ref_rhs_fn rhs,
                 ref_enforce_fn enforce, ref_norm_fn norm, ref_veto_fn veto, void* user, double* dense_out,
                 double* dense_t, int64_t max_dense, int64_t* stats) {
    Series s;
    s.emplace_back(t0, Vec{std::vector<double>(y0, y0 + n)});
    int64_t attempts = 0, accepted = 0, rhs_evals = 0;
    auto time_op = [&](double t, const Vec& y) {
        Vec out{std::vector<double>(size_t(n))};
        rhs(user, t, y.v.data(), out.v.data());
        ++rhs_evals;
        return out;
    };
    auto enforce_value = [&](double t, const Vec& y) {
        Vec r{y.v};
        enforce(user, t, r.v.data());
        return r;
    };
    auto norm_error = [&](const Vec& err, const Vec& y) {
        const double e = norm(user, err.v.data(), y.v.data());
        ++attempts;
        if (e <= 1.) ++accepted;
        return e;
    };
    auto output = [](double, const Vec&) {};
    auto vetoer = [&](std::vector<double> times, double dense) {
        return veto(user, times.data(), int(times.size()), dense);
    };
    // (the integrator reports every attempt on std::cout)
    Tortoise::Algorithms::dormandPrince54(s, tf, dense_step, time_op, enforce_value, norm_error, output, vetoer);
    std::cout.flush();
    const int64_t nd = int64_t(s.t.size()) - 1;
    for (int64_t i = 0; i < nd && i < max_dense; ++i) {
        dense_t[i] = s.t[size_t(i) + 1];
        std::copy(s.y[size_t(i) + 1].v.begin(), s.y[size_t(i) + 1].v.end(), dense_out + i * n);
    }
    stats[0] = attempts;
    stats[1] = accepted;
    stats[2] = attempts - accepted;
    stats[3] = rhs_evals;
    return nd;
}

}  // extern "C"
