// ref_gauss_harness.cpp -- TEST INFRASTRUCTURE: the reference's Gauss
// quadrature constants (include/Geometry/GeometryCore/GaussQuadratureConst.hpp,
// compiled from the reference tree where it lies) read out through a C ABI,
// so the tests can check the values the oracle and the CUDA library use
// against the reference's own.  The header only needs the ArrayPoint type of
// Point.hpp (an Eigen fixed-size matrix, filled by brace or comma
// initialisation); a minimal stand-in with those two initialisations is
// given here, so neither Eigen nor anything else of the reference is needed.
// Built by `make -C oracle ref` into oracle/_ref/ when the reference tree is
// present; nothing in the product links it.
#include <initializer_list>

namespace Tortoise {

// D x N values, row-major fill as Eigen's comma initialiser does.
template <int D, int N>
struct ArrayPoint {
    double a[D][N] = {};
    ArrayPoint() {}
    ArrayPoint(std::initializer_list<double> l) {
        int k = 0;
        for (double v : l) { a[k / N][k % N] = v; ++k; }
    }
    struct Comma {
        ArrayPoint* p;
        int k;
        Comma& operator,(double v) {
            p->a[k / N][k % N] = v;
            ++k;
            return *this;
        }
    };
    Comma operator<<(double v) {
        a[0][0] = v;
        return Comma{this, 1};
    }
};

}  // namespace Tortoise

#include "Geometry/GeometryCore/GaussQuadratureConst.hpp"

extern "C" {

// The order-2 rule on the reference triangle: points (x, y) of its three
// nodes and their weights.
void ref_gauss_triangle_order2(double* points, double* weights) {
    using namespace Tortoise::GeometryCore;
    for (int q = 0; q < 3; ++q) {
        points[2 * q] = gaussPoints<2, 2>.a[0][q];
        points[2 * q + 1] = gaussPoints<2, 2>.a[1][q];
        weights[q] = gaussWeigths<2, 2>.a[0][q];
    }
}

// The order-2 rule on [0, 1].
void ref_gauss_interval_order2(double* points, double* weights) {
    using namespace Tortoise::GeometryCore;
    for (int q = 0; q < 2; ++q) {
        points[q] = gaussPoints<1, 2>.a[0][q];
        weights[q] = gaussWeigths<1, 2>.a[0][q];
    }
}

}  // extern "C"
