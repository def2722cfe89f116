// problems.cpp -- the three analytic test problems of the reference, selected at compile time
// with -DPROBLEM1 / -DPROBLEM2 / -DPROBLEM3 (default 1), as the reference's Makefile does
// (Makefile:28-32).  Each defines the link-time plug-ins Poisson::ufun (exact solution),
// ffun (its Laplacian, the right-hand side) and the first derivatives used as Neumann data
// (README "Test Problems"; include/problem_definition.h:8-18).
#include <cmath>

#include "problem_definition.h"

#if !defined(PROBLEM1) && !defined(PROBLEM2) && !defined(PROBLEM3)
#define PROBLEM1
#endif

namespace Poisson {
#if defined(PROBLEM1)
// u = sin(kx x) sin(ky y) sin(kz z), kx=3, ky=5.3, kz=-7.8
static const double KX = 3.0, KY = 5.3, KZ = -7.8;
double_t ufun(double_t x, double_t y, double_t z) { return sin(KX * x) * sin(KY * y) * sin(KZ * z); }
double_t ffun(double_t x, double_t y, double_t z) {
    return -(KX * KX + KY * KY + KZ * KZ) * sin(KX * x) * sin(KY * y) * sin(KZ * z);
}
double_t dudxfun(double_t x, double_t y, double_t z) { return KX * cos(KX * x) * sin(KY * y) * sin(KZ * z); }
double_t dudyfun(double_t x, double_t y, double_t z) { return KY * sin(KX * x) * cos(KY * y) * sin(KZ * z); }
double_t dudzfun(double_t x, double_t y, double_t z) { return KZ * sin(KX * x) * sin(KY * y) * cos(KZ * z); }
#elif defined(PROBLEM2)
// u = x^3 y^2 z
double_t ufun(double_t x, double_t y, double_t z) { return x * x * x * y * y * z; }
double_t ffun(double_t x, double_t y, double_t z) { return 2.0 * x * x * x * z + 6.0 * x * y * y * z; }
double_t dudxfun(double_t x, double_t y, double_t z) { return 3.0 * x * x * y * y * z; }
double_t dudyfun(double_t x, double_t y, double_t z) { return 2.0 * x * x * x * y * z; }
double_t dudzfun(double_t x, double_t y, double_t z) { return x * x * x * y * y; }
#else
// u = cos(x z^2) sin(y^3)
double_t ufun(double_t x, double_t y, double_t z) { return cos(x * z * z) * sin(y * y * y); }
double_t ffun(double_t x, double_t y, double_t z) {
    return ((-4.0 * x * x * z * z - 9.0 * y * y * y * y - z * z * z * z) * sin(y * y * y) + 6.0 * y * cos(y * y * y)) *
               cos(x * z * z) -
           2.0 * x * sin(x * z * z) * sin(y * y * y);
}
double_t dudxfun(double_t x, double_t y, double_t z) { return -z * z * sin(x * z * z) * sin(y * y * y); }
double_t dudyfun(double_t x, double_t y, double_t z) { return 3.0 * cos(x * z * z) * y * y * cos(y * y * y); }
double_t dudzfun(double_t x, double_t y, double_t z) { return -2 * x * z * sin(x * z * z) * sin(y * y * y); }
#endif
}  // namespace Poisson
