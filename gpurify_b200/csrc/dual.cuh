// Forward-mode dual numbers (value + directional derivative) for the
// geometric sensitivities: the panel integrals, centroids, areas and
// Chebyshev weights are evaluated on Dual inputs x + eps * dx/dp, and the eps
// part of the result is the exact derivative of the same floating-point
// formula along the parameter's vertex velocity field.
#pragma once
#include <cmath>

namespace gpx {

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double x) : v(x), d(0.0) {}
    __host__ __device__ Dual(double x, double dx) : v(x), d(dx) {}
    // Elementary functions as hidden friends: found only by argument-dependent
    // lookup on Dual arguments, so calls on double in this namespace still
    // resolve to the CUDA math library.
    friend __host__ __device__ inline Dual sqrt(Dual a) {
        const double s = ::sqrt(a.v);
        return {s, s > 0.0 ? a.d / (2.0 * s) : 0.0};
    }
    friend __host__ __device__ inline Dual log1p(Dual a) { return {::log1p(a.v), a.d / (1.0 + a.v)}; }
    friend __host__ __device__ inline Dual atan(Dual a) { return {::atan(a.v), a.d / (1.0 + a.v * a.v)}; }
    friend __host__ __device__ inline Dual fabs(Dual a) { return a.v < 0.0 ? Dual{-a.v, -a.d} : a; }
};

__host__ __device__ inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__host__ __device__ inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__host__ __device__ inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
__host__ __device__ inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__host__ __device__ inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
__host__ __device__ inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__host__ __device__ inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__host__ __device__ inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__host__ __device__ inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__host__ __device__ inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__host__ __device__ inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__host__ __device__ inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__host__ __device__ inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
__host__ __device__ inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
__host__ __device__ inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }

__host__ __device__ inline bool operator<(Dual a, double b) { return a.v < b; }
__host__ __device__ inline bool operator>(Dual a, double b) { return a.v > b; }
__host__ __device__ inline bool operator>=(Dual a, double b) { return a.v >= b; }
__host__ __device__ inline bool operator<=(Dual a, double b) { return a.v <= b; }
__host__ __device__ inline bool operator==(Dual a, double b) { return a.v == b; }
__host__ __device__ inline bool operator!=(Dual a, double b) { return a.v != b; }

// Value and derivative parts for the generic code paths.
__host__ __device__ inline double value_of(double x) { return x; }
__host__ __device__ inline double value_of(Dual x) { return x.v; }

}  // namespace gpx
