// Forward-mode dual numbers (value, directional derivative) for the pointwise
// functional code: instantiating a template written for double with Dual
// gives, in .d, the exact derivative of its result along the tangent carried
// by the inputs.  Used by the Hessian-vector product of the free energy: the
// directional derivative of dPhi/dn at the weighted densities of rho along
// the weighted densities of v.
#pragma once

struct Dual {
  double v, d;
  __host__ __device__ Dual(double value = 0.0, double deriv = 0.0) : v(value), d(deriv) {}
};

__device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator+(const Dual& a, double b) { return Dual(a.v + b, a.d); }
__device__ __forceinline__ Dual operator+(double a, const Dual& b) { return Dual(a + b.v, b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(const Dual& a, double b) { return Dual(a.v - b, a.d); }
__device__ __forceinline__ Dual operator-(double a, const Dual& b) { return Dual(a - b.v, -b.d); }
__device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
  return Dual(a.v * b.v, a.d * b.v + a.v * b.d);
}
__device__ __forceinline__ Dual operator*(const Dual& a, double b) { return Dual(a.v * b, a.d * b); }
__device__ __forceinline__ Dual operator*(double a, const Dual& b) { return Dual(a * b.v, a * b.d); }
__device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual operator/(const Dual& a, double b) { return Dual(a.v / b, a.d / b); }
__device__ __forceinline__ Dual operator/(double a, const Dual& b) {
  const double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
__device__ __forceinline__ Dual& operator+=(Dual& a, const Dual& b) { a = a + b; return a; }
__device__ __forceinline__ Dual& operator-=(Dual& a, const Dual& b) { a = a - b; return a; }
__device__ __forceinline__ Dual& operator*=(Dual& a, const Dual& b) { a = a * b; return a; }
__device__ __forceinline__ bool operator<=(const Dual& a, double b) { return a.v <= b; }
__device__ __forceinline__ Dual log(const Dual& a) { return Dual(::log(a.v), a.d / a.v); }
__device__ __forceinline__ Dual exp(const Dual& a) {
  const double e = ::exp(a.v);
  return Dual(e, e * a.d);
}
// clipping: the derivative of the selected branch (0 where the bound is taken)
__device__ __forceinline__ Dual fmin(const Dual& a, double b) { return (a.v <= b) ? a : Dual(b, 0.0); }
__device__ __forceinline__ Dual fmax(const Dual& a, double b) { return (a.v >= b) ? a : Dual(b, 0.0); }
