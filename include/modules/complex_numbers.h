// complex<T>: the complex type of the LaughlinEdge API (host and device).
//
// Drop-in for the reference's modules/complex_numbers.h: same free-function
// names (re, im, conj, norm, cabs, arg, clog, cexp, icpow, cpow) so user code
// written against the reference -- in particular excitation potentials such
// as [] __device__ (complex<float>* z) { ... re(z[i]) ... } -- compiles
// unchanged.  Layout: two consecutive T (x, y), so complex<float> aliases
// CUDA's float2 and the library's walker positions.  icpow(z, n) is the exact
// binary-powering product for every n >= 0 (the reference switches to a polar
// formula for n >= 3; both give z^n, this one without transcendentals).
#ifndef LAUGHLINEDGE_COMPLEX_NUMBERS_H
#define LAUGHLINEDGE_COMPLEX_NUMBERS_H

#include <cmath>

#if defined(__CUDACC__)
#define LEMC_HDI __host__ __device__ inline
#else
#define LEMC_HDI inline
#endif

template <typename T>
class complex {
 public:
  T x, y;
  LEMC_HDI complex() : x(0), y(0) {}
  LEMC_HDI complex(T r) : x(r), y(0) {}
  LEMC_HDI complex(T r, T i) : x(r), y(i) {}
  template <typename U>
  LEMC_HDI complex(const complex<U>& o) : x(T(o.x)), y(T(o.y)) {}

  LEMC_HDI T real() const { return x; }
  LEMC_HDI T imag() const { return y; }
  LEMC_HDI T* pointer_to_real() { return &x; }
  LEMC_HDI T* pointer_to_imag() { return &y; }

  LEMC_HDI complex& operator+=(const complex& o) { x += o.x; y += o.y; return *this; }
  LEMC_HDI complex& operator-=(const complex& o) { x -= o.x; y -= o.y; return *this; }
  LEMC_HDI complex& operator*=(const complex& o) {
    const T r = x * o.x - y * o.y;
    y = x * o.y + y * o.x;
    x = r;
    return *this;
  }
  LEMC_HDI complex& operator/=(const complex& o) {
    const T d = o.x * o.x + o.y * o.y;
    const T r = (x * o.x + y * o.y) / d;
    y = (y * o.x - x * o.y) / d;
    x = r;
    return *this;
  }
  LEMC_HDI complex& operator*=(T s) { x *= s; y *= s; return *this; }
  LEMC_HDI complex& operator/=(T s) { x /= s; y /= s; return *this; }

  LEMC_HDI friend complex operator+(complex a, const complex& b) { return a += b; }
  LEMC_HDI friend complex operator-(complex a, const complex& b) { return a -= b; }
  LEMC_HDI friend complex operator*(complex a, const complex& b) { return a *= b; }
  LEMC_HDI friend complex operator/(complex a, const complex& b) { return a /= b; }
  LEMC_HDI friend complex operator*(complex a, T s) { return a *= s; }
  LEMC_HDI friend complex operator*(T s, complex a) { return a *= s; }
  LEMC_HDI friend complex operator/(complex a, T s) { return a /= s; }
  LEMC_HDI friend complex operator-(const complex& a) { return complex(-a.x, -a.y); }
  LEMC_HDI friend bool operator==(const complex& a, const complex& b) { return a.x == b.x && a.y == b.y; }
  LEMC_HDI friend bool operator!=(const complex& a, const complex& b) { return !(a == b); }

  LEMC_HDI friend T re(const complex& z) { return z.x; }
  LEMC_HDI friend T im(const complex& z) { return z.y; }
  LEMC_HDI friend complex conj(const complex& z) { return complex(z.x, -z.y); }
  LEMC_HDI friend T norm(const complex& z) { return z.x * z.x + z.y * z.y; }
  LEMC_HDI friend T cabs(const complex& z) { return std::sqrt(z.x * z.x + z.y * z.y); }
  LEMC_HDI friend T arg(const complex& z) { return std::atan2(z.y, z.x); }
  LEMC_HDI friend complex clog(const complex& z) { return complex(std::log(cabs(z)), arg(z)); }
  LEMC_HDI friend complex cexp(const complex& z) {
    const T e = std::exp(z.x);
    return complex(e * std::cos(z.y), e * std::sin(z.y));
  }
  LEMC_HDI friend complex icpow(const complex& z, int n) {
    complex r(1), b = z;
    while (n > 0) {
      if (n & 1) r *= b;
      n >>= 1;
      if (n) b *= b;
    }
    return r;
  }
  LEMC_HDI friend complex cpow(const complex& z, const T& alpha) {
    const T th = arg(z) * alpha, m = std::pow(cabs(z), alpha);
    return complex(m * std::cos(th), m * std::sin(th));
  }
};

#endif
