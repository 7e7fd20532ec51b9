// Minimal complex arithmetic for the SIE kernels (FP64 and FP32), usable on the
// host and the device.  Complex values are stored interleaved (re, im) so device
// arrays are plain double2 / float2 streams.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

template <typename T>
struct cx {
  T re, im;
};
typedef cx<double> zc;  // complex128
typedef cx<float> cc;   // complex64

#define SIE_HD __host__ __device__ __forceinline__

template <typename T>
SIE_HD cx<T> mk(T r, T i) {
  cx<T> z;
  z.re = r;
  z.im = i;
  return z;
}
template <typename T>
SIE_HD cx<T> operator+(cx<T> a, cx<T> b) { return mk<T>(a.re + b.re, a.im + b.im); }
template <typename T>
SIE_HD cx<T> operator-(cx<T> a, cx<T> b) { return mk<T>(a.re - b.re, a.im - b.im); }
template <typename T>
SIE_HD cx<T> operator-(cx<T> a) { return mk<T>(-a.re, -a.im); }
template <typename T>
SIE_HD cx<T> operator*(cx<T> a, cx<T> b) {
  return mk<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
SIE_HD cx<T> operator*(cx<T> a, T s) { return mk<T>(a.re * s, a.im * s); }
template <typename T>
SIE_HD cx<T> operator*(T s, cx<T> a) { return mk<T>(a.re * s, a.im * s); }
template <typename T>
SIE_HD cx<T>& operator+=(cx<T>& a, cx<T> b) {
  a.re += b.re;
  a.im += b.im;
  return a;
}
template <typename T>
SIE_HD cx<T>& operator-=(cx<T>& a, cx<T> b) {
  a.re -= b.re;
  a.im -= b.im;
  return a;
}
template <typename T>
SIE_HD cx<T> conj(cx<T> a) { return mk<T>(a.re, -a.im); }
template <typename T>
SIE_HD cx<T> operator/(cx<T> a, cx<T> b) {
  // Smith's algorithm
  if (fabs(b.re) >= fabs(b.im)) {
    T r = b.im / b.re, d = b.re + b.im * r;
    return mk<T>((a.re + a.im * r) / d, (a.im - a.re * r) / d);
  } else {
    T r = b.re / b.im, d = b.re * r + b.im;
    return mk<T>((a.re * r + a.im) / d, (a.im * r - a.re) / d);
  }
}
template <typename T>
SIE_HD cx<T> operator/(cx<T> a, T s) { return mk<T>(a.re / s, a.im / s); }
template <typename T>
SIE_HD T cabs2(cx<T> a) { return a.re * a.re + a.im * a.im; }
// a*b + c
template <typename T>
SIE_HD cx<T> cfma(cx<T> a, cx<T> b, cx<T> c) {
  return mk<T>(fma(a.re, b.re, fma(-a.im, b.im, c.re)), fma(a.re, b.im, fma(a.im, b.re, c.im)));
}
// conj(a)*b + c
template <typename T>
SIE_HD cx<T> cfma_conj(cx<T> a, cx<T> b, cx<T> c) {
  return mk<T>(fma(a.re, b.re, fma(a.im, b.im, c.re)), fma(a.re, b.im, fma(-a.im, b.re, c.im)));
}

// Loads of data that is streamed once per product (near panels, radiation patterns):
// marked evict-first in L2 and not kept in L1, so they do not push the level
// coefficients, which the translation kernels re-read many times, out of L2.
__device__ __forceinline__ unsigned long long l2_evict_first_policy() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ cx<double> ld_stream(const cx<double>* a, unsigned long long pol) {
  double r, i;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n"
               : "=d"(r), "=d"(i)
               : "l"(a), "l"(pol));
  return mk<double>(r, i);
}
// Loads of data re-read from L2 many times (the SR's level coefficients): evict-last.
__device__ __forceinline__ unsigned long long l2_evict_last_policy() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ cx<double> ld_keep(const cx<double>* a, unsigned long long pol) {
  double r, i;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;\n"
               : "=d"(r), "=d"(i)
               : "l"(a), "l"(pol));
  return mk<double>(r, i);
}
// Stores of results read once later (the SR's D): streaming, evict-first.
__device__ __forceinline__ void st_stream(cx<double>* a, cx<double> v) {
  asm volatile("st.global.cs.v2.f64 [%0], {%1, %2};\n" ::"l"(a), "d"(v.re), "d"(v.im) : "memory");
}
// complex64 streams: a plain load measured faster (8-byte accesses)
__device__ __forceinline__ cx<float> ld_stream(const cx<float>* a, unsigned long long) { return *a; }

// widen to complex128
SIE_HD zc cvt_z(zc a) { return a; }
SIE_HD zc cvt_z(cc a) { return mk<double>((double)a.re, (double)a.im); }

// exp(i * t) for real t
SIE_HD zc cexpi(double t) {
  double s, c;
  sincos(t, &s, &c);
  return mk<double>(c, s);
}
SIE_HD cc cexpi(float t) {
  float s, c;
  sincosf(t, &s, &c);
  return mk<float>(c, s);
}
// exp(z)
SIE_HD zc cexp(zc z) {
  double s, c;
  sincos(z.im, &s, &c);
  double e = exp(z.re);
  return mk<double>(e * c, e * s);
}
SIE_HD cc cexp(cc z) {
  float s, c;
  sincosf(z.im, &s, &c);
  float e = expf(z.re);
  return mk<float>(e * c, e * s);
}
// exp(-i k t) for complex k and real t:  exp(Im(k) t) * exp(-i Re(k) t)
SIE_HD zc cexp_mik(zc k, double t) {
  double s, c;
  sincos(-k.re * t, &s, &c);
  double e = exp(k.im * t);
  return mk<double>(e * c, e * s);
}
SIE_HD cc cexp_mik(cc k, float t) {
  float s, c;
  sincosf(-k.re * t, &s, &c);
  float e = expf(k.im * t);
  return mk<float>(e * c, e * s);
}

template <typename T>
struct v3t {
  T x, y, z;
};
typedef v3t<double> vd;
typedef v3t<float> vf;
template <typename T>
SIE_HD v3t<T> mkv(T a, T b, T c) {
  v3t<T> v;
  v.x = a;
  v.y = b;
  v.z = c;
  return v;
}
template <typename T>
SIE_HD v3t<T> operator+(v3t<T> a, v3t<T> b) { return mkv<T>(a.x + b.x, a.y + b.y, a.z + b.z); }
template <typename T>
SIE_HD v3t<T> operator-(v3t<T> a, v3t<T> b) { return mkv<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T>
SIE_HD v3t<T> operator*(v3t<T> a, T s) { return mkv<T>(a.x * s, a.y * s, a.z * s); }
template <typename T>
SIE_HD v3t<T> operator/(v3t<T> a, T s) { return mkv<T>(a.x / s, a.y / s, a.z / s); }
template <typename T>
SIE_HD T dot(v3t<T> a, v3t<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename T>
SIE_HD v3t<T> cross(v3t<T> a, v3t<T> b) {
  return mkv<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T>
SIE_HD T vlen(v3t<T> a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

// complex 3-vectors
template <typename T>
struct c3t {
  cx<T> x, y, z;
};
typedef c3t<double> zv;
template <typename T>
SIE_HD c3t<T> c3zero() {
  c3t<T> r;
  r.x = r.y = r.z = mk<T>(0, 0);
  return r;
}
template <typename T>
SIE_HD c3t<T> operator+(c3t<T> a, c3t<T> b) {
  c3t<T> r;
  r.x = a.x + b.x;
  r.y = a.y + b.y;
  r.z = a.z + b.z;
  return r;
}
template <typename T>
SIE_HD c3t<T> operator*(v3t<T> a, cx<T> s) {
  c3t<T> r;
  r.x = s * a.x;
  r.y = s * a.y;
  r.z = s * a.z;
  return r;
}
template <typename T>
SIE_HD c3t<T> operator*(c3t<T> a, cx<T> s) {
  c3t<T> r;
  r.x = a.x * s;
  r.y = a.y * s;
  r.z = a.z * s;
  return r;
}
template <typename T>
SIE_HD cx<T> rdot(v3t<T> a, c3t<T> b) { return b.x * a.x + b.y * a.y + b.z * a.z; }
