// fft3.cuh -- register DFTs of small lengths with compile-time twiddles.
//
// RD<T2, R, SG>::run(v) replaces v[0..R) (natural order) by its DFT
//   X[k] = sum_n v[n] exp(SG * 2 pi i n k / R)      (SG = -1 forward, +1 inverse)
// in natural order.  Lengths 2, 3, 4, 8 use the butterflies of fft_ct.cuh;
// 6, 12, 16, 24 are four-step compositions R = R1 R2 whose twiddles are
// constants computed by the compiler (Taylor series of cos and sin of the
// angle reduced to the first octant, exact at multiples of pi/2), so no
// table is read.
#pragma once
#include <type_traits>

#include "fft_ct.cuh"

namespace ct {

constexpr double kPi3 = 3.14159265358979323846264338327950288;

// Taylor series of cos and sin for |x| <= pi/4, where every term is below
// 0.31 in magnitude: the sums are within about one ulp
__host__ __device__ constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; ++n) {
    term *= -x * x / ((2.0 * n - 1.0) * (2.0 * n));
    sum += term;
  }
  return sum;
}
__host__ __device__ constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 14; ++n) {
    term *= -x * x / ((2.0 * n) * (2.0 * n + 1.0));
    sum += term;
  }
  return sum;
}
// cos (c = true) or sin of 2 pi e / R: the angle is brought to the first
// octant with integer arithmetic, 8 e = o R + r, theta = (pi/4)(o + r/R) =
// q pi/2 + s t with t = (pi/4) r/R (o even, s = +1) or (pi/4)(R - r)/R (o
// odd, s = -1) and q = (o + (o odd)) / 2; then cos(q pi/2 + s t) and
// sin(q pi/2 + s t) are +-cos t or +-sin t
__host__ __device__ constexpr double cs2pi(int e, int R, bool c) {
  long k = 8L * (((long)e % R + R) % R);
  const int o = (int)(k / R);
  const long r = k - (long)o * R;
  const bool odd = o % 2 != 0;
  const double t = (kPi3 / 4.0) * ((double)(odd ? R - r : r) / (double)R);
  const double ct = taylor_cos(t), st = odd ? -taylor_sin(t) : taylor_sin(t);
  switch (((o + (odd ? 1 : 0)) / 2) % 4) {
    case 0: return c ? ct : st;
    case 1: return c ? -st : ct;
    case 2: return c ? -ct : -st;
    default: return c ? st : -ct;
  }
}
__host__ __device__ constexpr double cos2pi(int e, int R) { return cs2pi(e, R, true); }
__host__ __device__ constexpr double sin2pi(int e, int R) { return cs2pi(e, R, false); }

// compile-time loop: f(std::integral_constant<int, I>) for I in [B, E)
template <int B, int E, typename F>
__device__ __forceinline__ void sfor(F&& f) {
  if constexpr (B < E) {
    f(std::integral_constant<int, B>{});
    sfor<B + 1, E>(f);
  }
}

// z * exp(SG * 2 pi i E / R)
template <typename T2, int R, int E, int SG>
__device__ __forceinline__ T2 twc(T2 z) {
  typedef typename CT<T2>::R Rt;
  constexpr int e = ((E % R) + R) % R;
  if constexpr (e == 0) {
    return z;
  } else if constexpr (4 * e == R) {
    return mul_si(z, SG);
  } else if constexpr (2 * e == R) {
    return CT<T2>::mk(-z.x, -z.y);
  } else if constexpr (4 * e == 3 * R) {
    return mul_si(z, -SG);
  } else {
    constexpr Rt c = (Rt)cos2pi(e, R);
    constexpr Rt s = (Rt)(SG * sin2pi(e, R));
    return CT<T2>::mk(z.x * c - z.y * s, z.x * s + z.y * c);
  }
}

template <typename T2, int R, int SG>
struct RD;

// R = R1 R2: n = n2 + R2 n1, k = k1 + R1 k2
template <typename T2, int R1, int R2, int SG>
__device__ __forceinline__ void comp_dft(T2 (&v)[R1 * R2]) {
  T2 t[R1 * R2];
  sfor<0, R2>([&](auto n2c) {
    constexpr int n2 = decltype(n2c)::value;
    T2 a[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) a[n1] = v[n2 + R2 * n1];
    RD<T2, R1, SG>::run(a);
    sfor<0, R1>([&](auto k1c) {
      constexpr int k1 = decltype(k1c)::value;
      t[k1 * R2 + n2] = twc<T2, R1 * R2, n2 * k1, SG>(a[k1]);
    });
  });
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    T2 b[R2];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) b[n2] = t[k1 * R2 + n2];
    RD<T2, R2, SG>::run(b);
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = b[k2];
  }
}

template <typename T2, int SG>
struct RD<T2, 1, SG> {
  static __device__ __forceinline__ void run(T2 (&)[1]) {}
};
template <typename T2, int SG>
struct RD<T2, 2, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[2]) { Dft<T2, 2>::run(v, SG); }
};
template <typename T2, int SG>
struct RD<T2, 3, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[3]) { Dft<T2, 3>::run(v, SG); }
};
template <typename T2, int SG>
struct RD<T2, 4, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[4]) { Dft<T2, 4>::run(v, SG); }
};
template <typename T2, int SG>
struct RD<T2, 8, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[8]) { Dft<T2, 8>::run(v, SG); }
};
template <typename T2, int SG>
struct RD<T2, 6, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[6]) { comp_dft<T2, 2, 3, SG>(v); }
};
template <typename T2, int SG>
struct RD<T2, 12, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[12]) { comp_dft<T2, 4, 3, SG>(v); }
};
template <typename T2, int SG>
struct RD<T2, 16, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[16]) { comp_dft<T2, 4, 4, SG>(v); }
};
template <typename T2, int SG>
struct RD<T2, 24, SG> {
  static __device__ __forceinline__ void run(T2 (&v)[24]) { comp_dft<T2, 8, 3, SG>(v); }
};

// Two-step split of a length N = R1 R2 on one column of a shared-memory
// slab (element n at col[n * stride]): n = n2 + R2 n1, k = k1 + R1 k2, and
// max(R1, R2) threads per column.  Step 1, thread h = n2 < R2: the R1-point
// DFT over n1 of x[h + R2 n1], times W_N^(SG h k1) (tw[e] = exp(-2 pi i e /
// N)), written back over the same R1 slots, at h + R2 k1.  Step 2 (after a
// barrier), thread h = k1 < R1: the R2-point DFT over n2 of the slots R2 h ..
// R2 h + R2 - 1, which is X[h + R1 k2] in v[k2].  Two shared-memory passes
// instead of one per radix pass, and the results leave from registers.
template <int R1, int R2, int SG>
__device__ __forceinline__ void dft2_step1(double2* col, int stride, int h, const double2* __restrict__ tw) {
  if (h >= R2) return;
  double2 v[R1];
#pragma unroll
  for (int n1 = 0; n1 < R1; ++n1) v[n1] = col[(h + R2 * n1) * stride];
  RD<double2, R1, SG>::run(v);
  col[h * stride] = v[0];
#pragma unroll
  for (int k1 = 1; k1 < R1; ++k1) {
    double2 w = __ldg(tw + h * k1);
    if (SG > 0) w.y = -w.y;
    col[(h + R2 * k1) * stride] = mul(v[k1], w);
  }
}
template <int R1, int R2, int SG>
__device__ __forceinline__ void dft2_step2(const double2* col, int stride, int h, double2 (&v)[R2]) {
  if (h >= R1) return;
#pragma unroll
  for (int n2 = 0; n2 < R2; ++n2) v[n2] = col[(n2 + R2 * h) * stride];
  RD<double2, R2, SG>::run(v);
}
// the first factor of the two-step split of the radial lengths with a
// compile-time transform (0: radix passes)
__host__ __device__ constexpr int split2_r1(int n) {
  return n == 16 ? 4 : n == 32 ? 8 : n == 48 ? 12 : n == 64 ? 8 : n == 96 ? 12 : n == 128 ? 16 : n == 192 ? 16
       : n == 256 ? 16 : 0;
}
__host__ __device__ constexpr int split2_tpc(int n) {  // threads per column
  return split2_r1(n) == 0 ? 0 : (split2_r1(n) > n / split2_r1(n) ? split2_r1(n) : n / split2_r1(n));
}

// Three-step split of a phi length N = A M, M = B C: A = 16, B the
// power-of-two part of M capped at 16, C the rest.
__host__ __device__ constexpr int pow2_part_cap16(int m) {
  int b = 1;
  while (b < 16 && m % (2 * b) == 0) b *= 2;
  return b;
}

}  // namespace ct
