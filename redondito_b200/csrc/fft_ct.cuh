// fft_ct.cuh -- shared-memory FFTs with the length fixed at compile time.
//
// The same in-place decimation-in-frequency / decimation-in-time scheme as
// fft_engine.cuh (frequency k at position rev[k] after fft_dif), but with
// the radix sequence, spans and butterfly indices known to the compiler, so
// no runtime divisions are left in the passes, and with twiddles read from
// a per-pass table laid out [pass][j][r-1] = W_L^{j r} (L = R*s the pass's
// block length), so the R-1 factors of one butterfly are contiguous and
// neighbouring butterflies read neighbouring entries.
//
// Radix order (host and device agree): 8 while the remaining length is a
// multiple of 8, else 4, else 2, else 3.  Lengths of the form 2^a 3^b fit.
#pragma once
#include "fft_engine.cuh"

namespace ct {

__host__ __device__ constexpr int radix_of(int n) {
  return n % 8 == 0 ? 8 : n % 4 == 0 ? 4 : n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n;
}
// number of twiddle entries used by the passes that start at block length L
__host__ __device__ constexpr int tw_entries(int L) {
  return L <= 1 ? 0 : (L / radix_of(L)) * (radix_of(L) - 1) + tw_entries(L / radix_of(L));
}
__host__ __device__ constexpr bool supported(int n) {
  return n <= 1 ? true : (radix_of(n) <= 8 ? supported(n / radix_of(n)) : false);
}

template <typename T2>
struct CT;
template <>
struct CT<double2> {
  typedef double R;
  static __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
};
template <>
struct CT<float2> {
  typedef float R;
  static __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
};

template <typename T2>
__device__ __forceinline__ T2 add(T2 a, T2 b) { return CT<T2>::mk(a.x + b.x, a.y + b.y); }
template <typename T2>
__device__ __forceinline__ T2 sub(T2 a, T2 b) { return CT<T2>::mk(a.x - b.x, a.y - b.y); }
template <typename T2>
__device__ __forceinline__ T2 mul(T2 a, T2 b) {
  return CT<T2>::mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T2>
__device__ __forceinline__ T2 mul_si(T2 a, int sign) {  // (sign * i) a
  return sign > 0 ? CT<T2>::mk(-a.y, a.x) : CT<T2>::mk(a.y, -a.x);
}

template <typename T2, int R>
struct Dft;
template <typename T2>
struct Dft<T2, 2> {
  static __device__ __forceinline__ void run(T2 (&v)[2], int) {
    T2 a = v[0], b = v[1];
    v[0] = add(a, b);
    v[1] = sub(a, b);
  }
};
template <typename T2>
struct Dft<T2, 4> {
  static __device__ __forceinline__ void run(T2 (&v)[4], int sign) {
    T2 s02 = add(v[0], v[2]), d02 = sub(v[0], v[2]);
    T2 s13 = add(v[1], v[3]), d13 = mul_si(sub(v[1], v[3]), sign);
    v[0] = add(s02, s13);
    v[1] = add(d02, d13);
    v[2] = sub(s02, s13);
    v[3] = sub(d02, d13);
  }
};
template <typename T2>
struct Dft<T2, 8> {
  static __device__ __forceinline__ void run(T2 (&v)[8], int sign) {
    typedef typename CT<T2>::R Rt;
    const Rt h = (Rt)0.70710678118654752440084436210485;
    T2 e[4] = {v[0], v[2], v[4], v[6]};
    T2 o[4] = {v[1], v[3], v[5], v[7]};
    Dft<T2, 4>::run(e, sign);
    Dft<T2, 4>::run(o, sign);
    T2 o1 = o[1], o3 = o[3];
    T2 w1 = CT<T2>::mk(h * (o1.x - sign * o1.y), h * (o1.y + sign * o1.x));
    T2 w2 = mul_si(o[2], sign);
    T2 w3 = CT<T2>::mk(h * (-o3.x - sign * o3.y), h * (-o3.y + sign * o3.x));
    v[0] = add(e[0], o[0]);
    v[4] = sub(e[0], o[0]);
    v[1] = add(e[1], w1);
    v[5] = sub(e[1], w1);
    v[2] = add(e[2], w2);
    v[6] = sub(e[2], w2);
    v[3] = add(e[3], w3);
    v[7] = sub(e[3], w3);
  }
};
template <typename T2>
struct Dft<T2, 3> {
  static __device__ __forceinline__ void run(T2 (&v)[3], int sign) {
    typedef typename CT<T2>::R Rt;
    const Rt c = (Rt)0.86602540378443864676372317075294;
    T2 t = add(v[1], v[2]);
    T2 s = sub(v[1], v[2]);
    T2 a = CT<T2>::mk(v[0].x - (Rt)0.5 * t.x, v[0].y - (Rt)0.5 * t.y);
    T2 b = mul_si(CT<T2>::mk(c * s.x, c * s.y), sign);
    v[0] = add(v[0], t);
    v[1] = add(a, b);
    v[2] = sub(a, b);
  }
};

// Layout: element e of sequence b at buf[b*BS + E(e)*ES], E(e) = e + PAD*(e>>3).
// JFAST: consecutive threads take consecutive butterflies of one sequence.
template <int N, int PAD, bool JFAST>
struct Geo {
  int batch, bs, es;
  __device__ __forceinline__ int addr(int b, int e) const { return b * bs + (e + PAD * (e >> 3)) * es; }
};

template <typename T2>
__device__ __forceinline__ T2 twl(const T2* __restrict__ t, int sign) {
  T2 w = t[0];
  if (sign > 0) w.y = -w.y;
  return w;
}

// one pass, block length L, radix R = radix_of(L), span S = L/R
template <typename T2, int N, int L, bool DIT, int PAD, bool JFAST>
__device__ __forceinline__ void pass(T2* buf, const Geo<N, PAD, JFAST>& g, const T2* __restrict__ twp,
                                     int sign) {
  constexpr int R = radix_of(L), S = L / R, NQ = N / R;
  // twiddles of this pass start after those of the passes with longer blocks
  constexpr int TOFF = tw_entries(N) - tw_entries(L);
  const int nb = g.batch * NQ;
  for (int beta = threadIdx.x; beta < nb; beta += blockDim.x) {
    int b, q;
    if (JFAST) {
      b = beta / NQ;
      q = beta - b * NQ;
    } else {
      q = beta / g.batch;
      b = beta - q * g.batch;
    }
    const int blk = q / S, j = q - blk * S;
    const int e0 = blk * L + j;
    T2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[g.addr(b, e0 + r * S)];
    const T2* tw = twp + TOFF + j * (R - 1);
    if (DIT && S > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = mul(v[r], twl(tw + r - 1, sign));
    }
    Dft<T2, R>::run(v, sign);
    if (!DIT && S > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = mul(v[r], twl(tw + r - 1, sign));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) buf[g.addr(b, e0 + r * S)] = v[r];
  }
  __syncthreads();
}

// position of frequency k after dif<N> (the rev[] table, computed from the
// compile-time radix sequence): k = q0 + R0 (q1 + R1 (...)), pos = sum q_p s_p
template <int N, int L = N>
__host__ __device__ constexpr int rev_pos(int k) {
  constexpr int R = radix_of(L), S = L / R;
  if constexpr (S == 1) {
    return k;  // last digit, span 1
  } else {
    const int q = k % R;
    return q * S + rev_pos<N, S>(k / R);
  }
}

// Serial in-register decimation-in-frequency FFT of length R on v[R]
// (natural order in; frequency k out at v[rev_pos<R>(k)]), the same passes
// and twiddle table layout (pass_twiddles of length R) as the shared-memory
// version, every index known at compile time so v stays in registers.
template <typename T2, int R, int L = R>
__device__ __forceinline__ void reg_dif(T2 (&v)[R], const T2* __restrict__ twp, int sign) {
  constexpr int RR = radix_of(L), S = L / RR;
  constexpr int TOFF = tw_entries(R) - tw_entries(L);
#pragma unroll
  for (int blk = 0; blk < R / L; ++blk) {
#pragma unroll
    for (int j = 0; j < S; ++j) {
      T2 x[RR];
#pragma unroll
      for (int r = 0; r < RR; ++r) x[r] = v[blk * L + j + r * S];
      Dft<T2, RR>::run(x, sign);
      if constexpr (S > 1) {
#pragma unroll
        for (int r = 1; r < RR; ++r) x[r] = mul(x[r], twl(twp + TOFF + j * (RR - 1) + r - 1, sign));
      }
#pragma unroll
      for (int r = 0; r < RR; ++r) v[blk * L + j + r * S] = x[r];
    }
  }
  if constexpr (S > 1) reg_dif<T2, R, S>(v, twp, sign);
}

// Four-step split of a phi length N = N1 * N2 (N1 the power-of-two part,
// at most 32): N1-point DFTs over the stride-N2 subsequences, the twiddle
// W_N^(n2 k1), then N2-point DFTs; frequency k1 + N1 k2.
__host__ __device__ constexpr int split_n1(int n) {
  return n % 32 == 0 ? 32 : n % 16 == 0 ? 16 : n % 8 == 0 ? 8 : n % 4 == 0 ? 4 : n % 2 == 0 ? 2 : 1;
}

template <typename T2, int N, int L, int PAD, bool JFAST>
__device__ __forceinline__ void dif(T2* buf, const Geo<N, PAD, JFAST>& g, const T2* __restrict__ twp, int sign) {
  pass<T2, N, L, false>(buf, g, twp, sign);
  if constexpr (L / radix_of(L) > 1) dif<T2, N, L / radix_of(L)>(buf, g, twp, sign);
}

template <typename T2, int N, int L, int PAD, bool JFAST>
__device__ __forceinline__ void dit(T2* buf, const Geo<N, PAD, JFAST>& g, const T2* __restrict__ twp, int sign) {
  if constexpr (L / radix_of(L) > 1) dit<T2, N, L / radix_of(L)>(buf, g, twp, sign);
  pass<T2, N, L, true>(buf, g, twp, sign);
}

}  // namespace ct
