// fft_engine.cuh -- batched complex FFTs held in shared memory.
//
// A CTA owns `batch` sequences of length n; element e of sequence b lives at
// buf[b*bs + E(e)*es] with E(e) = e + pad*(e >> 3) (pad = 1 skews short-stride
// passes across banks).  Transforms are in place, one CTA-wide barrier per
// pass, and each butterfly reads and writes the same R slots, so a thread
// holds only R values at a time:
//   fft_dif: natural-order input -> spectrum in digit-reversed order
//            (Sande-Tukey: butterfly, then twiddle);
//   fft_dit: digit-reversed input -> natural-order output
//            (Cooley-Tukey: twiddle, then butterfly; the passes of fft_dif
//             transposed and run in reverse).
// Frequency k sits at position rev[k] = sum_p q_p s_p, where
// k = q_0 + R_0 (q_1 + R_1 (q_2 + ...)) and s_p = n / (R_0 ... R_p).
// Callers read or write spectra through rev[], so no reordering pass runs.
#pragma once
#include "sph_internal.cuh"

struct FftGeom {
  int n, batch, bs, es, pad;
  bool jfast;  // true: consecutive threads walk one sequence; false: across sequences
  __device__ __forceinline__ int addr(int b, int e) const { return b * bs + (e + pad * (e >> 3)) * es; }
};

template <int R>
__device__ __forceinline__ void dft_reg(double2 (&v)[R], int sign);

template <>
__device__ __forceinline__ void dft_reg<2>(double2 (&v)[2], int) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <>
__device__ __forceinline__ void dft_reg<4>(double2 (&v)[4], int sign) {
  // W = exp(sign*2*pi*i/4) = sign*i
  double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
  double2 s13 = cadd(v[1], v[3]), d13 = cmul_si(csub(v[1], v[3]), sign);
  v[0] = cadd(s02, s13);
  v[1] = cadd(d02, d13);
  v[2] = csub(s02, s13);
  v[3] = csub(d02, d13);
}

template <>
__device__ __forceinline__ void dft_reg<8>(double2 (&v)[8], int sign) {
  const double h = 0.70710678118654752440084436210485;  // sqrt(1/2)
  double2 e[4] = {v[0], v[2], v[4], v[6]};
  double2 o[4] = {v[1], v[3], v[5], v[7]};
  dft_reg<4>(e, sign);
  dft_reg<4>(o, sign);
  // W8 = h (1 + sign i), W8^2 = sign i, W8^3 = h (-1 + sign i)
  double2 o1 = o[1], o3 = o[3];
  double2 w1 = make_double2(h * (o1.x - sign * o1.y), h * (o1.y + sign * o1.x));
  double2 w2 = cmul_si(o[2], sign);
  double2 w3 = make_double2(h * (-o3.x - sign * o3.y), h * (-o3.y + sign * o3.x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], w1);
  v[5] = csub(e[1], w1);
  v[2] = cadd(e[2], w2);
  v[6] = csub(e[2], w2);
  v[3] = cadd(e[3], w3);
  v[7] = csub(e[3], w3);
}

template <>
__device__ __forceinline__ void dft_reg<3>(double2 (&v)[3], int sign) {
  // W3 = -1/2 + sign i sqrt(3)/2
  const double c = 0.86602540378443864676372317075294;  // sqrt(3)/2
  double2 t = cadd(v[1], v[2]);
  double2 s = csub(v[1], v[2]);
  double2 a = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
  double2 b = cmul_si(make_double2(c * s.x, c * s.y), sign);
  v[0] = cadd(v[0], t);
  v[1] = cadd(a, b);
  v[2] = csub(a, b);
}

__device__ __forceinline__ double2 tw_load(const double2* __restrict__ tw, int e, int sign) {
  double2 w = __ldg(tw + e);
  if (sign > 0) w.y = -w.y;
  return w;
}

__device__ __forceinline__ void bfly_index(const FftGeom& g, int beta, int nq, int& b, int& q) {
  if (g.jfast) {
    b = beta / nq;
    q = beta - b * nq;
  } else {
    q = beta / g.batch;
    b = beta - q * g.batch;
  }
}

// One pass of span s (block length L = R*s).  DIT == false: butterfly then
// twiddle W_L^{j r}; DIT == true: twiddle then butterfly.
template <int R, bool DIT>
__device__ __forceinline__ void fft_pass(double2* buf, const FftGeom& g, int s,
                                         const double2* __restrict__ tw, int sign) {
  const int n = g.n, L = R * s, nq = n / R, nb = g.batch * nq, tstep = n / L;
  for (int beta = threadIdx.x; beta < nb; beta += blockDim.x) {
    int b, q;
    bfly_index(g, beta, nq, b, q);
    const int blk = q / s, j = q - blk * s;
    const int e0 = blk * L + j;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[g.addr(b, e0 + r * s)];
    if (DIT && j > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_load(tw, j * r * tstep, sign));
    }
    dft_reg<R>(v, sign);
    if (!DIT && j > 0) {
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw_load(tw, j * r * tstep, sign));
    }
#pragma unroll
    for (int r = 0; r < R; ++r) buf[g.addr(b, e0 + r * s)] = v[r];
  }
  __syncthreads();
}

// Any radix (odd primes >= 5): direct length-R DFT from a local array.
template <bool DIT>
__device__ __noinline__ void fft_pass_generic(double2* buf, const FftGeom& g, int R, int s,
                                              const double2* __restrict__ tw, int sign) {
  const int n = g.n, L = R * s, nq = n / R, nb = g.batch * nq, tstep = n / L, wR = n / R;
  double2 x[64], y[64];
  for (int beta = threadIdx.x; beta < nb; beta += blockDim.x) {
    int b, q;
    bfly_index(g, beta, nq, b, q);
    const int blk = q / s, j = q - blk * s;
    const int e0 = blk * L + j;
    for (int r = 0; r < R; ++r) {
      x[r] = buf[g.addr(b, e0 + r * s)];
      if (DIT && j > 0 && r > 0) x[r] = cmul(x[r], tw_load(tw, j * r * tstep, sign));
    }
    for (int qq = 0; qq < R; ++qq) {
      double2 acc = x[0];
      for (int r = 1; r < R; ++r) {
        int e = (r * qq) % R;
        acc = cadd(acc, e ? cmul(x[r], tw_load(tw, e * wR, sign)) : x[r]);
      }
      y[qq] = acc;
    }
    for (int r = 0; r < R; ++r) {
      double2 v = y[r];
      if (!DIT && j > 0 && r > 0) v = cmul(v, tw_load(tw, j * r * tstep, sign));
      buf[g.addr(b, e0 + r * s)] = v;
    }
  }
  __syncthreads();
}

template <bool DIT>
__device__ __forceinline__ void run_pass(double2* buf, const FftGeom& g, int R, int s,
                                         const double2* __restrict__ tw, int sign) {
  switch (R) {
    case 2: fft_pass<2, DIT>(buf, g, s, tw, sign); break;
    case 3: fft_pass<3, DIT>(buf, g, s, tw, sign); break;
    case 4: fft_pass<4, DIT>(buf, g, s, tw, sign); break;
    case 8: fft_pass<8, DIT>(buf, g, s, tw, sign); break;
    default: fft_pass_generic<DIT>(buf, g, R, s, tw, sign); break;
  }
}

// natural order in, digit-reversed spectrum out
__device__ __forceinline__ void fft_dif(double2* buf, const FftDesc& fd, const FftGeom& g, int sign) {
  int s = fd.n;
  for (int ip = 0; ip < fd.npass; ++ip) {
    const int R = fd.pass[ip].R;
    s /= R;
    run_pass<false>(buf, g, R, s, fd.tw, sign);
  }
}

// digit-reversed spectrum in, natural order out
__device__ __forceinline__ void fft_dit(double2* buf, const FftDesc& fd, const FftGeom& g, int sign) {
  int s = 1;
  for (int ip = fd.npass - 1; ip >= 0; --ip) {
    const int R = fd.pass[ip].R;
    run_pass<true>(buf, g, R, s, fd.tw, sign);
    s *= R;
  }
}
