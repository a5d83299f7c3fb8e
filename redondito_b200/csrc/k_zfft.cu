// k_zfft.cu -- radial (z) transforms on the (lm, z) spectral layout.
//
// One CTA owns LB consecutive lm columns and all nz rows in shared memory
// (row-major: element (k, c) at sm[k*LB + c]), so every global access is a
// contiguous LB*16-byte run of one row.  The reference's steps, each a
// separate pass over HBM there, are fused here into one read and one write:
//   fftp1d_real_to_complex_z (src/sphp/sphp_sca.F90:332-397): continuation
//     of the last C rows from rows 1..d and N-d+1..N (sphp_sca.F90:369-381,
//     same summation order), DFT sign -1, divide by nz;
//   fftp1d_complex_to_real_z (sphp_sca.F90:495-530): DFT sign +1;
//   derivr_r (src/pseudo/pseudospec_hd.f90:101-135): forward, (i kz)^p,
//     inverse, without the reference's temporary copy;
//   fc_filter_r (pseudospec_hd.f90:443-467) and dlr (pseudospec_hd.f90:254-288)
//     likewise.
// Two kernels do the transform in shared memory: zfft2_kernel for the
// lengths N = R1 R2 with a two-step register split (every compile-time
// length up to 256: two shared-memory passes, results stored from
// registers), zfft_kernel with radix passes for the others (nz 512, lengths
// without a compile-time transform, tuned column widths).  Batches run the
// forward transforms of all their problems with one z length as one launch
// of zfft2_group_kernel (the same body, one column block per CTA).
#include <algorithm>
#include <mutex>

#include "fft3.cuh"
#include "fft_ct.cuh"

namespace {

constexpr int ZTHREADS = 256;
constexpr int ZMAXCOL = 4096;  // LB*nz complex values per CTA (64 KB)

template <int IO>
struct ZIo {
  static constexpr bool FIN = IO == ZIO_FF || IO == ZIO_FD, FOUT = IO == ZIO_FF || IO == ZIO_DF;
};

struct ZArgs {
  const void* in;
  void* out;
  int nlm, nz, N, C, d, LB, order;
  const double* dir;      // C x d column-major
  const double2* kfac;    // (i kz)^order, nz entries
  const double* filt;     // nz
  const double* zinv2;    // nz
  const int* ell;         // nlm
  FftDesc fd;
};

template <int CTN>
struct ZGeo {
  typedef ct::Geo<CTN, 0, false> type;
  static __device__ __forceinline__ type make(int LB, int) { return type{LB, 1, LB}; }
};
template <>
struct ZGeo<0> {
  typedef FftGeom type;
  static __device__ __forceinline__ type make(int LB, int n) {
    FftGeom g;
    g.n = n;
    g.batch = LB;
    g.bs = 1;
    g.es = LB;
    g.pad = 0;
    g.jfast = false;
    return g;
  }
};

// 16-byte global -> shared copy that lands asynchronously; src_bytes 0
// writes zeros (src is then not read but must be a valid address)
__device__ __forceinline__ void cp_async16z(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}

// column element (row r, column lm) of the input, widened to FP64
template <int IO>
__device__ __forceinline__ double2 zin(const ZArgs& a, size_t idx) {
  if constexpr (ZIo<IO>::FIN) {
    const float2 v = __ldg(static_cast<const float2*>(a.in) + idx);
    return make_double2((double)v.x, (double)v.y);
  } else {
    return __ldg(static_cast<const double2*>(a.in) + idx);
  }
}

// one column element into shared memory: by cp.async when the input is
// FP64, else loaded, widened and stored; zero past nlm
template <int IO>
__device__ __forceinline__ void zload(const ZArgs& a, double2* dst, size_t idx, bool in) {
  if constexpr (ZIo<IO>::FIN) {
    *dst = in ? zin<IO>(a, idx) : make_double2(0.0, 0.0);
  } else {
    const double2* src = static_cast<const double2*>(a.in);
    cp_async16z(dst, in ? src + idx : src, in ? 16 : 0);
  }
}

template <int IO>
__device__ __forceinline__ void zstore(const ZArgs& a, size_t idx, double2 v) {
  if constexpr (ZIo<IO>::FOUT)
    static_cast<float2*>(a.out)[idx] = make_float2((float)v.x, (float)v.y);
  else
    static_cast<double2*>(a.out)[idx] = v;
}

template <int MODE, int CTN, int IO>
__global__ void __launch_bounds__(ZTHREADS) zfft_kernel(ZArgs a) {
  extern __shared__ double2 sm[];
  const int LB = a.LB, nz = a.nz, nlm = a.nlm;
  const int lm0 = blockIdx.x * LB;
  const int tid = threadIdx.x;
  const bool cont = (MODE != Z_INV) && a.C > 0;
  const int nload = cont ? a.N : nz;
  double2* orig = sm + (size_t)LB * nz;  // D_l keeps the input column for the l(l+1)/r^2 term

  const int* __restrict__ rev = a.fd.rev;
  // every copy of the slab is in flight at once (no registers held); columns
  // past nlm are zero-filled
  for (int idx = tid; idx < nload * LB; idx += ZTHREADS) {
    int r = idx / LB, c = idx - r * LB;
    int lm = lm0 + c;
    // the inverse transform takes its input in digit-reversed order
    zload<IO>(a, sm + (MODE == Z_INV ? __ldg(rev + r) : r) * LB + c, (size_t)r * nlm + lm, lm < nlm);
  }
  if (MODE == Z_DLR) {
    for (int idx = tid; idx < nz * LB; idx += ZTHREADS) {
      int r = idx / LB, c = idx - r * LB;
      int lm = lm0 + c;
      zload<IO>(a, orig + idx, (size_t)r * nlm + lm, lm < nlm);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();

  if (cont) {
    // inout(n-C+ii) = sum_jj dir(ii,jj) inout(n-C-d+jj) + dir(C-ii+1,jj) inout(d-jj+1)
    const int C = a.C, d = a.d, N = a.N;
    for (int idx = tid; idx < C * LB; idx += ZTHREADS) {
      int ii = idx / LB, c = idx - ii * LB;  // ii is 0-based
      double2 acc;
      {
        double wr = __ldg(a.dir + ii), wl = __ldg(a.dir + (C - 1 - ii));
        double2 xr = sm[(N - d) * LB + c], xl = sm[(d - 1) * LB + c];
        acc = make_double2(wr * xr.x + wl * xl.x, wr * xr.y + wl * xl.y);
      }
      for (int jj = 1; jj < d; ++jj) {
        double wr = __ldg(a.dir + ii + C * jj), wl = __ldg(a.dir + (C - 1 - ii) + C * jj);
        double2 xr = sm[(N - d + jj) * LB + c], xl = sm[(d - 1 - jj) * LB + c];
        acc.x = (acc.x + wr * xr.x) + wl * xl.x;
        acc.y = (acc.y + wr * xr.y) + wl * xl.y;
      }
      sm[(N + ii) * LB + c] = acc;
    }
    __syncthreads();
  }

  const auto g = ZGeo<CTN>::make(LB, nz);
  if (MODE == Z_INV) {
    if constexpr (CTN > 0) ct::dit<double2, CTN, CTN>(sm, g, a.fd.twp, +1);
    else fft_dit(sm, a.fd, g, +1);
  } else {
    if constexpr (CTN > 0) ct::dif<double2, CTN, CTN>(sm, g, a.fd.twp, -1);
    else fft_dif(sm, a.fd, g, -1);
  }

  if (MODE == Z_DERIV || MODE == Z_FILTER || MODE == Z_DLR) {
    // spectral multiply in place (frequency k sits at row rev[k]), then back
    for (int idx = tid; idx < nz * LB; idx += ZTHREADS) {
      int k = idx / LB, c = idx - k * LB;
      int o = __ldg(rev + k) * LB + c;
      double2 v = div_nz(sm[o], nz);
      if (MODE == Z_FILTER) v = cscale(v, a.filt[k]);
      else v = cmul(a.kfac[k], v);
      sm[o] = v;
    }
    __syncthreads();
    if constexpr (CTN > 0) ct::dit<double2, CTN, CTN>(sm, g, a.fd.twp, +1);
    else fft_dit(sm, a.fd, g, +1);
  }

  for (int idx = tid; idx < nz * LB; idx += ZTHREADS) {
    int r = idx / LB, c = idx - r * LB;
    int lm = lm0 + c;
    if (lm >= nlm) continue;
    double2 v;
    if (MODE == Z_FWD) {
      v = div_nz(sm[__ldg(rev + r) * LB + c], nz);
    } else {
      v = sm[idx];
    }
    if (MODE == Z_DLR) {
      // b = b + z^-2 * (-l(l+1) a)   (laplang, multr(-2), saxpby_c)
      double lf = -(double)(a.ell[lm] * (a.ell[lm] + 1));
      double2 o = orig[idx];
      double zi = a.zinv2[r];
      v.x = v.x + zi * (lf * o.x);
      v.y = v.y + zi * (lf * o.y);
    }
    zstore<IO>(a, (size_t)r * nlm + lm, v);
  }
}

// Lengths with a two-step split N = R1 R2 (ct::split2_r1, fft3.cuh): every
// mode, max(R1, R2) threads per column, the column slab in shared memory as
// in zfft_kernel (same loads and continuation, the inverse's input in
// natural order).  A plain transform is the two register steps, its results
// stored from registers; the spectral modes run the forward steps, multiply
// in registers, put the spectrum back in natural order and run the inverse
// steps.
// The columns per CTA are those launch_zfft_io picks by default for the
// length (32 KB slabs), fixed at compile time; other choices take the radix
// kernel.  Registers are held to 80 per thread for the plain transforms
// (six CTAs of 128 threads per SM at nz 256; 1.66 against 1.68 ms for eight
// transforms with five) and 128 for the spectral modes (four).
__host__ __device__ constexpr int z2_lb(int nz) {
  int lb = 64;
  while (lb > 1 && lb * nz > ZMAXCOL / 2) lb >>= 1;
  return lb;
}
template <int MODE, int NZ, int TPC>
struct Z2Geo {
  static constexpr int LB = z2_lb(NZ), THREADS = LB * TPC;
  static constexpr bool PLAIN = MODE == Z_FWD || MODE == Z_INV;
  static constexpr int RPT = PLAIN ? 84 : 128;
  static constexpr int MINB = 65536 / (THREADS * RPT) > 1 ? 65536 / (THREADS * RPT) : 1;
};

// column block blk of the spectra a describes
template <int MODE, int R1, int R2, int IO>
__device__ __forceinline__ void zfft2_body(const ZArgs& a, int blk) {
  constexpr int NZ = R1 * R2, TPC = R1 > R2 ? R1 : R2;
  using GZ = Z2Geo<MODE, NZ, TPC>;
  constexpr bool PLAIN = GZ::PLAIN;
  constexpr int SG = MODE == Z_INV ? 1 : -1;  // first transform's sign
  constexpr int LB = GZ::LB, nthreads = GZ::THREADS;
  extern __shared__ double2 sm[];
  const int nlm = a.nlm, tid = threadIdx.x, lm0 = blk * LB;
  const bool cont = MODE != Z_INV && a.C > 0;
  const int nload = cont ? a.N : NZ;
  double2* orig = sm + (size_t)LB * NZ;  // D_l keeps the input column for the l(l+1)/r^2 term
  for (int idx = tid; idx < nload * LB; idx += nthreads) {
    const int r = idx / LB, c = idx - r * LB, lm = lm0 + c;
    zload<IO>(a, sm + idx, (size_t)r * nlm + lm, lm < nlm);
  }
  if (MODE == Z_DLR) {
    for (int idx = tid; idx < NZ * LB; idx += nthreads) {
      const int r = idx / LB, c = idx - r * LB, lm = lm0 + c;
      zload<IO>(a, orig + idx, (size_t)r * nlm + lm, lm < nlm);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  if (cont) {  // as in zfft_kernel
    const int C = a.C, d = a.d, N = a.N;
    for (int idx = tid; idx < C * LB; idx += nthreads) {
      const int ii = idx / LB, c = idx - ii * LB;
      sm[(N + ii) * LB + c] = fc_cont_elem(a.dir, C, d, N, ii, sm + c, LB);
    }
    __syncthreads();
  }
  const int c = tid % LB, h = tid / LB, lm = lm0 + c;
  double2* col = sm + c;
  ct::dft2_step1<R1, R2, SG>(col, LB, h, a.fd.tw);
  __syncthreads();
  double2 v[R2];
  ct::dft2_step2<R1, R2, SG>(col, LB, h, v);
  if constexpr (!PLAIN) {
    // X[k] / nz times (i kz)^p or the filter, k = h + R1 k2; back in natural
    // order once every thread has read its step-2 slots; then the inverse
    __syncthreads();
    if (h < R1) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const int k = h + R1 * k2;
        double2 x = div_nz(v[k2], NZ);
        if (MODE == Z_FILTER) x = cscale(x, a.filt[k]);
        else x = cmul(a.kfac[k], x);
        col[k * LB] = x;
      }
    }
    __syncthreads();
    ct::dft2_step1<R1, R2, 1>(col, LB, h, a.fd.tw);
    __syncthreads();
    ct::dft2_step2<R1, R2, 1>(col, LB, h, v);
  }
  if (h < R1 && lm < nlm) {
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) {
      const int r = h + R1 * k2;
      double2 x = MODE == Z_FWD ? div_nz(v[k2], NZ) : v[k2];
      if (MODE == Z_DLR) {
        // b = b + z^-2 * (-l(l+1) a)   (laplang, multr(-2), saxpby_c)
        const double lf = -(double)(a.ell[lm] * (a.ell[lm] + 1));
        const double2 o = orig[r * LB + c];
        const double zi = a.zinv2[r];
        x.x = x.x + zi * (lf * o.x);
        x.y = x.y + zi * (lf * o.y);
      }
      zstore<IO>(a, (size_t)r * nlm + lm, x);
    }
  }
}

template <int MODE, int R1, int R2, int IO>
__global__ void __launch_bounds__(Z2Geo<MODE, R1 * R2, (R1 > R2 ? R1 : R2)>::THREADS,
                                  Z2Geo<MODE, R1 * R2, (R1 > R2 ? R1 : R2)>::MINB) zfft2_kernel(ZArgs a) {
  zfft2_body<MODE, R1, R2, IO>(a, blockIdx.x);
}

// The same over the spectra of several plans with one z length (batches):
// job j owns the CTAs prefix[j] .. prefix[j+1]-1, one column block each.
template <int MODE, int R1, int R2, int IO>
__global__ void __launch_bounds__(Z2Geo<MODE, R1 * R2, (R1 > R2 ? R1 : R2)>::THREADS,
                                  Z2Geo<MODE, R1 * R2, (R1 > R2 ? R1 : R2)>::MINB)
    zfft2_group_kernel(const ZArgs* __restrict__ jobs, const int* __restrict__ prefix, int njobs) {
  int lo = 0, hi = njobs - 1;  // last job whose first CTA is <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(prefix + mid) <= (int)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  zfft2_body<MODE, R1, R2, IO>(jobs[lo], (int)blockIdx.x - __ldg(prefix + lo));
}

template <int MODE, int CTN, int IO>
int launch_ct(const ZArgs& a, int nblocks, size_t smem, cudaStream_t st) {
  static DeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(zfft_kernel<MODE, CTN, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    200 * 1024) == cudaSuccess &&
               cudaFuncSetAttribute(zfft_kernel<MODE, CTN, IO>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    100) == cudaSuccess;
      }))
    return SPH_ECUDA;
  if constexpr (CTN > 0 && ct::split2_r1(CTN) > 0) {
    constexpr int R1 = ct::split2_r1(CTN), R2 = CTN / R1;
    using GZ = Z2Geo<MODE, CTN, ct::split2_tpc(CTN)>;
    if (a.LB == GZ::LB) {
      static DeviceOnce once2;
      if (!once2.run([] {
            return cudaFuncSetAttribute(zfft2_kernel<MODE, R1, R2, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        200 * 1024) == cudaSuccess &&
                   cudaFuncSetAttribute(zfft2_kernel<MODE, R1, R2, IO>,
                                        cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
          }))
        return SPH_ECUDA;
      zfft2_kernel<MODE, R1, R2, IO><<<nblocks, GZ::THREADS, smem, st>>>(a);
      SPH_LAUNCH_OK();
      return SPH_OK;
    }
  }
  zfft_kernel<MODE, CTN, IO><<<nblocks, ZTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

#define Z_SIZES(X) X(16) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(512)

// the lengths that take the two-step split
bool zsplit_length(int nz) {
  switch (nz) {
#define CASE(n) \
  case n: return ct::split2_r1(n) > 0;
    Z_SIZES(CASE)
#undef CASE
  }
  return false;
}

template <int MODE, int IO>
int launch_mode(const ZArgs& a, int nblocks, size_t smem, cudaStream_t st) {
  switch (a.nz) {
#define CASE(n) \
  case n: return launch_ct<MODE, n, IO>(a, nblocks, smem, st);
    Z_SIZES(CASE)
#undef CASE
    default: return launch_ct<MODE, 0, IO>(a, nblocks, smem, st);
  }
}

// the element types used with each mode: FP64 everywhere; single precision
// in and out for every mode; FP64 in, single out for the forward transform
// (after the analysis in FP64); single in, FP64 out for the inverse (before
// the synthesis)
template <int MODE>
int launch_mode_io(const ZArgs& a, int io, int nblocks, size_t smem, cudaStream_t st) {
  switch (io) {
    case ZIO_DD: return launch_mode<MODE, ZIO_DD>(a, nblocks, smem, st);
    case ZIO_FF: return launch_mode<MODE, ZIO_FF>(a, nblocks, smem, st);
    case ZIO_DF:
      if constexpr (MODE == Z_FWD) return launch_mode<MODE, ZIO_DF>(a, nblocks, smem, st);
      break;
    case ZIO_FD:
      if constexpr (MODE == Z_INV) return launch_mode<MODE, ZIO_FD>(a, nblocks, smem, st);
      break;
  }
  return SPH_EINVAL;
}

}  // namespace

int launch_zfft(const sph_plan* p, int mode, const double2* in, double2* out, int order,
                cudaStream_t st, bool cont) {
  return launch_zfft_io(p, mode, in, out, ZIO_DD, order, st, cont);
}

namespace {

// The arguments of one z transform of plan p's spectra and its CTA count.
int make_zargs(const sph_plan* p, int mode, const void* in, void* out, int order, bool cont, ZArgs* ap,
               int* nblocks) {
  ZArgs& a = *ap;
  a.in = in;
  a.out = out;
  a.nlm = p->nlmv;  // the caller's lm columns [lm0, lm0 + nlmv)
  a.nz = p->nz;
  a.N = cont ? p->N : p->nz;
  a.C = cont ? p->C : 0;
  a.d = p->d;
  a.order = order;
  a.dir = p->d_dir;
  a.kfac = (order >= 1 && order <= 4) ? p->kfac + (size_t)(order - 1) * p->nz : nullptr;
  a.filt = p->filt;
  a.zinv2 = p->zinv2;
  a.ell = p->d_ell + p->lm0;
  a.fd = p->fz;
  // columns per CTA: a power of two with LB*nz <= ZMAXCOL/2, at most 64
  // (32 KB slabs: 4 CTAs per SM, still full 128-byte lines per row at nz = 256)
  int LB = 64;
  while (LB > 1 && LB * p->nz > ZMAXCOL / 2) LB >>= 1;
  // a tuned width, except for the lengths with the two-step split, whose
  // kernel is compiled for the default width
  if (p->tile_lb && !zsplit_length(p->nz)) LB = p->tile_lb;
  if (LB * p->nz > ZMAXCOL) return SPH_EINVAL;
  a.LB = LB;
  *nblocks = (p->nlmv + LB - 1) / LB;
  if (mode == Z_DLR) a.kfac = p->kfac + (size_t)1 * p->nz;  // (i kz)^2
  return SPH_OK;
}

}  // namespace

int launch_zfft_io(const sph_plan* p, int mode, const void* in, void* out, int io, int order, cudaStream_t st,
                   bool cont) {
  ZArgs a;
  int nblocks = 0;
  const int rc = make_zargs(p, mode, in, out, order, cont, &a, &nblocks);
  if (rc != SPH_OK) return rc;
  size_t smem = (size_t)a.LB * p->nz * sizeof(double2) * (mode == Z_DLR ? 2 : 1);
  TimedLaunch tl(p, T_ZFFT, st);
  switch (mode) {
    case Z_FWD: return launch_mode_io<Z_FWD>(a, io, nblocks, smem, st);
    case Z_INV: return launch_mode_io<Z_INV>(a, io, nblocks, smem, st);
    case Z_DERIV:
      if (!a.kfac) return SPH_EINVAL;
      return launch_mode_io<Z_DERIV>(a, io, nblocks, smem, st);
    case Z_FILTER: return launch_mode_io<Z_FILTER>(a, io, nblocks, smem, st);
    case Z_DLR: return launch_mode_io<Z_DLR>(a, io, nblocks, smem, st);
  }
  return SPH_EINVAL;
}

// ---------------------------------------------------------------- grouped forward z (batches)
namespace {

template <int R1, int R2>
int zgroup_launch_len(const ZGroupLen& L, cudaStream_t st) {
  constexpr int NZ = R1 * R2;
  using GZ = Z2Geo<Z_FWD, NZ, ct::split2_tpc(NZ)>;
  static DeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(zfft2_group_kernel<Z_FWD, R1, R2, ZIO_DD>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) == cudaSuccess &&
               cudaFuncSetAttribute(zfft2_group_kernel<Z_FWD, R1, R2, ZIO_DD>,
                                    cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
      }))
    return SPH_ECUDA;
  const size_t smem = (size_t)GZ::LB * NZ * sizeof(double2);
  zfft2_group_kernel<Z_FWD, R1, R2, ZIO_DD>
      <<<L.total, GZ::THREADS, smem, st>>>(static_cast<const ZArgs*>(L.jobs), L.prefix, L.njobs);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

// the two-step lengths only (the others never reach a grouped launch)
template <int NZ>
int zgroup_launch_nz(const ZGroupLen& L, cudaStream_t st) {
  if constexpr (ct::split2_r1(NZ) > 0) {
    return zgroup_launch_len<ct::split2_r1(NZ), NZ / ct::split2_r1(NZ)>(L, st);
  } else {
    return SPH_EINVAL;
  }
}

}  // namespace

int zfwd_group_prepare(const std::vector<ZJob>& jobs, ZGroupLaunch* g, std::vector<int>* rest) {
  if (!g || !rest) return SPH_EINVAL;
  rest->clear();
  std::vector<int> lens;  // z lengths, in order of first appearance
  std::vector<std::vector<ZArgs>> args;
  std::vector<std::vector<int>> prefix;
  for (int k = 0; k < (int)jobs.size(); ++k) {
    const sph_plan* p = jobs[k].p;
    ZArgs a;
    int nb = 0;
    if (!p || !jobs[k].spec || !zsplit_length(p->nz) ||
        make_zargs(p, Z_FWD, jobs[k].spec, jobs[k].spec, 0, jobs[k].cont, &a, &nb) != SPH_OK || nb < 1 ||
        a.LB != z2_lb(p->nz)) {
      rest->push_back(k);
      continue;
    }
    int li = (int)(std::find(lens.begin(), lens.end(), p->nz) - lens.begin());
    if (li == (int)lens.size()) {
      lens.push_back(p->nz);
      args.emplace_back();
      prefix.emplace_back(1, 0);
    }
    args[li].push_back(a);
    prefix[li].push_back(prefix[li].back() + nb);
  }
  for (size_t li = 0; li < lens.size(); ++li) {
    ZGroupLen L;
    L.nz = lens[li];
    L.njobs = (int)args[li].size();
    L.total = prefix[li].back();
    g->lens.push_back(L);
    ZGroupLen& G = g->lens.back();
    if (cudaMalloc(&G.jobs, args[li].size() * sizeof(ZArgs)) != cudaSuccess ||
        cudaMalloc((void**)&G.prefix, prefix[li].size() * sizeof(int)) != cudaSuccess)
      return SPH_ENOMEM;
    if (cudaMemcpy(G.jobs, args[li].data(), args[li].size() * sizeof(ZArgs), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(G.prefix, prefix[li].data(), prefix[li].size() * sizeof(int), cudaMemcpyHostToDevice) !=
            cudaSuccess)
      return SPH_ECUDA;
  }
  return SPH_OK;
}

int zfwd_group_launch(const ZGroupLaunch& g, cudaStream_t st) {
  for (const ZGroupLen& L : g.lens) {
    int rc = SPH_EINVAL;
    switch (L.nz) {
#define CASE(n)                    \
  case n:                          \
    rc = zgroup_launch_nz<n>(L, st); \
    break;
      Z_SIZES(CASE)
#undef CASE
    }
    if (rc != SPH_OK) return rc;
  }
  return SPH_OK;
}

void zgroup_free(ZGroupLaunch* g) {
  for (ZGroupLen& L : g->lens) {
    if (L.jobs) cudaFree(L.jobs);
    if (L.prefix) cudaFree(L.prefix);
  }
  g->lens.clear();
}

// ---------------------------------------------------------------- no-alloc derivative
// Radial derivative for callers that cannot allocate device memory: the
// device-resident tables the fused derivative kernel reads (twiddles,
// digit-reversal order, (i kz)^p factors, the FC-Gram operator) live in one
// file-scope array instead of a plan's cudaMalloc'd buffers.  The host side
// stages them in fixed static buffers, so the call allocates nothing on the
// host either.
namespace {

constexpr int NA_MAX_NZ = 4096;  // longest radial transform
constexpr int NA_MAX_CD = 2048;  // largest Cz*oz
constexpr size_t NA_TW = 0;                                              // double2[nz]
constexpr size_t NA_TWP = NA_TW + (size_t)NA_MAX_NZ * sizeof(double2);   // double2[< nz]
constexpr size_t NA_KF = NA_TWP + (size_t)NA_MAX_NZ * sizeof(double2);   // double2[nz]
constexpr size_t NA_DIR = NA_KF + (size_t)NA_MAX_NZ * sizeof(double2);   // double[Cz*oz]
constexpr size_t NA_REV = NA_DIR + (size_t)NA_MAX_CD * sizeof(double);   // int[nz]
constexpr size_t NA_BYTES = NA_REV + (size_t)NA_MAX_NZ * sizeof(int);    // 224 KiB

static __device__ __align__(256) unsigned char g_noalloc_tables[NA_BYTES];

// host staging, laid out like the device array; serialised by na_mutex
static unsigned char na_host[NA_BYTES];
static std::mutex na_mutex;
static void* na_dev[64];  // device address of g_noalloc_tables, per device

int na_setup(int dev) {
  if (dev < 0 || dev >= 64) return SPH_EINVAL;
  if (na_dev[dev]) return SPH_OK;
  void* ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, g_noalloc_tables) != cudaSuccess || !ptr) return SPH_ECUDA;
  na_dev[dev] = ptr;
  return SPH_OK;
}

}  // namespace

extern "C" int sph_derivr_noalloc(const double* a, double* b, int nlm, int nz, int Cz, int oz, double rint,
                                  double rext, const double* dir, int p, void* stream) {
  if (!a || !b || nlm < 1 || nz < 2 || nz > NA_MAX_NZ || p < 1 || p > 4) return SPH_EINVAL;
  if (Cz < 0 || oz < 0 || (Cz > 0 && (oz < 1 || nz - Cz < oz || !dir)) || (size_t)Cz * oz > NA_MAX_CD)
    return SPH_EINVAL;
  // radix plan (8s, then 4, 2, 3, other primes), as sph_plan_create builds it
  FftDesc fd = {};
  fd.n = nz;
  {
    int r = nz, Ns = 1;
    for (int q : {8, 4, 2, 3})
      while (r % q == 0) {
        if (fd.npass >= SPH_MAX_PASSES) return SPH_EINVAL;
        fd.pass[fd.npass++] = {q, Ns};
        Ns *= q;
        r /= q;
      }
    for (int q = 5; r > 1; q += 2)
      while (r % q == 0) {
        if (q > 64 || fd.npass >= SPH_MAX_PASSES) return SPH_EINVAL;
        fd.pass[fd.npass++] = {q, Ns};
        Ns *= q;
        r /= q;
      }
  }
  int LB = 64;
  // the column blocks of the plan path (so that both run the same kernel)
  while (LB > 1 && LB * nz > ZMAXCOL / 2) LB >>= 1;
  if (LB * nz > ZMAXCOL) return SPH_EINVAL;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SPH_ECUDA;
  std::lock_guard<std::mutex> lock(na_mutex);
  int rc = na_setup(dev);
  if (rc != SPH_OK) return rc;

  const long double pi = 3.141592653589793238462643383279502884L;
  double2* tw = reinterpret_cast<double2*>(na_host + NA_TW);
  double2* twp = reinterpret_cast<double2*>(na_host + NA_TWP);
  double2* kf = reinterpret_cast<double2*>(na_host + NA_KF);
  double* dr = reinterpret_cast<double*>(na_host + NA_DIR);
  int* rev = reinterpret_cast<int*>(na_host + NA_REV);
  for (int e = 0; e < nz; ++e) {
    long double ang = -2.0L * pi * e / nz;
    tw[e] = make_double2((double)cosl(ang), (double)sinl(ang));
  }
  int ntp = 0;  // per-pass twiddles [pass][j][r-1] = W_L^{j r}
  for (int L = nz; L > 1;) {
    int R = L % 8 == 0 ? 8 : L % 4 == 0 ? 4 : L % 2 == 0 ? 2 : L % 3 == 0 ? 3 : L;
    int S = L / R;
    for (int j = 0; j < S; ++j)
      for (int r = 1; r < R; ++r) {
        long double ang = -2.0L * pi * (long double)((long)j * r) / L;
        twp[ntp++] = make_double2((double)cosl(ang), (double)sinl(ang));
      }
    L = S;
  }
  for (int k = 0; k < nz; ++k) {
    int t = k, s = nz, pos = 0;
    for (int ip = 0; ip < fd.npass; ++ip) {
      s /= fd.pass[ip].R;
      pos += (t % fd.pass[ip].R) * s;
      t /= fd.pass[ip].R;
    }
    rev[k] = pos;
  }
  // kz as box_init builds it (src/pseudo/pseudospec_mod.f90:196-227), times i^p
  const int N = nz - Cz;
  const double dz = N > 1 ? (rext - rint) / (nz - Cz - 1) : 1.0;
  const double Dkz = 2.0 * 3.14159265358979323846 / (dz * nz);
  for (int k = 0; k < nz; ++k) {
    double kzk;
    if (nz % 2 == 0) kzk = (double)(k < nz / 2 ? k : k - nz) * Dkz;
    else kzk = (double)(k < (nz + 1) / 2 ? k : k - nz) * Dkz;
    double kp = 1.0;
    for (int q = 0; q < p; ++q) kp *= kzk;
    double re = (p % 4 == 0) ? 1 : (p % 4 == 2) ? -1 : 0;
    double im = (p % 4 == 1) ? 1 : (p % 4 == 3) ? -1 : 0;
    kf[k] = make_double2(re * kp, im * kp);
  }
  for (int q = 0; q < Cz * oz; ++q) dr[q] = dir[q];

  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* dbase = static_cast<unsigned char*>(na_dev[dev]);
  const size_t spans[][2] = {{NA_TW, (size_t)nz * sizeof(double2)},
                             {NA_TWP, (size_t)(ntp > 0 ? ntp : 1) * sizeof(double2)},
                             {NA_KF, (size_t)nz * sizeof(double2)},
                             {NA_DIR, (size_t)(Cz * oz > 0 ? Cz * oz : 1) * sizeof(double)},
                             {NA_REV, (size_t)nz * sizeof(int)}};
  for (auto& sp : spans)
    if (cudaMemcpyAsync(dbase + sp[0], na_host + sp[0], sp[1], cudaMemcpyHostToDevice, st) != cudaSuccess)
      return SPH_ECUDA;

  fd.tw = reinterpret_cast<const double2*>(dbase + NA_TW);
  fd.twp = reinterpret_cast<const double2*>(dbase + NA_TWP);
  fd.rev = reinterpret_cast<const int*>(dbase + NA_REV);
  ZArgs z = {};
  z.in = reinterpret_cast<const double2*>(a);
  z.out = reinterpret_cast<double2*>(b);
  z.nlm = nlm;
  z.nz = nz;
  z.N = N;
  z.C = Cz;
  z.d = oz;
  z.LB = LB;
  z.order = p;
  z.dir = reinterpret_cast<const double*>(dbase + NA_DIR);
  z.kfac = reinterpret_cast<const double2*>(dbase + NA_KF);
  z.fd = fd;
  const int nblocks = (nlm + LB - 1) / LB;
  const size_t smem = (size_t)LB * nz * sizeof(double2);
  return launch_mode<Z_DERIV, ZIO_DD>(z, nblocks, smem, st);
}
