// k_phifft.cu -- azimuthal (phi) transforms between the physical grid and
// the folded Fourier coefficients the Legendre GEMMs consume.
//
// The reference does the phi FFT inside SHTns, plane by plane
// (spat_to_SH / SH_to_spat at src/sphp/sphp_sca.F90:311-313,484-486; on the
// GPU cu_spat_to_SH per plane at src/sphp-gpu/sphp_sca.F90:84-86).  Here one
// launch covers every plane and field.  A CTA owns NP northern rings i and
// their mirrors nlat-1-i of one plane: ring i and its mirror are the real
// and imaginary parts of one complex length-nphi FFT.  The forward kernel
// writes, for m <= lmax,
//   G[m][0][k][i] = W_i (F_m(i) + F_m(mirror))   (even part, pairs with l-m even)
//   G[m][1][k][i] = W_i (F_m(i) - F_m(mirror))   (odd part)
// with W_i = w_i 2 pi / nphi; the inverse kernel reads the same layout
// (synthesised even/odd sums) and writes both rings of the grid.
// Lengths 2^a 3^b use the compile-time FFT of fft_ct.cuh; others the
// runtime engine of fft_engine.cuh.
#include "fft_ct.cuh"

namespace {

constexpr int PTHREADS = 512;
constexpr int PMAXC = 8192;  // NP*nphi complex values per CTA
constexpr int UNR = 8;       // independent global loads in flight per thread

// sequence stride in shared memory: E(e) = e + e/8 skews short-span passes,
// and an odd stride spreads the per-ring stores of the load phase over banks
__host__ __device__ inline int seq_stride(int nphi) {
  int s = nphi + (nphi + 7) / 8;
  return s | 1;
}

struct PhiArgs {
  const double* gin[SPH_MAX_FIELDS];
  double* gout[SPH_MAX_FIELDS];
  double2* G;
  const double2* Gc;
  size_t Gfield;
  int nlat, nlat2, ldn, nphi, nz, lmax, NP;
  const double* wfold;
  FftDesc fd;
};

// The geometry type of a length: compile-time for CTN > 0, runtime otherwise.
template <int CTN>
struct PhiGeo {
  typedef ct::Geo<CTN, 1, true> type;
  static __device__ __forceinline__ type make(int NP, int ss, int) { return type{NP, ss, 1}; }
};
template <>
struct PhiGeo<0> {
  typedef FftGeom type;
  static __device__ __forceinline__ type make(int NP, int ss, int n) {
    FftGeom g;
    g.n = n;
    g.batch = NP;
    g.bs = ss;
    g.es = 1;
    g.pad = 1;
    g.jfast = true;
    return g;
  }
};

template <int CTN>
__global__ void __launch_bounds__(PTHREADS, 2) phi_fwd_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const double* plane = a.gin[f] + (size_t)k * nphi * nlat;
  const int np = min(NP, nlat2 - p0);
  const auto g = PhiGeo<CTN>::make(NP, seq_stride(nphi), nphi);
  double* smd = reinterpret_cast<double*>(sm);

  // rings p0..p0+np-1 (real part) and their mirrors (imaginary part);
  // consecutive threads read consecutive theta addresses
  const int total = nphi * 2 * NP;
  for (int base = tid; base < total; base += PTHREADS * UNR) {
    double v[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      int idx = base + u * PTHREADS;
      v[u] = 0.0;
      if (idx < total) {
        int j = idx / (2 * NP), q = idx - j * 2 * NP;
        int b = q < NP ? q : NP - 1 - (q - NP);  // mirrors in ascending address order
        int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
        if (b < np) v[u] = __ldg(plane + (size_t)j * nlat + ring);
      }
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      int idx = base + u * PTHREADS;
      if (idx < total) {
        int j = idx / (2 * NP), q = idx - j * 2 * NP;
        int b = q < NP ? q : NP - 1 - (q - NP);
        smd[2 * g.addr(b, j) + (q < NP ? 0 : 1)] = v[u];
      }
    }
  }
  __syncthreads();
  if constexpr (CTN > 0) ct::dif<double2, CTN, CTN>(sm, g, a.fd.twp, -1);
  else fft_dif(sm, a.fd, g, -1);
  const int* __restrict__ rev = a.fd.rev;

  double2* G = a.G + (size_t)f * a.Gfield;
  const int M = a.lmax + 1;
  for (int idx = tid; idx < M * 2 * NP; idx += PTHREADS) {
    int b = idx % NP;
    int rest = idx / NP;
    int par = rest & 1, m = rest >> 1;
    if (b >= np) continue;
    double2 Z = sm[g.addr(b, __ldg(rev + m))];
    double2 Zc = sm[g.addr(b, __ldg(rev + (m == 0 ? 0 : nphi - m)))];
    Zc.y = -Zc.y;
    // F(i) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
    double2 Fi = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y + Zc.y));
    double2 Fm = make_double2(0.5 * (Z.y - Zc.y), -0.5 * (Z.x - Zc.x));
    double W = __ldg(a.wfold + p0 + b);
    double2 gv = par ? csub(Fi, Fm) : cadd(Fi, Fm);
    G[(((size_t)m * 2 + par) * a.nz + k) * a.ldn + p0 + b] = cscale(gv, W);
  }
}

template <int CTN>
__global__ void __launch_bounds__(PTHREADS, 2) phi_inv_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const int np = min(NP, nlat2 - p0);
  const int M = a.lmax + 1;
  const double2* G = a.Gc + (size_t)f * a.Gfield;
  const auto g = PhiGeo<CTN>::make(NP, seq_stride(nphi), nphi);
  const int* __restrict__ rev = a.fd.rev;

  // the band between the two Hermitian halves is zero
  for (int idx = tid; idx < NP * nphi; idx += PTHREADS) {
    int b = idx / nphi, m = idx - b * nphi;
    if (m >= M && m <= nphi - M) sm[g.addr(b, __ldg(rev + m))] = make_double2(0.0, 0.0);
  }
  for (int base = tid; base < M * NP; base += PTHREADS * (UNR / 2)) {
    double2 se[UNR / 2], so[UNR / 2];
#pragma unroll
    for (int u = 0; u < UNR / 2; ++u) {
      int idx = base + u * PTHREADS;
      se[u] = so[u] = make_double2(0.0, 0.0);
      int b = idx % NP, m = idx / NP;
      if (idx < M * NP && b < np) {
        se[u] = __ldg(G + (((size_t)m * 2 + 0) * a.nz + k) * a.ldn + p0 + b);
        so[u] = __ldg(G + (((size_t)m * 2 + 1) * a.nz + k) * a.ldn + p0 + b);
      }
    }
#pragma unroll
    for (int u = 0; u < UNR / 2; ++u) {
      int idx = base + u * PTHREADS;
      if (idx >= M * NP) continue;
      int b = idx % NP, m = idx / NP;
      double2 Fi = cadd(se[u], so[u]), Fm = csub(se[u], so[u]);
      if (m == 0) {
        sm[g.addr(b, __ldg(rev))] = make_double2(Fi.x, Fm.x);
      } else {
        // z = x + i y with x, y the real fields of ring i and its mirror
        sm[g.addr(b, __ldg(rev + m))] = make_double2(Fi.x - Fm.y, Fi.y + Fm.x);
        sm[g.addr(b, __ldg(rev + nphi - m))] = make_double2(Fi.x + Fm.y, -Fi.y + Fm.x);
      }
    }
  }
  __syncthreads();
  if constexpr (CTN > 0) ct::dit<double2, CTN, CTN>(sm, g, a.fd.twp, +1);
  else fft_dit(sm, a.fd, g, +1);

  double* plane = a.gout[f] + (size_t)k * nphi * nlat;
  const double* smd = reinterpret_cast<const double*>(sm);
  for (int idx = tid; idx < nphi * 2 * NP; idx += PTHREADS) {
    int j = idx / (2 * NP), q = idx - j * 2 * NP;
    if (q < NP) {
      if (q < np) plane[(size_t)j * nlat + p0 + q] = smd[2 * g.addr(q, j)];
    } else {
      int b = NP - 1 - (q - NP);
      if (b < np) plane[(size_t)j * nlat + (nlat - 1 - (p0 + b))] = smd[2 * g.addr(b, j) + 1];
    }
  }
}

int pairs_per_cta(const sph_plan* p) {
  int cap = PMAXC / p->nphi;
  if (cap > 8) cap = 8;
  for (int np = cap; np >= 1; --np)
    if (p->nlat2 % np == 0) return np;
  return 1;
}

template <typename K>
bool smem_attr(K fn) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) == cudaSuccess &&
         cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
}

template <int CTN>
int launch_fwd_n(const PhiArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
  static bool once = smem_attr(phi_fwd_kernel<CTN>);
  if (!once) return SPH_ECUDA;
  phi_fwd_kernel<CTN><<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

template <int CTN>
int launch_inv_n(const PhiArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
  static bool once = smem_attr(phi_inv_kernel<CTN>);
  if (!once) return SPH_ECUDA;
  phi_inv_kernel<CTN><<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

#define PHI_SIZES(X) X(12) X(24) X(48) X(96) X(192) X(384) X(768) X(1536) X(3072) X(6144)

PhiArgs make_args(const sph_plan* p) {
  PhiArgs a = {};
  a.G = p->G;
  a.Gc = p->G;
  a.Gfield = p->Gfield;
  a.nlat = p->nlat;
  a.nlat2 = p->nlat2;
  a.ldn = p->ldn;
  a.nphi = p->nphi;
  a.nz = p->nz;
  a.lmax = p->lmax;
  a.NP = pairs_per_cta(p);
  a.wfold = p->wfold;
  a.fd = p->fphi;
  return a;
}

}  // namespace

int launch_phi_fwd(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st) {
  if (nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  if (p->nphi > PMAXC) return SPH_EINVAL;
  PhiArgs a = make_args(p);
  for (int f = 0; f < nfields; ++f) a.gin[f] = grids[f];
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_FWD, st);
  switch (p->nphi) {
#define CASE(n) \
  case n: return launch_fwd_n<n>(a, grid, smem, st);
    PHI_SIZES(CASE)
#undef CASE
    default: return launch_fwd_n<0>(a, grid, smem, st);
  }
}

int launch_phi_inv(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st) {
  if (nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  if (p->nphi > PMAXC) return SPH_EINVAL;
  PhiArgs a = make_args(p);
  for (int f = 0; f < nfields; ++f) a.gout[f] = grids[f];
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_INV, st);
  switch (p->nphi) {
#define CASE(n) \
  case n: return launch_inv_n<n>(a, grid, smem, st);
    PHI_SIZES(CASE)
#undef CASE
    default: return launch_inv_n<0>(a, grid, smem, st);
  }
}
