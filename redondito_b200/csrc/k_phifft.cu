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
#include "fft_engine.cuh"

namespace {

constexpr int PTHREADS = 512;
constexpr int PMAXC = 8192;  // NP*nphi complex values per CTA

// sequence stride in shared memory: E(e) = e + e/8 skews short-span passes
__host__ __device__ inline int seq_stride(int nphi) { return nphi + (nphi + 7) / 8; }

struct PhiArgs {
  const double* gin[SPH_MAX_FIELDS];
  double* gout[SPH_MAX_FIELDS];
  double2* G;
  const double2* Gc;
  size_t Gfield;
  int nlat, nlat2, nphi, nz, lmax, NP;
  const double* wfold;
  FftDesc fd;
};

__global__ void __launch_bounds__(PTHREADS) phi_fwd_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const double* plane = a.gin[f] + (size_t)k * nphi * nlat;
  const int np = min(NP, nlat2 - p0);
  FftGeom g;
  g.n = nphi; g.batch = NP; g.bs = seq_stride(nphi); g.es = 1; g.pad = 1; g.jfast = true;
  double* smd = reinterpret_cast<double*>(sm);

  // rings p0..p0+np-1 (real part) and their mirrors (imaginary part);
  // consecutive threads read consecutive theta addresses
  for (int idx = tid; idx < nphi * 2 * NP; idx += PTHREADS) {
    int j = idx / (2 * NP), q = idx - j * 2 * NP;
    if (q < NP) {
      smd[2 * g.addr(q, j)] = q < np ? plane[(size_t)j * nlat + p0 + q] : 0.0;
    } else {
      int b = NP - 1 - (q - NP);  // ascending address order
      smd[2 * g.addr(b, j) + 1] = b < np ? plane[(size_t)j * nlat + (nlat - 1 - (p0 + b))] : 0.0;
    }
  }
  __syncthreads();
  fft_dif(sm, a.fd, g, -1);
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
    G[(((size_t)m * 2 + par) * a.nz + k) * nlat2 + p0 + b] = cscale(gv, W);
  }
}

__global__ void __launch_bounds__(PTHREADS) phi_inv_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const int np = min(NP, nlat2 - p0);
  const int M = a.lmax + 1;
  const double2* G = a.Gc + (size_t)f * a.Gfield;

  FftGeom g;
  g.n = nphi; g.batch = NP; g.bs = seq_stride(nphi); g.es = 1; g.pad = 1; g.jfast = true;
  const int* __restrict__ rev = a.fd.rev;
  // the band between the two Hermitian halves is zero
  for (int idx = tid; idx < NP * nphi; idx += PTHREADS) {
    int b = idx / nphi, m = idx - b * nphi;
    if (m >= M && m <= nphi - M) sm[g.addr(b, __ldg(rev + m))] = make_double2(0.0, 0.0);
  }
  for (int idx = tid; idx < M * NP; idx += PTHREADS) {
    int b = idx % NP, m = idx / NP;
    double2 Fi = make_double2(0.0, 0.0), Fm = Fi;
    if (b < np) {
      double2 Se = G[(((size_t)m * 2 + 0) * a.nz + k) * nlat2 + p0 + b];
      double2 So = G[(((size_t)m * 2 + 1) * a.nz + k) * nlat2 + p0 + b];
      Fi = cadd(Se, So);
      Fm = csub(Se, So);
    }
    if (m == 0) {
      sm[g.addr(b, __ldg(rev))] = make_double2(Fi.x, Fm.x);
    } else {
      // z = x + i y with x, y the real fields of ring i and its mirror
      sm[g.addr(b, __ldg(rev + m))] = make_double2(Fi.x - Fm.y, Fi.y + Fm.x);
      sm[g.addr(b, __ldg(rev + nphi - m))] = make_double2(Fi.x + Fm.y, -Fi.y + Fm.x);
    }
  }
  __syncthreads();
  fft_dit(sm, a.fd, g, +1);

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

bool smem_attr(const void* fn) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
         cudaSuccess;
}

}  // namespace

int launch_phi_fwd(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st) {
  if (nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  if (p->nphi > PMAXC) return SPH_EINVAL;
  PhiArgs a = {};
  for (int f = 0; f < nfields; ++f) a.gin[f] = grids[f];
  a.G = p->G;
  a.Gfield = p->Gfield;
  a.nlat = p->nlat; a.nlat2 = p->nlat2; a.nphi = p->nphi; a.nz = p->nz; a.lmax = p->lmax;
  a.NP = pairs_per_cta(p);
  a.wfold = p->wfold;
  a.fd = p->fphi;
  static bool once = smem_attr((const void*)phi_fwd_kernel);
  if (!once) return SPH_ECUDA;
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_FWD, st);
  phi_fwd_kernel<<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_phi_inv(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st) {
  if (nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  if (p->nphi > PMAXC) return SPH_EINVAL;
  PhiArgs a = {};
  for (int f = 0; f < nfields; ++f) a.gout[f] = grids[f];
  a.Gc = p->G;
  a.Gfield = p->Gfield;
  a.nlat = p->nlat; a.nlat2 = p->nlat2; a.nphi = p->nphi; a.nz = p->nz; a.lmax = p->lmax;
  a.NP = pairs_per_cta(p);
  a.wfold = p->wfold;
  a.fd = p->fphi;
  static bool once = smem_attr((const void*)phi_inv_kernel);
  if (!once) return SPH_ECUDA;
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_INV, st);
  phi_inv_kernel<<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
