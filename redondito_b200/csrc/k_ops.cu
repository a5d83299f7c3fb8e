// k_ops.cu -- pointwise pseudospectral operators, the no-slip boundary and
// the FP64 energy reduction.  Memory-bound kernels over the (lm, z) and
// (theta, phi, z) layouts; grids are sized as a multiple of the SM count by
// grid-stride loops.
#include <algorithm>

#include "sph_internal.cuh"

namespace {

constexpr int EW_THREADS = 256;

int ew_blocks(size_t n) {
  size_t b = (n + EW_THREADS - 1) / EW_THREADS;
  const size_t cap = 148 * 16;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

// derivr_k (src/pseudo/pseudospec_hd.f90:60-98): b = (i kz)^p a
__global__ void kmul_kernel(const double2* __restrict__ a, double2* __restrict__ b,
                            const double2* __restrict__ f, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    b[q] = cmul(f[q / nlm], a[q]);
}

// fc_filter_k (pseudospec_hd.f90:407-440)
__global__ void rowscale_kernel(double2* a, const double* __restrict__ f, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    a[q] = cscale(a[q], f[q / nlm]);
}

// laplang (pseudospec_hd.f90:138-172): b = -l(l+1) a
__global__ void laplang_kernel(const double2* __restrict__ a, double2* __restrict__ b,
                               const int* __restrict__ ell, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int l = ell[q % nlm];
    b[q] = cscale(a[q], (double)(-l * (l + 1)));
  }
}

// multr (pseudospec_hd.f90:175-208): b = z^p a, integer p as Fortran's z**p
__global__ void multr_kernel(const double2* __restrict__ a, double2* __restrict__ b,
                             const double* __restrict__ z, int power, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double zk = z[q / nlm], zp = 1.0;
    int ap = power < 0 ? -power : power;
    for (int i = 0; i < ap; ++i) zp *= zk;
    if (power < 0) zp = 1.0 / zp;
    b[q] = cscale(a[q], zp);
  }
}

// saxpby_c / saxpby_r (pseudospec_hd.f90:291-366): z = a x + b y
__global__ void saxpby_kernel(double* z, const double* x, double a, const double* y, double b, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    z[q] = a * x[q] + b * y[q];
}

// prodvec (pseudospec_hd.f90:211-251): C = A x B on planes k < N; zero beyond.
__global__ void prodvec_kernel(const double* __restrict__ ar, const double* __restrict__ at,
                               const double* __restrict__ ap, const double* __restrict__ br,
                               const double* __restrict__ bt, const double* __restrict__ bp,
                               double* cr, double* ct, double* cp, size_t nphys, size_t ntot) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ntot; q += (size_t)gridDim.x * blockDim.x) {
    if (q < nphys) {
      double xr = ar[q], xt = at[q], xp = ap[q], yr = br[q], yt = bt[q], yp = bp[q];
      cr[q] = xt * yp - xp * yt;
      ct[q] = xp * yr - xr * yp;
      cp[q] = xr * yt - xt * yr;
    } else {
      cr[q] = 0.0;
      ct[q] = 0.0;
      cp[q] = 0.0;
    }
  }
}

// dirichlet (src/boundary/boundary_mod.f90:62-93): rows 1 and N
__global__ void dirichlet_kernel(double2* a, int nlm, int N) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    a[lm] = make_double2(0.0, 0.0);
    a[(size_t)(N - 1) * nlm + lm] = make_double2(0.0, 0.0);
  }
}

// One wall value of column lm from the d-1 values inside it, the reference's
// reconstruction loop (fcgram_mod.f90:368-650, z boundaries): acc = neu(d) g
// + sum_k neu(k) f(interior k), divided by a neu(d) + 1 for Robin.  Rows
// (0-based) of the interior points: d - k at the inner wall, N - 1 - d + k at
// the outer one.
__device__ __forceinline__ double2 reconstruct_col(const double2* f, int lm, int nlm, int N, int d, int boun,
                                                   const double* neu, bool robin, double a, double2 g) {
  double2 acc = cscale(g, neu[d - 1]);
  for (int k = 1; k <= d - 1; ++k) {
    const int row = boun == 0 ? d - k : N - 1 - d + k;
    const double2 v = f[(size_t)row * nlm + lm];
    acc = make_double2(acc.x + neu[k - 1] * v.x, acc.y + neu[k - 1] * v.y);
  }
  if (robin) {
    const double s = a * neu[d - 1] + 1.0;
    acc = make_double2(acc.x / s, acc.y / s);
  }
  return acc;
}

__global__ void reconstruct_kernel(double2* f, const double* __restrict__ neu, const double* __restrict__ a,
                                   int nlm, int N, int d, int boun, int robin) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    const int b = boun == 0 ? 0 : N - 1;
    const double2 g = f[(size_t)b * nlm + lm];
    f[(size_t)b * nlm + lm] = reconstruct_col(f, lm, nlm, N, d, boun, neu, robin != 0, robin ? a[lm] : 0.0, g);
  }
}

// the toroidal condition at both walls: Z = 0 (noslip), or Z' - 2 Z/r = 0
// (freeslip) by the Robin reconstruction with g = 0, a = +2/rint inside and
// -2/rext outside (outward normal derivatives)
__global__ void bc_walls_kernel(double2* tor, const double* __restrict__ neu, int nlm, int N, int d, int kin,
                                int kout, double ain, double aout) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    for (int w = 0; w < 2; ++w) {
      const int b = w == 0 ? 0 : N - 1;
      const int kind = w == 0 ? kin : kout;
      double2 v = make_double2(0.0, 0.0);
      if (kind == 1) v = reconstruct_col(tor, lm, nlm, N, d, w, neu, true, w == 0 ? ain : aout, v);
      tor[(size_t)b * nlm + lm] = v;
    }
  }
}

// invDl (boundary_mod.f90:244-292): W(1:N) = M_l phi(3:N-2) for all m of one
// l, the reference's DGEMM with two columns (re, im) per mode.  CTA: one l and
// up to 32 m; phi rows staged in shared memory, M_l streamed from L2.  The
// arrays are the caller's lm columns [lm0, lm0 + nlm); modes outside are
// skipped.
constexpr int IDL_M = 32;
__global__ void __launch_bounds__(256) invdl_kernel(const double2* __restrict__ phi, double2* __restrict__ w,
                                                    const double* __restrict__ binv,
                                                    const int* __restrict__ mbase, int lm0, int nlm, int N) {
  extern __shared__ double2 Ph[];  // [(N-4)][IDL_M]
  const int l = blockIdx.x + 1;
  const int m0 = blockIdx.y * IDL_M;
  if (m0 > l) return;
  const int nm = min(IDL_M, l + 1 - m0);
  const int K = N - 4;
  for (int idx = threadIdx.x; idx < K * IDL_M; idx += blockDim.x) {
    int j = idx / IDL_M, mm = idx - j * IDL_M;
    double2 v = make_double2(0.0, 0.0);
    if (mm < nm) {
      const int lm = mbase[m0 + mm] + (l - m0 - mm) - lm0;  // column of the caller's slab
      if (lm >= 0 && lm < nlm) v = phi[(size_t)(j + 2) * nlm + lm];
    }
    Ph[idx] = v;
  }
  __syncthreads();
  const double* M = binv + (size_t)(l - 1) * N * K;
  for (int idx = threadIdx.x; idx < N * nm; idx += blockDim.x) {
    int i = idx % N, mm = idx / N;
    double sr = 0.0, si = 0.0;
    for (int j = 0; j < K; ++j) {
      double c = __ldg(M + i + (size_t)N * j);
      double2 v = Ph[j * IDL_M + mm];
      sr += c * v.x;
      si += c * v.y;
    }
    const int lm = mbase[m0 + mm] + (l - m0 - mm) - lm0;
    if (lm >= 0 && lm < nlm) w[(size_t)i * nlm + lm] = make_double2(sr, si);
  }
}

// v_imposebc_fast step 3 (src/boundary/vboundary.f90:117-127)
__global__ void bc_fast_kernel(double2* phi, const double2* __restrict__ w, const double* __restrict__ d2bor,
                               const int* __restrict__ ell, const double* __restrict__ z, int nlm, int nz,
                               int N) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    int l = ell[lm];
    if (l == 0) {
      for (int k = 0; k < nz; ++k) phi[(size_t)k * nlm + lm] = make_double2(0.0, 0.0);
      continue;
    }
    const int rows[4] = {0, 1, N - 2, N - 1};
    double2 s[4];
    for (int r = 0; r < 4; ++r) s[r] = make_double2(0.0, 0.0);
    for (int j = 0; j < N; ++j) {
      double2 v = w[(size_t)j * nlm + lm];
      for (int r = 0; r < 4; ++r) {
        double c = d2bor[r + 4 * j];
        s[r].x += c * v.x;
        s[r].y += c * v.y;
      }
    }
    double lf = (double)(l * (l + 1));
    for (int r = 0; r < 4; ++r) {
      int i = rows[r];
      double zi = z[i];
      double2 wi = w[(size_t)i * nlm + lm];
      phi[(size_t)i * nlm + lm] = make_double2(s[r].x - lf * wi.x / (zi * zi), s[r].y - lf * wi.y / (zi * zi));
    }
  }
}

// QST potentials of u and curl u: out = sc * z^rpow * (l(l+1) if lfac) * in
__global__ void qst_scale_kernel(const double2* __restrict__ a, double2* __restrict__ b,
                                 const double* __restrict__ z, const int* __restrict__ ell, int rpow,
                                 int lfac, double sc, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int l = ell[q % nlm];
    double f = sc * pow(z[q / nlm], (double)rpow) * (lfac ? (double)(l * (l + 1)) : 1.0);
    b[q] = cscale(a[q], f);
  }
}

// 0.5 * sum_k c_k r_k^2 dz sum_{j,i} w_i (2 pi/nphi) |u|^2 over k < N (FP64)
__global__ void energy_kernel(const double* __restrict__ ur, const double* __restrict__ ut,
                              const double* __restrict__ up, const double* __restrict__ w,
                              const double* __restrict__ z, int nlat, int nphi, int N, double scale,
                              double* acc) {
  __shared__ double red[EW_THREADS / 32];
  const size_t plane = (size_t)nlat * nphi;
  const size_t n = plane * N;
  double s = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int k = (int)(q / plane);
    int i = (int)(q % nlat);
    double ck = (k == 0 || k == N - 1) ? 0.5 : 1.0;
    double rk = z[k];
    double v = ur[q] * ur[q] + ut[q] * ut[q] + up[q] * up[q];
    s += ck * rk * rk * w[i] * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (EW_THREADS / 32) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) atomicAdd(acc, s * scale);
  }
}

}  // namespace

int launch_kmul(const sph_plan* p, const double2* a, double2* b, int order, cudaStream_t st) {
  if (order < 0 || order > 4) return SPH_EINVAL;
  size_t n = spec_view(p);
  if (order == 0) {
    if (a != b) SPH_CUDA_OK(cudaMemcpyAsync(b, a, n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    return SPH_OK;
  }
  TimedLaunch tl(p, T_OPS, st);
  kmul_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(a, b, p->kfac + (size_t)(order - 1) * p->nz, p->nlmv, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_filter_k(const sph_plan* p, double2* a, cudaStream_t st) {
  size_t n = spec_view(p);
  TimedLaunch tl(p, T_OPS, st);
  rowscale_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(a, p->filt, p->nlmv, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_laplang(const sph_plan* p, const double2* a, double2* b, cudaStream_t st) {
  size_t n = spec_view(p);
  TimedLaunch tl(p, T_OPS, st);
  laplang_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(a, b, p->d_ell + p->lm0, p->nlmv, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_multr(const sph_plan* p, const double2* a, double2* b, int power, cudaStream_t st) {
  size_t n = spec_view(p);
  TimedLaunch tl(p, T_OPS, st);
  multr_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(a, b, p->d_z, power, p->nlmv, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_saxpby(const sph_plan* p, double* z, const double* x, double a, const double* y, double b,
                  size_t n, cudaStream_t st) {
  TimedLaunch tl(p, T_OPS, st);
  saxpby_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(z, x, a, y, b, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_prodvec(const sph_plan* p, const double* const* A, const double* const* B,
                   double* const* Cout, cudaStream_t st) {
  // the caller's planes [k0, k0 + nzv); physical where k < N
  size_t plane = (size_t)p->nlat * p->nphi;
  const int nphys_planes = std::max(0, std::min(p->nzv, p->N - p->k0));
  size_t ntot = plane * p->nzv, nphys = plane * nphys_planes;
  TimedLaunch tl(p, T_OPS, st);
  prodvec_kernel<<<ew_blocks(ntot), EW_THREADS, 0, st>>>(A[0], A[1], A[2], B[0], B[1], B[2], Cout[0],
                                                        Cout[1], Cout[2], nphys, ntot);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_dirichlet(const sph_plan* p, double2* a, cudaStream_t st) {
  TimedLaunch tl(p, T_OPS, st);
  dirichlet_kernel<<<ew_blocks(p->nlmv), EW_THREADS, 0, st>>>(a, p->nlmv, p->N);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_bc_walls(const sph_plan* p, double2* tor, cudaStream_t st) {
  if ((p->bck[0] || p->bck[1]) && (!p->d_neu || p->neu[0].empty())) return SPH_ENOTREADY;
  TimedLaunch tl(p, T_OPS, st);
  bc_walls_kernel<<<ew_blocks(p->nlmv), EW_THREADS, 0, st>>>(tor, p->d_neu, p->nlmv, p->N, p->d, p->bck[0],
                                                             p->bck[1], 2.0 / p->z[0], -2.0 / p->z[p->N - 1]);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_reconstruct(const sph_plan* p, double2* f, int boun, int ord, const double* a, cudaStream_t st) {
  if ((boun != 0 && boun != 1) || (ord != 1 && ord != 2)) return SPH_EINVAL;
  if (!p->d_neu || p->neu[ord - 1].empty() || p->N < p->d) return SPH_ENOTREADY;
  TimedLaunch tl(p, T_OPS, st);
  reconstruct_kernel<<<ew_blocks(p->nlmv), EW_THREADS, 0, st>>>(f, p->d_neu + (size_t)(ord - 1) * p->d, a, p->nlmv,
                                                               p->N, p->d, boun, a != nullptr);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_invDl(const sph_plan* p, const double2* phi, double2* w, cudaStream_t st) {
  SPH_CUDA_OK(cudaMemsetAsync(w, 0, spec_view(p) * sizeof(double2), st));
  if (p->lmax < 1) return SPH_OK;
  size_t smem = (size_t)(p->N - 4) * IDL_M * sizeof(double2);
  if (smem > 200 * 1024) return SPH_EINVAL;
  static DeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(invdl_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) ==
               cudaSuccess;
      }))
    return SPH_ECUDA;
  dim3 grid(p->lmax, (p->lmax + 1 + IDL_M - 1) / IDL_M);
  TimedLaunch tl(p, T_OPS, st);
  invdl_kernel<<<grid, 256, smem, st>>>(phi, w, p->binv, p->d_mbase, p->lm0, p->nlmv, p->N);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_bc_fast_rows(const sph_plan* p, double2* phi, const double2* w, cudaStream_t st) {
  TimedLaunch tl(p, T_OPS, st);
  bc_fast_kernel<<<ew_blocks(p->nlmv), EW_THREADS, 0, st>>>(phi, w, p->d2bor, p->d_ell + p->lm0, p->d_z, p->nlmv,
                                                            p->nz, p->N);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_qst_scale(const sph_plan* p, const double2* in, double2* out, int rpow, int lfac, double sc,
                     cudaStream_t st) {
  size_t n = spec_elems(p);
  TimedLaunch tl(p, T_OPS, st);
  qst_scale_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(in, out, p->d_z, p->d_ell, rpow, lfac, sc, p->nlm, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_energy(const sph_plan* p, const double* ur, const double* ut, const double* up, double* acc,
                  cudaStream_t st) {
  size_t n = (size_t)p->nlat * p->nphi * p->N;
  double scale = 0.5 * p->dz * 2.0 * 3.14159265358979323846 / p->nphi;
  TimedLaunch tl(p, T_OPS, st);
  energy_kernel<<<ew_blocks(n), EW_THREADS, 0, st>>>(ur, ut, up, p->wfull, p->d_z, p->nlat, p->nphi, p->N,
                                                     scale, acc);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
