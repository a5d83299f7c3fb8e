// sph_f32.cu -- single-precision entry points: the arrays of a
// GSINGLE_PRECISION build of the reference (src/sphp/fprecision_mod.F90:13-18,
// REAL(KIND=GP) and COMPLEX(KIND=GP) with GP = 4) on an SPH_MIXED plan.
//
// The reference's single build runs every step in single precision.  Here
// the arrays at the interface are float (grids) and float pairs (spectra),
// and the plan's mixed engine does the work: fp32 phi FFTs that read and
// write the float grids directly (half the bytes of an FP64 grid), bf16x3
// tensor-core Legendre contractions, FP64 z transforms that read and write
// the float spectra (widened in shared memory), FP64 continuation.  Where a
// step needs FP64 spectra in between (the Legendre contractions' outputs and
// inputs, the boundary solve, the nonlinear step), they live in the plan's
// own scratch.
//
// Each entry point has the name and arguments of its FP64 counterpart with
// float arrays; they take whole fields only (no slab views).
#include "sph_internal.cuh"

namespace {

#define RCF(x)                \
  do {                        \
    const int rc_ = (x);      \
    if (rc_ != SPH_OK) return rc_; \
  } while (0)

inline cudaStream_t st_of(void* s) { return (cudaStream_t)s; }

// single-precision entry points need a mixed plan over whole fields
inline bool f32_ok(const sph_plan* p) { return p && p->precision == SPH_MIXED && slab_whole(p); }

__global__ void widen_kernel(const float* __restrict__ in, double* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)__ldg(in + i);
}
__global__ void narrow_kernel(const double* __restrict__ in, float* __restrict__ out, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (float)__ldg(in + i);
}

int blocks_for(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

// n reals float -> FP64 / FP64 -> float
int widen(const float* in, double* out, size_t n, cudaStream_t st) {
  if (n == 0) return SPH_OK;
  widen_kernel<<<blocks_for(n), 256, 0, st>>>(in, out, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
int narrow(const double* in, float* out, size_t n, cudaStream_t st) {
  if (n == 0) return SPH_OK;
  narrow_kernel<<<blocks_for(n), 256, 0, st>>>(in, out, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

// FP64 spectral scratch i (0..4) of the plan, allocated on first use
int scratch(sph_plan* p, int i, double2** out) {
  if (!p->fsp[i] && cudaMalloc((void**)&p->fsp[i], spec_elems(p) * sizeof(double2)) != cudaSuccess)
    return SPH_ENOMEM;
  *out = p->fsp[i];
  return SPH_OK;
}

// pointwise operators on float arrays, computed in FP64
// (pseudospec_hd.f90:138-251,291-366; boundary_mod.f90:62-93)
__global__ void laplang_f32(const float2* __restrict__ a, float2* __restrict__ b, const int* __restrict__ ell,
                            int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int l = ell[q % nlm];
    const double f = -(double)(l * (l + 1));
    const float2 v = a[q];
    b[q] = make_float2((float)(f * v.x), (float)(f * v.y));
  }
}
__global__ void multr_f32(const float2* __restrict__ a, float2* __restrict__ b, const double* __restrict__ z,
                          int power, int nlm, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double zk = z[q / nlm], zp = 1.0;
    const int ap = power < 0 ? -power : power;
    for (int i = 0; i < ap; ++i) zp *= zk;
    if (power < 0) zp = 1.0 / zp;
    const float2 v = a[q];
    b[q] = make_float2((float)(zp * v.x), (float)(zp * v.y));
  }
}
__global__ void saxpby_f32(float* z, const float* x, double a, const float* y, double b, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    z[q] = (float)(a * (double)x[q] + b * (double)y[q]);
}
__global__ void prodvec_f32(const float* __restrict__ ar, const float* __restrict__ at, const float* __restrict__ ap,
                            const float* __restrict__ br, const float* __restrict__ bt, const float* __restrict__ bp,
                            float* cr, float* ct, float* cp, size_t nphys, size_t ntot) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ntot; q += (size_t)gridDim.x * blockDim.x) {
    if (q < nphys) {
      const double xr = ar[q], xt = at[q], xp = ap[q], yr = br[q], yt = bt[q], yp = bp[q];
      cr[q] = (float)(xt * yp - xp * yt);
      ct[q] = (float)(xp * yr - xr * yp);
      cp[q] = (float)(xr * yt - xt * yr);
    } else {
      cr[q] = ct[q] = cp[q] = 0.0f;
    }
  }
}
__global__ void dirichlet_f32(float2* a, int nlm, int N) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    a[lm] = make_float2(0.f, 0.f);
    a[(size_t)(N - 1) * nlm + lm] = make_float2(0.f, 0.f);
  }
}

// float spectra -> FP64 scratch i
int widen_spec(sph_plan* p, const float* in, int i, double2** out, cudaStream_t st) {
  RCF(scratch(p, i, out));
  return widen(in, reinterpret_cast<double*>(*out), 2 * spec_elems(p), st);
}
int narrow_spec(const sph_plan* p, const double2* in, float* out, cudaStream_t st) {
  return narrow(reinterpret_cast<const double*>(in), out, 2 * spec_elems(p), st);
}

// the analysis of nv fields (1: scalar, 3: vector) from float grids g into
// FP64 spectra o (the physical continuation first when `cont`)
int analysis(sph_plan* p, const float* const* g, int nv, double2* const* o, bool cont, cudaStream_t st) {
  const void* gv[SPH_MAX_FIELDS] = {};
  for (int f = 0; f < nv; ++f) gv[f] = g[f];
  if (cont) {
    const void* gh[SPH_MAX_FIELDS] = {};
    for (int f = 0; f < nv; ++f) gh[f] = reinterpret_cast<const float*>(p->contg) + (size_t)f * p->C * p->nphi * p->nlat;
    RCF(launch_cont_phys_g(p, gv, nv, st, true));
    RCF(launch_phi_fwd32_g(p, gv, nv, st, gh, true));
  } else {
    RCF(launch_phi_fwd32_g(p, gv, nv, st, nullptr, true));
  }
  RCF(launch_tc_analysis(p, 0, o[0], nullptr, st));
  if (nv == 3) RCF(launch_tc_analysis(p, 1, o[1], o[2], st));
  return SPH_OK;
}

// the synthesis of nv fields from FP64 spectra i into float grids g
int synthesis(sph_plan* p, const double2* const* i, int nv, float* const* g, cudaStream_t st) {
  RCF(launch_tc_synthesis(p, 0, i[0], nullptr, st));
  if (nv == 3) RCF(launch_tc_synthesis(p, 1, i[1], i[2], st));
  void* gv[SPH_MAX_FIELDS] = {};
  for (int f = 0; f < nv; ++f) gv[f] = g[f];
  return launch_phi_inv32_g(p, gv, nv, st, true);
}

}  // namespace

// ---------------------------------------------------------------- transforms
extern "C" int sph_fftp2d_real_to_complex_xy_f32(sph_plan* p, const float* in, float* out, void* s) {
  if (!f32_ok(p) || !in || !out) return SPH_EINVAL;
  double2* o;
  RCF(scratch(p, 0, &o));
  RCF(analysis(p, &in, 1, &o, false, st_of(s)));
  return narrow(reinterpret_cast<const double*>(o), out, 2 * spec_elems(p), st_of(s));
}

extern "C" int sph_fftp2d_complex_to_real_xy_f32(sph_plan* p, const float* in, float* out, void* s) {
  if (!f32_ok(p) || !in || !out) return SPH_EINVAL;
  double2* i;
  RCF(scratch(p, 0, &i));
  RCF(widen(in, reinterpret_cast<double*>(i), 2 * spec_elems(p), st_of(s)));
  return synthesis(p, &i, 1, &out, st_of(s));
}

extern "C" int sph_fftp1d_real_to_complex_z_f32(sph_plan* p, float* inout, void* s) {
  if (!f32_ok(p) || !inout) return SPH_EINVAL;
  return launch_zfft_io(p, Z_FWD, inout, inout, ZIO_FF, 0, st_of(s));
}

extern "C" int sph_fftp1d_complex_to_real_z_f32(sph_plan* p, float* inout, void* s) {
  if (!f32_ok(p) || !inout) return SPH_EINVAL;
  return launch_zfft_io(p, Z_INV, inout, inout, ZIO_FF, 0, st_of(s));
}

// grid -> (lm, kz): the physical continuation and the analysis write FP64
// spectra to scratch, the z transform reads them and writes the float output
extern "C" int sph_fftp3d_real_to_complex_f32(sph_plan* p, const float* in, float* out, void* s) {
  if (!f32_ok(p) || !in || !out) return SPH_EINVAL;
  double2* o;
  RCF(scratch(p, 0, &o));
  const bool cont = p->C > 0 && p->contg;
  RCF(analysis(p, &in, 1, &o, cont, st_of(s)));
  return launch_zfft_io(p, Z_FWD, o, out, ZIO_DF, 0, st_of(s), !cont);
}

// (lm, kz) -> grid: the z inverse reads the float spectra and writes FP64
// scratch for the synthesis; the input is preserved
extern "C" int sph_fftp3d_complex_to_real_f32(sph_plan* p, const float* in, float* out, void* s) {
  if (!f32_ok(p) || !in || !out) return SPH_EINVAL;
  if (zinv_tiles_ok(p)) {  // the z inverse writes the synthesis tiles directly
    RCF(launch_zinv_tiles_g(p, in, 0, st_of(s), true));
    RCF(launch_tc_synthesis_tiles(p, 0, st_of(s)));
    void* g[1] = {out};
    return launch_phi_inv32_g(p, g, 1, st_of(s), true);
  }
  double2* i;
  RCF(scratch(p, 0, &i));
  RCF(launch_zfft_io(p, Z_INV, in, i, ZIO_FD, 0, st_of(s)));
  return synthesis(p, &i, 1, &out, st_of(s));
}

extern "C" int sph_fftp2d_vec_to_qst_f32(sph_plan* p, const float* vr, const float* vt, const float* vp, float* q,
                                         float* sO, float* t, void* s) {
  if (!f32_ok(p) || !vr || !vt || !vp || !q || !sO || !t) return SPH_EINVAL;
  double2* o[3];
  for (int f = 0; f < 3; ++f) RCF(scratch(p, f, &o[f]));
  const float* g[3] = {vr, vt, vp};
  RCF(analysis(p, g, 3, o, false, st_of(s)));
  float* out[3] = {q, sO, t};
  for (int f = 0; f < 3; ++f) RCF(narrow(reinterpret_cast<const double*>(o[f]), out[f], 2 * spec_elems(p), st_of(s)));
  return SPH_OK;
}

extern "C" int sph_fftp2d_qst_to_vec_f32(sph_plan* p, const float* q, const float* sI, const float* t, float* vr,
                                         float* vt, float* vp, void* s) {
  if (!f32_ok(p) || !q || !sI || !t || !vr || !vt || !vp) return SPH_EINVAL;
  double2* i[3];
  const float* in[3] = {q, sI, t};
  for (int f = 0; f < 3; ++f) {
    RCF(scratch(p, f, &i[f]));
    RCF(widen(in[f], reinterpret_cast<double*>(i[f]), 2 * spec_elems(p), st_of(s)));
  }
  float* g[3] = {vr, vt, vp};
  return synthesis(p, i, 3, g, st_of(s));
}

extern "C" int sph_fftp3d_vec_to_qst_f32(sph_plan* p, const float* vr, const float* vt, const float* vp, float* q,
                                         float* sO, float* t, void* s) {
  if (!f32_ok(p) || !vr || !vt || !vp || !q || !sO || !t) return SPH_EINVAL;
  double2* o[3];
  for (int f = 0; f < 3; ++f) RCF(scratch(p, f, &o[f]));
  const float* g[3] = {vr, vt, vp};
  const bool cont = p->C > 0 && p->contg;
  RCF(analysis(p, g, 3, o, cont, st_of(s)));
  float* out[3] = {q, sO, t};
  for (int f = 0; f < 3; ++f) RCF(launch_zfft_io(p, Z_FWD, o[f], out[f], ZIO_DF, 0, st_of(s), !cont));
  return SPH_OK;
}

extern "C" int sph_fftp3d_qst_to_vec_f32(sph_plan* p, const float* q, const float* sI, const float* t, float* vr,
                                         float* vt, float* vp, void* s) {
  if (!f32_ok(p) || !q || !sI || !t || !vr || !vt || !vp) return SPH_EINVAL;
  if (zinv_tiles_ok(p)) {
    RCF(launch_zinv_tiles_g(p, q, 0, st_of(s), true));
    RCF(launch_tc_synthesis_tiles(p, 0, st_of(s)));
    RCF(launch_zinv_tiles_g(p, sI, 0, st_of(s), true));
    RCF(launch_zinv_tiles_g(p, t, 1, st_of(s), true));
    RCF(launch_tc_synthesis_tiles(p, 1, st_of(s)));
    void* g[3] = {vr, vt, vp};
    return launch_phi_inv32_g(p, g, 3, st_of(s), true);
  }
  double2* i[3];
  const float* in[3] = {q, sI, t};
  for (int f = 0; f < 3; ++f) {
    RCF(scratch(p, f, &i[f]));
    RCF(launch_zfft_io(p, Z_INV, in[f], i[f], ZIO_FD, 0, st_of(s)));
  }
  float* g[3] = {vr, vt, vp};
  return synthesis(p, i, 3, g, st_of(s));
}

// ---------------------------------------------------------------- radial operators
// derivr (src/pseudo/pseudospec_hd.f90:101-135) in physical space: one fused
// z transform reading and writing float spectra
extern "C" int sph_derivr_f32(sph_plan* p, const float* a, float* b, int order, char esp, void* s) {
  if (!f32_ok(p) || !a || !b || order < 0 || order > 4 || (esp != 'r' && esp != 'k')) return SPH_EINVAL;
  if (esp == 'k' || order == 0) {  // (i kz)^p in place of the spectral coefficients, or forward and back
    double2* x;
    RCF(scratch(p, 0, &x));
    RCF(widen(a, reinterpret_cast<double*>(x), 2 * spec_elems(p), st_of(s)));
    RCF(sph_derivr(p, reinterpret_cast<const double*>(x), reinterpret_cast<double*>(x), order, esp, s));
    return narrow(reinterpret_cast<const double*>(x), b, 2 * spec_elems(p), st_of(s));
  }
  return launch_zfft_io(p, Z_DERIV, a, b, ZIO_FF, order, st_of(s));
}

extern "C" int sph_dlr_f32(sph_plan* p, const float* a, float* b, void* s) {
  if (!f32_ok(p) || !a || !b) return SPH_EINVAL;
  return launch_zfft_io(p, Z_DLR, a, b, ZIO_FF, 2, st_of(s));
}

extern "C" int sph_fc_filter_f32(sph_plan* p, float* a, char esp, void* s) {
  if (!f32_ok(p) || !a || (esp != 'r' && esp != 'k')) return SPH_EINVAL;
  if (esp == 'r') return launch_zfft_io(p, Z_FILTER, a, a, ZIO_FF, 0, st_of(s));
  double2* x;
  RCF(scratch(p, 0, &x));
  RCF(widen(a, reinterpret_cast<double*>(x), 2 * spec_elems(p), st_of(s)));
  RCF(sph_fc_filter(p, reinterpret_cast<double*>(x), 'k', s));
  return narrow(reinterpret_cast<const double*>(x), a, 2 * spec_elems(p), st_of(s));
}

// ---------------------------------------------------------------- pointwise operators
extern "C" int sph_laplang_f32(sph_plan* p, const float* a, float* b, void* s) {
  if (!f32_ok(p) || !a || !b) return SPH_EINVAL;
  const size_t n = spec_elems(p);
  laplang_f32<<<blocks_for(n), 256, 0, st_of(s)>>>(reinterpret_cast<const float2*>(a), reinterpret_cast<float2*>(b),
                                                    p->d_ell, p->nlm, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

extern "C" int sph_multr_f32(sph_plan* p, const float* a, float* b, int pw, void* s) {
  if (!f32_ok(p) || !a || !b) return SPH_EINVAL;
  const size_t n = spec_elems(p);
  multr_f32<<<blocks_for(n), 256, 0, st_of(s)>>>(reinterpret_cast<const float2*>(a), reinterpret_cast<float2*>(b),
                                                  p->d_z, pw, p->nlm, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

extern "C" int sph_saxpby_c_f32(sph_plan* p, float* z, const float* x, double a, const float* y, double b, void* s) {
  if (!f32_ok(p) || !z || !x || !y) return SPH_EINVAL;
  const size_t n = 2 * spec_elems(p);
  saxpby_f32<<<blocks_for(n), 256, 0, st_of(s)>>>(z, x, a, y, b, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

extern "C" int sph_saxpby_r_f32(sph_plan* p, float* z, const float* x, double a, const float* y, double b, void* s) {
  if (!f32_ok(p) || !z || !x || !y) return SPH_EINVAL;
  const size_t n = grid_elems(p);
  saxpby_f32<<<blocks_for(n), 256, 0, st_of(s)>>>(z, x, a, y, b, n);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

extern "C" int sph_copy_f32(sph_plan* p, const float* a, float* b, void* s) {
  if (!f32_ok(p) || !a || !b) return SPH_EINVAL;
  if (a != b && cudaMemcpyAsync(b, a, spec_elems(p) * 2 * sizeof(float), cudaMemcpyDeviceToDevice, st_of(s)) !=
                    cudaSuccess)
    return SPH_ECUDA;
  return SPH_OK;
}

extern "C" int sph_prodvec_f32(sph_plan* p, const float* ar, const float* at, const float* ap, const float* br,
                               const float* bt, const float* bp, float* cr, float* ct, float* cp, void* s) {
  if (!f32_ok(p) || !ar || !at || !ap || !br || !bt || !bp || !cr || !ct || !cp) return SPH_EINVAL;
  const size_t plane = (size_t)p->nlat * p->nphi, ntot = plane * p->nz, nphys = plane * p->N;
  prodvec_f32<<<blocks_for(ntot), 256, 0, st_of(s)>>>(ar, at, ap, br, bt, bp, cr, ct, cp, nphys, ntot);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

extern "C" int sph_dirichlet_f32(sph_plan* p, float* a, void* s) {
  if (!f32_ok(p) || !a) return SPH_EINVAL;
  dirichlet_f32<<<blocks_for(p->nlm), 256, 0, st_of(s)>>>(reinterpret_cast<float2*>(a), p->nlm, p->N);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

// ---------------------------------------------------------------- boundary, NL step
// The boundary solve and the nonlinear step run on FP64 copies of the float
// spectra in the plan's scratch (the state of a step is FP64 by design; the
// copies are a small share of a step's traffic).
extern "C" int sph_invDl_f32(sph_plan* p, const float* phi, float* w, void* s) {
  if (!f32_ok(p) || !phi || !w) return SPH_EINVAL;
  double2 *f, *x;
  RCF(widen_spec(p, phi, 0, &f, st_of(s)));
  RCF(scratch(p, 1, &x));
  RCF(sph_invDl(p, reinterpret_cast<const double*>(f), reinterpret_cast<double*>(x), s));
  return narrow_spec(p, x, w, st_of(s));
}

namespace {
int imposebc_f32(sph_plan* p, float* tor, float* phi, float* pol, void* s, bool fast) {
  if (!f32_ok(p) || !tor || !phi || !pol) return SPH_EINVAL;
  double2 *t, *f, *w;
  RCF(widen_spec(p, tor, 0, &t, st_of(s)));
  RCF(widen_spec(p, phi, 1, &f, st_of(s)));
  RCF(widen_spec(p, pol, 2, &w, st_of(s)));  // v_imposebc_fast keeps pol's rows it does not set
  double *td = reinterpret_cast<double*>(t), *fd = reinterpret_cast<double*>(f), *wd = reinterpret_cast<double*>(w);
  RCF(fast ? sph_v_imposebc_fast(p, td, fd, wd, s) : sph_v_imposebc(p, td, fd, wd, s));
  RCF(narrow_spec(p, t, tor, st_of(s)));
  RCF(narrow_spec(p, f, phi, st_of(s)));
  return narrow_spec(p, w, pol, st_of(s));
}
}  // namespace

extern "C" int sph_v_imposebc_f32(sph_plan* p, float* tor, float* phi, float* pol, void* s) {
  return imposebc_f32(p, tor, phi, pol, s, false);
}

extern "C" int sph_v_imposebc_fast_f32(sph_plan* p, float* tor, float* phi, float* pol, void* s) {
  return imposebc_f32(p, tor, phi, pol, s, true);
}

extern "C" int sph_nl_rhs_f32(sph_plan* p, const float* Z, const float* W, const float* phi, double nu, float* rhs_z,
                              float* rhs_phi, double* energy, void* s) {
  if (!f32_ok(p) || !Z || !W || !phi || !rhs_z || !rhs_phi) return SPH_EINVAL;
  double2 *z, *w, *f, *rz, *rf;
  RCF(widen_spec(p, Z, 0, &z, st_of(s)));
  RCF(widen_spec(p, W, 1, &w, st_of(s)));
  RCF(widen_spec(p, phi, 2, &f, st_of(s)));
  RCF(scratch(p, 3, &rz));
  RCF(scratch(p, 4, &rf));
  RCF(sph_nl_rhs(p, reinterpret_cast<const double*>(z), reinterpret_cast<const double*>(w),
                 reinterpret_cast<const double*>(f), nu, reinterpret_cast<double*>(rz), reinterpret_cast<double*>(rf),
                 energy, s));
  RCF(narrow_spec(p, rz, rhs_z, st_of(s)));
  return narrow_spec(p, rf, rhs_phi, st_of(s));
}

extern "C" int sph_rk3_step_f32(sph_plan* p, float* Z, float* W, float* phi, double nu, double dt, double* energy,
                                void* s) {
  if (!f32_ok(p) || !Z || !W || !phi) return SPH_EINVAL;
  double2 *z, *w, *f;
  RCF(widen_spec(p, Z, 0, &z, st_of(s)));
  RCF(widen_spec(p, W, 1, &w, st_of(s)));
  RCF(widen_spec(p, phi, 2, &f, st_of(s)));
  RCF(sph_rk3_step(p, reinterpret_cast<double*>(z), reinterpret_cast<double*>(w), reinterpret_cast<double*>(f), nu,
                   dt, energy, s));
  RCF(narrow_spec(p, z, Z, st_of(s)));
  RCF(narrow_spec(p, w, W, st_of(s)));
  return narrow_spec(p, f, phi, st_of(s));
}
