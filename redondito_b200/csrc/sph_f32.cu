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

// FP64 spectral scratch i (0..2) of the plan, allocated on first use
int scratch(sph_plan* p, int i, double2** out) {
  if (!p->fsp[i] && cudaMalloc((void**)&p->fsp[i], spec_elems(p) * sizeof(double2)) != cudaSuccess)
    return SPH_ENOMEM;
  *out = p->fsp[i];
  return SPH_OK;
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
