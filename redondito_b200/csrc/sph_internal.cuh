// sph_internal.cuh -- plan layout, device helpers and launcher declarations
// shared by the CUDA sources of the transform core.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/sph_b200.h"

#define SPH_MAX_FIELDS 3
#define SPH_MAX_PASSES 16

// One Stockham pass: radix R applied after Ns points have been combined.
struct FftPass {
  int R, Ns;
};

// A length-n complex FFT in shared memory.  tw[e] = exp(-2 pi i e / n);
// rev[k] = position of frequency k after the decimation-in-frequency passes.
struct FftDesc {
  int n, npass;
  FftPass pass[SPH_MAX_PASSES];
  const double2* tw;
  const float2* twf;  // same table in fp32 (mixed-precision path)
  const int* rev;
  const double2* twp;   // per-pass table [pass][j][r-1] = W_L^{j r} (compile-time lengths)
  const float2* twpf;
};

// Legendre GEMM work tile: one (m, row block) pair.
struct LegTile {
  int m, r0;
};

// Mixed-precision (tcgen05) work item: one m, one parity (or output fold),
// one block of at most 256 MMA rows; its Legendre table tiles sit in HBM as
// nk consecutive blocks of [hi | lo] fp16 (2 x nr x 32 halves each, 8x8 core
// matrices, K-major), pre-scaled by the power of two tscale.
struct TcItem {
  int m, par, r0, nr, nvalid, nk, nk1, out;
  long long boff;  // first table block, in halves
  float tscale;
  int pad_;
};

struct TcSet {
  TcItem* items = nullptr;  // device
  int nitems = 0;
  __half* blocks = nullptr;  // device
  size_t nhalves = 0;
};

struct sph_plan {
  // sizes
  int lmax, nlat, nlat2, nphi, nz, C, d, nlm, N, precision;
  int ldn;  // node stride of the tables and folded buffers: nlat/2 rounded up to 4
  double rint, rext, dz, Dkz;
  // host copies of the grid (box_init)
  std::vector<double> theta, ct, w, phi, z, kz, dir;
  std::vector<int> ell, emm, mbase;
  // device tables
  double* P = nullptr;    // [nlm][ldn]  Pbar_lm(x_i), northern nodes (0 past nlat/2)
  double* dP = nullptr;   // [nlm][ldn]  d Pbar_lm / d theta
  double* mPs = nullptr;  // [nlm][ldn]  m Pbar_lm / sin theta
  double* wfold = nullptr;  // [nlat2] w_i * 2 pi / nphi
  double* wfull = nullptr;  // [nlat] Gauss weights
  double* d_dir = nullptr;  // [C*d] column-major
  double* d_z = nullptr;    // [nz]
  double2* kfac = nullptr;  // [4][nz] (i kz)^p for p = 1..4
  double* filt = nullptr;   // [nz] exponential filter factors
  double* zinv2 = nullptr;  // [nz] 1/z^2
  int* d_ell = nullptr;     // [nlm]
  int* d_mbase = nullptr;   // [lmax+2]
  double2* twz = nullptr;   // [nz]
  double2* twphi = nullptr; // [nphi]
  float2* twzf = nullptr;
  float2* twphif = nullptr;
  int* revz = nullptr;      // [nz]
  int* revphi = nullptr;    // [nphi]
  double2* twpz = nullptr;  // per-pass twiddles (see fft_ct.cuh)
  double2* twpphi = nullptr;
  float2* twpzf = nullptr;
  float2* twpphif = nullptr;
  FftDesc fz, fphi;
  // Legendre work lists (device)
  LegTile* tilesA = nullptr;   // analysis: (m, l0) blocks of 64 l
  int ntilesA = 0;
  LegTile* tilesA32 = nullptr; // vector analysis: blocks of 32 l
  int ntilesA32 = 0;
  LegTile* tilesS = nullptr;   // synthesis: (m, i0) blocks of 64 nodes
  int ntilesS = 0;
  LegTile* tilesS32 = nullptr; // vector synthesis: blocks of 32 nodes
  int ntilesS32 = 0;
  // scratch: folded Fourier coefficients, per field [lmax+1][2][nz][ldn] complex
  double2* G = nullptr;
  size_t Gfield = 0;  // elements per field
  // spectral scratch (nz*nlm complex each)
  double2* sp[12] = {nullptr};
  int nsp = 0;
  // grid scratch for the NL step (nz*nphi*nlat doubles each)
  double* gr[9] = {nullptr};
  int ngr = 0;
  // boundary
  int bc_ready = 0;
  double* binv = nullptr;   // [lmax][N-4][N]  M_l column-major per l
  double* d2bor = nullptr;  // [N][4]
  double* energy = nullptr; // device accumulator (1 double)
  // mixed precision: fp16 hi/lo tables for the tcgen05 GEMMs, fp32 folded
  // coefficients G32 (reusing the G allocation), running data maxima
  TcSet tcAS, tcAV, tcSS, tcSV;  // analysis scalar/vector, synthesis scalar/vector
  int ldn8 = 0;                  // node stride of G32 (nlat/2 rounded up to 8)
  size_t G32field = 0;           // float2 elements per G32 field
  float* dmax = nullptr;         // [4] max |value| per data operand (bit-compared)
  int* dflag = nullptr;          // device status word (bounded waits that gave up)
  // stage timers (sph_timer_*): event pairs recorded around each launch
  int timing = 0;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<int> ev_class;  // class of the i-th recorded pair
  int ev_used = 0;
};

// Records a start event for kernel class `cls` on `st` when timing is on;
// returns the slot to close with timer_stop (or -1).
int timer_start(const sph_plan* p, int cls, cudaStream_t st);
void timer_stop(const sph_plan* p, int slot, cudaStream_t st);

struct TimedLaunch {
  const sph_plan* p;
  int slot;
  cudaStream_t st;
  TimedLaunch(const sph_plan* p_, int cls, cudaStream_t st_) : p(p_), slot(timer_start(p_, cls, st_)), st(st_) {}
  ~TimedLaunch() { timer_stop(p, slot, st); }
};
enum { T_PHI_FWD = 0, T_PHI_INV, T_LEG_ANA, T_LEG_SYN, T_VEC_ANA, T_VEC_SYN, T_ZFFT, T_OPS };

static inline size_t spec_elems(const sph_plan* p) { return (size_t)p->nz * p->nlm; }
static inline size_t grid_elems(const sph_plan* p) { return (size_t)p->nz * p->nphi * p->nlat; }

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by (sign * i)
__device__ __forceinline__ double2 cmul_si(double2 a, int sign) {
  return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// ---------------------------------------------------------------- launchers
// z transforms (k_zfft.cu)
enum ZMode { Z_FWD = 0, Z_INV = 1, Z_DERIV = 2, Z_FILTER = 3, Z_DLR = 4 };
int launch_zfft(const sph_plan* p, int mode, const double2* in, double2* out, int order,
                cudaStream_t st);

// phi transforms (k_phifft.cu): grid fields -> folded coefficients and back
int launch_phi_fwd(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st);
int launch_phi_inv(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st);

// Legendre contractions (k_legendre.cu)
int launch_leg_analysis(const sph_plan* p, int gfield, double2* spec, cudaStream_t st);
int launch_leg_synthesis(const sph_plan* p, const double2* spec, int gfield, cudaStream_t st);
int launch_vec_analysis(const sph_plan* p, double2* s, double2* t, cudaStream_t st);
int launch_vec_synthesis(const sph_plan* p, const double2* s, const double2* t, cudaStream_t st);

// elementwise operators and boundary (k_ops.cu)
int launch_kmul(const sph_plan* p, const double2* a, double2* b, int order, cudaStream_t st);
int launch_filter_k(const sph_plan* p, double2* a, cudaStream_t st);
int launch_laplang(const sph_plan* p, const double2* a, double2* b, cudaStream_t st);
int launch_multr(const sph_plan* p, const double2* a, double2* b, int power, cudaStream_t st);
int launch_saxpby(const sph_plan* p, double* z, const double* x, double a, const double* y, double b,
                  size_t n, cudaStream_t st);
int launch_prodvec(const sph_plan* p, const double* const* A, const double* const* B,
                   double* const* Cout, cudaStream_t st);
int launch_dirichlet(const sph_plan* p, double2* a, cudaStream_t st);
int launch_invDl(const sph_plan* p, const double2* phi, double2* w, cudaStream_t st);
int launch_bc_fast_rows(const sph_plan* p, double2* phi, const double2* w, cudaStream_t st);
int launch_qst_scale(const sph_plan* p, const double2* in, double2* out, int rpow, int lfac,
                     double sc, cudaStream_t st);
int launch_energy(const sph_plan* p, const double* ur, const double* ut, const double* up,
                  double* acc, cudaStream_t st);

// mixed precision (k_mixed.cu)
int mixed_setup(sph_plan* p, const std::vector<double>& hP, const std::vector<double>& hdP,
                const std::vector<double>& hmPs);
void mixed_free(sph_plan* p);
int launch_phi_fwd32(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st);
int launch_phi_inv32(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st);
int launch_tc_analysis(const sph_plan* p, int vector, double2* out, double2* out2, cudaStream_t st);
int launch_tc_synthesis(const sph_plan* p, int vector, const double2* in, const double2* in2,
                        cudaStream_t st);
int mixed_status(const sph_plan* p);
bool mixed_nphi_ok(int nphi);  // phi lengths the fp32 phi kernels are built for

#define SPH_CUDA_OK(call)                     \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) return SPH_ECUDA;  \
  } while (0)

#define SPH_LAUNCH_OK()                                   \
  do {                                                    \
    if (cudaGetLastError() != cudaSuccess) return SPH_ECUDA; \
  } while (0)
