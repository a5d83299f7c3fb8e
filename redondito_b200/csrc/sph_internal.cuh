// sph_internal.cuh -- plan layout, device helpers and launcher declarations
// shared by the CUDA sources of the transform core.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <memory>
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
// one block of at most 128 (scalar) or 64 (vector) MMA rows; its Legendre
// table tiles sit in HBM as nk consecutive blocks of [hi | mid | lo] bf16
// (3 x nr x 32 values each, 8x8 core matrices, K-major).  Vector items come
// in twins (out = 0: S or Vt, out = 1: T or Vp) sharing their blocks; their
// first nk1 K steps are the dP part, the rest the mPs part.
struct TcItem {
  int m, par, r0, nr, nvalid, nk, nk1, out;
  long long boff;  // first table block, in halves
  float tscale;
  int pad_;
};

struct TcSet {
  TcItem* items = nullptr;  // device
  int nitems = 0;
  uint16_t* blocks = nullptr;  // device, bf16 bit patterns
  size_t nhalves = 0;
};

// Device tables a plan shares with its clones (sph_plan_clone): everything a
// plan reads but never writes after creation.  Freed with the last plan.
struct PlanTables {
  std::vector<void*> dev;      // plain table allocations
  TcSet tc[4];                 // mixed table tiles (tcAS, tcAV, tcSS, tcSV)
  double* binv = nullptr;      // boundary tables (sph_setup_bc), shared once built
  double* d2bor = nullptr;
  int bc_kinds = -1;           // the wall kinds binv was built for (inner + 2 outer)
  ~PlanTables();
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
  // four-step phi FFT (nphi = N1 N2): pass twiddles of length N1, then N2 at tw4off
  float2* tw4f = nullptr;
  double2* tw4d = nullptr;
  int tw4off = 0;
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
  // (m, 16-degree chunk) items of the fused z inverse into synthesis tiles (mixed)
  int2* d_ztitems = nullptr;
  int nztitems = 0;
  // FP64 spectral scratch of the single-precision entry points (allocated on first use)
  double2* fsp[5] = {nullptr};
  // boundary: kinds at the inner and outer wall (0 noslip, 1 freeslip); the
  // plan owns binv/d2bor when its kinds differ from the shared tables'
  int bck[2] = {0, 0};
  int bc_own = 0;
  // Neumann reconstructors (sph_plan_set_neumann): host neu[0] first and
  // neu[1] second normal derivative, d values each (empty: not set); device
  // copy [2][d]
  std::vector<double> neu[2];
  double* d_neu = nullptr;
  int bc_ready = 0;
  double* binv = nullptr;   // [lmax][N-4][N]  M_l column-major per l
  double* d2bor = nullptr;  // [N][4]
  double* energy = nullptr; // device accumulator (1 double)
  double* spectrum = nullptr;  // device [lmax+1][2] per-degree energies (sph_energy_spectrum)
  std::shared_ptr<PlanTables> tables;  // owner of the read-only tables (shared by clones)
  // mixed precision: bf16 table tiles for the tcgen05 GEMMs, bf16 data tiles
  // (analysis: written by the phi FFT; synthesis: from the spectra), fp32
  // folded coefficients G32 of the synthesis (reusing the G allocation)
  TcSet tcAS, tcAV, tcSS, tcSV;  // analysis scalar/vector, synthesis scalar/vector
  int ldn8 = 0;                  // node stride of G32 (nlat/2 rounded up to 8)
  int nkn = 0;                   // K tiles of 32 nodes
  size_t G32field = 0;           // float2 elements per G32 field
  uint16_t* Tana = nullptr;      // [3][m][fold][plane block][node tile] x 24 KB
  uint16_t* Tsyn = nullptr;      // [2][m][parity][plane block][l tile] x 24 KB
  size_t Tsynfield = 0;          // bf16 values per synthesis field
  long long* d_toff = nullptr;   // [lmax+1][2] first synthesis tile of each block
  int* dflag = nullptr;          // device status word (bounded waits that gave up)
  int nsm = 0;                   // SMs of the plan's device (persistent grids)
  // planes that feed the FC-Gram continuation ([0, oz) and [N-oz, N)); a
  // mixed plan transforms them again in FP64, because the continuation
  // operator (norm ~1e4) amplifies their round-off into every radial mode
  int* d_bplanes = nullptr;
  int nbplanes = 0;
  // plane selection of the FP64 phi and Legendre launchers (nullptr: all nz)
  mutable const int* sel_kz = nullptr;
  mutable int sel_n = 0;
  mutable int bpass = 0;         // mixed 2D transforms recompute d_bplanes in FP64
  // tile shapes (0: the built-in choice; sph_plan_set_tiles)
  int tile_nr = 0;               // mixed scalar items: MMA rows (32, 64, 128)
  int tile_np = 0;               // phi transforms: ring pairs per CTA (1, 2, 4, 8)
  int tile_lb = 0;               // z transforms: lm columns per CTA (1..64, power of two)
  double* contg = nullptr;       // [3][Cz][nphi][nlat] physically continued planes (mixed)
  // two-pass forward phi transform (mixed): tile images of phi2_planes plane-fields
  float2* phi2 = nullptr;
  int phi2_planes = 0;
  // the caller's slab (sph_plan_set_slab; the whole field by default): the
  // radial transforms, spectral operators and boundary act on the lm
  // columns [lm0, lm0 + nlmv) of (nlmv, nz) arrays; the 2D angular
  // transforms on the planes [k0, k0 + nzv) of (nlat, nphi, nzv) and
  // (nlm, nzv) arrays (the reference's per-rank arrays in, carr1)
  int k0 = 0, nzv = 0, lm0 = 0, nlmv = 0;
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
// the caller's slab: (nlmv, nz) spectral and (nlat, nphi, nzv) physical arrays
static inline size_t spec_view(const sph_plan* p) { return (size_t)p->nz * p->nlmv; }
static inline size_t grid_view(const sph_plan* p) { return (size_t)p->nzv * p->nphi * p->nlat; }
static inline bool slab_whole(const sph_plan* p) {
  return p->k0 == 0 && p->nzv == p->nz && p->lm0 == 0 && p->nlmv == p->nlm;
}

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// v / nz: a multiplication by the exact reciprocal when nz is a power of
// two (the same result bit for bit, without the cost of a double division)
__device__ __forceinline__ double2 div_nz(double2 v, int nz) {
  if ((nz & (nz - 1)) == 0) {
    const double r = 1.0 / (double)nz;
    return make_double2(v.x * r, v.y * r);
  }
  return make_double2(v.x / (double)nz, v.y / (double)nz);
}
// continued element ii (0-based) of a column (element r at col[r * stride])
// from its first and last d physical ones: sum_jj dir(ii,jj) x(N-d+jj) +
// dir(C-1-ii,jj) x(d-1-jj), dir C x d column-major, the summation order of
// the reference's continuation (sphp_sca.F90:369-381)
__device__ __forceinline__ double2 fc_cont_elem(const double* __restrict__ dir, int C, int d, int N, int ii,
                                                const double2* col, int stride) {
  double2 acc;
  {
    const double wr = __ldg(dir + ii), wl = __ldg(dir + (C - 1 - ii));
    const double2 xr = col[(N - d) * stride], xl = col[(d - 1) * stride];
    acc = make_double2(wr * xr.x + wl * xl.x, wr * xr.y + wl * xl.y);
  }
  for (int jj = 1; jj < d; ++jj) {
    const double wr = __ldg(dir + ii + C * jj), wl = __ldg(dir + (C - 1 - ii) + C * jj);
    const double2 xr = col[(N - d + jj) * stride], xl = col[(d - 1 - jj) * stride];
    acc.x = (acc.x + wr * xr.x) + wl * xl.x;
    acc.y = (acc.y + wr * xr.y) + wl * xl.y;
  }
  return acc;
}
// multiply by (sign * i)
__device__ __forceinline__ double2 cmul_si(double2 a, int sign) {
  return sign > 0 ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// ---------------------------------------------------------------- launchers
// z transforms (k_zfft.cu)
enum ZMode { Z_FWD = 0, Z_INV = 1, Z_DERIV = 2, Z_FILTER = 3, Z_DLR = 4 };
// cont = false: the planes past N are taken as given (already continued)
int launch_zfft(const sph_plan* p, int mode, const double2* in, double2* out, int order,
                cudaStream_t st, bool cont = true);
// element types of the spectra a z transform reads and writes: FP64
// (double2) or single precision (float2, the single-precision entry
// points); the transform itself runs in FP64 in shared memory
enum { ZIO_DD = 0, ZIO_FF = 1, ZIO_DF = 2, ZIO_FD = 3 };
int launch_zfft_io(const sph_plan* p, int mode, const void* in, void* out, int io, int order, cudaStream_t st,
                   bool cont = true);

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
// the toroidal condition of each wall by its kind: Z = 0 (noslip) or the
// Robin reconstruction of Z' - 2Z/r = 0 (freeslip)
int launch_bc_walls(const sph_plan* p, double2* tor, cudaStream_t st);
// neumann_reconstruct / robin_reconstruct on a radial boundary (boun 0 inner,
// 1 outer) of the caller's lm columns; a: device Robin coefficients or null
int launch_reconstruct(const sph_plan* p, double2* f, int boun, int ord, const double* a, cudaStream_t st);
int launch_invDl(const sph_plan* p, const double2* phi, double2* w, cudaStream_t st);
int launch_bc_fast_rows(const sph_plan* p, double2* phi, const double2* w, cudaStream_t st);
int launch_qst_scale(const sph_plan* p, const double2* in, double2* out, int rpow, int lfac,
                     double sc, cudaStream_t st);
int launch_energy(const sph_plan* p, const double* ur, const double* ut, const double* up,
                  double* acc, cudaStream_t st);

// mixed precision (k_mixed.cu)
int mixed_setup(sph_plan* p, const std::vector<double>& hP, const std::vector<double>& hdP,
                const std::vector<double>& hmPs);
int mixed_alloc_scratch(sph_plan* p);  // the per-plan buffers of a mixed plan (also for clones)
void mixed_free_scratch(sph_plan* p);
void mixed_free_tables(sph_plan* p);
// grids_hi: planes k >= N of field f come from grids_hi[f] + (k - N) planes
int launch_phi_fwd32(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st,
                     const double* const* grids_hi = nullptr);
// FC-Gram continuation of physical fields: planes N..nz-1 of each field into
// p->contg (field f at f * Cz planes), from its planes 0..oz-1 and N-oz..N-1
int launch_cont_phys(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st);
// the same on grids of float (f32) or FP64 values (the single-precision entry points)
int launch_cont_phys_g(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st, bool f32);
int launch_phi_fwd32_g(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st,
                       const void* const* grids_hi, bool f32);
int launch_phi_inv32_g(const sph_plan* p, void* const* grids, int nfields, cudaStream_t st, bool f32);
int launch_phi_inv32(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st);
int launch_tc_analysis(const sph_plan* p, int vector, double2* out, double2* out2, cudaStream_t st);
int launch_tc_synthesis(const sph_plan* p, int vector, const double2* in, const double2* in2,
                        cudaStream_t st);
int mixed_status(const sph_plan* p);
int mixed_retile(sph_plan* p);  // rebuild the scalar work sets for tile_nr
bool mixed_nphi_ok(int nphi);  // phi lengths the fp32 phi kernels are built for

// grouped launches over several plans' work sets (batches): one job per
// (plan, field); the spectra are the synthesis input or the analysis output
struct GroupJob {
  const sph_plan* p;
  int field;
  double2* spec;
};
struct GroupLaunch {
  void* jobs = nullptr;   // device array of the kernel's per-job arguments
  int* prefix = nullptr;  // device [njobs]: first CTA (FP64) or work unit (mixed) of each job
  int njobs = 0, total = 0, grid = 0;
  bool analysis = false;
};
int leg_group_prepare(bool analysis, const std::vector<GroupJob>& jobs, GroupLaunch* g);
int leg_group_launch(const GroupLaunch& g, cudaStream_t st);
int tc_group_prepare(bool analysis, const std::vector<GroupJob>& jobs, int nsm, GroupLaunch* g);
int tc_group_launch(const GroupLaunch& g, int* flag, cudaStream_t st);
void group_free(GroupLaunch* g);
// the in-place forward z transforms of several plans' spectra (batches):
// one grouped launch per z length whose two-step kernel runs at the plan's
// column width, each CTA one column block of one job; cont as in
// launch_zfft.  The indices of the jobs it does not take go to `rest`.
struct ZJob {
  const sph_plan* p;
  double2* spec;
  bool cont;
};
struct ZGroupLen {
  int nz = 0;
  void* jobs = nullptr;   // device array of the jobs' kernel arguments
  int* prefix = nullptr;  // device [njobs + 1]: first CTA of each job
  int njobs = 0, total = 0;
};
struct ZGroupLaunch {
  std::vector<ZGroupLen> lens;
};
int zfwd_group_prepare(const std::vector<ZJob>& jobs, ZGroupLaunch* g, std::vector<int>* rest);
int zfwd_group_launch(const ZGroupLaunch& g, cudaStream_t st);
void zgroup_free(ZGroupLaunch* g);
// spectra -> synthesis data tiles of field slot `field` (mixed plans)
int launch_spec_to_tiles_field(const sph_plan* p, const double2* in, int field, cudaStream_t st);
// the z inverse of FP64 spectra (fftp1d_complex_to_real_z) written straight
// into synthesis tiles of field `field` (the input is preserved); SPH_EINVAL
// where it does not apply (nz without a compile-time transform length)
bool zinv_tiles_ok(const sph_plan* p);
// the z inverse of field `field`'s spectra straight into its synthesis
// tiles; with out, also the radial-space spectra (out may be in: in place);
// with dout (zinv_der_ok), also their radial derivative derivr(., 1, 'r')
int launch_zinv_tiles(const sph_plan* p, const double2* in, int field, cudaStream_t st, double2* out = nullptr,
                      double2* dout = nullptr);
bool zinv_der_ok(const sph_plan* p);
int launch_zinv_tiles_g(const sph_plan* p, const void* in, int field, cudaStream_t st, bool f32,
                        double2* out = nullptr, double2* dout = nullptr);
// the tensor-core synthesis from tiles already in place
int launch_tc_synthesis_tiles(const sph_plan* p, int vector, cudaStream_t st);

// Runs a set-up step (typically cudaFuncSetAttribute: a kernel's dynamic
// shared-memory limit) once per device.  Function attributes belong to the
// context of the device current at the call, so a process that drives
// several GPUs must set them on each; devices 0..63 are remembered, others
// repeat the step on every call.
struct DeviceOnce {
  std::atomic<unsigned long long> mask{0};
  template <typename F>
  bool run(F&& step) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
    if (bit && (mask.load(std::memory_order_acquire) & bit)) return true;
    if (!step()) return false;
    if (bit) mask.fetch_or(bit, std::memory_order_acq_rel);
    return true;
  }
};

#define SPH_CUDA_OK(call)                     \
  do {                                        \
    cudaError_t e_ = (call);                  \
    if (e_ != cudaSuccess) return SPH_ECUDA;  \
  } while (0)

#define SPH_LAUNCH_OK()                                   \
  do {                                                    \
    if (cudaGetLastError() != cudaSuccess) return SPH_ECUDA; \
  } while (0)
