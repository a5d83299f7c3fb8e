// k_legendre.cu -- per-m Legendre contractions as FP64 tensor-core GEMMs.
//
// The reference does these inside SHTns, one plane at a time (spat_to_SH /
// SH_to_spat / spat_to_SHqst / SHqst_to_spat at src/sphp/sphp_sca.F90:312,485
// and src/sphp/sphp_vec.F90:89-91,157-159).  Here every plane and field is a
// column of one GEMM per m, so each Legendre table tile is read once per
// (m, row block) for all nz planes:
//   analysis   a[l][n]   = sum_i Pbar_lm(x_i) G_(l-m)%2[i][n]          K = nlat/2
//   synthesis  S_q[i][n] = sum_{l: (l-m)%2 = q} Pbar_lm(x_i) a[l][n]    K = lmax+1-m
// with n = (plane, re/im); folding mirror rings into even/odd parts halves K.
// The vector transforms fold their complex factors into the operand loads:
//   S_l  = 1/(l(l+1)) sum_i [ dP_l Vt_(1-p) + mPs_l (-i Vp_p) ]
//   T_l  = 1/(l(l+1)) sum_i [ mPs_l (-i Vt_p) - dP_l Vp_(1-p) ]
//   Vt_q = sum_(p=1-q) dP_l S_l + sum_(p=q) mPs_l (i T_l)
//   Vp_q = sum_(p=1-q) dP_l (-T_l) + sum_(p=q) mPs_l (i S_l)
// (p = (l-m)%2, fold 0 = F(i)+F(mirror), fold 1 = F(i)-F(mirror); Pbar has
// the parity of p, dPbar the opposite), so each output is one accumulator
// over a K twice as long.
//
// Every kernel streams its tiles through a 3-stage cp.async pipeline into
// padded shared memory (conflict-free fragment loads) and runs FP64
// mma.sync.m8n8k4 on the DMMA pipe; output tiles are staged through shared
// memory so global writes are contiguous rows.
#include "sph_internal.cuh"

namespace {

// ---------------------------------------------------------------- primitives
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// 16-byte global->shared copy; pred == false fills zeros (no global read).
__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool pred) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = pred ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int MT, int NT>
__device__ __forceinline__ void zero_acc(double (&acc)[MT][NT][2]) {
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
}

// B-operand forms applied at fragment-load time to an interleaved complex
// column pair (column 2k = re, 2k+1 = im of the same value v):
//   PLAIN: v    NEG: -v    MULI: i v    MULMI: -i v
enum BForm { PLAIN = 0, NEG = 1, MULI = 2, MULMI = 3 };

// Fragment b for column n of a complex operand stored as doubles where the
// (re, im) pair of column n>>1 sits at base[0], base[1].
template <int FORM>
__device__ __forceinline__ double bform(const double* pair, int c) {
  if (FORM == PLAIN) return pair[c];
  if (FORM == NEG) return -pair[c];
  if (FORM == MULI) return c ? pair[0] : -pair[1];  // (i v).re = -v.im, (i v).im = v.re
  return c ? -pair[0] : pair[1];                    // (-i v).re = v.im, (-i v).im = -v.re
}

struct LegArgs {
  const double* P;     // [nlm][ldn]
  const double* dP;    // [nlm][ldn]
  const double* mPs;   // [nlm][ldn]
  const double2* G;    // folded coefficients [field][m][2][nz][ldn]
  double2* Gw;
  size_t Gfield;
  int gfield;
  const double2* spec;  // (nz, nlm)
  const double2* spec2;
  double2* out;
  double2* out2;
  const LegTile* tiles;
  const int* mbase;
  const int* kzl;  // planes to transform (nullptr: all nz)
  int lmax, ldn, nz, nlm, nkz;
  int ntiles;      // tiles of this work set (grouped launches)
};

// Grouped launches: the CTAs of several plans' work sets in one grid; job j
// owns CTAs prefix[j] .. prefix[j+1]-1, laid out (plane block, tile).
struct LegGroup {
  const LegArgs* jobs;
  const int* prefix;
  int njobs;
};

// This CTA's arguments and (tile, plane block) indices.
template <bool G>
__device__ __forceinline__ void leg_cta(const LegArgs& a0, const LegGroup& grp, LegArgs& a, int& bx, int& by) {
  if constexpr (!G) {
    a = a0;
    bx = blockIdx.x;
    by = blockIdx.y;
  } else {
    int lo = 0, hi = grp.njobs - 1;
    const int c = blockIdx.x;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(grp.prefix + mid) <= c) lo = mid;
      else hi = mid - 1;
    }
    a = grp.jobs[lo];
    const int local = c - __ldg(grp.prefix + lo);
    bx = local % a.ntiles;
    by = local / a.ntiles;
  }
}

// plane of local index kl (blockIdx.y * KZ + offset); ok = within the selection
__device__ __forceinline__ int plane_of(const LegArgs& a, int kl, bool& ok) {
  ok = kl < a.nkz;
  return a.kzl ? (ok ? __ldg(a.kzl + kl) : 0) : kl;
}

constexpr int STAGES = 3;

// ================================================================ scalar analysis
// CTA: 64 consecutive l (rows split by parity, 32 each) x 32 planes (64
// columns); K tile 16 nodes.  4 warps = (parity, column half), 32x32 each.
namespace an {
constexpr int L = 64, KZ = 32, K = 16, LDA = K + 4, LDB = K + 4;  // LDB in complex units
constexpr int A_SZ = 2 * 32 * LDA;          // doubles
constexpr int B_SZ = 2 * KZ * LDB * 2;      // doubles
constexpr int STAGE = A_SZ + B_SZ;
constexpr int SMEM = STAGES * STAGE * 8;
}  // namespace an

template <bool GROUP>
__global__ void __launch_bounds__(128) leg_analysis_kernel(LegArgs a0, LegGroup grp) {
  using namespace an;
  extern __shared__ __align__(16) double sm[];
  LegArgs a;
  int bx, by;
  leg_cta<GROUP>(a0, grp, a, bx, by);
  const LegTile tile = a.tiles[bx];
  const int m = tile.m, l0 = tile.r0;
  const int kz0 = by * KZ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int par = warp >> 1, nh = warp & 1;
  const double2* G = a.G + (size_t)a.gfield * a.Gfield + (size_t)m * 2 * a.nz * a.ldn;
  const size_t base_lm = (size_t)a.mbase[m] - m;
  const int nk = (a.ldn + K - 1) / K;

  auto load = [&](int st, int k0) {
    double* As = sm + st * STAGE;
    double* Bs = As + A_SZ;
    for (int c = tid; c < L * (K / 2); c += 128) {  // A: 64 rows x 8 chunks
      int row = c >> 3, cc = c & 7;
      int l = l0 + row, i = k0 + 2 * cc;
      bool ok = l <= a.lmax && i < a.ldn;
      const double* src = ok ? a.P + (base_lm + l) * a.ldn + i : a.P;
      cp16(As + ((row & 1) * 32 + (row >> 1)) * LDA + 2 * cc, src, ok);
    }
    for (int c = tid; c < 2 * KZ * K; c += 128) {  // B: [par][plane][node] complex
      int i_ = c % K, r = c / K, kzl = r % KZ, pr = r / KZ;
      bool ok;
      int kz = plane_of(a, kz0 + kzl, ok), i = k0 + i_;
      ok = ok && i < a.ldn;
      const double2* src = ok ? G + ((size_t)pr * a.nz + kz) * a.ldn + i : a.G;
      cp16(Bs + ((pr * KZ + kzl) * LDB + i_) * 2, src, ok);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, s * K);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* As = sm + (kt % STAGES) * STAGE + par * 32 * LDA;
    const double* Bs = sm + (kt % STAGES) * STAGE + A_SZ + (par * KZ + nh * 16) * LDB * 2;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 4) {
      double av[4], bv[4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) av[mt] = As[(mt * 8 + g) * LDA + k0 + t];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) bv[nt] = Bs[((nt * 4 + (g >> 1)) * LDB + k0 + t) * 2 + (g & 1)];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], av[mt], bv[nt]);
    }
    int nx = kt + STAGES - 1;
    if (nx < nk) load(nx % STAGES, nx * K);
    cp_commit();
  }
  cp_wait<0>();
  __syncthreads();

  // Cs[plane][l] then contiguous rows of the (nz, nlm) output
  double2* Cs = reinterpret_cast<double2*>(sm);
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int row = mt * 8 + g;
      int pl = nh * 16 + nt * 4 + t;
      Cs[pl * L + 2 * row + par] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
  __syncthreads();
  const int nvalid = min(L, a.lmax + 1 - l0);
  for (int idx = tid; idx < KZ * L; idx += 128) {
    int pl = idx / L, ll = idx - pl * L;
    bool okz;
    int kz = plane_of(a, kz0 + pl, okz);
    if (!okz || ll >= nvalid) continue;
    double2 v = Cs[idx];
    if (m == 0) v.y = 0.0;  // m = 0 coefficients of a real field are real
    a.out[(size_t)kz * a.nlm + base_lm + l0 + ll] = v;
  }
}

// ================================================================ scalar synthesis
// CTA: 64 nodes x 32 planes; K tile 16 consecutive l (8 per parity).
// 8 warps = (parity, node half, column half), 32x32 each.
namespace sy {
constexpr int I = 64, KZ = 32, K = 16, LDA = I + 4, LDB = 2 * KZ + 4;
constexpr int A_SZ = K * LDA, B_SZ = K * LDB;
constexpr int STAGE = A_SZ + B_SZ;
constexpr int SMEM = STAGES * STAGE * 8;
}  // namespace sy

template <bool GROUP>
__global__ void __launch_bounds__(256) leg_synthesis_kernel(LegArgs a0, LegGroup grp) {
  using namespace sy;
  extern __shared__ __align__(16) double sm[];
  LegArgs a;
  int bx, by;
  leg_cta<GROUP>(a0, grp, a, bx, by);
  const LegTile tile = a.tiles[bx];
  const int m = tile.m, i0 = tile.r0;
  const int kz0 = by * KZ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int par = warp >> 2, mh = (warp >> 1) & 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;
  const int nk = (a.lmax + 1 - m + K - 1) / K;

  auto load = [&](int st, int lk) {
    double* As = sm + st * STAGE;  // [par][q][node]  (K-major)
    double* Bs = As + A_SZ;        // [par][q][col]   (K x N)
    for (int c = tid; c < K * (I / 2); c += 256) {
      int cc = c % (I / 2), q = c / (I / 2);
      int l = lk + q, i = i0 + 2 * cc;
      bool ok = l <= a.lmax && i < a.ldn;
      const double* src = ok ? a.P + (base_lm + l) * a.ldn + i : a.P;
      cp16(As + ((q & 1) * (K / 2) + (q >> 1)) * LDA + 2 * cc, src, ok);
    }
    for (int c = tid; c < K * KZ; c += 256) {
      int q = c % K, pl = c / K;
      bool ok;
      int l = lk + q, kz = plane_of(a, kz0 + pl, ok);
      ok = ok && l <= a.lmax;
      const double2* src = ok ? a.spec + (size_t)kz * a.nlm + base_lm + l : a.spec;
      cp16(Bs + ((q & 1) * (K / 2) + (q >> 1)) * LDB + 2 * pl, src, ok);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, m + s * K);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* As = sm + (kt % STAGES) * STAGE + par * (K / 2) * LDA + mh * 32;
    const double* Bs = sm + (kt % STAGES) * STAGE + A_SZ + par * (K / 2) * LDB + nh * 32;
#pragma unroll
    for (int k0 = 0; k0 < K / 2; k0 += 4) {
      double av[4], bv[4];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) av[mt] = As[(k0 + t) * LDA + mt * 8 + g];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) bv[nt] = Bs[(k0 + t) * LDB + nt * 8 + g];
#pragma unroll
      for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], av[mt], bv[nt]);
    }
    int nx = kt + STAGES - 1;
    if (nx < nk) load(nx % STAGES, m + nx * K);
    cp_commit();
  }
  cp_wait<0>();

  double2* G = a.Gw + (size_t)a.gfield * a.Gfield + ((size_t)m * 2 + par) * a.nz * a.ldn;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int i = i0 + mh * 32 + mt * 8 + g;
      bool okz;
      int kz = plane_of(a, kz0 + nh * 16 + nt * 4 + t, okz);
      if (i < a.ldn && okz) G[(size_t)kz * a.ldn + i] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
}

// ================================================================ vector analysis
// CTA: 64 consecutive l x 32 planes; K tile 8 nodes.  8 warps =
// (parity, output S/T, column half), 32x32 each.  Each output is one
// accumulator over the dP block (nodes x Vt/Vp fold 1-p) and the mPs block
// (nodes x Vt/Vp fold p).
namespace va {
constexpr int L = 64, KZ = 32, K = 8, LDA = K + 4, LDB = K + 4;  // LDB complex units
constexpr int A_SZ = 2 * 2 * 32 * LDA;   // [table][par][row][k]
constexpr int B_SZ = 2 * 2 * KZ * LDB * 2;  // [field][fold][plane][k] complex
constexpr int STAGE = A_SZ + B_SZ;
constexpr int SMEM = STAGES * STAGE * 8;
}  // namespace va

template <int FORM>
__device__ __forceinline__ void mma_block_nmaj(double (&acc)[4][4][2], const double* As, int lda,
                                               const double* Bs, int ldbc, int g, int t) {
#pragma unroll
  for (int k0 = 0; k0 < 8; k0 += 4) {
    double av[4], bv[4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) av[mt] = As[(mt * 8 + g) * lda + k0 + t];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) bv[nt] = bform<FORM>(Bs + ((nt * 4 + (g >> 1)) * ldbc + k0 + t) * 2, g & 1);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], av[mt], bv[nt]);
  }
}

__global__ void __launch_bounds__(256) vec_analysis_kernel(LegArgs a) {
  using namespace va;
  extern __shared__ __align__(16) double sm[];
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, l0 = tile.r0;
  const int kz0 = blockIdx.y * KZ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int par = warp >> 2, outT = (warp >> 1) & 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;
  const size_t moff = (size_t)m * 2 * a.nz * a.ldn;
  const double2* Gt = a.G + 1 * a.Gfield + moff;  // v_theta
  const double2* Gp = a.G + 2 * a.Gfield + moff;  // v_phi
  const int nk = (a.ldn + K - 1) / K;

  auto load = [&](int st, int k0) {
    double* As = sm + st * STAGE;
    double* Bs = As + A_SZ;
    for (int c = tid; c < 2 * L * (K / 2); c += 256) {  // 2 tables x 64 rows x 4 chunks
      int cc = c & 3, r = c >> 2, row = r % L, tb = r / L;
      int l = l0 + row, i = k0 + 2 * cc;
      bool ok = l <= a.lmax && i < a.ldn;
      const double* tab = tb ? a.mPs : a.dP;
      const double* src = ok ? tab + (base_lm + l) * a.ldn + i : a.dP;
      cp16(As + ((tb * 2 + (row & 1)) * 32 + (row >> 1)) * LDA + 2 * cc, src, ok);
    }
    for (int c = tid; c < 2 * 2 * KZ * K; c += 256) {  // 2 fields x 2 folds x 32 planes x 8 nodes
      int i_ = c % K, r = c / K, kzl = r % KZ, r2 = r / KZ, fo = r2 & 1, fl = r2 >> 1;
      bool ok;
      int kz = plane_of(a, kz0 + kzl, ok), i = k0 + i_;
      ok = ok && i < a.ldn;
      const double2* Gf = fl ? Gp : Gt;
      const double2* src = ok ? Gf + ((size_t)fo * a.nz + kz) * a.ldn + i : a.G;
      cp16(Bs + (((fl * 2 + fo) * KZ + kzl) * LDB + i_) * 2, src, ok);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, s * K);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* As = sm + (kt % STAGES) * STAGE;
    const double* Bs = As + A_SZ;
    const double* Ad = As + ((0 * 2 + par) * 32) * LDA;  // dP rows of this parity
    const double* Am = As + ((1 * 2 + par) * 32) * LDA;  // mPs rows
    auto B = [&](int fl, int fo) { return Bs + ((fl * 2 + fo) * KZ + nh * 16) * LDB * 2; };
    if (!outT) {
      // S: dP x Vt_(1-p)  +  mPs x (-i Vp_p)
      mma_block_nmaj<PLAIN>(acc, Ad, LDA, B(0, 1 - par), LDB, g, t);
      mma_block_nmaj<MULMI>(acc, Am, LDA, B(1, par), LDB, g, t);
    } else {
      // T: mPs x (-i Vt_p)  -  dP x Vp_(1-p)
      mma_block_nmaj<MULMI>(acc, Am, LDA, B(0, par), LDB, g, t);
      mma_block_nmaj<NEG>(acc, Ad, LDA, B(1, 1 - par), LDB, g, t);
    }
    int nx = kt + STAGES - 1;
    if (nx < nk) load(nx % STAGES, nx * K);
    cp_commit();
  }
  cp_wait<0>();
  __syncthreads();

  double2* Cs = reinterpret_cast<double2*>(sm);  // [out][plane][l]
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int row = mt * 8 + g;
      int pl = nh * 16 + nt * 4 + t;
      Cs[(outT * KZ + pl) * L + 2 * row + par] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
  __syncthreads();
  const int nvalid = min(L, a.lmax + 1 - l0);
  for (int idx = tid; idx < 2 * KZ * L; idx += 256) {
    int ll = idx % L, r = idx / L, pl = r % KZ, o = r / KZ;
    bool okz;
    int kz = plane_of(a, kz0 + pl, okz);
    if (!okz || ll >= nvalid) continue;
    int l = l0 + ll;
    double f = l ? 1.0 / ((double)l * (double)(l + 1)) : 0.0;
    double2 v = Cs[idx];
    v.x *= f;
    v.y *= f;
    if (m == 0) v.y = 0.0;
    (o ? a.out2 : a.out)[(size_t)kz * a.nlm + base_lm + l] = v;
  }
}

// ================================================================ vector synthesis
// CTA: 32 nodes x 32 planes; K tile 16 consecutive l.  8 warps =
// (fold q, output Vt/Vp, column half), 32x32 each.
namespace vs {
constexpr int I = 32, KZ = 32, K = 16, LDA = I + 4, LDB = 2 * KZ + 4;
constexpr int A_SZ = 2 * K * LDA;  // [table][par][q][node]
constexpr int B_SZ = 2 * K * LDB;  // [field S/T][par][q][col]
constexpr int STAGE = A_SZ + B_SZ;
constexpr int SMEM = STAGES * STAGE * 8;
}  // namespace vs

template <int FORM>
__device__ __forceinline__ void mma_block_kmaj(double (&acc)[4][4][2], const double* As, int lda,
                                               const double* Bs, int ldb, int g, int t) {
#pragma unroll
  for (int k0 = 0; k0 < 8; k0 += 4) {
    double av[4], bv[4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) av[mt] = As[(k0 + t) * lda + mt * 8 + g];
    // column n = nt*8 + g of an interleaved (re, im) row
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) bv[nt] = bform<FORM>(Bs + (k0 + t) * ldb + nt * 8 + (g & ~1), g & 1);
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma(acc[mt][nt], av[mt], bv[nt]);
  }
}

__global__ void __launch_bounds__(256) vec_synthesis_kernel(LegArgs a) {
  using namespace vs;
  extern __shared__ __align__(16) double sm[];
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, i0 = tile.r0;
  const int kz0 = blockIdx.y * KZ;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  const int q = warp >> 2, outP = (warp >> 1) & 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;
  const int nk = (a.lmax + 1 - m + K - 1) / K;

  auto load = [&](int st, int lk) {
    double* As = sm + st * STAGE;
    double* Bs = As + A_SZ;
    for (int c = tid; c < 2 * K * (I / 2); c += 256) {
      int cc = c % (I / 2), r = c / (I / 2), qq = r % K, tb = r / K;
      int l = lk + qq, i = i0 + 2 * cc;
      bool ok = l <= a.lmax && i < a.ldn;
      const double* tab = tb ? a.mPs : a.dP;
      const double* src = ok ? tab + (base_lm + l) * a.ldn + i : a.dP;
      cp16(As + (tb * K + (qq & 1) * (K / 2) + (qq >> 1)) * LDA + 2 * cc, src, ok);
    }
    for (int c = tid; c < 2 * K * KZ; c += 256) {
      int qq = c % K, r = c / K, pl = r % KZ, fl = r / KZ;
      bool ok;
      int l = lk + qq, kz = plane_of(a, kz0 + pl, ok);
      ok = ok && l <= a.lmax && l > 0;
      const double2* sp = fl ? a.spec2 : a.spec;
      const double2* src = ok ? sp + (size_t)kz * a.nlm + base_lm + l : a.spec;
      cp16(Bs + (fl * K + (qq & 1) * (K / 2) + (qq >> 1)) * LDB + 2 * pl, src, ok);
    }
  };

  double acc[4][4][2];
  zero_acc(acc);
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < nk) load(s, m + s * K);
    cp_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const double* As = sm + (kt % STAGES) * STAGE;
    const double* Bs = As + A_SZ;
    // rows of parity 1-q through dP, rows of parity q through mPs
    const double* Ad = As + (0 * K + (1 - q) * (K / 2)) * LDA;
    const double* Am = As + (1 * K + q * (K / 2)) * LDA;
    const double* BS_d = Bs + (0 * K + (1 - q) * (K / 2)) * LDB + nh * 32;
    const double* BT_d = Bs + (1 * K + (1 - q) * (K / 2)) * LDB + nh * 32;
    const double* BS_m = Bs + (0 * K + q * (K / 2)) * LDB + nh * 32;
    const double* BT_m = Bs + (1 * K + q * (K / 2)) * LDB + nh * 32;
    if (!outP) {
      // Vt_q = dP S + mPs (i T)
      mma_block_kmaj<PLAIN>(acc, Ad, LDA, BS_d, LDB, g, t);
      mma_block_kmaj<MULI>(acc, Am, LDA, BT_m, LDB, g, t);
    } else {
      // Vp_q = dP (-T) + mPs (i S)
      mma_block_kmaj<NEG>(acc, Ad, LDA, BT_d, LDB, g, t);
      mma_block_kmaj<MULI>(acc, Am, LDA, BS_m, LDB, g, t);
    }
    int nx = kt + STAGES - 1;
    if (nx < nk) load(nx % STAGES, m + nx * K);
    cp_commit();
  }
  cp_wait<0>();

  double2* G = a.Gw + (size_t)(1 + outP) * a.Gfield + ((size_t)m * 2 + q) * a.nz * a.ldn;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int i = i0 + mt * 8 + g;
      bool okz;
      int kz = plane_of(a, kz0 + nh * 16 + nt * 4 + t, okz);
      if (okz && i < a.ldn) G[(size_t)kz * a.ldn + i] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
}

LegArgs base_args(const sph_plan* p) {
  LegArgs a = {};
  a.P = p->P;
  a.dP = p->dP;
  a.mPs = p->mPs;
  a.G = p->G;
  a.Gw = p->G;
  a.Gfield = p->Gfield;
  a.mbase = p->d_mbase;
  a.lmax = p->lmax;
  a.ldn = p->ldn;
  a.nz = p->nz;
  a.nlm = p->nlm;
  a.kzl = p->sel_kz;
  a.nkz = p->sel_kz ? p->sel_n : p->nz;
  return a;
}

template <typename K>
bool set_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess &&
         cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
}

}  // namespace

int launch_leg_analysis(const sph_plan* p, int gfield, double2* spec, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.gfield = gfield;
  a.out = spec;
  a.tiles = p->tilesA;
  static DeviceOnce once;
  if (!once.run([] { return set_smem(leg_analysis_kernel<false>, an::SMEM); })) return SPH_ECUDA;
  dim3 grid(p->ntilesA, (a.nkz + an::KZ - 1) / an::KZ);
  TimedLaunch tl(p, T_LEG_ANA, st);
  leg_analysis_kernel<false><<<grid, 128, an::SMEM, st>>>(a, LegGroup{});
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_leg_synthesis(const sph_plan* p, const double2* spec, int gfield, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.gfield = gfield;
  a.spec = spec;
  a.tiles = p->tilesS;
  static DeviceOnce once;
  if (!once.run([] { return set_smem(leg_synthesis_kernel<false>, sy::SMEM); })) return SPH_ECUDA;
  dim3 grid(p->ntilesS, (a.nkz + sy::KZ - 1) / sy::KZ);
  TimedLaunch tl(p, T_LEG_SYN, st);
  leg_synthesis_kernel<false><<<grid, 256, sy::SMEM, st>>>(a, LegGroup{});
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_vec_analysis(const sph_plan* p, double2* s, double2* t, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.out = s;
  a.out2 = t;
  a.tiles = p->tilesA;
  static DeviceOnce once;
  if (!once.run([] { return set_smem(vec_analysis_kernel, va::SMEM); })) return SPH_ECUDA;
  dim3 grid(p->ntilesA, (a.nkz + va::KZ - 1) / va::KZ);
  TimedLaunch tl(p, T_VEC_ANA, st);
  vec_analysis_kernel<<<grid, 256, va::SMEM, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_vec_synthesis(const sph_plan* p, const double2* s, const double2* t, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.spec = s;
  a.spec2 = t;
  a.tiles = p->tilesS32;
  static DeviceOnce once;
  if (!once.run([] { return set_smem(vec_synthesis_kernel, vs::SMEM); })) return SPH_ECUDA;
  dim3 grid(p->ntilesS32, (a.nkz + vs::KZ - 1) / vs::KZ);
  TimedLaunch tl(p, T_VEC_SYN, st);
  vec_synthesis_kernel<<<grid, 256, vs::SMEM, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

// ---------------------------------------------------------------- grouped launches
int leg_group_prepare(bool analysis, const std::vector<GroupJob>& jobs, GroupLaunch* g) {
  std::vector<LegArgs> args;
  std::vector<int> prefix;
  long long total = 0;
  for (const GroupJob& j : jobs) {
    if (j.p->precision != SPH_FP64 || j.field < 0 || j.field >= SPH_MAX_FIELDS) return SPH_EINVAL;
    LegArgs a = base_args(j.p);
    a.gfield = j.field;
    if (analysis) {
      a.out = j.spec;
      a.tiles = j.p->tilesA;
      a.ntiles = j.p->ntilesA;
    } else {
      a.spec = j.spec;
      a.tiles = j.p->tilesS;
      a.ntiles = j.p->ntilesS;
    }
    const int kz = analysis ? an::KZ : sy::KZ;
    prefix.push_back((int)total);
    total += (long long)a.ntiles * ((a.nkz + kz - 1) / kz);
    args.push_back(a);
  }
  if (total > (1ll << 30)) return SPH_EINVAL;
  g->analysis = analysis;
  g->njobs = (int)jobs.size();
  g->total = (int)total;
  g->grid = (int)total;
  if (jobs.empty()) return SPH_OK;
  if (cudaMalloc(&g->jobs, args.size() * sizeof(LegArgs)) != cudaSuccess ||
      cudaMalloc((void**)&g->prefix, prefix.size() * sizeof(int)) != cudaSuccess)
    return SPH_ENOMEM;
  if (cudaMemcpy(g->jobs, args.data(), args.size() * sizeof(LegArgs), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->prefix, prefix.data(), prefix.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return SPH_ECUDA;
  return SPH_OK;
}

int leg_group_launch(const GroupLaunch& g, cudaStream_t st) {
  if (g.total == 0) return SPH_OK;
  const LegGroup grp{static_cast<const LegArgs*>(g.jobs), g.prefix, g.njobs};
  if (g.analysis) {
    static DeviceOnce once;
    if (!once.run([] { return set_smem(leg_analysis_kernel<true>, an::SMEM); })) return SPH_ECUDA;
    leg_analysis_kernel<true><<<g.grid, 128, an::SMEM, st>>>(LegArgs{}, grp);
  } else {
    static DeviceOnce once;
    if (!once.run([] { return set_smem(leg_synthesis_kernel<true>, sy::SMEM); })) return SPH_ECUDA;
    leg_synthesis_kernel<true><<<g.grid, 256, sy::SMEM, st>>>(LegArgs{}, grp);
  }
  SPH_LAUNCH_OK();
  return SPH_OK;
}

void group_free(GroupLaunch* g) {
  if (g->jobs) cudaFree(g->jobs);
  if (g->prefix) cudaFree(g->prefix);
  g->jobs = nullptr;
  g->prefix = nullptr;
  g->njobs = g->total = g->grid = 0;
}
