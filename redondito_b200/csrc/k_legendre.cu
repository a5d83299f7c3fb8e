// k_legendre.cu -- per-m Legendre contractions as FP64 tensor-core GEMMs.
//
// The reference does these inside SHTns, one plane at a time (spat_to_SH /
// SH_to_spat / spat_to_SHqst / SHqst_to_spat at src/sphp/sphp_sca.F90:312,485
// and src/sphp/sphp_vec.F90:89-91,157-159).  Here every plane and field is a
// column of one GEMM per m, so the Legendre table tile is loaded once per
// (m, l-block) for all nz planes:
//   analysis   a[l][n] = sum_i  Pbar_lm(x_i) G_par(l)[i][n]      (K = nlat/2)
//   synthesis  S_q[i][n] = sum_{l: (l-m)%2 = q} Pbar_lm(x_i) a[l][n]  (K = lmax+1-m)
// with n = (plane, re/im) and the even/odd folding of mirror rings halving K.
// FP64 tiles run on the DMMA pipe through mma.sync.m8n8k4.f64.
#include "sph_internal.cuh"

namespace {

// D (8x8) += A (8x4, row) * B (4x8, col), FP64.  Fragments: a = A[g][t],
// b = B[t][g], c = {C[g][2t], C[g][2t+1]}, g = lane/4, t = lane%4.
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// Warp tile (8*MT) x (8*NT) += A (8*MT x K) * B (K x 8*NT) from shared memory.
// A_KMAJOR: A stored as As[k*lda + row], else As[row*lda + k].
// B_NMAJOR: B stored as Bs[col*ldb + k], else Bs[k*ldb + col].
template <int MT, int NT, bool A_KMAJOR, bool B_NMAJOR>
__device__ __forceinline__ void warp_mma(double (&acc)[MT][NT][2], const double* As, int lda,
                                         const double* Bs, int ldb, int K) {
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  for (int k0 = 0; k0 < K; k0 += 4) {
    double a[MT], b[NT];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
      a[mt] = A_KMAJOR ? As[(k0 + t) * lda + mt * 8 + g] : As[(mt * 8 + g) * lda + k0 + t];
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
      b[nt] = B_NMAJOR ? Bs[(nt * 8 + g) * ldb + k0 + t] : Bs[(k0 + t) * ldb + nt * 8 + g];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) dmma(acc[mt][nt], a[mt], b[nt]);
  }
}

template <int MT, int NT>
__device__ __forceinline__ void zero_acc(double (&acc)[MT][NT][2]) {
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
}

struct LegArgs {
  const double* P;     // [nlm][nlat2]
  const double* dP;    // [nlm][nlat2]
  const double* mPs;   // [nlm][nlat2]
  const double2* G;    // folded coefficients, field 0 (read)
  double2* Gw;         // folded coefficients (written by synthesis)
  size_t Gfield;
  int gfield;          // which G field
  const double2* spec; // (nz, nlm) input (synthesis)
  const double2* spec2;
  double2* out;        // (nz, nlm) output (analysis)
  double2* out2;
  const LegTile* tiles;
  const int* mbase;
  int lmax, nlat2, nz, nlm;
};

// ---------------------------------------------------------------- scalar analysis
// CTA: 64 consecutive l (32 even-offset rows, 32 odd) x 64 columns (32 planes).
constexpr int AT_L = 64, AT_N = 64, AT_K = 16, AT_LDA = AT_K + 4, AT_LDB = AT_K + 4;

__global__ void __launch_bounds__(128) leg_analysis_kernel(LegArgs a) {
  __shared__ __align__(16) double smem[2 * 32 * AT_LDA + 2 * AT_N * AT_LDB > 32 * 64 * 2
                                           ? 2 * 32 * AT_LDA + 2 * AT_N * AT_LDB
                                           : 32 * 64 * 2];
  double* As = smem;                    // [par][32][AT_LDA]
  double* Bs = smem + 2 * 32 * AT_LDA;  // [par][AT_N][AT_LDB]  (N-major)
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, l0 = tile.r0;
  const int n0 = blockIdx.y * AT_N;  // column = 2*plane + re/im
  const int kz0 = n0 / 2;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int par = warp >> 1, nh = warp & 1;
  const double2* G = a.G + (size_t)a.gfield * a.Gfield;
  const size_t base_lm = (size_t)a.mbase[m] - m;

  double acc[4][4][2];
  zero_acc(acc);

  for (int k0 = 0; k0 < a.nlat2; k0 += AT_K) {
    // A: rows l0 .. l0+63, nodes k0 .. k0+15 (row-major per parity)
    for (int idx = tid; idx < AT_L * AT_K; idx += 128) {
      int row = idx / AT_K, kk = idx - row * AT_K;
      int l = l0 + row, i = k0 + kk;
      double v = (l <= a.lmax && i < a.nlat2) ? __ldg(a.P + (base_lm + l) * a.nlat2 + i) : 0.0;
      As[((row & 1) * 32 + (row >> 1)) * AT_LDA + kk] = v;
    }
    // B: G[m][par][plane][node] -> Bs[par][2*plane + c][node]
    for (int idx = tid; idx < 2 * (AT_N / 2) * AT_K; idx += 128) {
      int kk = idx % AT_K, rest = idx / AT_K;
      int pl = rest % (AT_N / 2), pr = rest / (AT_N / 2);
      int kz = kz0 + pl, i = k0 + kk;
      double2 v = make_double2(0.0, 0.0);
      if (kz < a.nz && i < a.nlat2) v = G[(((size_t)m * 2 + pr) * a.nz + kz) * a.nlat2 + i];
      Bs[(pr * AT_N + 2 * pl) * AT_LDB + kk] = v.x;
      Bs[(pr * AT_N + 2 * pl + 1) * AT_LDB + kk] = v.y;
    }
    __syncthreads();
    warp_mma<4, 4, false, true>(acc, As + par * 32 * AT_LDA, AT_LDA,
                                Bs + (par * AT_N + nh * 32) * AT_LDB, AT_LDB, AT_K);
    __syncthreads();
  }

  // stage C through shared memory: Cs[plane][l] (double2), then contiguous rows
  double2* Cs = reinterpret_cast<double2*>(smem);  // [32 planes][64 l]
  const int lane = tid & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int row = mt * 8 + g;             // row within parity
      int col = nh * 32 + nt * 8 + 2 * t;  // even column -> (re, im) of one plane
      int lloc = 2 * row + par;
      Cs[(col >> 1) * AT_L + lloc] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
  __syncthreads();
  const int nvalid = min(AT_L, a.lmax + 1 - l0);
  for (int idx = tid; idx < (AT_N / 2) * AT_L; idx += 128) {
    int pl = idx / AT_L, ll = idx - pl * AT_L;
    int kz = kz0 + pl;
    if (kz >= a.nz || ll >= nvalid) continue;
    double2 v = Cs[idx];
    if (m == 0) v.y = 0.0;  // m = 0 coefficients are real
    a.out[(size_t)kz * a.nlm + base_lm + l0 + ll] = v;
  }
}

// ---------------------------------------------------------------- scalar synthesis
// CTA: 64 nodes x 64 columns, both parities; K loop over l in steps of 16
// (8 per parity).  8 warps: (parity, node half, column half), 32x32 each.
constexpr int ST_I = 64, ST_N = 64, ST_K = 16, ST_LDA = ST_I + 4, ST_LDB = ST_N + 4;

__global__ void __launch_bounds__(256) leg_synthesis_kernel(LegArgs a) {
  __shared__ __align__(16) double As[2 * (ST_K / 2) * ST_LDA];  // [par][q][node]  K-major
  __shared__ __align__(16) double Bs[2 * (ST_K / 2) * ST_LDB];  // [par][q][col]   K x N
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, i0 = tile.r0;
  const int n0 = blockIdx.y * ST_N, kz0 = n0 / 2;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int par = warp >> 2, mh = (warp >> 1) & 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;

  double acc[4][4][2];
  zero_acc(acc);

  for (int lk = m; lk <= a.lmax; lk += ST_K) {
    for (int idx = tid; idx < ST_K * ST_I; idx += 256) {
      int q = idx / ST_I, ii = idx - q * ST_I;
      int l = lk + q, i = i0 + ii;
      double v = (l <= a.lmax && i < a.nlat2) ? __ldg(a.P + (base_lm + l) * a.nlat2 + i) : 0.0;
      As[((q & 1) * (ST_K / 2) + (q >> 1)) * ST_LDA + ii] = v;
    }
    for (int idx = tid; idx < (ST_N / 2) * ST_K; idx += 256) {
      int q = idx % ST_K, pl = idx / ST_K;
      int l = lk + q, kz = kz0 + pl;
      double2 v = make_double2(0.0, 0.0);
      if (l <= a.lmax && kz < a.nz) v = a.spec[(size_t)kz * a.nlm + base_lm + l];
      if (m == 0) v.y = 0.0;  // only Re a_l0 enters a real field
      double* row = Bs + ((q & 1) * (ST_K / 2) + (q >> 1)) * ST_LDB;
      row[2 * pl] = v.x;
      row[2 * pl + 1] = v.y;
    }
    __syncthreads();
    warp_mma<4, 4, true, false>(acc, As + par * (ST_K / 2) * ST_LDA + mh * 32, ST_LDA,
                                Bs + par * (ST_K / 2) * ST_LDB + nh * 32, ST_LDB, ST_K / 2);
    __syncthreads();
  }

  double2* G = a.Gw + (size_t)a.gfield * a.Gfield;
  const int lane = tid & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int i = i0 + mh * 32 + mt * 8 + g;
      int kz = kz0 + (nh * 32 + nt * 8 + 2 * t) / 2;
      if (i < a.nlat2 && kz < a.nz)
        G[(((size_t)m * 2 + par) * a.nz + kz) * a.nlat2 + i] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
}

// ---------------------------------------------------------------- vector analysis
// S_l = 1/(l(l+1)) sum_i [dP_l Vt_(1-p) - i mPs_l Vp_p]
// T_l = 1/(l(l+1)) sum_i [-i mPs_l Vt_p - dP_l Vp_(1-p)]
// (p = (l-m)%2; fold 0 = F(i)+F(mirror), fold 1 = F(i)-F(mirror);
//  Pbar has the parity of p, dPbar the opposite.)
// CTA: 32 consecutive l (16 per parity) x 64 columns; 4 warps (parity, half).
constexpr int VA_L = 32, VA_N = 64, VA_K = 16, VA_LDA = VA_K + 4, VA_LDB = VA_K + 4;

__global__ void __launch_bounds__(128) vec_analysis_kernel(LegArgs a) {
  extern __shared__ __align__(16) double vsm[];
  double* Ad = vsm;                          // dP   [par][16][VA_LDA]
  double* Am = Ad + 2 * 16 * VA_LDA;         // mPs  [par][16][VA_LDA]
  double* Bt = Am + 2 * 16 * VA_LDA;         // Vt   [fold][VA_N][VA_LDB]
  double* Bp = Bt + 2 * VA_N * VA_LDB;       // Vp   [fold][VA_N][VA_LDB]
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, l0 = tile.r0;
  const int n0 = blockIdx.y * VA_N, kz0 = n0 / 2;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int par = warp >> 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;
  const double2* Gt = a.G + (size_t)1 * a.Gfield;  // field 1: v_theta
  const double2* Gp = a.G + (size_t)2 * a.Gfield;  // field 2: v_phi

  double x1[2][4][2], x2[2][4][2], x3[2][4][2], x4[2][4][2];
  zero_acc(x1); zero_acc(x2); zero_acc(x3); zero_acc(x4);

  for (int k0 = 0; k0 < a.nlat2; k0 += VA_K) {
    for (int idx = tid; idx < VA_L * VA_K; idx += 128) {
      int row = idx / VA_K, kk = idx - row * VA_K;
      int l = l0 + row, i = k0 + kk;
      bool ok = (l <= a.lmax && i < a.nlat2);
      size_t off = (base_lm + l) * a.nlat2 + i;
      int so = ((row & 1) * 16 + (row >> 1)) * VA_LDA + kk;
      Ad[so] = ok ? __ldg(a.dP + off) : 0.0;
      Am[so] = ok ? __ldg(a.mPs + off) : 0.0;
    }
    for (int idx = tid; idx < 2 * (VA_N / 2) * VA_K; idx += 128) {
      int kk = idx % VA_K, rest = idx / VA_K;
      int pl = rest % (VA_N / 2), fo = rest / (VA_N / 2);
      int kz = kz0 + pl, i = k0 + kk;
      double2 vt = make_double2(0.0, 0.0), vp = vt;
      if (kz < a.nz && i < a.nlat2) {
        size_t off = (((size_t)m * 2 + fo) * a.nz + kz) * a.nlat2 + i;
        vt = Gt[off];
        vp = Gp[off];
      }
      Bt[(fo * VA_N + 2 * pl) * VA_LDB + kk] = vt.x;
      Bt[(fo * VA_N + 2 * pl + 1) * VA_LDB + kk] = vt.y;
      Bp[(fo * VA_N + 2 * pl) * VA_LDB + kk] = vp.x;
      Bp[(fo * VA_N + 2 * pl + 1) * VA_LDB + kk] = vp.y;
    }
    __syncthreads();
    const double* ad = Ad + par * 16 * VA_LDA;
    const double* am = Am + par * 16 * VA_LDA;
    const int cofs = nh * 32;
    warp_mma<2, 4, false, true>(x1, ad, VA_LDA, Bt + ((1 - par) * VA_N + cofs) * VA_LDB, VA_LDB, VA_K);
    warp_mma<2, 4, false, true>(x2, am, VA_LDA, Bp + (par * VA_N + cofs) * VA_LDB, VA_LDB, VA_K);
    warp_mma<2, 4, false, true>(x3, ad, VA_LDA, Bp + ((1 - par) * VA_N + cofs) * VA_LDB, VA_LDB, VA_K);
    warp_mma<2, 4, false, true>(x4, am, VA_LDA, Bt + (par * VA_N + cofs) * VA_LDB, VA_LDB, VA_K);
    __syncthreads();
  }

  const int lane = tid & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int row = mt * 8 + g;
      int l = l0 + 2 * row + par;
      int kz = kz0 + (nh * 32 + nt * 8 + 2 * t) / 2;
      if (l > a.lmax || kz >= a.nz) continue;
      double f = l ? 1.0 / ((double)l * (double)(l + 1)) : 0.0;
      // S = X1 - i X2 ; T = -X3 - i X4
      double2 S = make_double2(x1[mt][nt][0] + x2[mt][nt][1], x1[mt][nt][1] - x2[mt][nt][0]);
      double2 T = make_double2(-x3[mt][nt][0] + x4[mt][nt][1], -x3[mt][nt][1] - x4[mt][nt][0]);
      S = cscale(S, f);
      T = cscale(T, f);
      if (m == 0) { S.y = 0.0; T.y = 0.0; }
      size_t o = (size_t)kz * a.nlm + base_lm + l;
      a.out[o] = S;
      a.out2[o] = T;
    }
}

// ---------------------------------------------------------------- vector synthesis
// Vt_q = sum_{p=1-q} dP_l S_l + i sum_{p=q} mPs_l T_l
// Vp_q = -sum_{p=1-q} dP_l T_l + i sum_{p=q} mPs_l S_l
// CTA: 32 nodes x 64 columns; 8 warps: (fold q, theta/phi, column half).
constexpr int VS_I = 32, VS_N = 64, VS_K = 16, VS_LDA = VS_I + 4, VS_LDB = VS_N + 4;

__global__ void __launch_bounds__(256) vec_synthesis_kernel(LegArgs a) {
  __shared__ __align__(16) double Ad[2 * 8 * VS_LDA];   // dP  [par][q8][node]
  __shared__ __align__(16) double Am[2 * 8 * VS_LDA];   // mPs
  __shared__ __align__(16) double Bsv[2 * 8 * VS_LDB];  // S   [par][q8][col]
  __shared__ __align__(16) double Btv[2 * 8 * VS_LDB];  // T
  const LegTile tile = a.tiles[blockIdx.x];
  const int m = tile.m, i0 = tile.r0;
  const int n0 = blockIdx.y * VS_N, kz0 = n0 / 2;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int q = warp >> 2, comp = (warp >> 1) & 1, nh = warp & 1;
  const size_t base_lm = (size_t)a.mbase[m] - m;

  double xa[4][4][2], xb[4][4][2];
  zero_acc(xa);
  zero_acc(xb);

  for (int lk = m; lk <= a.lmax; lk += VS_K) {
    for (int idx = tid; idx < VS_K * VS_I; idx += 256) {
      int qq = idx / VS_I, ii = idx - qq * VS_I;
      int l = lk + qq, i = i0 + ii;
      bool ok = (l <= a.lmax && i < a.nlat2);
      size_t off = (base_lm + l) * a.nlat2 + i;
      int so = ((qq & 1) * 8 + (qq >> 1)) * VS_LDA + ii;
      Ad[so] = ok ? __ldg(a.dP + off) : 0.0;
      Am[so] = ok ? __ldg(a.mPs + off) : 0.0;
    }
    for (int idx = tid; idx < (VS_N / 2) * VS_K; idx += 256) {
      int qq = idx % VS_K, pl = idx / VS_K;
      int l = lk + qq, kz = kz0 + pl;
      double2 s = make_double2(0.0, 0.0), tt = s;
      if (l <= a.lmax && kz < a.nz && l > 0) {
        size_t o = (size_t)kz * a.nlm + base_lm + l;
        s = a.spec[o];
        tt = a.spec2[o];
      }
      if (m == 0) { s.y = 0.0; tt.y = 0.0; }
      int ro = ((qq & 1) * 8 + (qq >> 1)) * VS_LDB;
      Bsv[ro + 2 * pl] = s.x;
      Bsv[ro + 2 * pl + 1] = s.y;
      Btv[ro + 2 * pl] = tt.x;
      Btv[ro + 2 * pl + 1] = tt.y;
    }
    __syncthreads();
    // rows of parity 1-q through dP, rows of parity q through mPs
    const double* ad = Ad + (1 - q) * 8 * VS_LDA;
    const double* am = Am + q * 8 * VS_LDA;
    const double* bA = (comp == 0 ? Bsv : Btv) + (1 - q) * 8 * VS_LDB + nh * 32;
    const double* bB = (comp == 0 ? Btv : Bsv) + q * 8 * VS_LDB + nh * 32;
    warp_mma<4, 4, true, false>(xa, ad, VS_LDA, bA, VS_LDB, 8);
    warp_mma<4, 4, true, false>(xb, am, VS_LDA, bB, VS_LDB, 8);
    __syncthreads();
  }

  double2* G = a.Gw + (size_t)(1 + comp) * a.Gfield;
  const int lane = tid & 31, g = lane >> 2, t = lane & 3;
  const double sa = comp == 0 ? 1.0 : -1.0;
#pragma unroll
  for (int mt = 0; mt < 4; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
      int i = i0 + mt * 8 + g;
      int kz = kz0 + (nh * 32 + nt * 8 + 2 * t) / 2;
      if (i >= a.nlat2 || kz >= a.nz) continue;
      // V = sa * Xa + i * Xb
      double2 v = make_double2(sa * xa[mt][nt][0] - xb[mt][nt][1], sa * xa[mt][nt][1] + xb[mt][nt][0]);
      G[(((size_t)m * 2 + q) * a.nz + kz) * a.nlat2 + i] = v;
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
  a.nlat2 = p->nlat2;
  a.nz = p->nz;
  a.nlm = p->nlm;
  return a;
}

}  // namespace

int launch_leg_analysis(const sph_plan* p, int gfield, double2* spec, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.gfield = gfield;
  a.out = spec;
  a.tiles = p->tilesA;
  dim3 grid(p->ntilesA, (2 * p->nz + AT_N - 1) / AT_N);
  TimedLaunch tl(p, T_LEG_ANA, st);
  leg_analysis_kernel<<<grid, 128, 0, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_leg_synthesis(const sph_plan* p, const double2* spec, int gfield, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.gfield = gfield;
  a.spec = spec;
  a.tiles = p->tilesS;
  dim3 grid(p->ntilesS, (2 * p->nz + ST_N - 1) / ST_N);
  TimedLaunch tl(p, T_LEG_SYN, st);
  leg_synthesis_kernel<<<grid, 256, 0, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_vec_analysis(const sph_plan* p, double2* s, double2* t, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.out = s;
  a.out2 = t;
  a.tiles = p->tilesA32;
  size_t smem = (size_t)(4 * 16 * VA_LDA + 4 * VA_N * VA_LDB) * sizeof(double);
  static bool once = cudaFuncSetAttribute(vec_analysis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem) == cudaSuccess;
  if (!once) return SPH_ECUDA;
  dim3 grid(p->ntilesA32, (2 * p->nz + VA_N - 1) / VA_N);
  TimedLaunch tl(p, T_VEC_ANA, st);
  vec_analysis_kernel<<<grid, 128, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int launch_vec_synthesis(const sph_plan* p, const double2* s, const double2* t, cudaStream_t st) {
  LegArgs a = base_args(p);
  a.spec = s;
  a.spec2 = t;
  a.tiles = p->tilesS32;
  dim3 grid(p->ntilesS32, (2 * p->nz + VS_N - 1) / VS_N);
  TimedLaunch tl(p, T_VEC_SYN, st);
  vec_synthesis_kernel<<<grid, 256, 0, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
