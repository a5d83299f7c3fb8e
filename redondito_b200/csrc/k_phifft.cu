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
#include <algorithm>

#include "fft3.cuh"
#include "fft_ct.cuh"
#include "tc05.cuh"
#include "tma.cuh"
#include "cluster.cuh"

namespace {

constexpr int PTHREADS = 512;
constexpr int PMAXC = 8192;  // NP*nphi complex values per CTA

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
  const int* kzl;  // planes to transform (nullptr: all nz)
  const double* wfold;
  FftDesc fd;
  int* flag;  // set when a bounded wait gives up (cluster three-step forward)
};

// ---------------------------------------------------------------- lengths 2^a 3^b
// N (phi length) and NP (ring pairs per CTA) fixed at compile time: every
// thread keeps one ring (load/store) or one ring pair (spectrum) and walks
// the other index with a constant stride, so no runtime divisions remain.
template <int N, int NP>
__global__ void __launch_bounds__(PTHREADS, 2) phi_fwd_ct(PhiArgs a) {
  extern __shared__ double2 sm[];
  constexpr int Q = 2 * NP;             // rings per CTA
  constexpr int JSTEP = PTHREADS / Q;   // phi stride of one thread
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = a.kzl ? __ldg(a.kzl + blockIdx.y) : blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x;
  const double* plane = a.gin[f] + (size_t)k * N * nlat;
  const ct::Geo<N, 1, true> g{NP, seq_stride(N), 1};
  double* smd = reinterpret_cast<double*>(sm);
  {
    // ring slot q: 0..NP-1 northern rings p0+q (real part), NP..2NP-1 their
    // mirrors in ascending address order (imaginary part of pair 2NP-1-q)
    const int q = tid % Q, j0 = tid / Q;
    const int b = q < NP ? q : 2 * NP - 1 - q;
    const int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
    const int half = q < NP ? 0 : 1;
    constexpr int NJ = (N + JSTEP - 1) / JSTEP;
    constexpr int U = 8;
#pragma unroll
    for (int u0 = 0; u0 < NJ; u0 += U) {
      double v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int j = j0 + (u0 + u) * JSTEP;
        v[u] = (u0 + u < NJ && j < N) ? __ldg(plane + (size_t)j * nlat + ring) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int j = j0 + (u0 + u) * JSTEP;
        if (u0 + u < NJ && j < N) smd[2 * g.addr(b, j) + half] = v[u];
      }
    }
  }
  __syncthreads();
  ct::dif<double2, N, N>(sm, g, a.fd.twp, -1);

  // both parities of one (m, pair) from one read of Z(m), Z(-m)
  double2* G = a.G + (size_t)f * a.Gfield + (size_t)k * a.ldn + p0;
  const size_t mstride = (size_t)2 * a.nz * a.ldn, pstride = (size_t)a.nz * a.ldn;
  const int b = tid % NP;
  const double W = __ldg(a.wfold + p0 + b);
  for (int m = tid / NP; m <= a.lmax; m += PTHREADS / NP) {
    double2 Z = sm[g.addr(b, ct::rev_pos<N>(m))];
    double2 Zc = sm[g.addr(b, ct::rev_pos<N>(m == 0 ? 0 : N - m))];
    // F(i) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
    double2 Fi = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y - Zc.y));
    double2 Fm = make_double2(0.5 * (Z.y + Zc.y), -0.5 * (Z.x - Zc.x));
    G[m * mstride + b] = cscale(cadd(Fi, Fm), W);
    G[m * mstride + pstride + b] = cscale(csub(Fi, Fm), W);
  }
}

template <int N, int NP>
__global__ void __launch_bounds__(PTHREADS, 2) phi_inv_ct(PhiArgs a) {
  extern __shared__ double2 sm[];
  constexpr int Q = 2 * NP;
  constexpr int JSTEP = PTHREADS / Q;
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = a.kzl ? __ldg(a.kzl + blockIdx.y) : blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x;
  const ct::Geo<N, 1, true> g{NP, seq_stride(N), 1};
  const int M = a.lmax + 1;

  // zero everything, then scatter the 2 lmax + 1 nonzero frequencies
  {
    double2* s4 = sm;
    const int tot = NP * seq_stride(N);
    for (int i = tid; i < tot; i += PTHREADS) s4[i] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  {
    const double2* G = a.Gc + (size_t)f * a.Gfield + (size_t)k * a.ldn + p0;
    const size_t mstride = (size_t)2 * a.nz * a.ldn, pstride = (size_t)a.nz * a.ldn;
    const int b = tid % NP;
    constexpr int U = 4;
    for (int m0 = tid / NP; m0 < M; m0 += U * (PTHREADS / NP)) {
      double2 se[U], so[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int m = m0 + u * (PTHREADS / NP);
        se[u] = so[u] = make_double2(0.0, 0.0);
        if (m < M) {
          se[u] = __ldg(G + m * mstride + b);
          so[u] = __ldg(G + m * mstride + pstride + b);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int m = m0 + u * (PTHREADS / NP);
        if (m >= M) continue;
        double2 Fi = cadd(se[u], so[u]), Fm = csub(se[u], so[u]);
        if (m == 0) {
          sm[g.addr(b, 0)] = make_double2(Fi.x, Fm.x);
        } else {
          // z = x + i y with x, y the real fields of ring i and its mirror
          sm[g.addr(b, ct::rev_pos<N>(m))] = make_double2(Fi.x - Fm.y, Fi.y + Fm.x);
          sm[g.addr(b, ct::rev_pos<N>(N - m))] = make_double2(Fi.x + Fm.y, -Fi.y + Fm.x);
        }
      }
    }
  }
  __syncthreads();
  ct::dit<double2, N, N>(sm, g, a.fd.twp, +1);

  double* plane = a.gout[f] + (size_t)k * N * nlat;
  const double* smd = reinterpret_cast<const double*>(sm);
  const int q = tid % Q, j0 = tid / Q;
  const int b = q < NP ? q : 2 * NP - 1 - q;
  const int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
  const int half = q < NP ? 0 : 1;
  for (int j = j0; j < N; j += JSTEP) plane[(size_t)j * nlat + ring] = smd[2 * g.addr(b, j) + half];
}

// ---------------------------------------------------------------- other lengths
template <int CTN>
__global__ void __launch_bounds__(PTHREADS, 2) phi_fwd_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = a.kzl ? __ldg(a.kzl + blockIdx.y) : blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const double* plane = a.gin[f] + (size_t)k * nphi * nlat;
  const int np = min(NP, nlat2 - p0);
  FftGeom g;
  g.n = nphi; g.batch = NP; g.bs = seq_stride(nphi); g.es = 1; g.pad = 1; g.jfast = true;
  double* smd = reinterpret_cast<double*>(sm);
  const int total = nphi * 2 * NP;
  for (int idx = tid; idx < total; idx += PTHREADS) {
    int j = idx / (2 * NP), q = idx - j * 2 * NP;
    int b = q < NP ? q : NP - 1 - (q - NP);
    int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
    smd[2 * g.addr(b, j) + (q < NP ? 0 : 1)] = b < np ? __ldg(plane + (size_t)j * nlat + ring) : 0.0;
  }
  __syncthreads();
  fft_dif(sm, a.fd, g, -1);
  const int* __restrict__ rev = a.fd.rev;
  double2* G = a.G + (size_t)f * a.Gfield;
  const int M = a.lmax + 1;
  for (int idx = tid; idx < M * NP; idx += PTHREADS) {
    int b = idx % NP, m = idx / NP;
    if (b >= np) continue;
    double2 Z = sm[g.addr(b, __ldg(rev + m))];
    double2 Zc = sm[g.addr(b, __ldg(rev + (m == 0 ? 0 : nphi - m)))];
    double2 Fi = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y - Zc.y));
    double2 Fm = make_double2(0.5 * (Z.y + Zc.y), -0.5 * (Z.x - Zc.x));
    double W = __ldg(a.wfold + p0 + b);
    G[(((size_t)m * 2 + 0) * a.nz + k) * a.ldn + p0 + b] = cscale(cadd(Fi, Fm), W);
    G[(((size_t)m * 2 + 1) * a.nz + k) * a.ldn + p0 + b] = cscale(csub(Fi, Fm), W);
  }
}

template <int CTN>
__global__ void __launch_bounds__(PTHREADS, 2) phi_inv_kernel(PhiArgs a) {
  extern __shared__ double2 sm[];
  const int NP = a.NP, nphi = a.nphi, nlat = a.nlat, nlat2 = a.nlat2;
  const int p0 = blockIdx.x * NP;
  const int k = a.kzl ? __ldg(a.kzl + blockIdx.y) : blockIdx.y;
  const int f = blockIdx.z;
  const int tid = threadIdx.x;
  const int np = min(NP, nlat2 - p0);
  const int M = a.lmax + 1;
  const double2* G = a.Gc + (size_t)f * a.Gfield;
  FftGeom g;
  g.n = nphi; g.batch = NP; g.bs = seq_stride(nphi); g.es = 1; g.pad = 1; g.jfast = true;
  const int* __restrict__ rev = a.fd.rev;
  for (int i = tid; i < NP * g.bs; i += PTHREADS) sm[i] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int idx = tid; idx < M * NP; idx += PTHREADS) {
    int b = idx % NP, m = idx / NP;
    if (b >= np) continue;
    double2 Se = G[(((size_t)m * 2 + 0) * a.nz + k) * a.ldn + p0 + b];
    double2 So = G[(((size_t)m * 2 + 1) * a.nz + k) * a.ldn + p0 + b];
    double2 Fi = cadd(Se, So), Fm = csub(Se, So);
    if (m == 0) {
      sm[g.addr(b, __ldg(rev))] = make_double2(Fi.x, Fm.x);
    } else {
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

// ---------------------------------------------------------------- three-step inverse (FP64)
// Persistent kernel over tiles of NP ring pairs of one (plane, field): the
// folded coefficients of the tile (lmax + 1 degrees x 2 parities x NP nodes,
// double2) arrive by cp.async, are assembled into Z(m) of each ring pair
// (x = ring + i mirror, zero past lmax), and go through the three-step
// inverse DFT N = A M, M = B C (A = 16): (C') C-point DFTs over kc of
// Z(ka + A (kb + B kc)), the twiddle W_M^-(c kb); (B') B-point DFTs over kb;
// (A') the twiddle W_N^-(nm ka) and A-point DFTs over ka, written to the
// grid rows x[nm + M n1].  One staged tile per CTA; two CTAs per SM where
// shared memory allows, so that one loads while the other computes.  Shared
// memory accesses are 16 bytes wide, so a quarter warp must hit distinct
// 16-byte slots mod 8: the row pitch PR is odd, the ring-pair stride SB is
// 8/NP (mod 8), and staged rows swap their parity halves every 4/NP rows.
constexpr int up_mod16(int x, int r) { return x + (((r - x) % 16) + 16) % 16; }

template <int N, int NP>
struct P3d {
  static constexpr int A = 16, M = N / A, B = ct::pow2_part_cap16(M), C = M / B;
  static constexpr int ITEMS_A = NP * M, ITEMS_B = NP * A * C, ITEMS_C = NP * A * B;
  static constexpr int THREADS = ITEMS_A <= 64 ? 64 : (ITEMS_A + 31) / 32 * 32;
  static constexpr int PR = M | 1;
  static constexpr int SB = up_mod16(A * PR, 8 / NP);
  static constexpr size_t XBYTES = (size_t)NP * SB * sizeof(double2);
  // transform area, twiddles W_N^e, one staged tile for the largest lmax (N/2 - 1)
  static constexpr size_t SMEM_MAX = XBYTES + (size_t)N * sizeof(double2) + (size_t)N * NP * sizeof(double2);
  static constexpr int MINB = SMEM_MAX <= 113 * 1024 && THREADS <= 512 ? 2 : 1;
  static size_t smem(int lmax) {
    return XBYTES + (size_t)N * sizeof(double2) + (size_t)(lmax + 1) * 2 * NP * sizeof(double2);
  }
  static_assert(N % A == 0 && NP >= 2 && NP <= 8 && XBYTES % 16 == 0, "three-step geometry");
};

template <int NP>
__device__ __forceinline__ int stage_swz64(int row) {
  return ((row * NP) >> 2) & 1;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}

template <int N, int NP>
__global__ void __launch_bounds__(P3d<N, NP>::THREADS, P3d<N, NP>::MINB) phi3_inv64(PhiArgs a, int ntiles) {
  using G = P3d<N, NP>;
  constexpr int A = G::A, M = G::M, B = G::B, C = G::C, T = G::THREADS;
  extern __shared__ __align__(1024) unsigned char sm3d[];
  double2* X = reinterpret_cast<double2*>(sm3d);
  double2* tw = reinterpret_cast<double2*>(sm3d + G::XBYTES);
  double2* st = tw + N;
  const int lmax = a.lmax, nlat = a.nlat, ngroups = nlat / 2 / NP;
  const int t = threadIdx.x;
  for (int i = t; i < N; i += T) tw[i] = __ldg(a.fd.tw + i);
  const size_t pstride = (size_t)a.nz * a.ldn;  // parity stride of the folded coefficients
  // the coefficients of a tile into the stage, by cp.async (every thread its share)
  auto issue = [&](int tile) {
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz;
    const double2* gs = a.Gc + (size_t)f * a.Gfield + (size_t)k * a.ldn + g * NP;
    const int total = (lmax + 1) * 2 * NP;
    for (int q = t; q < total; q += T) {
      const int b = q % NP, rr = q / NP, par = rr & 1, mm = rr >> 1;
      cp_async16(st + mm * 2 * NP + (par ^ stage_swz64<NP>(mm)) * NP + b, gs + (size_t)rr * pstride + b);
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  };
  if ((int)blockIdx.x < ntiles) issue(blockIdx.x);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz, p0 = g * NP;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();  // the tile's coefficients have landed; the last tile's step (A') is done with X
    auto zin = [&](int m, int b) {
      const bool lo = m <= lmax, hi = N - m <= lmax;
      if (!lo && !hi) return make_double2(0.0, 0.0);
      const int mm = lo ? m : N - m;
      const int sw = stage_swz64<NP>(mm);
      const double2 se = st[mm * 2 * NP + sw * NP + b], so = st[mm * 2 * NP + (1 - sw) * NP + b];
      const double2 Fi = make_double2(se.x + so.x, se.y + so.y), Fm = make_double2(se.x - so.x, se.y - so.y);
      if (m == 0) return make_double2(Fi.x, Fm.x);
      // z = x + i y with x, y the real fields of ring i and its mirror
      if (lo) return make_double2(Fi.x - Fm.y, Fi.y + Fm.x);
      return make_double2(Fi.x + Fm.y, -Fi.y + Fm.x);
    };
    auto conj = [](double2 z) { return make_double2(z.x, -z.y); };
    // (C')
    for (int it = t; it < G::ITEMS_C; it += T) {
      const int b = it % NP, rr = it / NP, ka = rr % A, kb = rr / A;
      double2 u[C];
#pragma unroll
      for (int kc = 0; kc < C; ++kc) u[kc] = zin(ka + A * (kb + B * kc), b);
      ct::RD<double2, C, 1>::run(u);
      double2* row = X + b * G::SB + ka * G::PR + C * kb;
#pragma unroll
      for (int c = 0; c < C; ++c) row[c] = (c && kb) ? ct::mul(u[c], conj(tw[A * c * kb])) : u[c];
    }
    __syncthreads();
    // step (C') was the last reader of the stage: the next tile's
    // coefficients load while steps (B') and (A') run
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
    if constexpr (B > 1) {  // (B'): stored at column c + C nb
      for (int it = t; it < G::ITEMS_B; it += T) {
        const int ka = it % A, rr = it / A, c = rr % C, b = rr / C;
        double2* row = X + b * G::SB + ka * G::PR + c;
        double2 w[B];
#pragma unroll
        for (int kb = 0; kb < B; ++kb) w[kb] = row[C * kb];
        ct::RD<double2, B, 1>::run(w);
#pragma unroll
        for (int nb = 0; nb < B; ++nb) row[C * nb] = w[nb];
      }
      __syncthreads();
    }
    // (A')
    if (t < G::ITEMS_A) {
      const int b = t % NP, nm = t / NP;
      double2 v[A];
      const double2* xi = X + b * G::SB + nm;
#pragma unroll
      for (int ka = 0; ka < A; ++ka) v[ka] = ka ? ct::mul(xi[ka * G::PR], conj(tw[nm * ka])) : xi[0];
      ct::RD<double2, A, 1>::run(v);
      double* plane = a.gout[f] + (size_t)k * N * nlat;
      double* pr = plane + p0 + b;
      double* pm = plane + (nlat - 1 - p0 - b);
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        const size_t j = (size_t)(nm + M * n1) * nlat;
        pr[j] = v[n1].x;
        pm[j] = v[n1].y;
      }
    }
  }
}

constexpr int PHI3D_UNSUPPORTED = 1000;

template <int N, int NP>
constexpr bool phi3d_ok() {
  if constexpr (N % 16 != 0 || N < 48 || NP * (N / 16) > 1024) {
    return false;
  } else {
    return P3d<N, NP>::SMEM_MAX <= 220 * 1024;
  }
}

template <int N, int NP>
int phi3d_run(const sph_plan* p, const PhiArgs& a, int nfields, cudaStream_t st) {
  if constexpr (!phi3d_ok<N, NP>()) {
    return PHI3D_UNSUPPORTED;
  } else {
    using G = P3d<N, NP>;
    const size_t smem = G::smem(p->lmax);
    const long long ntiles = (long long)(p->nlat2 / NP) * p->nz * nfields;
    if (ntiles == 0) return SPH_OK;
    if (ntiles > (1ll << 30)) return PHI3D_UNSUPPORTED;
    auto kern = phi3_inv64<N, NP>;
    int occ = 0, dev = 0, nsm = 0;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, G::THREADS, smem) != cudaSuccess ||
        cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return SPH_ECUDA;
    const int grid = (int)std::min<long long>(ntiles, (long long)std::max(1, occ) * std::max(1, nsm));
    kern<<<grid, G::THREADS, smem, st>>>(a, (int)ntiles);
    SPH_LAUNCH_OK();
    return SPH_OK;
  }
}

// ring pairs per tile: the most that fit, at most the tuned ring_pairs
template <int N>
int phi3d_dispatch_n(const sph_plan* p, const PhiArgs& a, int nfields, cudaStream_t st) {
  const int cap = p->tile_np ? p->tile_np : 8;
  if (phi3d_ok<N, 8>() && cap >= 8 && p->nlat2 % 8 == 0) return phi3d_run<N, 8>(p, a, nfields, st);
  if (phi3d_ok<N, 4>() && cap >= 4 && p->nlat2 % 4 == 0) return phi3d_run<N, 4>(p, a, nfields, st);
  if (phi3d_ok<N, 2>() && cap >= 2 && p->nlat2 % 2 == 0) return phi3d_run<N, 2>(p, a, nfields, st);
  return PHI3D_UNSUPPORTED;
}

// ---------------------------------------------------------------- three-step forward (FP64, cluster tiles)
// The forward transform reads NP consecutive rings and their NP mirrors from
// each of the N rows of a plane; a request carries 8 NP contiguous bytes,
// and the bandwidth an SM draws grows with that run (16, 32, 64 bytes:
// 1.1, 1.8, 2.7 TB/s).  An FP64 tile of 4 ring pairs already fills half of
// an SM's shared memory, so a tile of NPC = 4 CL ring pairs is shared by a
// cluster of CL CTAs: CTA rank r loads, by TMA, the rows [r N/CL, (r+1) N/CL)
// of all NPC rings and mirrors (runs of 8 NPC bytes: 64 B for CL = 2, 128 B
// for CL = 4), double buffered, and transforms ring pairs 4r .. 4r+3, whose
// samples it reads across the cluster from distributed shared memory in
// step (A).  Two cluster barriers per tile: (1) every CTA's rows have landed
// (or a bounded wait gave up, which every CTA then sees), (2) no CTA reads
// another's staged rows any more, so each overwrites its own with its
// transform area.  Steps (A), (B), (C) and the fold are those of the
// three-step inverse run forwards (sign -1); the fold writes the folded
// coefficients G[m][parity][k][node] like phi_fwd_ct.  Only warp 0, which
// stores nothing to global memory, arrives at barrier (1) with release
// semantics, and every warp arrives at (2) relaxed once its step-(A) loads
// have returned: the folding warps' stores are not drained at the barriers.
// The dispatcher uses clusters of 2.  The staged rows are swizzled by the
// TMA (16-byte chunk index XOR 128-byte row index), so the
// step-(A) reads of a half warp (4 ring pairs x 4 rows) spread over the
// banks; the transform area has an odd row pitch and a ring-pair stride of
// 2 (mod 8) 16-byte slots.
template <int N, int CL>
struct P3c {
  static constexpr int NPL = 4, NPC = NPL * CL;  // ring pairs per CTA, per cluster tile
  static constexpr int A = 16, M = N / A, B = ct::pow2_part_cap16(M), C = M / B;
  static constexpr int ROWS = N / CL;                          // phi rows staged by one CTA
  static constexpr int BR = largest_divisor_le(ROWS, 256);     // rows per TMA box
  static constexpr int ROWB = NPC * 8;                         // bytes per staged row
  static constexpr int SWB = ROWB >= 128 ? 3 : 2;               // swizzle: 2^SWB chunks of 16 bytes
  static constexpr int ITEMS_A = NPL * M, ITEMS_B = NPL * A * C, ITEMS_C = NPL * A * B;
  static constexpr int THREADS = ITEMS_A <= 64 ? 64 : (ITEMS_A + 31) / 32 * 32;
  static constexpr int PR = M | 1;
  static constexpr int SB = up_mod16(A * PR, 8 / NPL);
  static constexpr size_t XBYTES = (size_t)NPL * SB * sizeof(double2);
  static constexpr size_t TILE_BYTES = (size_t)2 * ROWS * ROWB;  // rings and mirrors
  static constexpr size_t STAGE = round_up(XBYTES > TILE_BYTES ? XBYTES : TILE_BYTES, 1024);
  static constexpr size_t SMEM = 2 * STAGE + (size_t)N * sizeof(double2) + 64;
  // byte offset of staged element (row, column) within one half of a stage
  static __device__ __forceinline__ uint32_t off(int row, int col) {
    const uint32_t o = (uint32_t)(row * ROWB + col * 8);
    return o ^ (((o >> 7) & ((1u << SWB) - 1)) << 4);
  }
};

template <int N, int CL>
constexpr bool phi3c_ok() {
  if constexpr (N % 16 != 0 || N < 48 || (CL != 2 && CL != 4)) {
    return false;
  } else {
    using G = P3c<N, CL>;
    // every TMA box and both halves of a stage start on a 1024-byte boundary (swizzle atoms)
    return G::THREADS <= 1024 && ((size_t)G::ROWS * G::ROWB) % 1024 == 0 && (G::BR * G::ROWB) % 1024 == 0 &&
           G::SMEM <= 227 * 1024;
  }
}

struct GridMaps {
  CUtensorMap m[SPH_MAX_FIELDS];
};

template <int N, int CL>
__global__ void __launch_bounds__(P3c<N, CL>::THREADS, 1)
    phi3c_fwd64(PhiArgs a, int ntiles, const __grid_constant__ GridMaps maps) {
  using G = P3c<N, CL>;
  constexpr int A = G::A, M = G::M, B = G::B, C = G::C, T = G::THREADS, NPL = G::NPL, NPC = G::NPC;
  constexpr int ROWS = G::ROWS, BR = G::BR;
  extern __shared__ __align__(1024) unsigned char sm3c[];
  double2* tws = reinterpret_cast<double2*>(sm3c + 2 * G::STAGE);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm3c + 2 * G::STAGE + (size_t)N * sizeof(double2));
  int* bad = reinterpret_cast<int*>(full + 2);  // this CTA's last wait gave up (read by the cluster)
  const int t = threadIdx.x, warp = t / 32;
  const uint32_t rank = cluster_rank();
  const int cid = blockIdx.x / CL, ncl = gridDim.x / CL;
  const int nlat = a.nlat, ngroups = nlat / 2 / NPC;
  for (int i = t; i < N; i += T) tws[i] = __ldg(a.fd.tw + i);
  auto tw = [&](int e) { return tws[e]; };  // W_N^e
  if (t == 0) {
    tc05::mbar_init(&full[0], 1);
    tc05::mbar_init(&full[1], 1);
    *bad = 0;
    tc05::mbar_fence_init();
  }
  __syncthreads();
  cluster_sync_all();  // every CTA of the cluster runs before any reads another's shared memory
  auto stage = [&](int w) { return sm3c + (size_t)w * G::STAGE; };
  // one thread: this CTA's rows of a tile, rings then mirrors
  auto issue = [&](int tile, int w) {
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz;
    unsigned char* st = stage(w);
    tma::expect_tx(&full[w], (uint32_t)G::TILE_BYTES);
    const int y0 = k * N + (int)rank * ROWS;
#pragma unroll 1
    for (int i = 0; i < ROWS / BR; ++i) {
      tma::load_2d(st + (size_t)i * BR * G::ROWB, &maps.m[f], g * NPC, y0 + i * BR, &full[w]);
      tma::load_2d(st + (size_t)(ROWS + i * BR) * G::ROWB, &maps.m[f], nlat - g * NPC - NPC, y0 + i * BR,
                   &full[w]);
    }
  };
  int tile = cid;
  if (t == 0 && tile < ntiles) issue(tile, 0);
  int s = 0;
  uint32_t phase = 0;  // bit s: parity of the next completion of stage s
  bool gave_up = false;
  for (; tile < ntiles; tile += ncl, s ^= 1) {
    const bool ok = tc05::mbar_wait(&full[s], (phase >> s) & 1);
    const int mine = __syncthreads_or(!ok);
    if (t == 0) *bad = mine;
    // (1) every CTA's rows of this tile have landed, or a wait gave up; warp 0
    // (which observed the copies' completion and wrote `bad`, and holds no
    // global stores) releases, the folding warps arrive relaxed so that their
    // stores of the last tile do not drain here
    cluster_sync_split(warp == 0);
    int any = 0;
#pragma unroll
    for (int r = 0; r < CL; ++r) any |= ld_cluster_s32(cluster_map(bad, r));
    if (any) {  // every CTA of the cluster leaves here, on the same tile
      gave_up = mine != 0;
      break;
    }
    phase ^= 1u << s;
    if (t == 0 && tile + ncl < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue(tile + ncl, s ^ 1);
    }
    const int g = tile % ngroups, rr = tile / ngroups, k = rr % a.nz, f = rr / a.nz;
    // (A) the samples x[nm + M n1] of local ring pair b (ring: real part, mirror: imaginary part)
    const bool act = t < G::ITEMS_A;
    // ring pair b of the CTA, row nm: with clusters of 2 a staged row is 64
    // bytes and this CTA reads 32 of them; a half warp takes rows
    // {q, q+1, q+4, q+5} (bits 1 and 2 of the row index swapped within blocks
    // of 8 rows), which the 64-byte swizzle puts in four distinct 32-byte bank
    // groups (rows q and q+2 would share one)
    const int b = t % NPL, g8 = t / NPL;
    const int nm = (CL == 2 && (g8 | 7) < M) ? ((g8 & ~7) | (g8 & 1) | ((g8 & 2) << 1) | ((g8 & 4) >> 1)) : g8;
    double2 v[A];
    if (act) {
      const int col = (int)rank * NPL + b;
      uint32_t base[CL];
#pragma unroll
      for (int o = 0; o < CL; ++o) base[o] = cluster_map(stage(s), o);
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        constexpr int PER = A / CL;  // n1 values per staged row range
        const int o = n1 / PER, jr = nm + M * (n1 - o * PER);
        v[n1] = make_double2(ld_cluster_f64(base[o] + G::off(jr, col)),
                             ld_cluster_f64(base[o] + (uint32_t)(ROWS * G::ROWB) + G::off(jr, NPC - 1 - col)));
      }
      ct::RD<double2, A, -1>::run(v);
    }
    // (2) no CTA reads another's staged rows any more: every sample has been
    // loaded (the arrival waits for v[0] = the sum of all of them)
    cluster_sync_split(false, act ? v[0].x + v[0].y : 0.0);
    double2* X = reinterpret_cast<double2*>(stage(s));
    if (act) {
      double2* xo = X + b * G::SB + nm;
#pragma unroll
      for (int ka = 0; ka < A; ++ka) xo[ka * G::PR] = ka ? ct::mul(v[ka], tw(nm * ka)) : v[ka];
    }
    __syncthreads();
    if constexpr (B > 1) {  // (B)
      for (int it = t; it < G::ITEMS_B; it += T) {
        const int ka = it % A, r2 = it / A, c = r2 % C, bb = r2 / C;
        double2* row = X + bb * G::SB + ka * G::PR + c;
        double2 w[B];
#pragma unroll
        for (int nb = 0; nb < B; ++nb) w[nb] = row[C * nb];
        ct::RD<double2, B, -1>::run(w);
#pragma unroll
        for (int kb = 0; kb < B; ++kb) row[C * kb] = (kb && c) ? ct::mul(w[kb], tw(A * c * kb)) : w[kb];
      }
      __syncthreads();
    }
    if constexpr (C > 1) {  // (C)
      for (int it = t; it < G::ITEMS_C; it += T) {
        const int ka = it % A, r2 = it / A, kb = r2 % B, bb = r2 / B;
        double2* row = X + bb * G::SB + ka * G::PR + C * kb;
        double2 u[C];
#pragma unroll
        for (int c = 0; c < C; ++c) u[c] = row[c];
        ct::RD<double2, C, -1>::run(u);
#pragma unroll
        for (int kc = 0; kc < C; ++kc) row[kc] = u[kc];
      }
      __syncthreads();
    }
    // fold both parities of one (m, pair) from Z(m), Z(-m), as phi_fwd_ct;
    // warp 0 takes no part: it holds no global stores at the releasing barrier
    if (warp > 0) {
      const int tf = t - 32;
      double2* Gp = a.G + (size_t)f * a.Gfield + (size_t)k * a.ldn + g * NPC + (int)rank * NPL + b;
      const size_t mstride = (size_t)2 * a.nz * a.ldn, pstride = (size_t)a.nz * a.ldn;
      const double W = __ldg(a.wfold + g * NPC + (int)rank * NPL + b);
      auto zpos = [&](int m) {
        const int q = m / A;
        return (m % A) * G::PR + C * (q % B) + q / B;
      };
      for (int m = tf / NPL; m <= a.lmax; m += (T - 32) / NPL) {
        const double2 Z = X[b * G::SB + zpos(m)];
        const double2 Zc = X[b * G::SB + zpos(m == 0 ? 0 : N - m)];
        // F(i) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
        double2 Fi = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y - Zc.y));
        double2 Fm = make_double2(0.5 * (Z.y + Zc.y), -0.5 * (Z.x - Zc.x));
        Gp[m * mstride] = cscale(cadd(Fi, Fm), W);
        Gp[m * mstride + pstride] = cscale(csub(Fi, Fm), W);
      }
    }
    // this stage is refilled by TMA (async proxy) after the next barrier
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  if (gave_up && t == 0) {  // report, and let the copy still in flight land before leaving
    atomicExch(a.flag, 1);
    tc05::mbar_wait(&full[s], (phase >> s) & 1);
  }
  cluster_sync_all();  // no CTA leaves while another may still read its shared memory
}

constexpr int PHI3C_UNSUPPORTED = 1000;

template <int N, int CL>
int phi3c_run(const sph_plan* p, const PhiArgs& a, int nfields, cudaStream_t st) {
  if constexpr (!phi3c_ok<N, CL>()) {
    return PHI3C_UNSUPPORTED;
  } else {
    using G = P3c<N, CL>;
    if (p->nlat2 % G::NPC || !a.flag) return PHI3C_UNSUPPORTED;
    const long long ntiles = (long long)(p->nlat2 / G::NPC) * p->nz * nfields;
    if (ntiles == 0) return SPH_OK;
    if (ntiles > (1ll << 30) || (long long)N * p->nz > (1ll << 31) - 1) return PHI3C_UNSUPPORTED;
    GridMaps maps;
    const CUtensorMapSwizzle swz = G::SWB == 3 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B;
    for (int f = 0; f < nfields; ++f)
      if (!tma::grid_map(&maps.m[f], a.gin[f], p->nlat, (long long)N * p->nz, G::NPC, G::BR,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, swz))
        return PHI3C_UNSUPPORTED;
    for (int f = nfields; f < SPH_MAX_FIELDS; ++f) maps.m[f] = maps.m[0];
    auto kern = phi3c_fwd64<N, CL>;
    static DeviceOnce once;
    if (!once.run([] {
          return cudaFuncSetAttribute(phi3c_fwd64<N, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)G::SMEM) == cudaSuccess &&
                 cudaFuncSetAttribute(phi3c_fwd64<N, CL>, cudaFuncAttributePreferredSharedMemoryCarveout, 100) ==
                     cudaSuccess;
        }))
      return SPH_ECUDA;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CL;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(G::THREADS);
    cfg.dynamicSmemBytes = G::SMEM;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cfg.gridDim = dim3(CL);
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters < 1)
      return PHI3C_UNSUPPORTED;
    const long long ncl = std::min<long long>(nclusters, (ntiles + 0));
    cfg.gridDim = dim3((unsigned)(ncl * CL));
    if (cudaLaunchKernelEx(&cfg, kern, a, (int)ntiles, maps) != cudaSuccess) return SPH_ECUDA;
    return SPH_OK;
  }
}

// clusters of 2 CTAs (64-byte runs): at nphi 1536 they place on all 148 SMs
// (clusters of 4 on 132) and their barriers are cheaper, 5.2 against 7.8 ms
// for the four fields of the benchmark pair; a plan with ring pairs set by
// sph_plan_set_tiles keeps the single-CTA kernels those settings were tuned on
template <int N>
int phi3c_dispatch_n(const sph_plan* p, const PhiArgs& a, int nfields, cudaStream_t st) {
  if (p->tile_np) return PHI3C_UNSUPPORTED;  // tuned ring pairs: the kernels they were tuned on
  if (p->nlat2 % 8 == 0) return phi3c_run<N, 2>(p, a, nfields, st);
  return PHI3C_UNSUPPORTED;
}

// ring pairs per CTA: the largest of 8, 4, 2, 1 that divides nlat/2 and
// keeps NP*nphi <= PMAXC
int pairs_per_cta(const sph_plan* p) {
  if (p->tile_np) return p->tile_np;
  for (int np = 8; np > 1; np >>= 1)
    if (p->nlat2 % np == 0 && np * p->nphi <= PMAXC) return np;
  return 1;
}

template <typename K>
bool smem_attr(K fn) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) == cudaSuccess &&
         cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100) == cudaSuccess;
}

template <typename K>
int run(K kernel, const PhiArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
  if (!smem_attr(kernel)) return SPH_ECUDA;
  kernel<<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

template <int N>
int launch_fwd_n(const PhiArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
  if constexpr (N > 0) {
    switch (a.NP) {
      case 8: if constexpr (8 * N <= PMAXC) return run(phi_fwd_ct<N, 8>, a, grid, smem, st); break;
      case 4: if constexpr (4 * N <= PMAXC) return run(phi_fwd_ct<N, 4>, a, grid, smem, st); break;
      case 2: if constexpr (2 * N <= PMAXC) return run(phi_fwd_ct<N, 2>, a, grid, smem, st); break;
      case 1: return run(phi_fwd_ct<N, 1>, a, grid, smem, st);
    }
  }
  return run(phi_fwd_kernel<0>, a, grid, smem, st);
}

template <int N>
int launch_inv_n(const PhiArgs& a, dim3 grid, size_t smem, cudaStream_t st) {
  if constexpr (N > 0) {
    switch (a.NP) {
      case 8: if constexpr (8 * N <= PMAXC) return run(phi_inv_ct<N, 8>, a, grid, smem, st); break;
      case 4: if constexpr (4 * N <= PMAXC) return run(phi_inv_ct<N, 4>, a, grid, smem, st); break;
      case 2: if constexpr (2 * N <= PMAXC) return run(phi_inv_ct<N, 2>, a, grid, smem, st); break;
      case 1: return run(phi_inv_ct<N, 1>, a, grid, smem, st);
    }
  }
  return run(phi_inv_kernel<0>, a, grid, smem, st);
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
  a.kzl = p->sel_kz;
  return a;
}

}  // namespace

int launch_phi_fwd(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st) {
  if (nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  if (p->nphi > PMAXC) return SPH_EINVAL;
  PhiArgs a = make_args(p);
  for (int f = 0; f < nfields; ++f) a.gin[f] = grids[f];
  dim3 grid(p->nlat2 / a.NP, p->sel_kz ? p->sel_n : p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_FWD, st);
  if (!p->sel_kz) {  // the cluster three-step kernel walks every plane
    a.flag = p->dflag;
    int rc = PHI3C_UNSUPPORTED;
    switch (p->nphi) {
#define CASE(n) \
  case n: rc = phi3c_dispatch_n<n>(p, a, nfields, st); break;
      PHI_SIZES(CASE)
#undef CASE
    }
    if (rc != PHI3C_UNSUPPORTED) return rc;
  }
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
  dim3 grid(p->nlat2 / a.NP, p->sel_kz ? p->sel_n : p->nz, nfields);
  size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(double2);
  TimedLaunch tl(p, T_PHI_INV, st);
  if (!p->sel_kz) {  // the three-step kernel walks every plane
    int rc = PHI3D_UNSUPPORTED;
    switch (p->nphi) {
#define CASE(n) \
  case n: rc = phi3d_dispatch_n<n>(p, a, nfields, st); break;
      PHI_SIZES(CASE)
#undef CASE
    }
    if (rc != PHI3D_UNSUPPORTED) return rc;
  }
  switch (p->nphi) {
#define CASE(n) \
  case n: return launch_inv_n<n>(a, grid, smem, st);
    PHI_SIZES(CASE)
#undef CASE
    default: return launch_inv_n<0>(a, grid, smem, st);
  }
}
