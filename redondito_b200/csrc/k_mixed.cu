// k_mixed.cu -- the mixed-precision form (SPH_MIXED) of the angular transforms.
//
// * phi FFTs in fp32 (twiddles derived in FP64 on the host) between the FP64
//   grid and fp32 folded coefficients G32[field][m][parity][plane][node].
// * Legendre contractions on the 5th-generation tensor cores
//   (tcgen05.mma kind::f16, fp32 accumulation in TMEM).  Each operand x is
//   scaled by a power of two s and split as x s = hi + lo (both fp16); the
//   product uses hi*hi + hi*lo + lo*hi, which keeps about 22 significant
//   bits of each operand.  The Legendre tables are split on the host, per
//   work item scaled by a power of two, and stored as ready-made
//   shared-memory tiles (8x8 core matrices, K-major) that one bulk copy
//   moves per K step.  The data operand is split on the fly by four producer
//   warps with a per-field power-of-two scale from the data's maximum.
// * Outputs are unscaled exactly (powers of two) and written in FP64
//   (spectra) or fp32 (G32).
//
// MMA orientation: M = 128 data columns (64 planes x re/im), N = rows of one
// parity (analysis: l; synthesis: nodes), K = nodes (analysis) or l
// (synthesis), so the triangular shape of one m wastes at most 15 rows.
#include <algorithm>
#include <cmath>
#include <thread>

#include "fft_ct.cuh"
#include "tc05.cuh"

namespace {

constexpr int TK = 32;          // K tile (two k16 MMA steps)
constexpr int MCOLS = 128;      // data columns per CTA (64 planes x re/im)
constexpr int PLANES = MCOLS / 2;
constexpr int NRMAX = 256;      // largest N of one work item
constexpr int STAGES = 4;
constexpr int A_BYTES = MCOLS * TK * 2;        // 8 KB (one of hi/lo)
constexpr int B_BYTES = 2 * NRMAX * TK * 2;    // 32 KB (hi | lo)
constexpr int STAGE_BYTES = 2 * A_BYTES + B_BYTES;
constexpr int TC_SMEM = STAGES * STAGE_BYTES + 256;
constexpr int NPROD = 128;               // producer / epilogue threads (warps 0-3)
constexpr int TC_THREADS = NPROD + 32;   // + one MMA-issue warp
constexpr int UNITS = PLANES * (TK / 8) / NPROD;  // 8-element chunks per producer thread per tile

enum { ANA_S = 0, ANA_V = 1, SYN_S = 2, SYN_V = 3 };

struct TcArgs {
  const TcItem* items;
  const __half* blocks;
  const float2* G32;     // folded coefficients (analysis input)
  float2* G32w;          // (synthesis output)
  size_t G32field;
  const double2* in;     // spectra (synthesis input)
  const double2* in2;
  double2* out;          // spectra (analysis output)
  double2* out2;
  const int* mbase;
  const float* dmax;     // maxima of the data operands
  int* flag;
  int lmax, nz, nlm, ldn8;
};

// largest power of two s with mx * s < 2^14 (fp16 max 65504 leaves room for
// the rounding of hi)
__device__ __forceinline__ float pow2_scale(float mx) {
  if (!(mx > 0.f) || !(mx < 3.0e38f)) return 1.f;
  int e;
  frexpf(mx, &e);  // mx = f 2^e, f in [0.5, 1)
  return ldexpf(1.f, 14 - e);
}

__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          tc05::smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(tc05::smem_u32(mbar))
      : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                   tc05::smem_u32(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__host__ __device__ inline uint32_t tmem_cols(int nr) {
  uint32_t c = 32;
  while ((int)c < nr) c <<= 1;
  return c;
}

// Split 8 scaled values into hi/lo fp16 and store one 16-byte chunk each.
__device__ __forceinline__ void store_split8(unsigned char* Ahi, unsigned char* Alo, int row, int chunk,
                                             const float (&v)[8]) {
  __align__(16) __half h[8], l[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) tc05::split16(v[j], h[j], l[j]);
  const uint32_t off = tc05::kmaj_off(row, chunk * 8, MCOLS);
  *reinterpret_cast<uint4*>(Ahi + off) = *reinterpret_cast<const uint4*>(h);
  *reinterpret_cast<uint4*>(Alo + off) = *reinterpret_cast<const uint4*>(l);
}

// forms of a complex data value: v, -v, i v, -i v
enum { F_PLAIN = 0, F_NEG = 1, F_MULI = 2, F_MULMI = 3 };
__device__ __forceinline__ float2 form_rt(float2 v, int f) {
  switch (f) {
    case F_NEG: return make_float2(-v.x, -v.y);
    case F_MULI: return make_float2(-v.y, v.x);
    case F_MULMI: return make_float2(v.y, -v.x);
    default: return v;
  }
}

// One CTA: one work item (blockIdx.y) x 64 planes (blockIdx.x).
template <int MODE>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm(TcArgs a) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* fullA = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);  // producers arrived
  uint64_t* fullB = fullA + STAGES;                                             // table copy landed
  uint64_t* empty = fullB + STAGES;                                             // MMAs of the stage done
  uint64_t* done = empty + STAGES;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
  int* abort_flag = reinterpret_cast<int*>(tslot + 1);

  constexpr bool analysis = (MODE == ANA_S || MODE == ANA_V);
  const TcItem it = a.items[blockIdx.y];
  const int k0 = blockIdx.x * PLANES;  // first plane
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // TMEM: the hi*lo + lo*hi accumulator at column 0 and one or two hi*hi
  // accumulators (alternate K tiles) at columns xoff, 2*xoff.  Keeping them
  // apart shortens the chains of fp32 roundings of each running sum.
  const uint32_t xoff = tmem_cols(it.nr);
  const int nmain = xoff <= 128 ? 2 : 1;
  const uint32_t ncols = tmem_cols((nmain + 1) * (int)xoff);

  // once any CTA of the plan has given up a wait, the rest do no work
  if (tid == 0) *abort_flag = *(volatile int*)a.flag;
  __syncthreads();
  if (*abort_flag) return;
  __syncthreads();

  if (warp == 0) tc05::tmem_alloc(tslot, ncols);
  if (tid == 32) {
    for (int s = 0; s < STAGES; ++s) {
      tc05::mbar_init(&fullA[s], NPROD);
      tc05::mbar_init(&fullB[s], 1);
      tc05::mbar_init(&empty[s], 1);
    }
    tc05::mbar_init(done, 1);
    *abort_flag = 0;
    tc05::mbar_fence_init();
  }
  tc05::fence_before();
  __syncthreads();
  tc05::fence_after();
  const uint32_t tbase = *tslot;

  float dscale;
  if (MODE == ANA_S) dscale = pow2_scale(a.dmax[0]);
  else if (MODE == ANA_V) dscale = pow2_scale(fmaxf(a.dmax[1], a.dmax[2]));
  else dscale = pow2_scale(a.dmax[3]);

  const uint32_t bbytes = (uint32_t)it.nr * TK * 2 * 2;
  const size_t base_lm = (size_t)a.mbase[it.m] - it.m;
  int issued = 0;  // table copies issued (thread 0)

  if (warp < 4) {
    // ------------------------------------------------------------ producers
    for (int kt = 0; kt < it.nk; ++kt) {
      const int s = kt % STAGES, use = kt / STAGES;
      if (use > 0 && !tc05::mbar_wait(&empty[s], (use - 1) & 1)) {
        atomicExch(a.flag, 1);
        *abort_flag = 1;
        break;
      }
      if (*abort_flag) break;
      unsigned char* Ahi = smem + s * STAGE_BYTES;
      unsigned char* Alo = Ahi + A_BYTES;
      unsigned char* Bs = Alo + A_BYTES;
      if (tid == 0) {
        mbar_arrive_tx(&fullB[s], bbytes);
        bulk_copy(Bs, a.blocks + it.boff + (size_t)kt * 2 * it.nr * TK, bbytes, &fullB[s]);
        issued = kt + 1;
      }
      // A tile: 64 planes x 4 chunks of 8 K values; the chunk index runs
      // fastest so that four lanes read 256 contiguous bytes of one plane
      float re[UNITS][8], im[UNITS][8];
#pragma unroll
      for (int u = 0; u < UNITS; ++u) {
        const int unit = tid + NPROD * u, ch = unit & 3, pl = unit >> 2, k = k0 + pl;
#pragma unroll
        for (int j = 0; j < 8; ++j) re[u][j] = im[u][j] = 0.f;
        if (k >= a.nz) continue;
        if (analysis) {
          int f = F_PLAIN, fold = it.par, node0, field = 0;
          if (MODE == ANA_S) {
            node0 = kt * TK + ch * 8;
          } else {
            // S: [dP . Vt_(1-p) ; mPs . (-i Vp_p)]   T: [dP . (-Vp_(1-p)) ; mPs . (-i Vt_p)]
            const bool first = kt < it.nk1;
            node0 = (first ? kt : kt - it.nk1) * TK + ch * 8;
            fold = first ? 1 - it.par : it.par;
            field = first ? (it.out ? 2 : 1) : (it.out ? 1 : 2);
            f = first ? (it.out ? F_NEG : F_PLAIN) : F_MULMI;
          }
          if (node0 < a.ldn8) {
            const float4* r4 = reinterpret_cast<const float4*>(
                a.G32 + (size_t)field * a.G32field + (((size_t)it.m * 2 + fold) * a.nz + k) * a.ldn8 + node0);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const float4 q = __ldg(r4 + j);
              const float2 v0 = form_rt(make_float2(q.x, q.y), f), v1 = form_rt(make_float2(q.z, q.w), f);
              re[u][2 * j] = v0.x * dscale;
              im[u][2 * j] = v0.y * dscale;
              re[u][2 * j + 1] = v1.x * dscale;
              im[u][2 * j + 1] = v1.y * dscale;
            }
          }
        } else {
          // K = l of one parity.  Vector: Vt_q = [dP . S ; mPs . (i T)], Vp_q = [dP . (-T) ; mPs . (i S)]
          int f = F_PLAIN, par = it.par, q0;
          const double2* spec = a.in;
          if (MODE == SYN_S) {
            q0 = kt * TK + ch * 8;
          } else {
            const bool first = kt < it.nk1;
            q0 = (first ? kt : kt - it.nk1) * TK + ch * 8;
            par = first ? 1 - it.par : it.par;
            if (first) {
              spec = it.out ? a.in2 : a.in;
              f = it.out ? F_NEG : F_PLAIN;
            } else {
              spec = it.out ? a.in : a.in2;
              f = F_MULI;
            }
          }
          const double2* col = spec + (size_t)k * a.nlm + base_lm;
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int l = it.m + par + 2 * (q0 + j);
            if (l <= a.lmax && (MODE == SYN_S || l > 0)) {
              const double2 d = __ldg(col + l);
              const float2 v =
                  form_rt(make_float2((float)(d.x * (double)dscale), (float)(d.y * (double)dscale)), f);
              re[u][j] = v.x;
              im[u][j] = v.y;
            }
          }
        }
      }
#pragma unroll
      for (int u = 0; u < UNITS; ++u) {
        const int unit = tid + NPROD * u, ch = unit & 3, pl = unit >> 2;
        store_split8(Ahi, Alo, 2 * pl, ch, re[u]);
        store_split8(Ahi, Alo, 2 * pl + 1, ch, im[u]);
      }
      fence_proxy_async();
      tc05::mbar_arrive(&fullA[s]);
    }
  } else if (warp == 4 && lane == 0) {
    // ------------------------------------------------------------ MMA issue
    const uint32_t idesc = tc05::idesc_f16(MCOLS, it.nr);
    const uint32_t lboA = (MCOLS / 8) * 128, lboB = (uint32_t)(it.nr / 8) * 128;
    for (int kt = 0; kt < it.nk; ++kt) {
      const int s = kt % STAGES, use = kt / STAGES;
      if (!tc05::mbar_wait(&fullA[s], use & 1) || !tc05::mbar_wait(&fullB[s], use & 1)) {
        atomicExch(a.flag, 1);
        *abort_flag = 1;
        break;
      }
      tc05::fence_after();
      unsigned char* Ahi = smem + s * STAGE_BYTES;
      unsigned char* Alo = Ahi + A_BYTES;
      unsigned char* Bhi = Alo + A_BYTES;
      unsigned char* Blo = Bhi + (size_t)it.nr * TK * 2;
#pragma unroll
      for (int j = 0; j < TK / 16; ++j) {
        const uint64_t ah = tc05::smem_desc(Ahi + j * 2 * lboA, lboA, 128);
        const uint64_t al = tc05::smem_desc(Alo + j * 2 * lboA, lboA, 128);
        const uint64_t bh = tc05::smem_desc(Bhi + j * 2 * lboB, lboB, 128);
        const uint64_t bl = tc05::smem_desc(Blo + j * 2 * lboB, lboB, 128);
        const int mi = 1 + (kt & (nmain - 1));
        tc05::mma_f16(tbase + mi * xoff, ah, bh, idesc, (kt >= nmain || j) ? 1u : 0u);
        tc05::mma_f16(tbase, ah, bl, idesc, (kt | j) ? 1u : 0u);
        tc05::mma_f16(tbase, al, bh, idesc, 1u);
      }
      tc05::commit(&empty[s]);
    }
    if (it.nk > 0) tc05::commit(done);
  }

  // ------------------------------------------------------------ epilogue
  if (warp < 4) {
    bool ok = it.nk == 0 || (!*abort_flag && tc05::mbar_wait(done, 0));
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) atomicExch(a.flag, 1);
    tc05::fence_after();
    if (ok) {
      const double inv = 1.0 / ((double)it.tscale * (double)dscale);
      const int n = 32 * warp + lane;  // data column: plane k0 + n/2, component n&1
      const int k = k0 + (n >> 1);
      for (int c = 0; c < it.nr; c += 16) {
        float v[16], x[16];
        if (it.nk > 0) {
          const uint32_t ta = tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)c;
          tc05::tmem_ld16(ta + xoff, v);
          tc05::tmem_ld16(ta, x);
          if (nmain == 2 && it.nk > 1) {
            float v2[16];
            tc05::tmem_ld16(ta + 2 * xoff, v2);
#pragma unroll
            for (int j = 0; j < 16; ++j) x[j] += v2[j];
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = x[j] = 0.f;  // empty fold: written as zeros
        }
        float w[16], y[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          w[j] = __shfl_xor_sync(0xffffffffu, v[j], 1);
          y[j] = __shfl_xor_sync(0xffffffffu, x[j], 1);
        }
        if ((lane & 1) || k >= a.nz) continue;
        if (analysis) {
          double2* out = (MODE == ANA_V && it.out) ? a.out2 : a.out;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int q = c + j;
            if (q >= it.nvalid) break;
            const int l = it.m + it.par + 2 * (it.r0 + q);
            double f = inv;
            if (MODE == ANA_V) f = l ? inv / ((double)l * (double)(l + 1)) : 0.0;
            out[(size_t)k * a.nlm + base_lm + l] =
                make_double2(((double)v[j] + (double)x[j]) * f, it.m == 0 ? 0.0 : ((double)w[j] + (double)y[j]) * f);
          }
        } else {
          const int field = (MODE == SYN_V) ? 1 + it.out : 0;
          float2* G = a.G32w + (size_t)field * a.G32field + (((size_t)it.m * 2 + it.par) * a.nz + k) * a.ldn8;
          const float finv = (float)inv;
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int i = it.r0 + c + j;
            if (i < a.ldn8) G[i] = make_float2((v[j] + x[j]) * finv, (w[j] + y[j]) * finv);
          }
        }
      }
    }
    // after a bounded wait gave up, table copies may still be in flight
    if (tid == 0 && *abort_flag)
      for (int kt = max(0, issued - STAGES); kt < issued; ++kt)
        tc05::mbar_wait(&fullB[kt % STAGES], (kt / STAGES) & 1, 100000000ull);
  }
  tc05::fence_before();
  __syncthreads();
  if (warp == 0) tc05::tmem_free(tbase, ncols);
}

// ---------------------------------------------------------------- fp32 phi FFTs
constexpr int PTHREADS = 512;
constexpr int PMAXC = 12288;  // NP*nphi complex values per CTA (two CTAs per SM)

__host__ __device__ inline int seq_stride(int nphi) {
  int s = nphi + (nphi + 7) / 8;
  return s | 1;
}

struct Phi32Args {
  const double* gin[SPH_MAX_FIELDS];
  double* gout[SPH_MAX_FIELDS];
  float2* G32;
  const float2* G32c;
  size_t G32field;
  float* dmax;  // per-field maxima of |G32| (forward)
  int nlat, ldn8, nz, lmax, NP;
  const double* wfold;
  const float2* twp;
};

__device__ __forceinline__ void atomic_max_pos(float* addr, float v) {
  atomicMax(reinterpret_cast<unsigned int*>(addr), __float_as_uint(v));
}

template <int N, int NP>
__global__ void __launch_bounds__(PTHREADS, 2) phi_fwd32(Phi32Args a) {
  extern __shared__ float2 sf[];
  constexpr int Q = 2 * NP, JSTEP = PTHREADS / Q;
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x;
  const double* plane = a.gin[f] + (size_t)k * N * nlat;
  const ct::Geo<N, 1, true> g{NP, seq_stride(N), 1};
  float* smf = reinterpret_cast<float*>(sf);
  {
    // ring slot q: NP northern rings (real part) and their mirrors (imaginary part)
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
        if (u0 + u < NJ && j < N) smf[2 * g.addr(b, j) + half] = (float)v[u];
      }
    }
  }
  __syncthreads();
  ct::dif<float2, N, N>(sf, g, a.twp, -1);

  float2* G = a.G32 + (size_t)f * a.G32field + (size_t)k * a.ldn8 + p0;
  const size_t mstride = (size_t)2 * a.nz * a.ldn8, pstride = (size_t)a.nz * a.ldn8;
  const int b = tid % NP;
  const float W = (float)__ldg(a.wfold + p0 + b);
  float mx = 0.f;
  for (int m = tid / NP; m <= a.lmax; m += PTHREADS / NP) {
    const float2 Z = sf[g.addr(b, ct::rev_pos<N>(m))];
    const float2 Zc = sf[g.addr(b, ct::rev_pos<N>(m == 0 ? 0 : N - m))];
    // F(ring) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
    const float2 Fi = make_float2(0.5f * (Z.x + Zc.x), 0.5f * (Z.y - Zc.y));
    const float2 Fm = make_float2(0.5f * (Z.y + Zc.y), -0.5f * (Z.x - Zc.x));
    const float2 ge = make_float2((Fi.x + Fm.x) * W, (Fi.y + Fm.y) * W);
    const float2 go = make_float2((Fi.x - Fm.x) * W, (Fi.y - Fm.y) * W);
    G[m * mstride + b] = ge;
    G[m * mstride + pstride + b] = go;
    mx = fmaxf(mx, fmaxf(fmaxf(fabsf(ge.x), fabsf(ge.y)), fmaxf(fabsf(go.x), fabsf(go.y))));
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((tid & 31) == 0 && mx > 0.f) atomic_max_pos(a.dmax + f, mx);
}

template <int N, int NP>
__global__ void __launch_bounds__(PTHREADS, 2) phi_inv32(Phi32Args a) {
  extern __shared__ float2 sf[];
  constexpr int Q = 2 * NP, JSTEP = PTHREADS / Q;
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x;
  const ct::Geo<N, 1, true> g{NP, seq_stride(N), 1};
  const int M = a.lmax + 1;
  for (int i = tid; i < NP * seq_stride(N); i += PTHREADS) sf[i] = make_float2(0.f, 0.f);
  __syncthreads();
  {
    const float2* G = a.G32c + (size_t)f * a.G32field + (size_t)k * a.ldn8 + p0;
    const size_t mstride = (size_t)2 * a.nz * a.ldn8, pstride = (size_t)a.nz * a.ldn8;
    const int b = tid % NP;
    for (int m = tid / NP; m < M; m += PTHREADS / NP) {
      const float2 se = __ldg(G + m * mstride + b), so = __ldg(G + m * mstride + pstride + b);
      const float2 Fi = make_float2(se.x + so.x, se.y + so.y), Fm = make_float2(se.x - so.x, se.y - so.y);
      if (m == 0) {
        sf[g.addr(b, 0)] = make_float2(Fi.x, Fm.x);
      } else {
        sf[g.addr(b, ct::rev_pos<N>(m))] = make_float2(Fi.x - Fm.y, Fi.y + Fm.x);
        sf[g.addr(b, ct::rev_pos<N>(N - m))] = make_float2(Fi.x + Fm.y, -Fi.y + Fm.x);
      }
    }
  }
  __syncthreads();
  ct::dit<float2, N, N>(sf, g, a.twp, +1);
  double* plane = a.gout[f] + (size_t)k * N * nlat;
  const float* smf = reinterpret_cast<const float*>(sf);
  const int q = tid % Q, j0 = tid / Q;
  const int b = q < NP ? q : 2 * NP - 1 - q;
  const int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
  const int half = q < NP ? 0 : 1;
  for (int j = j0; j < N; j += JSTEP) plane[(size_t)j * nlat + ring] = (double)smf[2 * g.addr(b, j) + half];
}

// maximum of |re|, |im| over one or two spectral fields (synthesis data scale)
__global__ void spec_max_kernel(const double2* a, const double2* b, size_t n, float* out) {
  float mx = 0.f;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double2 v = a[q];
    mx = fmaxf(mx, (float)fmax(fabs(v.x), fabs(v.y)));
    if (b) {
      v = b[q];
      mx = fmaxf(mx, (float)fmax(fabs(v.x), fabs(v.y)));
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.f) atomic_max_pos(out, mx);
}

// ---------------------------------------------------------------- host tables
// Builds one work set: items (heaviest first) and their fp16 hi/lo table
// blocks.  value(it, row, kt, kk) is the FP64 table entry of MMA row `row`,
// K element kt*32+kk.  An item with out = 1 right after its out = 0 twin
// shares the twin's blocks and scale.
template <typename ItemsFn, typename ValFn>
int build_set(TcSet& set, ItemsFn make_items, ValFn value) {
  std::vector<TcItem> raw;
  make_items(raw);
  auto is_twin = [&](int x) { return x > 0 && raw[x].out == 1 && raw[x - 1].out == 0; };
  std::vector<int> heads;
  for (int x = 0; x < (int)raw.size(); ++x)
    if (!is_twin(x)) heads.push_back(x);
  std::stable_sort(heads.begin(), heads.end(), [&](int u, int v) {
    return (long long)raw[u].nr * std::max(1, raw[u].nk) > (long long)raw[v].nr * std::max(1, raw[v].nk);
  });
  std::vector<TcItem> items;
  std::vector<int> own;  // items that own their blocks
  size_t total = 0;
  for (int h : heads) {
    TcItem it = raw[h];
    it.boff = (long long)total;
    total += (size_t)it.nk * 2 * it.nr * TK;
    own.push_back((int)items.size());
    items.push_back(it);
    if (h + 1 < (int)raw.size() && is_twin(h + 1)) {
      TcItem tw = raw[h + 1];
      tw.boff = it.boff;
      items.push_back(tw);
    }
  }
  std::vector<__half> hb(total);
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (int t = 0; t < nth; ++t)
    th.emplace_back([&, t]() {
      std::vector<double> tile;
      for (size_t x = t; x < own.size(); x += nth) {
        TcItem& it = items[own[x]];
        double mx = 0.0;
        tile.assign((size_t)it.nk * it.nr * TK, 0.0);
        for (int kt = 0; kt < it.nk; ++kt)
          for (int r = 0; r < it.nr; ++r)
            for (int kk = 0; kk < TK; ++kk) {
              const double v = r < it.nvalid ? value(it, r, kt, kk) : 0.0;
              tile[((size_t)kt * it.nr + r) * TK + kk] = v;
              mx = std::max(mx, std::fabs(v));
            }
        int e = 0;
        if (mx > 0) std::frexp(mx, &e);
        const double s = mx > 0 ? std::ldexp(1.0, 14 - e) : 1.0;
        it.tscale = (float)s;
        for (int kt = 0; kt < it.nk; ++kt) {
          __half* hi = hb.data() + it.boff + (size_t)kt * 2 * it.nr * TK;
          __half* lo = hi + (size_t)it.nr * TK;
          for (int r = 0; r < it.nr; ++r)
            for (int kk = 0; kk < TK; ++kk) {
              const double v = tile[((size_t)kt * it.nr + r) * TK + kk] * s;
              const __half h = __double2half(v);
              const __half l = __double2half(v - (double)__half2float(h));
              const uint32_t off = tc05::kmaj_off(r, kk, it.nr) / 2;
              hi[off] = h;
              lo[off] = l;
            }
        }
      }
    });
  for (auto& x : th) x.join();
  for (size_t x = 1; x < items.size(); ++x)
    if (items[x].out == 1 && items[x].boff == items[x - 1].boff) items[x].tscale = items[x - 1].tscale;
  set.nitems = (int)items.size();
  set.nhalves = total;
  if (cudaMalloc((void**)&set.items, std::max<size_t>(1, items.size()) * sizeof(TcItem)) != cudaSuccess)
    return SPH_ENOMEM;
  if (cudaMalloc((void**)&set.blocks, std::max<size_t>(1, total) * sizeof(__half)) != cudaSuccess)
    return SPH_ENOMEM;
  if (!items.empty() &&
      cudaMemcpy(set.items, items.data(), items.size() * sizeof(TcItem), cudaMemcpyHostToDevice) != cudaSuccess)
    return SPH_ECUDA;
  if (total && cudaMemcpy(set.blocks, hb.data(), total * sizeof(__half), cudaMemcpyHostToDevice) != cudaSuccess)
    return SPH_ECUDA;
  return SPH_OK;
}

inline int round16(int x) { return (x + 15) & ~15; }

#define PHI32_SIZES(X) X(12) X(24) X(48) X(96) X(192) X(384) X(768) X(1536) X(3072) X(6144)

}  // namespace

bool mixed_nphi_ok(int nphi) {
  switch (nphi) {
#define CASE(n) case n:
    PHI32_SIZES(CASE)
#undef CASE
    return true;
  }
  return false;
}

int mixed_setup(sph_plan* p, const std::vector<double>& hP, const std::vector<double>& hdP,
                const std::vector<double>& hmPs) {
  const int lmax = p->lmax, ldn = p->ldn, n2 = p->nlat2;
  p->ldn8 = (n2 + 7) & ~7;
  p->G32field = (size_t)(lmax + 1) * 2 * p->nz * p->ldn8;
  if (p->G32field * sizeof(float2) > p->Gfield * sizeof(double2)) return SPH_EINVAL;
  const int nkn = (p->ldn8 + TK - 1) / TK;  // K tiles over the nodes
  // synthesis node blocks: as few as keep N <= 256, of equal size
  const int nblk = (n2 + NRMAX - 1) / NRMAX;
  const int iblk = round16((n2 + nblk - 1) / nblk);
  auto lm = [&](int l, int m) { return (size_t)p->mbase[m] + (l - m); };
  auto rows = [&](int m, int par) { return m + par > lmax ? 0 : (lmax - m - par) / 2 + 1; };

  // analysis: rows = l of one parity, K = nodes (vector: [dP nodes | mPs nodes])
  auto ana_items = [&](bool vec) {
    return [&, vec](std::vector<TcItem>& v) {
      for (int m = 0; m <= lmax; ++m)
        for (int par = 0; par < 2; ++par) {
          const int L = rows(m, par);
          for (int r0 = 0; r0 < L; r0 += NRMAX) {
            TcItem it = {};
            it.m = m;
            it.par = par;
            it.r0 = r0;
            it.nvalid = std::min(NRMAX, L - r0);
            it.nr = round16(it.nvalid);
            it.nk = vec ? 2 * nkn : nkn;
            it.nk1 = nkn;
            v.push_back(it);
            if (vec) {
              it.out = 1;
              v.push_back(it);
            }
          }
        }
    };
  };
  auto ana_val = [&](bool vec) {
    return [&, vec](const TcItem& it, int r, int kt, int kk) -> double {
      const int l = it.m + it.par + 2 * (it.r0 + r);
      const bool second = vec && kt >= it.nk1;
      const int i = (second ? kt - it.nk1 : kt) * TK + kk;
      if (l > lmax || i >= n2) return 0.0;
      const std::vector<double>& T = vec ? (second ? hmPs : hdP) : hP;
      return T[lm(l, it.m) * ldn + i];
    };
  };
  // synthesis: rows = nodes, K = l of one parity (vector: [l of 1-q via dP | l of q via mPs])
  auto syn_items = [&](bool vec) {
    return [&, vec](std::vector<TcItem>& v) {
      for (int m = 0; m <= lmax; ++m)
        for (int q = 0; q < 2; ++q) {
          const int Lq = rows(m, q), L1 = rows(m, 1 - q);
          for (int i0 = 0; i0 < n2; i0 += iblk) {
            TcItem it = {};
            it.m = m;
            it.par = q;
            it.r0 = i0;
            it.nvalid = std::min(iblk, n2 - i0);
            it.nr = round16(it.nvalid);
            if (vec) {
              it.nk1 = (L1 + TK - 1) / TK;
              it.nk = it.nk1 + (Lq + TK - 1) / TK;
            } else {
              it.nk = (Lq + TK - 1) / TK;  // 0: the fold is written as zeros
              it.nk1 = it.nk;
            }
            v.push_back(it);
            if (vec) {
              it.out = 1;
              v.push_back(it);
            }
          }
        }
    };
  };
  auto syn_val = [&](bool vec) {
    return [&, vec](const TcItem& it, int r, int kt, int kk) -> double {
      const int i = it.r0 + r;
      if (i >= n2) return 0.0;
      if (!vec) {
        const int l = it.m + it.par + 2 * (kt * TK + kk);
        return l > lmax ? 0.0 : hP[lm(l, it.m) * ldn + i];
      }
      const bool second = kt >= it.nk1;
      const int par = second ? it.par : 1 - it.par;
      const int l = it.m + par + 2 * ((second ? kt - it.nk1 : kt) * TK + kk);
      if (l > lmax || l == 0) return 0.0;
      return (second ? hmPs : hdP)[lm(l, it.m) * ldn + i];
    };
  };

  int rc = build_set(p->tcAS, ana_items(false), ana_val(false));
  if (rc == SPH_OK) rc = build_set(p->tcAV, ana_items(true), ana_val(true));
  if (rc == SPH_OK) rc = build_set(p->tcSS, syn_items(false), syn_val(false));
  if (rc == SPH_OK) rc = build_set(p->tcSV, syn_items(true), syn_val(true));
  if (rc == SPH_OK && cudaMalloc((void**)&p->dmax, 4 * sizeof(float)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMalloc((void**)&p->dflag, sizeof(int)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(p->dflag, 0, sizeof(int)) != cudaSuccess) rc = SPH_ECUDA;
  if (rc == SPH_OK && cudaMemset(p->dmax, 0, 4 * sizeof(float)) != cudaSuccess) rc = SPH_ECUDA;
  return rc;
}

void mixed_free(sph_plan* p) {
  for (TcSet* s : {&p->tcAS, &p->tcAV, &p->tcSS, &p->tcSV}) {
    if (s->items) cudaFree(s->items);
    if (s->blocks) cudaFree(s->blocks);
    s->items = nullptr;
    s->blocks = nullptr;
  }
  if (p->dmax) cudaFree(p->dmax);
  if (p->dflag) cudaFree(p->dflag);
  p->dmax = nullptr;
  p->dflag = nullptr;
}

int mixed_status(const sph_plan* p) {
  int f = 0;
  if (p->dflag && cudaMemcpy(&f, p->dflag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SPH_ECUDA;
  return f ? SPH_ETIMEDOUT : SPH_OK;
}

namespace {

TcArgs tc_args(const sph_plan* p) {
  TcArgs a = {};
  a.G32 = reinterpret_cast<const float2*>(p->G);
  a.G32w = reinterpret_cast<float2*>(p->G);
  a.G32field = p->G32field;
  a.mbase = p->d_mbase;
  a.dmax = p->dmax;
  a.flag = p->dflag;
  a.lmax = p->lmax;
  a.nz = p->nz;
  a.nlm = p->nlm;
  a.ldn8 = p->ldn8;
  return a;
}

template <int MODE>
int run_tc(const TcSet& set, TcArgs a, int nz, cudaStream_t st) {
  static const bool attr_ok =
      cudaFuncSetAttribute(tc_gemm<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM) == cudaSuccess;
  if (!attr_ok) return SPH_ECUDA;
  if (set.nitems == 0) return SPH_OK;
  if (set.nitems > 65535) return SPH_EINVAL;
  a.items = set.items;
  a.blocks = set.blocks;
  dim3 grid((nz + PLANES - 1) / PLANES, set.nitems);
  tc_gemm<MODE><<<grid, TC_THREADS, TC_SMEM, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int phi_pairs(const sph_plan* p) {
  for (int np = 8; np > 1; np >>= 1)
    if (p->nlat2 % np == 0 && np * p->nphi <= PMAXC) return np;
  return 1;
}

template <typename K>
int run_phi(K kernel, const Phi32Args& a, dim3 grid, size_t smem, cudaStream_t st) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess ||
      cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
    return SPH_ECUDA;
  kernel<<<grid, PTHREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

template <int N, bool FWD>
int phi32_n(const Phi32Args& a, dim3 grid, size_t smem, cudaStream_t st) {
  switch (a.NP) {
    case 8:
      if constexpr (8 * N <= PMAXC) return run_phi(FWD ? phi_fwd32<N, 8> : phi_inv32<N, 8>, a, grid, smem, st);
      break;
    case 4:
      if constexpr (4 * N <= PMAXC) return run_phi(FWD ? phi_fwd32<N, 4> : phi_inv32<N, 4>, a, grid, smem, st);
      break;
    case 2:
      if constexpr (2 * N <= PMAXC) return run_phi(FWD ? phi_fwd32<N, 2> : phi_inv32<N, 2>, a, grid, smem, st);
      break;
    case 1: return run_phi(FWD ? phi_fwd32<N, 1> : phi_inv32<N, 1>, a, grid, smem, st);
  }
  return SPH_EINVAL;
}

template <bool FWD>
int phi32_dispatch(const sph_plan* p, const Phi32Args& a, dim3 grid, size_t smem, cudaStream_t st) {
  switch (p->nphi) {
#define CASE(n) \
  case n: return phi32_n<n, FWD>(a, grid, smem, st);
    PHI32_SIZES(CASE)
#undef CASE
  }
  return SPH_EINVAL;
}

Phi32Args phi32_args(const sph_plan* p) {
  Phi32Args a = {};
  a.G32 = reinterpret_cast<float2*>(p->G);
  a.G32c = reinterpret_cast<const float2*>(p->G);
  a.G32field = p->G32field;
  a.dmax = p->dmax;
  a.nlat = p->nlat;
  a.ldn8 = p->ldn8;
  a.nz = p->nz;
  a.lmax = p->lmax;
  a.NP = phi_pairs(p);
  a.wfold = p->wfold;
  a.twp = p->fphi.twpf;
  return a;
}

}  // namespace

int launch_phi_fwd32(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st) {
  Phi32Args a = phi32_args(p);
  for (int f = 0; f < nfields; ++f) a.gin[f] = grids[f];
  SPH_CUDA_OK(cudaMemsetAsync(p->dmax, 0, 3 * sizeof(float), st));  // field f -> maximum slot f
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  const size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(float2);
  TimedLaunch tl(p, T_PHI_FWD, st);
  return phi32_dispatch<true>(p, a, grid, smem, st);
}

int launch_phi_inv32(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st) {
  Phi32Args a = phi32_args(p);
  for (int f = 0; f < nfields; ++f) a.gout[f] = grids[f];
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  const size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(float2);
  TimedLaunch tl(p, T_PHI_INV, st);
  return phi32_dispatch<false>(p, a, grid, smem, st);
}

int launch_tc_analysis(const sph_plan* p, int vector, double2* out, double2* out2, cudaStream_t st) {
  TcArgs a = tc_args(p);
  a.out = out;
  a.out2 = out2;
  TimedLaunch tl(p, vector ? T_VEC_ANA : T_LEG_ANA, st);
  return vector ? run_tc<ANA_V>(p->tcAV, a, p->nz, st) : run_tc<ANA_S>(p->tcAS, a, p->nz, st);
}

int launch_tc_synthesis(const sph_plan* p, int vector, const double2* in, const double2* in2, cudaStream_t st) {
  TcArgs a = tc_args(p);
  a.in = in;
  a.in2 = in2;
  {
    TimedLaunch tl(p, T_OPS, st);
    SPH_CUDA_OK(cudaMemsetAsync(p->dmax + 3, 0, sizeof(float), st));
    const size_t n = spec_elems(p);
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 8);
    spec_max_kernel<<<blocks, 256, 0, st>>>(in, vector ? in2 : nullptr, n, p->dmax + 3);
    SPH_LAUNCH_OK();
  }
  TimedLaunch tl(p, vector ? T_VEC_SYN : T_LEG_SYN, st);
  return vector ? run_tc<SYN_V>(p->tcSV, a, p->nz, st) : run_tc<SYN_S>(p->tcSS, a, p->nz, st);
}
