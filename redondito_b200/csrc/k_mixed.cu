// k_mixed.cu -- the mixed-precision form (SPH_MIXED) of the angular transforms.
//
// * phi FFTs in fp32 (twiddles derived in FP64 on the host).
// * Legendre contractions on the 5th-generation tensor cores
//   (tcgen05.mma kind::f16 with bf16 operands, fp32 accumulation in TMEM).
//   Every operand value x is split into three bf16 pieces x = hi + mid + lo
//   (8 significant bits each, so an fp32 value is represented exactly and
//   no scaling is needed: bf16 has the fp32 exponent range).  A product
//   keeps the six piece products of order <= 2 (hi.hi, hi.mid, mid.hi,
//   hi.lo, mid.mid, lo.hi), about 24 bits.  The tensor cores align the
//   addends of one MMA to the largest exponent and truncate below it, so
//   hi.hi (16-bit products, kept exactly against the running sum) and the
//   five small products accumulate in two separate TMEM column ranges; the
//   epilogue adds them in FP64.
// * The data operand is split ONCE, by the kernel that produces it, into
//   ready-made shared-memory tiles: 3 pieces x [128 rows = 64 planes x
//   (re, im)] x [32 K] bf16 in the no-swizzle K-major core-matrix layout,
//   24 KB per tile, one bulk copy per K step.  The phi FFT writes the
//   analysis tiles (K = Gauss nodes); spec_to_tiles writes the synthesis
//   tiles (K = degrees l of one parity).  The Legendre tables are split on
//   the host into the same layout.
// * One persistent CTA per SM walks its work units (item x 64 planes).  For
//   scalar units TMEM holds two accumulator sets, so the epilogue of a unit
//   overlaps the main loop of the next.  Vector transforms keep the dP and
//   mPs parts in separate accumulators (128-column MMAs: the four
//   accumulators fill TMEM, one set) and apply the +-i factors in the
//   epilogue.
//
// Warp roles of the tensor-core kernel: 0 bulk copies (one lane), 1 TMEM
// allocation and MMA issue (one lane), 2-9 epilogue (TMEM lane quarters
// 2, 3, 0, 1, twice; the two warps of a quarter take alternate 16-column
// chunks).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>

#include "fft3.cuh"
#include "fft_ct.cuh"
#include "tc05.cuh"
#include "tma.cuh"

namespace {

constexpr int TK = 32;                              // K tile (two k16 MMA steps)
constexpr int MCOLS = 128;                          // data columns per unit (64 planes x re/im)
constexpr int PLANES = MCOLS / 2;
constexpr int NPIECE = 3;                           // bf16 pieces per value
constexpr int PIECE_HALVES = MCOLS * TK;            // 4096 (8 KB)
constexpr int TILE_HALVES = NPIECE * PIECE_HALVES;  // one data tile (24 KB)
constexpr int NR_S = 128;                           // MMA N of scalar items
constexpr int NR_V = 128;                           // MMA N of vector items (two parts)
constexpr int A_BYTES = TILE_HALVES * 2;
constexpr int B_BYTES = NPIECE * NR_S * TK * 2;     // 24 KB
constexpr int STAGES = 4;
constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
constexpr int STG_WORDS = 32 * 17;                  // epilogue staging per warp (doubles)
constexpr int OFF_STG = STAGES * STAGE_BYTES;
constexpr int NEPI_WARPS = 8;                       // epilogue warps: two per TMEM lane quarter
constexpr int OFF_BAR = OFF_STG + NEPI_WARPS * STG_WORDS * 8;
constexpr int NBARS = 2 * STAGES + 2 + 2 + 1;
constexpr int TC_SMEM = OFF_BAR + NBARS * 8 + 16;
constexpr int TC_THREADS = (2 + NEPI_WARPS) * 32;
constexpr int NEPI = NEPI_WARPS * 32;                // epilogue threads
constexpr int TMEM_COLS = 512;                      // two accumulator sets of 256 columns

enum { ANA_S = 0, ANA_V = 1, SYN_S = 2, SYN_V = 3 };

struct TcArgs {
  const TcItem* items;
  const __nv_bfloat16* blocks;  // table tiles
  const __nv_bfloat16* tiles;   // data tiles (analysis or synthesis layout)
  size_t tfield;                // halves per field of the synthesis data tiles
  const long long* toff;        // synthesis: [m][parity] first tile of the block
  float2* G32w;                 // synthesis output (folded coefficients)
  size_t G32field;
  double2* out;                 // analysis output (spectra)
  double2* out2;
  const int* mbase;
  int* flag;
  int lmax, nz, nlm, ldn8, nkn, ncb, nunits;
};

__host__ __device__ inline int rows_of(int lmax, int m, int par) {
  return m + par > lmax ? 0 : (lmax - m - par) / 2 + 1;
}
__host__ __device__ inline int ntiles_of(int lmax, int m, int par) { return (rows_of(lmax, m, par) + TK - 1) / TK; }

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

// x (fp32) = hi + mid + lo, each bf16 (round to nearest); exact for finite
// x whose pieces stay in the bf16 normal range (|x| > ~2^-110).
__device__ __forceinline__ void split3(float x, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
  h = __float2bfloat16_rn(x);
  const float r = x - __bfloat162float(h);
  m = __float2bfloat16_rn(r);
  l = __float2bfloat16_rn(r - __bfloat162float(m));
}

// Store NV consecutive K values of one row of a data tile, all three pieces.
template <int NV>
__device__ __forceinline__ void store_tile_row(__nv_bfloat16* tile, int row, int kk0, const float* v) {
  static_assert(NV == 1 || NV == 2 || NV == 4 || NV == 8, "row chunk");
  __align__(16) __nv_bfloat16 p[NPIECE][NV];
  if constexpr (NV == 1) {
    split3(v[0], p[0][0], p[1][0], p[2][0]);
  } else {
    // the same three roundings as split3, two values per conversion
#pragma unroll
    for (int j = 0; j < NV; j += 2) {
      const __nv_bfloat162 h = __floats2bfloat162_rn(v[j], v[j + 1]);
      const float2 hf = __bfloat1622float2(h);
      const float r0 = v[j] - hf.x, r1 = v[j + 1] - hf.y;
      const __nv_bfloat162 m = __floats2bfloat162_rn(r0, r1);
      const float2 mf = __bfloat1622float2(m);
      const __nv_bfloat162 l = __floats2bfloat162_rn(r0 - mf.x, r1 - mf.y);
      *reinterpret_cast<__nv_bfloat162*>(&p[0][j]) = h;
      *reinterpret_cast<__nv_bfloat162*>(&p[1][j]) = m;
      *reinterpret_cast<__nv_bfloat162*>(&p[2][j]) = l;
    }
  }
  const uint32_t off = tc05::kmaj_off(row, kk0, MCOLS) / 2;
#pragma unroll
  for (int s = 0; s < NPIECE; ++s) {
    __nv_bfloat16* d = tile + s * PIECE_HALVES + off;
    if constexpr (NV == 8) *reinterpret_cast<uint4*>(d) = *reinterpret_cast<const uint4*>(p[s]);
    if constexpr (NV == 4) *reinterpret_cast<uint2*>(d) = *reinterpret_cast<const uint2*>(p[s]);
    if constexpr (NV == 2) *reinterpret_cast<uint32_t*>(d) = *reinterpret_cast<const uint32_t*>(p[s]);
    if constexpr (NV == 1) *d = p[s][0];
  }
}

// ---------------------------------------------------------------- data tiles
// Analysis tiles: [field][m][fold][plane block][node tile]
__host__ __device__ inline size_t ana_tile(int lmax, int ncb, int nkn, int field, int m, int fold, int cb, int kt) {
  return ((((size_t)field * (lmax + 1) + m) * 2 + fold) * ncb + cb) * nkn + kt;
}
// Synthesis tiles: per field, [m][parity] blocks of ncb x ntiles(m, parity)
__device__ __forceinline__ size_t syn_tile(const long long* toff, int lmax, int m, int par, int cb, int kt) {
  return (size_t)toff[2 * m + par] + (size_t)cb * ntiles_of(lmax, m, par) + kt;
}

// data tile and part (0: dP or scalar, 1: mPs) of K step kt of an item
template <int MODE>
__device__ __forceinline__ const __nv_bfloat16* a_tile(const TcArgs& a, const TcItem& it, int cb, int kt) {
  if (MODE == ANA_S)
    return a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, 0, it.m, it.par, cb, kt) * TILE_HALVES;
  if (MODE == SYN_S) return a.tiles + syn_tile(a.toff, a.lmax, it.m, it.par, cb, kt) * TILE_HALVES;
  const bool first = kt < it.nk1;
  const int kk = first ? kt : kt - it.nk1;
  if (MODE == ANA_V) {
    // S: dP . Vt_(1-p) - i mPs . Vp_p      T: -dP . Vp_(1-p) - i mPs . Vt_p
    const int fold = first ? 1 - it.par : it.par;
    const int field = first ? (it.out ? 2 : 1) : (it.out ? 1 : 2);
    return a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, field, it.m, fold, cb, kk) * TILE_HALVES;
  }
  // Vt_q = dP . S + i mPs . T      Vp_q = -dP . T + i mPs . S   (fields S = 0, T = 1)
  const int par = first ? 1 - it.par : it.par;
  const int field = first ? (it.out ? 1 : 0) : (it.out ? 0 : 1);
  return a.tiles + (size_t)field * a.tfield + syn_tile(a.toff, a.lmax, it.m, par, cb, kk) * TILE_HALVES;
}

// A launch of the tensor-core kernel: one work set (`one`), or a group of
// work sets from several plans (`jobs`, job j owning the global units
// prefix[j] .. prefix[j+1]-1) walked by the same persistent CTAs.
struct TcLaunch {
  TcArgs one;
  const TcArgs* jobs;   // grouped launches (nullptr: `one`)
  const int* prefix;    // [njobs] first global unit of each job
  int njobs, total;     // total work units
  int* flag;            // status word of the launch
};

template <bool G>
__device__ __forceinline__ int job_of(const TcLaunch& L, int u) {
  if constexpr (!G) {
    return 0;
  } else {
    int lo = 0, hi = L.njobs - 1;  // last job whose first unit is <= u
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(L.prefix + mid) <= u) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
}

// The work unit u of a launch: its job's arguments, item and plane block.
template <bool G>
struct Unit {
  TcArgs a;
  TcItem it;
  int cb;
  __device__ __forceinline__ void load(const TcLaunch& L, int u) {
    int lu = u;
    if constexpr (G) {
      const int j = job_of<G>(L, u);
      a = L.jobs[j];
      lu = u - __ldg(L.prefix + j);
    } else {
      a = L.one;
    }
    it = a.items[lu / a.ncb];
    cb = lu % a.ncb;
  }
};

// Walks the K steps of this CTA's work units in order (units with no K
// steps are skipped).
template <bool G>
struct TileCur {
  int u, kt;
  Unit<G> w;
  __device__ void skip(const TcLaunch& L) {
    while (u < L.total && kt >= w.it.nk) {
      u += gridDim.x;
      kt = 0;
      if (u < L.total) w.load(L, u);
    }
  }
  __device__ void init(const TcLaunch& L) {
    u = blockIdx.x;
    kt = 0;
    if (u < L.total) w.load(L, u);
    skip(L);
  }
  __device__ void next(const TcLaunch& L) {
    ++kt;
    skip(L);
  }
  __device__ bool valid(const TcLaunch& L) const { return u < L.total; }
};

// ---------------------------------------------------------------- tensor-core kernel
template <int MODE, bool G>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_gemm(TcLaunch L) {
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + OFF_BAR);
  uint64_t* full = bars;                 // [STAGES] data + table tiles landed
  uint64_t* empty = full + STAGES;       // [STAGES] MMAs of the stage done
  uint64_t* accFull = empty + STAGES;    // [2] accumulator set complete
  uint64_t* accEmpty = accFull + 2;      // [2] accumulator set drained (count NEPI)
  uint64_t* fin = accEmpty + 2;          // all MMAs of this CTA done
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

  constexpr bool analysis = (MODE == ANA_S || MODE == ANA_V);
  constexpr bool vector = (MODE == ANA_V || MODE == SYN_V);
  // TMEM columns of one accumulator set: scalar modes main @0 and cross @128
  // (two sets, so the epilogue of one unit overlaps the MMAs of the next);
  // vector modes (128-column MMAs, two parts) main/cross @0/128 and
  // @256/384 -- all 512 columns, one set
  constexpr int NACC = vector ? 1 : 2;
  constexpr uint32_t PART = vector ? 256u : 128u, CROSS = 128u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // once any CTA of the launch's owner has given up a wait, later launches do no work
  if (tid == 0) *abort_flag = *(volatile int*)L.flag;
  __syncthreads();
  if (*abort_flag) return;
  __syncthreads();

  if (warp == 1) tc05::tmem_alloc(tslot, TMEM_COLS);
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      tc05::mbar_init(&full[s], 1);
      tc05::mbar_init(&empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      tc05::mbar_init(&accFull[s], 1);
      tc05::mbar_init(&accEmpty[s], NEPI);
    }
    tc05::mbar_init(fin, 1);
    tc05::mbar_fence_init();
  }
  tc05::fence_before();
  __syncthreads();
  tc05::fence_after();
  const uint32_t tbase = *tslot;
  auto fail = [&]() {
    atomicExch(L.flag, 1);
    *abort_flag = 1;
  };

  if (warp == 0) {
    // ------------------------------------------------------------ bulk copies
    if (lane == 0) {
      TileCur<G> cur;
      cur.init(L);
      int g = 0;
      for (; cur.valid(L); ++g, cur.next(L)) {
        const int s = g % STAGES, n = g / STAGES;
        if (n > 0 && (*abort_flag || !tc05::mbar_wait(&empty[s], (n - 1) & 1))) {
          fail();
          break;
        }
        const TcItem& it = cur.w.it;
        const __nv_bfloat16* At = a_tile<MODE>(cur.w.a, it, cur.w.cb, cur.kt);
        const uint32_t bbytes = (uint32_t)(NPIECE * it.nr * TK * 2);
        unsigned char* st = smem + s * STAGE_BYTES;
        mbar_arrive_tx(&full[s], A_BYTES + bbytes);
        bulk_copy(st, At, A_BYTES, &full[s]);
        bulk_copy(st + A_BYTES, cur.w.a.blocks + it.boff + (size_t)cur.kt * NPIECE * it.nr * TK, bbytes,
                  &full[s]);
      }
      // after a failure, copies may still be in flight: let them land
      if (*abort_flag)
        for (int t = max(0, g - STAGES); t < g; ++t)
          tc05::mbar_wait(&full[t % STAGES], (t / STAGES) & 1, 100000000ull);
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------ MMA issue
    if (lane == 0) {
      int g = 0, uc = 0;
      bool ok = true;
      for (int u = blockIdx.x; u < L.total && ok; u += gridDim.x, ++uc) {
        Unit<G> w;
        w.load(L, u);
        const TcItem& it = w.it;
        const int buf = uc % NACC, use = uc / NACC;
        if (use >= 1 && !tc05::mbar_wait(&accEmpty[buf], (use - 1) & 1)) {
          ok = false;
          break;
        }
        tc05::fence_after();
        const uint32_t tacc = tbase + (uint32_t)buf * 256;
        const uint32_t idesc = tc05::idesc_bf16(MCOLS, it.nr);
        const uint32_t lboA = (MCOLS / 8) * 128, lboB = (uint32_t)(it.nr / 8) * 128;
        const uint32_t bpiece = (uint32_t)it.nr * TK * 2;
        for (int kt = 0; kt < it.nk; ++kt, ++g) {
          const int s = g % STAGES;
          if (*abort_flag || !tc05::mbar_wait(&full[s], (g / STAGES) & 1)) {
            ok = false;
            break;
          }
          tc05::fence_after();
          const int part = (vector && kt >= it.nk1) ? 1 : 0;
          const bool first = kt == (part ? it.nk1 : 0);
          const uint32_t tmain = tacc + (uint32_t)part * PART;
          const uint32_t tcross = tmain + CROSS;
          unsigned char* At = smem + s * STAGE_BYTES;
          unsigned char* Bt = At + A_BYTES;
#pragma unroll
          for (int j = 0; j < TK / 16; ++j) {
            uint64_t ad[NPIECE], bd[NPIECE];
#pragma unroll
            for (int p = 0; p < NPIECE; ++p) {
              ad[p] = tc05::smem_desc(At + p * PIECE_HALVES * 2 + j * 2 * lboA, lboA, 128);
              bd[p] = tc05::smem_desc(Bt + p * bpiece + j * 2 * lboB, lboB, 128);
            }
            const uint32_t acc0 = (first && j == 0) ? 0u : 1u;
            tc05::mma_f16(tmain, ad[0], bd[0], idesc, acc0);
            tc05::mma_f16(tcross, ad[0], bd[1], idesc, acc0);
            tc05::mma_f16(tcross, ad[1], bd[0], idesc, 1u);
            tc05::mma_f16(tcross, ad[0], bd[2], idesc, 1u);
            tc05::mma_f16(tcross, ad[1], bd[1], idesc, 1u);
            tc05::mma_f16(tcross, ad[2], bd[0], idesc, 1u);
          }
          tc05::commit(&empty[s]);
        }
        if (!ok) break;
        tc05::commit(&accFull[buf]);
      }
      if (!ok) fail();
      tc05::commit(fin);
      tc05::mbar_wait(fin, 0, 100000000ull);
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    // Per chunk of 16 rows: TMEM -> registers (this lane's component), the
    // vector forms, then through a per-warp staging area so that the global
    // stores of a half-warp cover 16 consecutive rows of one plane.
    const int q = warp & 3;  // TMEM lane quarter of this warp
    const bool odd = lane & 1;
    double* stg = reinterpret_cast<double*>(smem + OFF_STG) + (warp - 2) * STG_WORDS;  // [32 lanes][17]
    const int j_out = lane & 15, ph = lane >> 4;  // store phase: row, plane half
    int uc = 0;
    for (int u = blockIdx.x; u < L.total; u += gridDim.x, ++uc) {
      Unit<G> w;
      w.load(L, u);
      const TcArgs& a = w.a;
      const TcItem& it = w.it;
      const int buf = uc % NACC, use = uc / NACC;
      bool ok = !*abort_flag && tc05::mbar_wait(&accFull[buf], use & 1);
      ok = __all_sync(0xffffffffu, ok);
      if (!ok) {
        fail();
        break;
      }
      tc05::fence_after();
      const int kbase = w.cb * PLANES + 16 * q;  // first plane of this warp
      const size_t base_lm = (size_t)a.mbase[it.m] - it.m;
      const uint32_t ta = tbase + (uint32_t)buf * 256 + ((uint32_t)(32 * q) << 16);
      const bool have0 = vector ? it.nk1 > 0 : it.nk > 0;
      const bool have1 = vector && it.nk > it.nk1;
      const int cfirst = 16 * ((warp - 2) / 4);  // the quarter's two warps alternate 16-column chunks
      // global stores of one chunk whose 16 values per lane are staged in stg:
      // 16 planes x 16 rows, lanes 0-15 rows of plane 2i, lanes 16-31 of plane 2i+1
      auto store_chunk = [&](int c) {
        __syncwarp();
#pragma unroll 4
        for (int i = 0; i < 8; ++i) {
          const int pl = 2 * i + ph, k = kbase + pl;
          const double re = stg[(2 * pl) * 17 + j_out], im = stg[(2 * pl + 1) * 17 + j_out];
          const int rr = c + j_out;
          if (k >= a.nz) continue;
          if (analysis) {
            if (rr >= it.nvalid) continue;
            const int l = it.m + it.par + 2 * (it.r0 + rr);
            double f = 1.0;
            if (MODE == ANA_V) f = l ? 1.0 / ((double)l * (double)(l + 1)) : 0.0;
            double2* out = (MODE == ANA_V && it.out) ? a.out2 : a.out;
            out[(size_t)k * a.nlm + base_lm + l] = make_double2(re * f, it.m == 0 ? 0.0 : im * f);
          } else {
            const int field = (MODE == SYN_V) ? 1 + it.out : 0;
            const int node = it.r0 + rr;
            if (node < a.ldn8)
              a.G32w[(size_t)field * a.G32field + (((size_t)it.m * 2 + it.par) * a.nz + k) * a.ldn8 + node] =
                  make_float2((float)re, (float)im);
          }
        }
        __syncwarp();
      };
      if constexpr (MODE == SYN_V) {
        // Vector synthesis fills all 512 TMEM columns with one unit, so the
        // next unit's MMAs wait until the accumulators are drained.  They are
        // drained first: every chunk of this warp is read and combined into
        // registers (the same float operations as below), the columns are
        // released, and the global stores run while the next unit's MMAs do.
        constexpr int NCH = NR_V / 32;
        float res[NCH][16];
        const float s0 = it.out ? -1.f : 1.f;
        const float sg = odd ? 1.f : -1.f;  // part 1 times +i: re' = -im, im' = re
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          const int c = cfirst + 32 * h;
          if (c < it.nr) {
            uint32_t v0[16], x0[16], v1[16], x1[16];
            if (have0) {
              tc05::tmem_ld16_nw(ta + c, v0);
              tc05::tmem_ld16_nw(ta + CROSS + c, x0);
            }
            if (have1) {
              tc05::tmem_ld16_nw(ta + PART + c, v1);
              tc05::tmem_ld16_nw(ta + PART + CROSS + c, x1);
            }
            tc05::tmem_wait_ld();
            tc05::tmem_regs(v0);
            tc05::tmem_regs(x0);
            tc05::tmem_regs(v1);
            tc05::tmem_regs(x1);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              float rf = have0 ? s0 * (__uint_as_float(v0[j]) + __uint_as_float(x0[j])) : 0.f;
              const float y = have1 ? __uint_as_float(v1[j]) + __uint_as_float(x1[j]) : 0.f;
              rf += sg * __shfl_xor_sync(0xffffffffu, y, 1);
              res[h][j] = rf;
            }
          }
        }
        tc05::fence_before();
        tc05::mbar_arrive(&accEmpty[buf]);
#pragma unroll
        for (int h = 0; h < NCH; ++h) {
          const int c = cfirst + 32 * h;
          if (c < it.nr) {
#pragma unroll
            for (int j = 0; j < 16; ++j) stg[lane * 17 + j] = (double)res[h][j];
            store_chunk(c);
          }
        }
        continue;
      }
      for (int c = cfirst; c < it.nr; c += 32) {
        uint32_t v0[16], x0[16], v1[16], x1[16];
        if (have0) {
          tc05::tmem_ld16_nw(ta + c, v0);
          tc05::tmem_ld16_nw(ta + CROSS + c, x0);
        }
        if (have1) {
          tc05::tmem_ld16_nw(ta + PART + c, v1);
          tc05::tmem_ld16_nw(ta + PART + CROSS + c, x1);
        }
        tc05::tmem_wait_ld();
        tc05::tmem_regs(v0);
        tc05::tmem_regs(x0);
        tc05::tmem_regs(v1);
        tc05::tmem_regs(x1);
        const double s0 = (vector && it.out) ? -1.0 : 1.0;  // part 0 form: +1 or -1
        // part 1 times -i (analysis: re' = im, im' = -re) or +i (synthesis:
        // re' = -im, im' = re): each lane takes its partner's value
        const double sg = (analysis != odd) ? 1.0 : -1.0;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          double r = 0.0;
          if (analysis) {
            if (have0) r = s0 * ((double)__uint_as_float(v0[j]) + (double)__uint_as_float(x0[j]));
            if (vector) {
              const double y = have1 ? (double)__uint_as_float(v1[j]) + (double)__uint_as_float(x1[j]) : 0.0;
              r += sg * __shfl_xor_sync(0xffffffffu, y, 1);
            }
          } else {
            float rf = have0 ? (float)s0 * (__uint_as_float(v0[j]) + __uint_as_float(x0[j])) : 0.f;
            if (vector) {
              const float y = have1 ? __uint_as_float(v1[j]) + __uint_as_float(x1[j]) : 0.f;
              rf += (float)sg * __shfl_xor_sync(0xffffffffu, y, 1);
            }
            r = rf;
          }
          stg[lane * 17 + j] = r;
        }
        store_chunk(c);
      }
      tc05::fence_before();
      tc05::mbar_arrive(&accEmpty[buf]);
    }
  }
  tc05::fence_before();
  __syncthreads();
  tc05::fence_after();
  if (warp == 1) tc05::tmem_free(tbase, TMEM_COLS);
}

// ---------------------------------------------------------------- fp32 phi FFTs
constexpr int PTHREADS = 512;
constexpr int PMAXC = 12288;  // NP*nphi complex values per CTA (two CTAs per SM)

__host__ __device__ inline int seq_stride(int nphi) {
  int s = nphi + (nphi + 7) / 8;
  return s | 1;
}

struct Phi32Args {
  // grids: double, or float for the single-precision entry points (the
  // kernels' GT template parameter says which)
  const void* gin[SPH_MAX_FIELDS];
  const void* gin_hi[SPH_MAX_FIELDS];  // planes k >= ksplit (continued planes)
  int ksplit;
  void* gout[SPH_MAX_FIELDS];
  __nv_bfloat16* tiles;  // analysis data tiles (forward output)
  const float2* G32c;    // folded coefficients (inverse input)
  size_t G32field;
  int nlat, ldn8, nz, lmax, NP, ncb, nkn;
  const double* wfold;
  const float2* twp;
  const float2* tw1;  // four-step kernels: pass twiddles of length N1 and N2,
  const float2* tw2;  // and W_N^e = exp(-2 pi i e / N)
  const float2* twN;
  int* flag;  // set when a bounded wait gives up (three-step forward)
};

// plane k of field f of the forward input: from the grid below ksplit, from
// the continued planes above
template <typename GT>
__device__ __forceinline__ const GT* in_plane(const Phi32Args& a, int f, int k, int N) {
  return k < a.ksplit ? static_cast<const GT*>(a.gin[f]) + (size_t)k * N * a.nlat
                      : static_cast<const GT*>(a.gin_hi[f]) + (size_t)(k - a.ksplit) * N * a.nlat;
}

// Four-step forward phi FFT geometry (N = N1 N2, NP ring pairs per CTA),
// the register-staged fallback for grids whose rows cannot be staged by TMA
// or for an odd number of ring pairs.  Shared memory: X[b][k1][n2] with row
// pitch = 1 (mod 16) and sequence stride = 4 (mod 16) float2 slots, so that
// the lanes of a warp (8 sequences x 4 rows) hit 32 distinct slots; the
// kernel overwrites each row k1 with its spectrum Z(k1 + N1 k2), k2 along
// the row.
constexpr int up_mod16(int x, int r) { return x + (((r - x) % 16) + 16) % 16; }
template <int N, int NP>
struct P4 {
  static constexpr int N1 = ct::split_n1(N), N2 = N / N1;
  // about two work items per thread, so that two CTAs fit an SM's registers
  static constexpr int THREADS = ((NP * (N1 > N2 ? N1 : N2) + 1) / 2 + 31) / 32 * 32;
  static constexpr int PF = up_mod16(N2, 1), SF = up_mod16(N1 * PF, 4);
  static constexpr size_t SMEM_FWD = (size_t)NP * SF * sizeof(float2);
};

// Forward, four-step: (1) thread (b, n2) loads x[n2 + N2 n1] of ring pair b
// straight from the grid into registers, an N1-point DFT, the twiddle
// W_N^(n2 k1), one store to X; (2) thread (b, k1) an N2-point DFT of row
// k1 giving Z(k1 + N1 k2), written back over the row; (3) thread m folds
// both parities of the NP nodes from Z(m), Z(-m) and writes them, split, as
// row chunks of the analysis tiles.
template <int N, int NP, typename GT>
__global__ void __launch_bounds__(P4<N, NP>::THREADS, 2) phi4_fwd32(Phi32Args a) {
  using C = P4<N, NP>;
  constexpr int N1 = C::N1, N2 = C::N2;
  extern __shared__ float2 sx[];
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = blockIdx.y, f = blockIdx.z;
  const int t = threadIdx.x;
  const GT* plane = in_plane<GT>(a, f, k, N);
  for (int it = t; it < NP * N2; it += C::THREADS) {
    const int b = it % NP, n2 = it / NP;
    const GT* pr = plane + p0 + b;               // ring p0 + b (real part)
    const GT* pm = plane + (nlat - 1 - p0 - b);  // its mirror (imaginary part)
    float2 v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) {
      const size_t j = (size_t)(n2 + N2 * n1) * nlat;
      v[n1] = make_float2((float)__ldg(pr + j), (float)__ldg(pm + j));
    }
    ct::reg_dif<float2, N1>(v, a.tw1, -1);
    float2* X = sx + b * C::SF + n2;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      float2 z = v[ct::rev_pos<N1>(k1)];
      if (k1) z = ct::mul(z, __ldg(a.twN + n2 * k1));
      X[k1 * C::PF] = z;
    }
  }
  __syncthreads();
  // step 2: each row X[b][k1][.] becomes the spectrum Z(k1 + N1 k2) in place
  for (int it = t; it < NP * N1; it += C::THREADS) {
    const int b2 = it % NP, k1 = it / NP;
    float2* X = sx + b2 * C::SF + k1 * C::PF;
    float2 w[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) w[n2] = X[n2];
    ct::reg_dif<float2, N2>(w, a.tw2, -1);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) X[k2] = w[ct::rev_pos<N2>(k2)];
  }
  __syncthreads();
  float W[NP];
#pragma unroll
  for (int b = 0; b < NP; ++b) W[b] = (float)__ldg(a.wfold + p0 + b);
  const int cb = k / PLANES, row = 2 * (k % PLANES), kt = p0 / TK, kk0 = p0 % TK;
  for (int m = t; m <= a.lmax; m += C::THREADS) {
    float er[NP], ei[NP], orr[NP], oi[NP];
#pragma unroll
    for (int b = 0; b < NP; ++b) {
      const int mc = m == 0 ? 0 : N - m;
      const float2 Z = sx[b * C::SF + (m % N1) * C::PF + m / N1];
      const float2 Zc = sx[b * C::SF + (mc % N1) * C::PF + mc / N1];
      // F(ring) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
      const float fir = 0.5f * (Z.x + Zc.x), fii = 0.5f * (Z.y - Zc.y);
      const float fmr = 0.5f * (Z.y + Zc.y), fmi = -0.5f * (Z.x - Zc.x);
      er[b] = (fir + fmr) * W[b];
      ei[b] = (fii + fmi) * W[b];
      orr[b] = (fir - fmr) * W[b];
      oi[b] = (fii - fmi) * W[b];
    }
    __nv_bfloat16* t0 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 0, cb, kt) * TILE_HALVES;
    __nv_bfloat16* t1 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 1, cb, kt) * TILE_HALVES;
    store_tile_row<NP>(t0, row, kk0, er);
    store_tile_row<NP>(t0, row + 1, kk0, ei);
    store_tile_row<NP>(t1, row, kk0, orr);
    store_tile_row<NP>(t1, row + 1, kk0, oi);
  }
}

// Forward: ring pairs p0..p0+NP-1 of plane k, field f.  The samples are
// placed at their digit-reversed positions and transformed by the
// decimation-in-time passes, so the spectrum comes out in natural order; the
// thread of degree m then reads Z(m), Z(-m) of its NP ring pairs from
// consecutive addresses, folds both parities and writes them, split, as row
// chunks of the analysis tiles.
template <int N, int NP, typename GT>
__global__ void __launch_bounds__(PTHREADS, 2) phi_fwd32(Phi32Args a) {
  extern __shared__ float2 sf[];
  constexpr int Q = 2 * NP, JSTEP = PTHREADS / Q;
  const int nlat = a.nlat;
  const int p0 = blockIdx.x * NP, k = blockIdx.y, f = blockIdx.z;
  const int tid = threadIdx.x;
  const GT* plane = in_plane<GT>(a, f, k, N);
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
      GT v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int j = j0 + (u0 + u) * JSTEP;
        v[u] = (u0 + u < NJ && j < N) ? __ldg(plane + (size_t)j * nlat + ring) : GT(0);
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        int j = j0 + (u0 + u) * JSTEP;
        if (u0 + u < NJ && j < N) smf[2 * g.addr(b, ct::rev_pos<N>(j)) + half] = (float)v[u];
      }
    }
  }
  __syncthreads();
  ct::dit<float2, N, N>(sf, g, a.twp, -1);

  float W[NP];
#pragma unroll
  for (int b = 0; b < NP; ++b) W[b] = (float)__ldg(a.wfold + p0 + b);
  const int cb = k / PLANES, row = 2 * (k % PLANES), kt = p0 / TK, kk0 = p0 % TK;
  for (int m = tid; m <= a.lmax; m += PTHREADS) {
    float er[NP], ei[NP], orr[NP], oi[NP];
#pragma unroll
    for (int b = 0; b < NP; ++b) {
      const float2 Z = sf[g.addr(b, m)];
      const float2 Zc = sf[g.addr(b, m == 0 ? 0 : N - m)];
      // F(ring) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
      const float fir = 0.5f * (Z.x + Zc.x), fii = 0.5f * (Z.y - Zc.y);
      const float fmr = 0.5f * (Z.y + Zc.y), fmi = -0.5f * (Z.x - Zc.x);
      er[b] = (fir + fmr) * W[b];
      ei[b] = (fii + fmi) * W[b];
      orr[b] = (fir - fmr) * W[b];
      oi[b] = (fii - fmi) * W[b];
    }
    __nv_bfloat16* t0 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 0, cb, kt) * TILE_HALVES;
    __nv_bfloat16* t1 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 1, cb, kt) * TILE_HALVES;
    store_tile_row<NP>(t0, row, kk0, er);
    store_tile_row<NP>(t0, row + 1, kk0, ei);
    store_tile_row<NP>(t1, row, kk0, orr);
    store_tile_row<NP>(t1, row + 1, kk0, oi);
  }
}

template <int N, int NP, typename GT>
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
  GT* plane = static_cast<GT*>(a.gout[f]) + (size_t)k * N * nlat;
  const float* smf = reinterpret_cast<const float*>(sf);
  const int q = tid % Q, j0 = tid / Q;
  const int b = q < NP ? q : 2 * NP - 1 - q;
  const int ring = q < NP ? p0 + q : nlat - 1 - (p0 + b);
  const int half = q < NP ? 0 : 1;
  for (int j = j0; j < N; j += JSTEP) plane[(size_t)j * nlat + ring] = (GT)smf[2 * g.addr(b, j) + half];
}

// ---------------------------------------------------------------- three-step phi FFTs
// Persistent kernels over tiles of NP ring pairs of one (plane, field).  The
// input of the tile after the current one is copied into shared memory while
// the current one is transformed -- TMA boxes of the grid for the forward
// transform (2 N / BR requests of NP x BR values instead of N NP / 2 16-byte
// copies, which the load path cannot keep in flight), cp.async for the
// inverse's folded coefficients -- so no registers are held by loads in flight.
//
// N = A M, M = B C (A = 16, B the power-of-two part of M up to 16, C the
// rest).  Forward: (A) A-point DFTs of the stride-M subsequences
// x[nm + M n1], the twiddle W_N^(nm ka), stored as row ka, column nm;
// (B) B-point DFTs of each row over its stride-C subsequences c + C nb,
// the twiddle W_M^(c kb), stored back at c + C kb; (C) C-point DFTs of the
// runs C kb .. C kb + C-1, stored back in place.  Frequency ka + A (kb + B kc)
// then sits in row ka, column C kb + kc.  The inverse runs the same steps
// backwards with conjugate twiddles.  The row pitch PR is odd and the
// ring-pair stride SB = 16/NP (mod 16), so the lanes of every half warp
// (NP ring pairs x 16/NP rows or columns) hit distinct banks in each step.
template <int N, int NP>
struct P3 {
  static constexpr int A = 16, M = N / A, B = ct::pow2_part_cap16(M), C = M / B;
  static constexpr int ITEMS_A = NP * M, ITEMS_B = NP * A * C, ITEMS_C = NP * A * B;
  static constexpr int THREADS = ITEMS_A <= 64 ? 64 : (ITEMS_A + 31) / 32 * 32;
  static constexpr int PR = M | 1;
  static constexpr int SB = up_mod16(A * PR, 16 / NP);
  static constexpr size_t XBYTES = (size_t)NP * SB * sizeof(float2);      // transform area
  static constexpr size_t STAGE_F = (size_t)N * 2 * NP * sizeof(double);  // one forward tile, fp64
  static constexpr size_t SMEM_F = 2 * STAGE_F + (size_t)N * sizeof(float2) + 2 * sizeof(uint64_t);
  // two CTAs per SM where two forward tiles fit (registers bounded to match)
  static constexpr int MINB = SMEM_F <= 110 * 1024 && THREADS <= 512 ? 2 : 1;
  static_assert(N % A == 0 && NP >= 2 && NP <= 16 && XBYTES % 16 == 0, "three-step geometry");
  // single-pass kernels: the transform area overlays one staged tile, one step-A item per thread
  static constexpr bool ONE_PASS = XBYTES <= STAGE_F && ITEMS_A <= THREADS && THREADS <= 1024;
  // inverse: transform area, twiddles, one staged coefficient tile of (lmax + 1) x 2 x NP float2;
  // two CTAs per SM where that fits for every lmax < N/2 (one loads while the other computes)
  __host__ __device__ static size_t smem_inv(int lmax) { return XBYTES + (size_t)N * sizeof(float2) + stage_inv(lmax) * sizeof(float2); }
  static constexpr int MINB_INV = XBYTES + (size_t)N * sizeof(float2) + (size_t)N * NP * sizeof(float2) <= 113 * 1024 && THREADS <= 512 ? 2 : 1;
  __host__ __device__ static int stage_inv(int lmax) { return (lmax + 1) * 2 * NP; }
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// staged rows of 2 NP values (rings | mirrors, or parity 0 | parity 1) swap
// their halves every 8/NP rows, so that 16/NP consecutive rows read by a
// half warp fall in distinct banks
template <int NP>
__device__ __forceinline__ int stage_swz(int row) {
  return ((row * NP) >> 3) & 1;
}

__device__ __forceinline__ float2 conj2(float2 z) { return make_float2(z.x, -z.y); }

// TMA views of the forward input: per field, the planes below ksplit (lo)
// and the continued planes from ksplit on (hi), each a 2D fp64 array of
// nlat columns (rings) and N x planes rows (phi samples); box NP x BR.
struct Phi3Maps {
  CUtensorMap lo[SPH_MAX_FIELDS], hi[SPH_MAX_FIELDS];
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* mbar) {
  tma::load_2d(dst, map, x, y, mbar);
}

template <int N>
__host__ __device__ constexpr int phi3_box_rows() {
  return N <= 256 ? N : (N % 256 == 0 ? 256 : 192);
}

template <int N, int NP, typename GT>
__global__ void __launch_bounds__(P3<N, NP>::THREADS, P3<N, NP>::MINB)
    phi3_fwd32(Phi32Args a, int ntiles, const __grid_constant__ Phi3Maps maps) {
  using G = P3<N, NP>;
  constexpr int A = G::A, M = G::M, B = G::B, C = G::C, T = G::THREADS, BR = phi3_box_rows<N>();
  static_assert(N % BR == 0 && G::ONE_PASS, "box rows, single-pass geometry");
  // [stage 0 | stage 1 | twiddles | 2 mbarriers]; a stage is [ring rows | mirror rows], rows of NP values
  extern __shared__ __align__(1024) unsigned char sm3[];
  float2* tw = reinterpret_cast<float2*>(sm3 + 2 * G::STAGE_F);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm3 + 2 * G::STAGE_F + (size_t)N * sizeof(float2));
  const int t = threadIdx.x;
  const int nlat = a.nlat, ngroups = nlat / 2 / NP;
  for (int i = t; i < N; i += T) tw[i] = __ldg(a.twN + i);
  if (t == 0) {
    tc05::mbar_init(&full[0], 1);
    tc05::mbar_init(&full[1], 1);
    tc05::mbar_fence_init();
  }
  __syncthreads();
  // a stage holds an FP64 tile (float grids use the first half of it)
  auto stage = [&](int which) { return reinterpret_cast<GT*>(sm3 + which * G::STAGE_F); };
  // one thread: the 2 N / BR boxes of a tile (its NP rings and their NP mirrors, all N samples)
  auto issue = [&](int tile, int which) {
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz;
    const bool lo = k < a.ksplit;
    const CUtensorMap* map = lo ? &maps.lo[f] : &maps.hi[f];
    const int y0 = (lo ? k : k - a.ksplit) * N;
    GT* st = stage(which);
    mbar_arrive_tx(&full[which], (uint32_t)(2 * N * NP * sizeof(GT)));
#pragma unroll 1
    for (int i = 0; i < N / BR; ++i) {
      tma_load_2d(st + (size_t)i * BR * NP, map, g * NP, y0 + i * BR, &full[which]);
      tma_load_2d(st + (size_t)(N + i * BR) * NP, map, nlat - g * NP - NP, y0 + i * BR, &full[which]);
    }
  };
  if (t == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
  int s = 0;
  uint32_t phase = 0;  // bit s: parity of the next completion of stage s
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, s ^= 1) {
    const bool ok = tc05::mbar_wait(&full[s], (phase >> s) & 1);
    if (__syncthreads_or(!ok)) {  // the tile never arrived: report, let the copies land, stop
      if (t == 0) {
        atomicExch(a.flag, 1);
        tc05::mbar_wait(&full[s], (phase >> s) & 1);
      }
      return;
    }
    phase ^= 1u << s;
    if (t == 0 && tile + (int)gridDim.x < ntiles) {
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      issue(tile + gridDim.x, s ^ 1);
    }
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz, p0 = g * NP;
    const GT* ring = stage(s);
    const GT* mir = ring + (size_t)N * NP;
    float2* X = reinterpret_cast<float2*>(stage(s));
    // (A) the samples x[nm + M n1] of ring pair bA (ring: real part, mirror: imaginary part)
    const bool act = t < G::ITEMS_A;
    const int bA = t % NP, nm = t / NP;
    float2 v[A];
    if (act) {
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        const int j = nm + M * n1;
        v[n1] = make_float2((float)ring[j * NP + bA], (float)mir[j * NP + (NP - 1 - bA)]);
      }
    }
    __syncthreads();  // the transform area overlays the staged samples
    if (act) {
      ct::RD<float2, A, -1>::run(v);
      float2* xo = X + bA * G::SB + nm;
#pragma unroll
      for (int ka = 0; ka < A; ++ka) xo[ka * G::PR] = ka ? ct::mul(v[ka], tw[nm * ka]) : v[ka];
    }
    __syncthreads();
    if constexpr (B > 1) {  // (B)
      for (int it = t; it < G::ITEMS_B; it += T) {
        const int ka = it % A, rr = it / A, c = rr % C, b = rr / C;
        float2* row = X + b * G::SB + ka * G::PR + c;
        float2 w[B];
#pragma unroll
        for (int nb = 0; nb < B; ++nb) w[nb] = row[C * nb];
        ct::RD<float2, B, -1>::run(w);
#pragma unroll
        for (int kb = 0; kb < B; ++kb) row[C * kb] = (kb && c) ? ct::mul(w[kb], tw[A * c * kb]) : w[kb];
      }
      __syncthreads();
    }
    if constexpr (C > 1) {  // (C)
      for (int it = t; it < G::ITEMS_C; it += T) {
        const int ka = it % A, rr = it / A, kb = rr % B, b = rr / B;
        float2* row = X + b * G::SB + ka * G::PR + C * kb;
        float2 u[C];
#pragma unroll
        for (int c = 0; c < C; ++c) u[c] = row[c];
        ct::RD<float2, C, -1>::run(u);
#pragma unroll
        for (int kc = 0; kc < C; ++kc) row[kc] = u[kc];
      }
      __syncthreads();
    }
    // fold both parities of the NP ring pairs from Z(m), Z(-m), weight, split, write tile rows
    float W[NP];
#pragma unroll
    for (int b = 0; b < NP; ++b) W[b] = (float)__ldg(a.wfold + p0 + b);
    const int cb = k / PLANES, row = 2 * (k % PLANES), kt = p0 / TK, kk0 = p0 % TK;
    auto zpos = [&](int m) {
      const int q = m / A;
      return (m % A) * G::PR + C * (q % B) + q / B;
    };
    for (int m = t; m <= a.lmax; m += T) {
      const int pz = zpos(m), pc = zpos(m == 0 ? 0 : N - m);
      float er[NP], ei[NP], orr[NP], oi[NP];
#pragma unroll
      for (int b = 0; b < NP; ++b) {
        const float2 Z = X[b * G::SB + pz], Zc = X[b * G::SB + pc];
        // F(ring) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
        const float fir = 0.5f * (Z.x + Zc.x), fii = 0.5f * (Z.y - Zc.y);
        const float fmr = 0.5f * (Z.y + Zc.y), fmi = -0.5f * (Z.x - Zc.x);
        er[b] = (fir + fmr) * W[b];
        ei[b] = (fii + fmi) * W[b];
        orr[b] = (fir - fmr) * W[b];
        oi[b] = (fii - fmi) * W[b];
      }
      __nv_bfloat16* t0 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 0, cb, kt) * TILE_HALVES;
      __nv_bfloat16* t1 = a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 1, cb, kt) * TILE_HALVES;
      store_tile_row<NP>(t0, row, kk0, er);
      store_tile_row<NP>(t0, row + 1, kk0, ei);
      store_tile_row<NP>(t1, row, kk0, orr);
      store_tile_row<NP>(t1, row + 1, kk0, oi);
    }
    // this stage is refilled by TMA (async proxy) after the next barrier
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
}

template <int N, int NP, typename GT>
__global__ void __launch_bounds__(P3<N, NP>::THREADS, P3<N, NP>::MINB_INV) phi3_inv32(Phi32Args a, int ntiles) {
  using G = P3<N, NP>;
  constexpr int A = G::A, M = G::M, B = G::B, C = G::C, T = G::THREADS;
  static_assert(G::ONE_PASS, "single-pass geometry");
  extern __shared__ __align__(1024) unsigned char sm3i[];
  float2* X = reinterpret_cast<float2*>(sm3i);
  float2* tw = reinterpret_cast<float2*>(sm3i + G::XBYTES);
  const int lmax = a.lmax, nlat = a.nlat, ngroups = nlat / 2 / NP;
  float2* stg = tw + N;
  const int t = threadIdx.x;
  for (int i = t; i < N; i += T) tw[i] = __ldg(a.twN + i);
  const size_t pstride = (size_t)a.nz * a.ldn8;  // parity stride of the folded coefficients
  auto issue = [&](int tile, float2* st) {
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz;
    const float2* gs = a.G32c + (size_t)f * a.G32field + (size_t)k * a.ldn8 + g * NP;
    constexpr int GR = NP / 2;
    const int total = (lmax + 1) * 2 * GR;
    for (int q = t; q < total; q += T) {
      const int gg = q % GR, rr = q / GR, par = rr & 1, mm = rr >> 1;
      cp_async16(st + mm * 2 * NP + (par ^ stage_swz<NP>(mm)) * NP + 2 * gg, gs + (size_t)rr * pstride + 2 * gg);
    }
    cp_async_commit();
  };
  if ((int)blockIdx.x < ntiles) issue(blockIdx.x, stg);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    cp_async_wait_all();
    __syncthreads();  // the tile's coefficients have landed; the last tile's step (A') is done with X
    const int g = tile % ngroups, r = tile / ngroups, k = r % a.nz, f = r / a.nz, p0 = g * NP;
    const float2* st = stg;
    // Z(m) of ring pair b (x = ring + i mirror) from the folded coefficients of both parities
    auto zin = [&](int m, int b) {
      const bool lo = m <= lmax, hi = N - m <= lmax;
      if (!lo && !hi) return make_float2(0.f, 0.f);
      const int mm = lo ? m : N - m;
      const int sw = stage_swz<NP>(mm);
      const float2 se = st[mm * 2 * NP + sw * NP + b], so = st[mm * 2 * NP + (1 - sw) * NP + b];
      const float2 Fi = make_float2(se.x + so.x, se.y + so.y), Fm = make_float2(se.x - so.x, se.y - so.y);
      if (m == 0) return make_float2(Fi.x, Fm.x);
      if (lo) return make_float2(Fi.x - Fm.y, Fi.y + Fm.x);
      return make_float2(Fi.x + Fm.y, -Fi.y + Fm.x);
    };
    // (C') C-point inverse DFTs over kc of Z(ka + A (kb + B kc)), the twiddle W_M^-(c kb)
    for (int it = t; it < G::ITEMS_C; it += T) {
      const int b = it % NP, rr = it / NP, ka = rr % A, kb = rr / A;
      float2 u[C];
#pragma unroll
      for (int kc = 0; kc < C; ++kc) u[kc] = zin(ka + A * (kb + B * kc), b);
      ct::RD<float2, C, 1>::run(u);
      float2* row = X + b * G::SB + ka * G::PR + C * kb;
#pragma unroll
      for (int c = 0; c < C; ++c) row[c] = (c && kb) ? ct::mul(u[c], conj2(tw[A * c * kb])) : u[c];
    }
    __syncthreads();
    // step (C') was the last reader of the stage: the next tile's
    // coefficients load while steps (B') and (A') run
    if (tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x, stg);
    if constexpr (B > 1) {  // (B') B-point inverse DFTs over kb, stored at column c + C nb
      for (int it = t; it < G::ITEMS_B; it += T) {
        const int ka = it % A, rr = it / A, c = rr % C, b = rr / C;
        float2* row = X + b * G::SB + ka * G::PR + c;
        float2 w[B];
#pragma unroll
        for (int kb = 0; kb < B; ++kb) w[kb] = row[C * kb];
        ct::RD<float2, B, 1>::run(w);
#pragma unroll
        for (int nb = 0; nb < B; ++nb) row[C * nb] = w[nb];
      }
      __syncthreads();
    }
    // (A') the twiddle W_N^-(nm ka), A-point inverse DFTs over ka, grid stores
    if (t < G::ITEMS_A) {
      const int b = t % NP, nm = t / NP;
      float2 v[A];
      const float2* xi = X + b * G::SB + nm;
#pragma unroll
      for (int ka = 0; ka < A; ++ka) v[ka] = ka ? ct::mul(xi[ka * G::PR], conj2(tw[nm * ka])) : xi[0];
      ct::RD<float2, A, 1>::run(v);
      GT* plane = static_cast<GT*>(a.gout[f]) + (size_t)k * N * nlat;
      GT* pr = plane + p0 + b;
      GT* pm = plane + (nlat - 1 - p0 - b);
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) {
        const size_t j = (size_t)(nm + M * n1) * nlat;
        pr[j] = (GT)v[n1].x;
        pm[j] = (GT)v[n1].y;
      }
    }
  }
}

// ---------------------------------------------------------------- two-pass forward phi FFT
// For lengths whose tile of 8 ring pairs does not fit shared memory twice,
// the forward transform runs in two passes, so that every HBM request is a
// full line: pass 1 reads whole grid rows (PB consecutive ring pairs per
// warp: 128-byte runs of rings and of mirrors) and does step (A) of the
// three-step transform for all ring pairs; it writes, through shared memory,
// each tile's transform area exactly as the single-pass kernel lays it out
// in shared memory ([b][ka][nm], pitches PR and SB), one contiguous image per
// (plane, tile).  Pass 2 bulk-copies an image into shared memory (double
// buffered) and finishes steps (B), (C), the fold and the tile rows.
// The passes alternate over batches of PHI2_BATCH plane-fields; pass 1
// reads whole grid rows.
// Batches of 16 plane-fields, whose images (77 MB at nphi 1536) stay in L2
// between the passes, were measured slower on the B200 (6.5 against 5.1 ms
// per pair): four times the launches, and a pass 2 of 768 tiles on 296 CTAs
// leaves 14% of its last wave idle.
constexpr int PHI2_PB = 16, PHI2_NMC = 16, PHI2_NP = 8, PHI2_BATCH = 64;

template <int N, typename GT>
__global__ void __launch_bounds__(PHI2_PB* PHI2_NMC, 2) phi2a_fwd32(Phi32Args a, float2* img, int q0) {
  using G = P3<N, PHI2_NP>;
  constexpr int A = G::A, M = G::M, PB = PHI2_PB, NMC = PHI2_NMC, SPB = A * NMC + 1;
  static_assert(M % NMC == 0, "nm chunks");
  __shared__ float2 S[PB * SPB];
  const int t = threadIdx.x, b = t % PB, nmi = t / PB;
  const int nlat = a.nlat, pair = blockIdx.x * PB + b, nm0 = blockIdx.y * NMC, nm = nm0 + nmi;
  const int q = q0 + blockIdx.z, k = q % a.nz, f = q / a.nz;
  const GT* pl = in_plane<GT>(a, f, k, N);
  float2 v[A];
#pragma unroll
  for (int n1 = 0; n1 < A; ++n1) {
    const GT* row = pl + (size_t)(nm + M * n1) * nlat;
    v[n1] = make_float2((float)__ldg(row + pair), (float)__ldg(row + (nlat - 1 - pair)));
  }
  ct::RD<float2, A, -1>::run(v);
#pragma unroll
  for (int ka = 0; ka < A; ++ka) S[b * SPB + ka * NMC + nmi] = ka ? ct::mul(v[ka], __ldg(a.twN + nm * ka)) : v[ka];
  __syncthreads();
  // rows (b, ka) of NMC consecutive columns into the tile images
  const int ntile = a.nlat / 2 / PHI2_NP;
  for (int e = t; e < PB * A * NMC; e += PB * NMC) {
    const int r = e / NMC, i = e % NMC, bb = r / A, ka = r % A;
    const int pr = blockIdx.x * PB + bb, tile = pr / PHI2_NP, b8 = pr % PHI2_NP;
    float2* dst = img + ((size_t)blockIdx.z * ntile + tile) * (PHI2_NP * G::SB);
    dst[b8 * G::SB + ka * G::PR + nm0 + i] = S[bb * SPB + ka * NMC + i];
  }
}

// pass-2 threads: two CTAs per SM, one tile image each.  Measured per pair
// at 768 x 1536 x 256 x 4 fields: 5.57 ms at 512 threads, 5.08 at 384,
// 4.99 at 256, 4.84 at 192, 4.91 at 128: fewer threads with more work each
// (the B-step items four per thread) keep more of each thread's loads in flight.
constexpr int PHI2_T = 192;
template <int N>
__host__ __device__ constexpr size_t phi2_smem() {
  return P3<N, PHI2_NP>::XBYTES + (size_t)P3<N, PHI2_NP>::M * sizeof(float2) + sizeof(uint64_t);
}

template <int N>
__global__ void __launch_bounds__(PHI2_T, 2) phi2b_fwd32(Phi32Args a, const float2* img, int q0, int nq, int ntiles) {
  using G = P3<N, PHI2_NP>;
  constexpr int NP = PHI2_NP, A = G::A, M = G::M, B = G::B, C = G::C, T = PHI2_T;
  constexpr int XF = NP * G::SB;  // float2 per tile image
  // [tile image | twiddles W_M^e | mbarrier]; the other CTA on the SM computes while this one loads
  extern __shared__ __align__(1024) unsigned char sm2[];
  float2* X = reinterpret_cast<float2*>(sm2);
  float2* tw = reinterpret_cast<float2*>(sm2 + G::XBYTES);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm2 + G::XBYTES + (size_t)M * sizeof(float2));
  const int t = threadIdx.x;
  const int ngroups = a.nlat / 2 / NP;
  for (int i = t; i < M; i += T) tw[i] = __ldg(a.twN + A * i);
  if (t == 0) {
    tc05::mbar_init(full, 1);
    tc05::mbar_fence_init();
  }
  __syncthreads();
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, phase ^= 1) {
    // planes fastest: the CTAs in flight write the tiles of one or two node
    // tiles (kt), a set that stays in L2 until every row of it is written
    const int g = tile / nq, ql = tile % nq, q = q0 + ql, k = q % a.nz, f = q / a.nz, p0 = g * NP;
    if (t == 0) {
      const float2* src = img + ((size_t)ql * ngroups + g) * XF;
      mbar_arrive_tx(full, (uint32_t)G::XBYTES);
      constexpr uint32_t PIECE = 32768;
      for (uint32_t o = 0; o < (uint32_t)G::XBYTES; o += PIECE) {
        const uint32_t n = (uint32_t)G::XBYTES - o < PIECE ? (uint32_t)G::XBYTES - o : PIECE;
        bulk_copy(reinterpret_cast<char*>(X) + o, reinterpret_cast<const char*>(src) + o, n, full);
      }
    }
    float W[NP];  // quadrature weights, loaded while the image arrives
#pragma unroll
    for (int b = 0; b < NP; ++b) W[b] = (float)__ldg(a.wfold + p0 + b);
    const bool ok = tc05::mbar_wait(full, phase);
    if (__syncthreads_or(!ok)) {  // the image never arrived: report, let the copy land, stop
      if (t == 0) {
        atomicExch(a.flag, 1);
        tc05::mbar_wait(full, phase);
      }
      return;
    }
    if constexpr (B > 1) {  // (B)
      for (int it = t; it < G::ITEMS_B; it += T) {
        const int ka = it % A, rr = it / A, c = rr % C, b = rr / C;
        float2* row = X + b * G::SB + ka * G::PR + c;
        float2 w[B];
#pragma unroll
        for (int nb = 0; nb < B; ++nb) w[nb] = row[C * nb];
        ct::RD<float2, B, -1>::run(w);
#pragma unroll
        for (int kb = 0; kb < B; ++kb) row[C * kb] = (kb && c) ? ct::mul(w[kb], tw[c * kb]) : w[kb];
      }
      __syncthreads();
    }
    if constexpr (C > 1) {  // (C)
      for (int it = t; it < G::ITEMS_C; it += T) {
        const int ka = it % A, rr = it / A, kb = rr % B, b = rr / B;
        float2* row = X + b * G::SB + ka * G::PR + C * kb;
        float2 u[C];
#pragma unroll
        for (int c = 0; c < C; ++c) u[c] = row[c];
        ct::RD<float2, C, -1>::run(u);
#pragma unroll
        for (int kc = 0; kc < C; ++kc) row[kc] = u[kc];
      }
      __syncthreads();
    }
    // fold: lanes 2i and 2i+1 take degree m's real (even and odd parity) and
    // imaginary rows, so each store instruction fills whole 32-byte sectors
    const int cb = k / PLANES, row = 2 * (k % PLANES), kt = p0 / TK, kk0 = p0 % TK;
    const int im = t & 1;
    auto zpos = [&](int m) {
      const int qq = m / A;
      return (m % A) * G::PR + C * (qq % B) + qq / B;
    };
    for (int m = t >> 1; m <= a.lmax; m += T / 2) {
      const int pz = zpos(m), pc = zpos(m == 0 ? 0 : N - m);
      float ev[NP], od[NP];
#pragma unroll
      for (int b = 0; b < NP; ++b) {
        const float2 Z = X[b * G::SB + pz], Zc = X[b * G::SB + pc];
        // F(ring) = (Z + conj Z(-m))/2, F(mirror) = -i (Z - conj Z(-m))/2
        const float fr = im ? 0.5f * (Z.y - Zc.y) : 0.5f * (Z.x + Zc.x);
        const float fm = im ? -0.5f * (Z.x - Zc.x) : 0.5f * (Z.y + Zc.y);
        ev[b] = (fr + fm) * W[b];
        od[b] = (fr - fm) * W[b];
      }
      store_tile_row<NP>(a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 0, cb, kt) * TILE_HALVES, row + im, kk0, ev);
      store_tile_row<NP>(a.tiles + ana_tile(a.lmax, a.ncb, a.nkn, f, m, 1, cb, kt) * TILE_HALVES, row + im, kk0, od);
    }
    // the image is refilled by the bulk copy (async proxy) after this barrier
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
  }
}

// FC-Gram continuation of physical planes (FP64), one grid point per
// thread: out(ii) = sum_jj dir(ii,jj) f(N-d+jj) + dir(C-1-ii,jj) f(d-1-jj),
// the same operator the z transform applies to spectral planes
// (fcgram_mod.f90 / pseudospec continuation step), here before the
// analysis so that its round-off is not amplified.
template <typename GT>
__global__ void cont_phys_kernel(const GT* __restrict__ f0, const GT* __restrict__ f1, const GT* __restrict__ f2,
                                 GT* out, const double* __restrict__ dir, int C, int d, int N, size_t npts) {
  const int f = blockIdx.y;
  const GT* in = f == 0 ? f0 : (f == 1 ? f1 : f2);
  GT* o = out + (size_t)f * C * npts;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < npts; x += (size_t)gridDim.x * blockDim.x) {
    double hi[32], lo[32];
#pragma unroll 8
    for (int jj = 0; jj < d; ++jj) {
      hi[jj] = (double)__ldg(in + (size_t)(N - d + jj) * npts + x);
      lo[jj] = (double)__ldg(in + (size_t)(d - 1 - jj) * npts + x);
    }
    for (int ii = 0; ii < C; ++ii) {
      double acc = 0.0;
      for (int jj = 0; jj < d; ++jj)
        acc = (acc + __ldg(dir + ii + C * jj) * hi[jj]) + __ldg(dir + (C - 1 - ii) + C * jj) * lo[jj];
      o[(size_t)ii * npts + x] = (GT)acc;
    }
  }
}

// The same continuation with the order d fixed at compile time: the matrix
// in shared memory (read as a broadcast), the 2 d input values of each point
// in registers, two points per thread (each matrix entry read once for both);
// every output is summed in the same order as above.
template <int D, typename GT>
__global__ void __launch_bounds__(256) cont_phys_d(const GT* __restrict__ f0, const GT* __restrict__ f1,
                                                   const GT* __restrict__ f2, GT* out,
                                                   const double* __restrict__ dir, int C, int N, size_t npts) {
  extern __shared__ double sdir[];  // dir(ii, jj) at ii + C jj
  for (int i = threadIdx.x; i < C * D; i += blockDim.x) sdir[i] = __ldg(dir + i);
  __syncthreads();
  const int f = blockIdx.y;
  const GT* in = f == 0 ? f0 : (f == 1 ? f1 : f2);
  GT* o = out + (size_t)f * C * npts;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < npts; x += 2 * stride) {
    const size_t x2 = x + stride;
    const bool two = x2 < npts;
    double hi0[D], lo0[D], hi1[D], lo1[D];
#pragma unroll
    for (int jj = 0; jj < D; ++jj) {
      hi0[jj] = (double)__ldg(in + (size_t)(N - D + jj) * npts + x);
      lo0[jj] = (double)__ldg(in + (size_t)(D - 1 - jj) * npts + x);
      hi1[jj] = two ? (double)__ldg(in + (size_t)(N - D + jj) * npts + x2) : 0.0;
      lo1[jj] = two ? (double)__ldg(in + (size_t)(D - 1 - jj) * npts + x2) : 0.0;
    }
    for (int ii = 0; ii < C; ++ii) {
      double a0 = 0.0, a1 = 0.0;
#pragma unroll
      for (int jj = 0; jj < D; ++jj) {
        const double w1 = sdir[ii + C * jj], w2 = sdir[(C - 1 - ii) + C * jj];
        a0 = (a0 + w1 * hi0[jj]) + w2 * lo0[jj];
        a1 = (a1 + w1 * hi1[jj]) + w2 * lo1[jj];
      }
      o[(size_t)ii * npts + x] = (GT)a0;
      if (two) o[(size_t)ii * npts + x2] = (GT)a1;
    }
  }
}

// Spectra (lm order) -> synthesis data tiles.  Thread c of block (m, k, field)
// takes l = m + 16c .. m + 16c + 15, i.e. 8 values of each parity (q = 8c ..
// 8c + 7), and writes one row chunk per parity and component; values past
// lmax are written as zeros.
__global__ void spec_to_tiles(const double2* __restrict__ in, const double2* __restrict__ in2,
                              __nv_bfloat16* tiles, size_t tfield, const long long* __restrict__ toff,
                              const int* __restrict__ mbase, int lmax, int nlm) {
  const int m = blockIdx.x, k = blockIdx.y, f = blockIdx.z;
  const double2* src = (f ? in2 : in) + (size_t)k * nlm + mbase[m] - m;
  __nv_bfloat16* T = tiles + (size_t)f * tfield;
  const int cb = k / PLANES, row = 2 * (k % PLANES);
  const int nc = ntiles_of(lmax, m, 0) * (TK / 8);  // chunks of 8 q (parity 0 has the most rows)
  for (int c = threadIdx.x; c < nc; c += blockDim.x) {
    double2 v[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int l = m + 16 * c + j;
      v[j] = l <= lmax ? __ldg(src + l) : make_double2(0.0, 0.0);
    }
    const int kt = c / (TK / 8), kk0 = (c % (TK / 8)) * 8;
#pragma unroll
    for (int par = 0; par < 2; ++par) {
      if (kt >= ntiles_of(lmax, m, par)) continue;
      float re[8], im[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        re[j] = (float)v[2 * j + par].x;
        im[j] = (float)v[2 * j + par].y;
      }
      __nv_bfloat16* t = T + syn_tile(toff, lmax, m, par, cb, kt) * TILE_HALVES;
      store_tile_row<8>(t, row, kk0, re);
      store_tile_row<8>(t, row + 1, kk0, im);
    }
  }
}

// z inverse (fftp1d_complex_to_real_z, src/sphp/sphp_sca.F90:495-530, sign
// +1) of the 16 columns l = m + 16c .. m + 16c + 15 of one m, written
// straight into the synthesis tiles the way spec_to_tiles writes them: one
// CTA per (m, c) item loads the columns in digit-reversed row order (zero
// past lmax), transforms them in shared memory by the passes of
// zfft_kernel<Z_INV> (the same operations per column, so the same bits), and
// each plane's 8 values of a parity go out as one 16-byte row chunk per piece.
// The column stride of 17 slots keeps the read-out conflict-free.  It saves
// the z inverse's write of the spectra and spec_to_tiles' read of them.
constexpr int ZT_COLS = 16, ZT_PITCH = 17, ZT_THREADS = 256;

struct ZtArgs {
  const void* in;  // double2, or float2 for the single-precision entry points
  __nv_bfloat16* tiles;
  const long long* toff;
  const int* mbase;
  const int2* items;
  int lmax, nlm, nz;
  const int* rev;
  const double2* twp;
  const double2* tw;  // W_nz^e, e < nz (the two-step split)
  double2* out;       // also the radial-space spectra, same layout as in (may be in); nullable
  // the radial derivative of those (derivr(., 1, 'r')), when the kernel is
  // instantiated for it: output, FC-Gram operator, i kz
  double2* dout;
  const double* dir;
  int C, d, N;
  const double2* kfac;
};

__device__ __forceinline__ void cp_async16zf(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}

// three CTAs per SM (80 registers); the derivative at nz 256 takes two
// (its 16-point steps spill heavily at 80)
template <int NZ, typename TI, bool DER = false>
__global__ void __launch_bounds__(ZT_THREADS, (DER && NZ >= 256) ? 2 : 3) zinv_tiles(ZtArgs a) {
  extern __shared__ double2 zs[];  // element e of column j at j + ZT_PITCH e
  const int2 it = a.items[blockIdx.x];
  const int m = it.x, c = it.y, t = threadIdx.x;
  const TI* base = static_cast<const TI*>(a.in) + (a.mbase[m] - m);  // column l of row r at base[r nlm + l]
  for (int idx = t; idx < NZ * ZT_COLS; idx += ZT_THREADS) {
    const int r = idx / ZT_COLS, j = idx % ZT_COLS, l = m + ZT_COLS * c + j;
    const bool in = l <= a.lmax;
    // the radix passes take the input digit-reversed; the two-step split in natural order
    double2* dst = zs + j + ZT_PITCH * (ct::split2_r1(NZ) > 0 ? r : __ldg(a.rev + r));
    if constexpr (sizeof(TI) == sizeof(double2)) {
      cp_async16zf(dst, in ? base + (size_t)r * a.nlm + l : a.in, in ? 16 : 0);
    } else {  // float input, widened
      const TI v = in ? __ldg(base + (size_t)r * a.nlm + l) : TI{0.f, 0.f};
      *dst = make_double2((double)v.x, (double)v.y);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  const ct::Geo<NZ, 0, false> g{ZT_COLS, 1, ZT_PITCH};
  if constexpr (ct::split2_r1(NZ) > 0 && ct::split2_tpc(NZ) * ZT_COLS <= ZT_THREADS) {
    // the arithmetic of the plain z inverse (zfft2_kernel), so that both
    // inverse paths agree bit for bit
    constexpr int R1 = ct::split2_r1(NZ), R2 = NZ / R1, TPC = ct::split2_tpc(NZ);
    const int j = t % ZT_COLS, h = t / ZT_COLS;
    if (h < TPC) ct::dft2_step1<R1, R2, 1>(zs + j, ZT_PITCH, h, a.tw);
    __syncthreads();
    double2 v[R2];
    if (h < TPC) ct::dft2_step2<R1, R2, 1>(zs + j, ZT_PITCH, h, v);
    __syncthreads();
    if (h < R1) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) zs[j + ZT_PITCH * (h + R1 * k2)] = v[k2];
    }
    __syncthreads();
  } else {
    ct::dit<double2, NZ, NZ>(zs, g, a.twp, +1);
  }
  if (a.out) {  // the z inverse itself, in the spectra's layout (rows of 16 consecutive lm)
    for (int idx = t; idx < NZ * ZT_COLS; idx += ZT_THREADS) {
      const int r = idx / ZT_COLS, j = idx % ZT_COLS, l = m + ZT_COLS * c + j;
      if (l <= a.lmax) a.out[(size_t)(a.mbase[m] - m) + (size_t)r * a.nlm + l] = zs[j + ZT_PITCH * r];
    }
  }
  const int kt = c / (TK / 8), kk0 = (c % (TK / 8)) * 8;
  for (int w = t; w < NZ * 2; w += ZT_THREADS) {
    const int k = w >> 1, par = w & 1;
    if (kt >= ntiles_of(a.lmax, m, par)) continue;
    float re[8], im[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double2 v = zs[2 * i + par + ZT_PITCH * k];
      re[i] = (float)v.x;
      im[i] = (float)v.y;
    }
    __nv_bfloat16* tt = a.tiles + syn_tile(a.toff, a.lmax, m, par, k / PLANES, kt) * TILE_HALVES;
    store_tile_row<8>(tt, 2 * (k % PLANES), kk0, re);
    store_tile_row<8>(tt, 2 * (k % PLANES) + 1, kk0, im);
  }
  if constexpr (DER && ct::split2_r1(NZ) > 0 && ct::split2_tpc(NZ) * ZT_COLS <= ZT_THREADS) {
    // derivr(., 1, 'r') of the radial-space columns, the arithmetic of
    // zfft2_kernel<Z_DERIV>: continuation of the last C rows, the forward
    // split, / nz times i kz, the inverse split
    constexpr int R1 = ct::split2_r1(NZ), R2 = NZ / R1, TPC = ct::split2_tpc(NZ);
    const int j = t % ZT_COLS, h = t / ZT_COLS;
    double2* col = zs + j;
    __syncthreads();  // every read of the radial values above is done
    if (a.C > 0) {
      for (int idx = t; idx < a.C * ZT_COLS; idx += ZT_THREADS) {
        const int ii = idx / ZT_COLS, jj = idx % ZT_COLS;
        zs[jj + ZT_PITCH * (a.N + ii)] = fc_cont_elem(a.dir, a.C, a.d, a.N, ii, zs + jj, ZT_PITCH);
      }
      __syncthreads();
    }
    if (h < TPC) ct::dft2_step1<R1, R2, -1>(col, ZT_PITCH, h, a.tw);
    __syncthreads();
    double2 v[R2];
    if (h < TPC) ct::dft2_step2<R1, R2, -1>(col, ZT_PITCH, h, v);
    __syncthreads();
    if (h < R1) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const int k = h + R1 * k2;
        col[k * ZT_PITCH] = cmul(a.kfac[k], div_nz(v[k2], NZ));
      }
    }
    __syncthreads();
    if (h < TPC) ct::dft2_step1<R1, R2, 1>(col, ZT_PITCH, h, a.tw);
    __syncthreads();
    if (h < TPC) ct::dft2_step2<R1, R2, 1>(col, ZT_PITCH, h, v);
    const int l = m + ZT_COLS * c + j;
    if (h < R1 && l <= a.lmax) {
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2)
        a.dout[(size_t)(a.mbase[m] - m) + (size_t)(h + R1 * k2) * a.nlm + l] = v[k2];
    }
  }
}

#define ZT_SIZES(X) X(16) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(512)

// ---------------------------------------------------------------- host tables
__host__ inline uint16_t bf16_bits(double x) {
  // x already rounded to 8 significant bits: exact in fp32 and bf16
  const float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (uint16_t)(u >> 16);
}
// round to 8 significant bits, nearest even; tiny values flush to zero
__host__ inline double round8(double x) {
  if (!(std::fabs(x) >= 0x1p-110)) return 0.0;
  int e;
  const double m = std::frexp(x, &e);  // |m| in [0.5, 1)
  return std::ldexp(std::nearbyint(std::ldexp(m, 8)), e - 8);
}

// Builds one work set: items (heaviest first) and their bf16 table blocks
// (per K step: [hi | mid | lo] x nr rows x 32, core-matrix K-major).
// value(it, row, kt, kk) is the FP64 table entry of MMA row `row`, K element
// kt*32+kk.  An item with out = 1 right after its out = 0 twin shares the
// twin's blocks.
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
    it.tscale = 1.f;
    total += (size_t)it.nk * NPIECE * it.nr * TK;
    own.push_back((int)items.size());
    items.push_back(it);
    if (h + 1 < (int)raw.size() && is_twin(h + 1)) {
      TcItem tw = raw[h + 1];
      tw.boff = it.boff;
      tw.tscale = 1.f;
      items.push_back(tw);
    }
  }
  std::vector<uint16_t> hb(total, 0);
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::thread> th;
  for (int t = 0; t < nth; ++t)
    th.emplace_back([&, t]() {
      for (size_t x = t; x < own.size(); x += nth) {
        const TcItem& it = items[own[x]];
        for (int kt = 0; kt < it.nk; ++kt) {
          uint16_t* blk = hb.data() + it.boff + (size_t)kt * NPIECE * it.nr * TK;
          for (int r = 0; r < it.nvalid; ++r)
            for (int kk = 0; kk < TK; ++kk) {
              const double v = value(it, r, kt, kk);
              const double h = round8(v), md = round8(v - h), lo = round8(v - h - md);
              const uint32_t off = tc05::kmaj_off(r, kk, it.nr) / 2;
              blk[off] = bf16_bits(h);
              blk[(size_t)it.nr * TK + off] = bf16_bits(md);
              blk[(size_t)2 * it.nr * TK + off] = bf16_bits(lo);
            }
        }
      }
    });
  for (auto& x : th) x.join();
  set.nitems = (int)items.size();
  set.nhalves = total;
  if (cudaMalloc((void**)&set.items, std::max<size_t>(1, items.size()) * sizeof(TcItem)) != cudaSuccess)
    return SPH_ENOMEM;
  if (cudaMalloc((void**)&set.blocks, std::max<size_t>(1, total) * 2) != cudaSuccess) return SPH_ENOMEM;
  if (!items.empty() &&
      cudaMemcpy(set.items, items.data(), items.size() * sizeof(TcItem), cudaMemcpyHostToDevice) != cudaSuccess)
    return SPH_ECUDA;
  if (total && cudaMemcpy(set.blocks, hb.data(), total * 2, cudaMemcpyHostToDevice) != cudaSuccess)
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

// The tensor-core work sets (items and table blocks) of a mixed plan from
// its host Legendre tables [nlm][ldn]; scalar and/or vector sets.
static int build_sets(sph_plan* p, const std::vector<double>& hP, const std::vector<double>& hdP,
                      const std::vector<double>& hmPs, bool scalar, bool vector) {
  const int lmax = p->lmax, ldn = p->ldn, n2 = p->nlat2, nkn = p->nkn;
  auto lm = [&](int l, int m) { return (size_t)p->mbase[m] + (l - m); };
  auto rows = [&](int m, int par) { return rows_of(lmax, m, par); };

  // analysis: rows = l of one parity, K = nodes (vector: [dP . fold 1-p | mPs . fold p])
  auto ana_items = [&](bool vec) {
    return [&, vec](std::vector<TcItem>& v) {
      const int NR = vec ? NR_V : (p->tile_nr ? p->tile_nr : NR_S);
      for (int m = 0; m <= lmax; ++m)
        for (int par = 0; par < 2; ++par) {
          const int L = rows(m, par);
          for (int r0 = 0; r0 < L; r0 += NR) {
            TcItem it = {};
            it.m = m;
            it.par = par;
            it.r0 = r0;
            it.nvalid = std::min(NR, L - r0);
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
  // synthesis: rows = nodes, K = l of one parity (vector: [dP . l of 1-q | mPs . l of q])
  auto syn_items = [&](bool vec) {
    return [&, vec](std::vector<TcItem>& v) {
      const int NR = vec ? NR_V : (p->tile_nr ? p->tile_nr : NR_S);
      for (int m = 0; m <= lmax; ++m)
        for (int q = 0; q < 2; ++q) {
          for (int i0 = 0; i0 < n2; i0 += NR) {
            TcItem it = {};
            it.m = m;
            it.par = q;
            it.r0 = i0;
            it.nvalid = std::min(NR, n2 - i0);
            it.nr = round16(it.nvalid);
            if (vec) {
              it.nk1 = ntiles_of(lmax, m, 1 - q);
              it.nk = it.nk1 + ntiles_of(lmax, m, q);
            } else {
              it.nk = ntiles_of(lmax, m, q);  // 0: the fold is written as zeros
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

  int rc = SPH_OK;
  if (scalar) rc = build_set(p->tcAS, ana_items(false), ana_val(false));
  if (rc == SPH_OK && vector) rc = build_set(p->tcAV, ana_items(true), ana_val(true));
  if (rc == SPH_OK && scalar) rc = build_set(p->tcSS, syn_items(false), syn_val(false));
  if (rc == SPH_OK && vector) rc = build_set(p->tcSV, syn_items(true), syn_val(true));
  return rc;
}

namespace {
size_t phi2_plane_floats(int nphi, int nlat2);
}  // namespace

int mixed_setup(sph_plan* p, const std::vector<double>& hP, const std::vector<double>& hdP,
                const std::vector<double>& hmPs) {
  const int lmax = p->lmax, n2 = p->nlat2;
  p->ldn8 = (n2 + 7) & ~7;
  p->G32field = (size_t)(lmax + 1) * 2 * p->nz * p->ldn8;
  if (p->G32field * sizeof(float2) > p->Gfield * sizeof(double2)) return SPH_EINVAL;
  const int nkn = (n2 + TK - 1) / TK;  // K tiles over the nodes
  const int ncb = (p->nz + PLANES - 1) / PLANES;
  p->nkn = nkn;
  int rc = build_sets(p, hP, hdP, hmPs, true, true);
  // data tiles: analysis [3 fields][m][fold][cb][nkn]; synthesis 2 fields of [m][par][cb][ntiles]
  std::vector<long long> off(2 * (lmax + 1));
  long long nsyn = 0;
  for (int m = 0; m <= lmax; ++m)
    for (int par = 0; par < 2; ++par) {
      off[2 * m + par] = nsyn;
      nsyn += (long long)ncb * ntiles_of(lmax, m, par);
    }
  p->Tsynfield = (size_t)nsyn * TILE_HALVES;
  if (rc == SPH_OK && cudaMalloc((void**)&p->d_toff, off.size() * sizeof(long long)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK &&
      cudaMemcpy(p->d_toff, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice) != cudaSuccess)
    rc = SPH_ECUDA;
  if (rc == SPH_OK) rc = mixed_alloc_scratch(p);
  int dev = 0;
  if (rc == SPH_OK && (cudaGetDevice(&dev) != cudaSuccess ||
                       cudaDeviceGetAttribute(&p->nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess))
    rc = SPH_ECUDA;
  return rc;
}

// The per-plan buffers: analysis and synthesis data tiles, the physically
// continued planes, the two-pass phi images and the status word.
int mixed_alloc_scratch(sph_plan* p) {
  const int lmax = p->lmax, ncb = (p->nz + PLANES - 1) / PLANES;
  const size_t nana = ana_tile(lmax, ncb, p->nkn, SPH_MAX_FIELDS, 0, 0, 0, 0) * TILE_HALVES;
  const size_t bytes_ana = nana * 2, bytes_syn = (size_t)SPH_MAX_FIELDS * p->Tsynfield * 2;
  int rc = SPH_OK;
  if (rc == SPH_OK && cudaMalloc((void**)&p->Tana, bytes_ana) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(p->Tana, 0, bytes_ana) != cudaSuccess) rc = SPH_ECUDA;
  if (rc == SPH_OK && cudaMalloc((void**)&p->Tsyn, std::max<size_t>(16, bytes_syn)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(p->Tsyn, 0, std::max<size_t>(16, bytes_syn)) != cudaSuccess) rc = SPH_ECUDA;
  if (rc == SPH_OK && p->C > 0 && p->d <= 32 &&
      cudaMalloc((void**)&p->contg, (size_t)SPH_MAX_FIELDS * p->C * p->nphi * p->nlat * sizeof(double)) !=
          cudaSuccess)
    rc = SPH_ENOMEM;
  if (rc == SPH_OK) {
    const size_t per = phi2_plane_floats(p->nphi, p->nlat2);
    if (per) {
      p->phi2_planes = std::min(PHI2_BATCH, p->nz * SPH_MAX_FIELDS);
      if (cudaMalloc((void**)&p->phi2, per * p->phi2_planes * sizeof(float2)) != cudaSuccess) rc = SPH_ENOMEM;
    }
  }
  if (rc == SPH_OK && cudaMalloc((void**)&p->dflag, sizeof(int)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(p->dflag, 0, sizeof(int)) != cudaSuccess) rc = SPH_ECUDA;
  if (rc == SPH_OK) {  // (m, 16-degree chunk) items of the fused z inverse
    std::vector<int2> items;
    for (int m = 0; m <= lmax; ++m)
      for (int c = 0; c * ZT_COLS <= lmax - m; ++c) items.push_back(make_int2(m, c));
    p->nztitems = (int)items.size();
    if (cudaMalloc((void**)&p->d_ztitems, items.size() * sizeof(int2)) != cudaSuccess) rc = SPH_ENOMEM;
    else if (cudaMemcpy(p->d_ztitems, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice) !=
             cudaSuccess)
      rc = SPH_ECUDA;
  }
  return rc;
}

// Rebuilds the scalar work sets with p->tile_nr rows per item, from the
// Legendre tables read back from the device.
int mixed_retile(sph_plan* p) {
  const size_t n = (size_t)p->nlm * p->ldn;
  std::vector<double> hP(n);
  SPH_CUDA_OK(cudaDeviceSynchronize());
  SPH_CUDA_OK(cudaMemcpy(hP.data(), p->P, n * sizeof(double), cudaMemcpyDeviceToHost));
  for (TcSet* s : {&p->tcAS, &p->tcSS}) {
    if (s->items) cudaFree(s->items);
    if (s->blocks) cudaFree(s->blocks);
    *s = TcSet();
  }
  const std::vector<double> none;
  return build_sets(p, hP, none, none, true, false);
}

void mixed_free_tables(sph_plan* p) {
  for (TcSet* s : {&p->tcAS, &p->tcAV, &p->tcSS, &p->tcSV}) {
    if (s->items) cudaFree(s->items);
    if (s->blocks) cudaFree(s->blocks);
    s->items = nullptr;
    s->blocks = nullptr;
  }
  if (p->d_toff) cudaFree(p->d_toff);
  p->d_toff = nullptr;
}

void mixed_free_scratch(sph_plan* p) {
  void* ptrs[] = {p->dflag, p->Tana, p->Tsyn, p->contg, p->phi2, p->d_ztitems};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  p->d_ztitems = nullptr;
  p->nztitems = 0;
  p->phi2 = nullptr;
  p->phi2_planes = 0;
  p->contg = nullptr;
  p->dflag = nullptr;
  p->Tana = nullptr;
  p->Tsyn = nullptr;
}

int mixed_status(const sph_plan* p) {
  int f = 0;
  if (p->dflag && cudaMemcpy(&f, p->dflag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SPH_ECUDA;
  return f ? SPH_ETIMEDOUT : SPH_OK;
}

namespace {

TcArgs tc_args(const sph_plan* p) {
  TcArgs a = {};
  a.G32w = reinterpret_cast<float2*>(p->G);
  a.G32field = p->G32field;
  a.toff = p->d_toff;
  a.tfield = p->Tsynfield;
  a.mbase = p->d_mbase;
  a.flag = p->dflag;
  a.lmax = p->lmax;
  a.nz = p->nz;
  a.nlm = p->nlm;
  a.ldn8 = p->ldn8;
  a.nkn = p->nkn;
  a.ncb = (p->nz + PLANES - 1) / PLANES;
  return a;
}

template <int MODE, bool G>
bool tc_attr() {
  static DeviceOnce once;
  return once.run([] {
    return cudaFuncSetAttribute(tc_gemm<MODE, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM) ==
           cudaSuccess;
  });
}

template <int MODE>
int run_tc(const sph_plan* p, const TcSet& set, TcArgs a, cudaStream_t st) {
  if (!tc_attr<MODE, false>()) return SPH_ECUDA;
  const long long nunits = (long long)set.nitems * a.ncb;
  if (nunits == 0) return SPH_OK;
  if (nunits > (1ll << 30)) return SPH_EINVAL;
  a.items = set.items;
  a.blocks = reinterpret_cast<const __nv_bfloat16*>(set.blocks);
  a.nunits = (int)nunits;
  TcLaunch L = {};
  L.one = a;
  L.total = (int)nunits;
  L.flag = p->dflag;
  const int grid = (int)std::min<long long>(nunits, std::max(1, p->nsm));
  tc_gemm<MODE, false><<<grid, TC_THREADS, TC_SMEM, st>>>(L);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

int phi_pairs(const sph_plan* p) {
  if (p->tile_np) return p->tile_np;
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

template <typename K>
int run_phi4(K kernel, const Phi32Args& a, dim3 grid, int threads, size_t smem, cudaStream_t st) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
      cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
    return SPH_ECUDA;
  kernel<<<grid, threads, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}

template <int N, int NP, bool FWD, typename GT>
int phi4_np(const Phi32Args& a, dim3 grid, cudaStream_t st) {
  static_assert(FWD, "the four-step form is forward only");
  using C = P4<N, NP>;
  return run_phi4(phi4_fwd32<N, NP, GT>, a, grid, C::THREADS, C::SMEM_FWD, st);
}

template <int N, bool FWD, typename GT>
int phi32_n(const Phi32Args& a, dim3 grid, size_t smem, cudaStream_t st) {
  // the four-step form for the forward transform; the inverse keeps the
  // shared-memory passes (more resident warps hide its grid stores better)
  if constexpr (FWD && N <= 1536) {
    if (a.tw1 && a.tw2) {
      switch (a.NP) {
        case 8: return phi4_np<N, 8, FWD, GT>(a, grid, st);
        case 4: return phi4_np<N, 4, FWD, GT>(a, grid, st);
        case 2: return phi4_np<N, 2, FWD, GT>(a, grid, st);
        case 1: return phi4_np<N, 1, FWD, GT>(a, grid, st);
      }
    }
  }
  switch (a.NP) {
    case 8:
      if constexpr (8 * N <= PMAXC)
        return run_phi(FWD ? phi_fwd32<N, 8, GT> : phi_inv32<N, 8, GT>, a, grid, smem, st);
      break;
    case 4:
      if constexpr (4 * N <= PMAXC)
        return run_phi(FWD ? phi_fwd32<N, 4, GT> : phi_inv32<N, 4, GT>, a, grid, smem, st);
      break;
    case 2:
      if constexpr (2 * N <= PMAXC)
        return run_phi(FWD ? phi_fwd32<N, 2, GT> : phi_inv32<N, 2, GT>, a, grid, smem, st);
      break;
    case 1: return run_phi(FWD ? phi_fwd32<N, 1, GT> : phi_inv32<N, 1, GT>, a, grid, smem, st);
  }
  return SPH_EINVAL;
}

template <bool FWD, typename GT>
int phi32_dispatch(const sph_plan* p, const Phi32Args& a, dim3 grid, size_t smem, cudaStream_t st) {
  switch (p->nphi) {
#define CASE(n) \
  case n: return phi32_n<n, FWD, GT>(a, grid, smem, st);
    PHI32_SIZES(CASE)
#undef CASE
  }
  return SPH_EINVAL;
}

constexpr int PHI3_UNSUPPORTED = 1000;
// 2D view [rows][nlat] of a grid array (FP64 or float), box NP x box_rows;
// unsupported where a box row is not a multiple of 16 bytes (float: NP < 4)
template <typename GT>
int phi3_map(CUtensorMap* map, const void* base, int nlat, int rows, int np, int box_rows) {
  return tma::grid_map(map, static_cast<const GT*>(base), nlat, rows, np, box_rows) ? SPH_OK : PHI3_UNSUPPORTED;
}

// three-step kernels: which (N, NP) fit (one step-A item per thread, both
// staged forward tiles and the twiddles in shared memory)
constexpr size_t PHI3_SMEM_MAX = 220 * 1024;
template <int N, int NP>
constexpr bool phi3_ok() {
  return N % 16 == 0 && N >= 48 && NP * (N / 16) <= 1024 &&
         (size_t)2 * N * 2 * NP * sizeof(double) + (size_t)N * sizeof(float2) <= PHI3_SMEM_MAX;
}

// the inverse holds one staged coefficient tile (for the largest lmax,
// N/2 - 1) instead of two forward tiles, so it takes 8 ring pairs at
// lengths whose forward does not: 32-byte runs of float grid rows, 64-byte
// runs of FP64 ones
template <int N, int NP>
constexpr bool phi3_inv_ok() {
  if constexpr (N % 16 != 0 || N < 48 || NP * (N / 16) > 1024) {
    return false;
  } else {
    return P3<N, NP>::XBYTES + (size_t)N * sizeof(float2) + (size_t)N * NP * sizeof(float2) <= PHI3_SMEM_MAX;
  }
}
template <int N, int NP, bool FWD>
constexpr bool phi3_fits() {
  if constexpr (FWD) {
    return phi3_ok<N, NP>();
  } else {
    return phi3_inv_ok<N, NP>();
  }
}

template <int N, int NP, bool FWD, typename GT>
int phi3_run(const sph_plan* p, const Phi32Args& a, int nfields, cudaStream_t st) {
  if constexpr (!phi3_fits<N, NP, FWD>()) {
    return PHI3_UNSUPPORTED;
  } else {
    using G = P3<N, NP>;
    const size_t smem = FWD ? G::SMEM_F : G::smem_inv(p->lmax);
    if (smem > PHI3_SMEM_MAX) return PHI3_UNSUPPORTED;
    const long long ntiles = (long long)(p->nlat2 / NP) * p->nz * nfields;
    if (ntiles == 0) return SPH_OK;
    if (ntiles > (1ll << 30)) return PHI3_UNSUPPORTED;
    int occ = 0;
    if constexpr (FWD) {
      Phi3Maps maps;
      if (!a.flag) return PHI3_UNSUPPORTED;
      for (int f = 0; f < nfields; ++f) {
        const int rc = phi3_map<GT>(&maps.lo[f], a.gin[f], p->nlat, N * a.ksplit, NP, phi3_box_rows<N>());
        if (rc != SPH_OK) return rc;
        const bool hi = a.ksplit < p->nz;
        const int rc2 = phi3_map<GT>(&maps.hi[f], hi ? a.gin_hi[f] : a.gin[f], p->nlat,
                                     N * (hi ? p->nz - a.ksplit : a.ksplit), NP, phi3_box_rows<N>());
        if (rc2 != SPH_OK) return rc2;
      }
      for (int f = nfields; f < SPH_MAX_FIELDS; ++f) maps.lo[f] = maps.hi[f] = maps.lo[0];
      auto kern = phi3_fwd32<N, NP, GT>;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, G::THREADS, smem) != cudaSuccess)
        return SPH_ECUDA;
      const int grid = (int)std::min<long long>(ntiles, (long long)std::max(1, occ) * std::max(1, p->nsm));
      kern<<<grid, G::THREADS, smem, st>>>(a, (int)ntiles, maps);
    } else {
      auto kern = phi3_inv32<N, NP, GT>;
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
          cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, G::THREADS, smem) != cudaSuccess)
        return SPH_ECUDA;
      const int grid = (int)std::min<long long>(ntiles, (long long)std::max(1, occ) * std::max(1, p->nsm));
      kern<<<grid, G::THREADS, smem, st>>>(a, (int)ntiles);
    }
    SPH_LAUNCH_OK();
    return SPH_OK;
  }
}

// two-pass forward: lengths whose 8-ring-pair tile fits shared memory only once
template <int N>
constexpr bool phi2_ok() {
  if constexpr (N % 256 != 0 || N < 768 || phi3_ok<N, 8>()) {
    return false;
  } else {
    return phi2_smem<N>() <= PHI3_SMEM_MAX;
  }
}

template <int N, typename GT>
int phi2_run(const sph_plan* p, const Phi32Args& a, int nfields, cudaStream_t st) {
  if constexpr (!phi2_ok<N>()) {
    return PHI3_UNSUPPORTED;
  } else {
    using G = P3<N, PHI2_NP>;
    if (!p->phi2 || p->phi2_planes < 1 || p->nlat2 % PHI2_PB || !a.flag) return PHI3_UNSUPPORTED;
    constexpr int T = PHI2_T;
    const size_t smem = phi2_smem<N>();
    auto kb = phi2b_fwd32<N>;
    int occ = 0;
    if (cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        cudaFuncSetAttribute(kb, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kb, T, smem) != cudaSuccess)
      return SPH_ECUDA;
    const int nq = p->nz * nfields, ngroups = p->nlat2 / PHI2_NP;
    for (int q0 = 0; q0 < nq; q0 += p->phi2_planes) {
      const int nb = std::min(p->phi2_planes, nq - q0);
      phi2a_fwd32<N, GT><<<dim3(p->nlat2 / PHI2_PB, G::M / PHI2_NMC, nb), PHI2_PB * PHI2_NMC, 0, st>>>(a, p->phi2,
                                                                                                      q0);
      SPH_LAUNCH_OK();
      const int ntiles = nb * ngroups;
      const int grid = std::min(ntiles, std::max(1, occ) * std::max(1, p->nsm));
      kb<<<grid, T, smem, st>>>(a, p->phi2, q0, nb, ntiles);
      SPH_LAUNCH_OK();
    }
    return SPH_OK;
  }
}

template <typename GT>
int phi2_dispatch(const sph_plan* p, const Phi32Args& a, int nfields, cudaStream_t st) {
  switch (p->nphi) {
#define CASE(n) \
  case n: return phi2_run<n, GT>(p, a, nfields, st);
    PHI32_SIZES(CASE)
#undef CASE
  }
  return PHI3_UNSUPPORTED;
}

template <int N>
size_t phi2_plane_floats_n(int nlat2) {
  if constexpr (phi2_ok<N>())
    return (size_t)(nlat2 / PHI2_NP) * PHI2_NP * P3<N, PHI2_NP>::SB;
  else
    return 0;
}

// float2 values of one plane's tile images (0: the two-pass form does not apply)
size_t phi2_plane_floats(int nphi, int nlat2) {
  if (nlat2 % PHI2_PB) return 0;
  switch (nphi) {
#define CASE(n) \
  case n: return phi2_plane_floats_n<n>(nlat2);
    PHI32_SIZES(CASE)
#undef CASE
  }
  return 0;
}

// ring pairs per tile: the most that fit, at most the tuned ring_pairs
template <int N, bool FWD>
int phi3_pairs(const sph_plan* p) {
  const int cap = p->tile_np ? p->tile_np : 8;
  if (phi3_fits<N, 8, FWD>() && cap >= 8 && p->nlat2 % 8 == 0) return 8;
  if (phi3_fits<N, 4, FWD>() && cap >= 4 && p->nlat2 % 4 == 0) return 4;
  if (phi3_fits<N, 2, FWD>() && cap >= 2 && p->nlat2 % 2 == 0) return 2;
  return 0;
}

template <bool FWD, typename GT>
int phi3_dispatch(const sph_plan* p, const Phi32Args& a, int nfields, cudaStream_t st) {
  switch (p->nphi) {
#define CASE(n)                                                  \
  case n:                                                        \
    switch (phi3_pairs<n, FWD>(p)) {                             \
      case 8: return phi3_run<n, 8, FWD, GT>(p, a, nfields, st); \
      case 4: return phi3_run<n, 4, FWD, GT>(p, a, nfields, st); \
      case 2: return phi3_run<n, 2, FWD, GT>(p, a, nfields, st); \
    }                                                            \
    return PHI3_UNSUPPORTED;
    PHI32_SIZES(CASE)
#undef CASE
  }
  return PHI3_UNSUPPORTED;
}

Phi32Args phi32_args(const sph_plan* p) {
  Phi32Args a = {};
  a.tiles = reinterpret_cast<__nv_bfloat16*>(p->Tana);
  a.G32c = reinterpret_cast<const float2*>(p->G);
  a.G32field = p->G32field;
  a.nlat = p->nlat;
  a.ldn8 = p->ldn8;
  a.nz = p->nz;
  a.lmax = p->lmax;
  a.NP = phi_pairs(p);
  a.ncb = (p->nz + PLANES - 1) / PLANES;
  a.nkn = p->nkn;
  a.wfold = p->wfold;
  a.twp = p->fphi.twpf;
  a.ksplit = p->nz;
  a.tw1 = p->tw4f;
  a.tw2 = p->tw4f ? p->tw4f + p->tw4off : nullptr;
  a.twN = p->twphif;
  a.flag = p->dflag;
  return a;
}

}  // namespace

namespace {

template <typename GT>
int cont_phys_t(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st) {
  const size_t npts = (size_t)p->nphi * p->nlat;
  const GT* f[SPH_MAX_FIELDS];
  for (int i = 0; i < SPH_MAX_FIELDS; ++i) f[i] = static_cast<const GT*>(grids[i < nfields ? i : 0]);
  GT* out = reinterpret_cast<GT*>(p->contg);  // float planes use the first half of the FP64 buffer
  TimedLaunch tl(p, T_OPS, st);
  const int blocks = (int)std::min<size_t>((npts + 255) / 256, 148 * 8);
  const size_t smem = (size_t)p->C * p->d * sizeof(double);
  switch (p->d) {
#define CASE(D)                                                                                               \
  case D:                                                                                                     \
    cont_phys_d<D, GT><<<dim3(blocks, nfields), 256, smem, st>>>(f[0], f[1], f[2], out, p->d_dir, p->C, p->N, \
                                                                  npts);                                     \
    break;
    CASE(1) CASE(2) CASE(3) CASE(4) CASE(5) CASE(6) CASE(7) CASE(8)
#undef CASE
    default:
      cont_phys_kernel<GT><<<dim3(blocks, nfields), 256, 0, st>>>(f[0], f[1], f[2], out, p->d_dir, p->C, p->d,
                                                                  p->N, npts);
  }
  SPH_LAUNCH_OK();
  return SPH_OK;
}

template <typename GT>
int phi_fwd32_t(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st,
                const void* const* grids_hi) {
  Phi32Args a = phi32_args(p);
  for (int f = 0; f < nfields; ++f) a.gin[f] = grids[f];
  a.ksplit = p->nz;
  if (grids_hi) {
    a.ksplit = p->N;
    for (int f = 0; f < nfields; ++f) a.gin_hi[f] = grids_hi[f];
  }
  TimedLaunch tl(p, T_PHI_FWD, st);
  bool aligned = (p->nlat * sizeof(GT)) % 16 == 0;
  for (int f = 0; f < nfields; ++f)
    aligned = aligned && reinterpret_cast<uintptr_t>(a.gin[f]) % 16 == 0 &&
              (!grids_hi || reinterpret_cast<uintptr_t>(a.gin_hi[f]) % 16 == 0);
  {
    const int rc = phi2_dispatch<GT>(p, a, nfields, st);
    if (rc != PHI3_UNSUPPORTED) return rc;
  }
  if (aligned) {
    const int rc = phi3_dispatch<true, GT>(p, a, nfields, st);
    if (rc != PHI3_UNSUPPORTED) return rc;
  }
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  const size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(float2);
  return phi32_dispatch<true, GT>(p, a, grid, smem, st);
}

template <typename GT>
int phi_inv32_t(const sph_plan* p, void* const* grids, int nfields, cudaStream_t st) {
  Phi32Args a = phi32_args(p);
  for (int f = 0; f < nfields; ++f) a.gout[f] = grids[f];
  TimedLaunch tl(p, T_PHI_INV, st);
  const int rc = phi3_dispatch<false, GT>(p, a, nfields, st);
  if (rc != PHI3_UNSUPPORTED) return rc;
  dim3 grid(p->nlat2 / a.NP, p->nz, nfields);
  const size_t smem = (size_t)a.NP * seq_stride(p->nphi) * sizeof(float2);
  return phi32_dispatch<false, GT>(p, a, grid, smem, st);
}

}  // namespace

int launch_cont_phys_g(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st, bool f32) {
  if (!p->contg || p->C <= 0 || p->d > 32 || nfields < 1 || nfields > SPH_MAX_FIELDS) return SPH_EINVAL;
  return f32 ? cont_phys_t<float>(p, grids, nfields, st) : cont_phys_t<double>(p, grids, nfields, st);
}

int launch_phi_fwd32_g(const sph_plan* p, const void* const* grids, int nfields, cudaStream_t st,
                       const void* const* grids_hi, bool f32) {
  return f32 ? phi_fwd32_t<float>(p, grids, nfields, st, grids_hi)
             : phi_fwd32_t<double>(p, grids, nfields, st, grids_hi);
}

int launch_phi_inv32_g(const sph_plan* p, void* const* grids, int nfields, cudaStream_t st, bool f32) {
  return f32 ? phi_inv32_t<float>(p, grids, nfields, st) : phi_inv32_t<double>(p, grids, nfields, st);
}

int launch_cont_phys(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st) {
  const void* g[SPH_MAX_FIELDS] = {};
  for (int f = 0; f < nfields && f < SPH_MAX_FIELDS; ++f) g[f] = grids[f];
  return launch_cont_phys_g(p, g, nfields, st, false);
}

int launch_phi_fwd32(const sph_plan* p, const double* const* grids, int nfields, cudaStream_t st,
                     const double* const* grids_hi) {
  const void* g[SPH_MAX_FIELDS] = {};
  const void* gh[SPH_MAX_FIELDS] = {};
  for (int f = 0; f < nfields && f < SPH_MAX_FIELDS; ++f) {
    g[f] = grids[f];
    if (grids_hi) gh[f] = grids_hi[f];
  }
  return launch_phi_fwd32_g(p, g, nfields, st, grids_hi ? gh : nullptr, false);
}

int launch_phi_inv32(const sph_plan* p, double* const* grids, int nfields, cudaStream_t st) {
  void* g[SPH_MAX_FIELDS] = {};
  for (int f = 0; f < nfields && f < SPH_MAX_FIELDS; ++f) g[f] = grids[f];
  return launch_phi_inv32_g(p, g, nfields, st, false);
}

int launch_tc_analysis(const sph_plan* p, int vector, double2* out, double2* out2, cudaStream_t st) {
  TcArgs a = tc_args(p);
  a.tiles = reinterpret_cast<const __nv_bfloat16*>(p->Tana);
  a.out = out;
  a.out2 = out2;
  TimedLaunch tl(p, vector ? T_VEC_ANA : T_LEG_ANA, st);
  return vector ? run_tc<ANA_V>(p, p->tcAV, a, st) : run_tc<ANA_S>(p, p->tcAS, a, st);
}

int launch_tc_synthesis(const sph_plan* p, int vector, const double2* in, const double2* in2, cudaStream_t st) {
  TcArgs a = tc_args(p);
  a.tiles = reinterpret_cast<const __nv_bfloat16*>(p->Tsyn);
  {
    TimedLaunch tl(p, T_OPS, st);
    spec_to_tiles<<<dim3(p->lmax + 1, p->nz, vector ? 2 : 1), 32, 0, st>>>(
        in, in2, reinterpret_cast<__nv_bfloat16*>(p->Tsyn), p->Tsynfield, p->d_toff, p->d_mbase, p->lmax, p->nlm);
    SPH_LAUNCH_OK();
  }
  TimedLaunch tl(p, vector ? T_VEC_SYN : T_LEG_SYN, st);
  return vector ? run_tc<SYN_V>(p, p->tcSV, a, st) : run_tc<SYN_S>(p, p->tcSS, a, st);
}

// ---------------------------------------------------------------- grouped launches
int tc_group_prepare(bool analysis, const std::vector<GroupJob>& jobs, int nsm, GroupLaunch* g) {
  std::vector<TcArgs> args;
  std::vector<int> prefix;
  long long total = 0;
  for (const GroupJob& j : jobs) {
    const sph_plan* p = j.p;
    if (p->precision != SPH_MIXED || j.field < 0 || j.field >= SPH_MAX_FIELDS) return SPH_EINVAL;
    TcArgs a = tc_args(p);
    const TcSet& set = analysis ? p->tcAS : p->tcSS;
    a.items = set.items;
    a.blocks = reinterpret_cast<const __nv_bfloat16*>(set.blocks);
    if (analysis) {
      const size_t per = ana_tile(p->lmax, a.ncb, a.nkn, 1, 0, 0, 0, 0) * TILE_HALVES;
      a.tiles = reinterpret_cast<const __nv_bfloat16*>(p->Tana) + (size_t)j.field * per;
      a.out = j.spec;
    } else {
      a.tiles = reinterpret_cast<const __nv_bfloat16*>(p->Tsyn) + (size_t)j.field * p->Tsynfield;
      a.G32w = reinterpret_cast<float2*>(p->G) + (size_t)j.field * p->G32field;
    }
    a.nunits = set.nitems * a.ncb;
    prefix.push_back((int)total);
    total += a.nunits;
    args.push_back(a);
  }
  if (total > (1ll << 30)) return SPH_EINVAL;
  g->analysis = analysis;
  g->njobs = (int)jobs.size();
  g->total = (int)total;
  g->grid = (int)std::min<long long>(total, std::max(1, nsm));
  if (jobs.empty()) return SPH_OK;
  if (cudaMalloc(&g->jobs, args.size() * sizeof(TcArgs)) != cudaSuccess ||
      cudaMalloc((void**)&g->prefix, prefix.size() * sizeof(int)) != cudaSuccess)
    return SPH_ENOMEM;
  if (cudaMemcpy(g->jobs, args.data(), args.size() * sizeof(TcArgs), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(g->prefix, prefix.data(), prefix.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    return SPH_ECUDA;
  return SPH_OK;
}

int tc_group_launch(const GroupLaunch& g, int* flag, cudaStream_t st) {
  if (g.total == 0) return SPH_OK;
  TcLaunch L = {};
  L.jobs = static_cast<const TcArgs*>(g.jobs);
  L.prefix = g.prefix;
  L.njobs = g.njobs;
  L.total = g.total;
  L.flag = flag;
  if (g.analysis) {
    if (!tc_attr<ANA_S, true>()) return SPH_ECUDA;
    tc_gemm<ANA_S, true><<<g.grid, TC_THREADS, TC_SMEM, st>>>(L);
  } else {
    if (!tc_attr<SYN_S, true>()) return SPH_ECUDA;
    tc_gemm<SYN_S, true><<<g.grid, TC_THREADS, TC_SMEM, st>>>(L);
  }
  SPH_LAUNCH_OK();
  return SPH_OK;
}

bool zinv_tiles_ok(const sph_plan* p) {
  if (p->precision != SPH_MIXED || !p->d_ztitems || p->nztitems < 1) return false;
  switch (p->nz) {
#define CASE(n) \
  case n:       \
    return true;
    ZT_SIZES(CASE)
#undef CASE
  }
  return false;
}

namespace {
template <int NZ, typename TI, bool DER = false>
int zinv_tiles_run(const sph_plan* p, const ZtArgs& a, cudaStream_t st) {
  const size_t smem = (size_t)ZT_PITCH * NZ * sizeof(double2);
  static DeviceOnce once;
  if (!once.run([] {
        return cudaFuncSetAttribute(zinv_tiles<NZ, TI, DER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)((size_t)ZT_PITCH * NZ * sizeof(double2))) == cudaSuccess &&
               cudaFuncSetAttribute(zinv_tiles<NZ, TI, DER>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    100) == cudaSuccess;
      }))
    return SPH_ECUDA;
  zinv_tiles<NZ, TI, DER><<<p->nztitems, ZT_THREADS, smem, st>>>(a);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
}  // namespace

int launch_zinv_tiles(const sph_plan* p, const double2* in, int field, cudaStream_t st, double2* out,
                      double2* dout) {
  return launch_zinv_tiles_g(p, in, field, st, false, out, dout);
}

int launch_zinv_tiles_g(const sph_plan* p, const void* in, int field, cudaStream_t st, bool f32, double2* out,
                        double2* dout) {
  if (!zinv_tiles_ok(p) || !in || field < 0 || field >= SPH_MAX_FIELDS || (f32 && (out || dout)) ||
      (dout && (!zinv_der_ok(p) || !p->kfac)))
    return SPH_EINVAL;
  ZtArgs a;
  a.in = in;
  a.out = out;
  a.dout = dout;
  a.dir = p->d_dir;
  a.C = p->C;
  a.d = p->d;
  a.N = p->N;
  a.kfac = p->kfac;  // (i kz)^1
  a.tiles = reinterpret_cast<__nv_bfloat16*>(p->Tsyn) + (size_t)field * p->Tsynfield;
  a.toff = p->d_toff;
  a.mbase = p->d_mbase;
  a.items = p->d_ztitems;
  a.lmax = p->lmax;
  a.nlm = p->nlm;
  a.nz = p->nz;
  a.rev = p->fz.rev;
  a.twp = p->fz.twp;
  a.tw = p->fz.tw;
  TimedLaunch tl(p, T_ZFFT, st);
  switch (p->nz) {
#define CASE(n)                                                                  \
  case n:                                                                        \
    if constexpr (ct::split2_r1(n) > 0) {                                        \
      if (dout) return zinv_tiles_run<n, double2, true>(p, a, st);               \
    }                                                                            \
    return f32 ? zinv_tiles_run<n, float2>(p, a, st) : zinv_tiles_run<n, double2>(p, a, st);
    ZT_SIZES(CASE)
#undef CASE
  }
  return SPH_EINVAL;
}

bool zinv_der_ok(const sph_plan* p) {
  if (!zinv_tiles_ok(p)) return false;
  switch (p->nz) {
#define CASE(n) \
  case n: return ct::split2_r1(n) > 0 && ct::split2_tpc(n) * ZT_COLS <= ZT_THREADS;
    ZT_SIZES(CASE)
#undef CASE
  }
  return false;
}

int launch_tc_synthesis_tiles(const sph_plan* p, int vector, cudaStream_t st) {
  TcArgs a = tc_args(p);
  a.tiles = reinterpret_cast<const __nv_bfloat16*>(p->Tsyn);
  TimedLaunch tl(p, vector ? T_VEC_SYN : T_LEG_SYN, st);
  return vector ? run_tc<SYN_V>(p, p->tcSV, a, st) : run_tc<SYN_S>(p, p->tcSS, a, st);
}

int launch_spec_to_tiles_field(const sph_plan* p, const double2* in, int field, cudaStream_t st) {
  if (p->precision != SPH_MIXED || field < 0 || field >= SPH_MAX_FIELDS) return SPH_EINVAL;
  spec_to_tiles<<<dim3(p->lmax + 1, p->nz, 1), 32, 0, st>>>(
      in, nullptr, reinterpret_cast<__nv_bfloat16*>(p->Tsyn) + (size_t)field * p->Tsynfield, p->Tsynfield,
      p->d_toff, p->d_mbase, p->lmax, p->nlm);
  SPH_LAUNCH_OK();
  return SPH_OK;
}
