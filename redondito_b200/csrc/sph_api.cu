// sph_api.cu -- plans, host-side tables and the C ABI of the transform core.
//
// Host-side setup is FP64 (80-bit long double where it matters): the
// Gauss-Legendre grid, the associated Legendre tables, FFT twiddles, the
// FC-Gram operator and the boundary LU.  Everything per-call runs on the
// device, stream-ordered, through the kernels of k_*.cu.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cstdlib>
#include <thread>

#include "fft_ct.cuh"
#include "sph_internal.cuh"

typedef long double ld;
static const ld kPi = 3.141592653589793238462643383279502884L;

// ---------------------------------------------------------------- host tables

// Gauss-Legendre nodes (descending cos theta: north pole first, the order of
// SHTns's Gauss grid, src/sphp/sphp_sca.F90:120-122) and weights.
static void gl_grid(int n, std::vector<double>& ct, std::vector<double>& w) {
  ct.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    ld x = cosl(kPi * (i + 0.75L) / (n + 0.5L));
    ld pn = 0, dpn = 1;
    for (int it = 0; it < 64; ++it) {
      ld a = 1, b = x;
      for (int k = 2; k <= n; ++k) {
        ld c = ((2 * k - 1) * x * b - (k - 1) * a) / k;
        a = b;
        b = c;
      }
      pn = b;
      dpn = n * (x * b - a) / (x * x - 1);
      ld step = pn / dpn;
      x -= step;
      if (fabsl(step) <= 4e-19L * fabsl(x)) break;
    }
    ld a = 1, b = x;
    for (int k = 2; k <= n; ++k) {
      ld c = ((2 * k - 1) * x * b - (k - 1) * a) / k;
      a = b;
      b = c;
    }
    dpn = n * (x * b - a) / (x * x - 1);
    ct[i] = (double)x;
    ct[n - 1 - i] = -(double)x;
    w[i] = w[n - 1 - i] = (double)(2.0L / ((1 - x * x) * dpn * dpn));
  }
}

// Pbar_lm (orthonormal, no Condon-Shortley phase), dPbar/dtheta and
// m Pbar/sin(theta) for one (m, node), l = m..lmax.  The sectoral start
// sin^m theta can be far below the double range near the poles; 80-bit
// arithmetic keeps it, and values that underflow double are their true 0.
static void legendre_column(int lmax, int m, ld x, ld s, double* P, double* dP, double* mPs) {
  const int L = lmax - m + 1;
  std::vector<ld> p(L);
  ld v = sqrtl(1.0L / (4.0L * kPi));
  for (int k = 1; k <= m; ++k) v *= s * sqrtl((2.0L * k + 1.0L) / (2.0L * k));
  p[0] = v;
  if (L > 1) p[1] = sqrtl(2.0L * m + 3.0L) * x * v;
  for (int l = m + 2; l <= lmax; ++l) {
    ld l2 = (ld)l * l, m2 = (ld)m * m, lm1 = (ld)(l - 1);
    ld a = sqrtl((4.0L * l2 - 1.0L) / (l2 - m2));
    ld b = sqrtl((lm1 * lm1 - m2) / (4.0L * lm1 * lm1 - 1.0L));
    p[l - m] = a * (x * p[l - m - 1] - b * p[l - m - 2]);
  }
  for (int l = m; l <= lmax; ++l) {
    ld pl = p[l - m];
    P[l - m] = (double)pl;
    ld prev = l > m ? p[l - m - 1] : 0.0L;
    ld c = l > m ? sqrtl((2.0L * l + 1.0L) * ((ld)l * l - (ld)m * m) / (2.0L * l - 1.0L)) : 0.0L;
    dP[l - m] = (double)((l * x * pl - c * prev) / s);
    mPs[l - m] = (double)(m * pl / s);
  }
}

// Radix plan for a length-n FFT: 8s first, then 4, 2, 3, any other prime.
static int fft_factor(int n, FftDesc& fd) {
  fd.n = n;
  fd.npass = 0;
  int r = n, Ns = 1;
  auto push = [&](int R) {
    if (fd.npass >= SPH_MAX_PASSES) return false;
    fd.pass[fd.npass].R = R;
    fd.pass[fd.npass].Ns = Ns;
    fd.npass++;
    Ns *= R;
    r /= R;
    return true;
  };
  while (r % 8 == 0) if (!push(8)) return 1;
  while (r % 4 == 0) if (!push(4)) return 1;
  while (r % 2 == 0) if (!push(2)) return 1;
  while (r % 3 == 0) if (!push(3)) return 1;
  for (int q = 5; r > 1; q += 2)
    while (r % q == 0) {
      if (q > 64) return 1;  // direct DFT passes stay short
      if (!push(q)) return 1;
    }
  return 0;
}

// position of frequency k after the decimation-in-frequency passes
static std::vector<int> digit_reversal(const FftDesc& fd) {
  std::vector<int> rev(fd.n);
  for (int k = 0; k < fd.n; ++k) {
    int t = k, s = fd.n, pos = 0;
    for (int ip = 0; ip < fd.npass; ++ip) {
      const int R = fd.pass[ip].R;
      s /= R;
      pos += (t % R) * s;
      t /= R;
    }
    rev[k] = pos;
  }
  return rev;
}

// per-pass twiddles [pass][j][r-1] = W_L^{j r}, DIF pass order (fft_ct.cuh)
static void pass_twiddles(int n, std::vector<double2>& tw, std::vector<float2>& twf) {
  tw.clear();
  twf.clear();
  for (int L = n; L > 1;) {
    int R = L % 8 == 0 ? 8 : L % 4 == 0 ? 4 : L % 2 == 0 ? 2 : L % 3 == 0 ? 3 : L;
    int S = L / R;
    for (int j = 0; j < S; ++j)
      for (int r = 1; r < R; ++r) {
        ld a = -2.0L * kPi * (ld)((long)j * r) / L;
        tw.push_back(make_double2((double)cosl(a), (double)sinl(a)));
        twf.push_back(make_float2((float)cosl(a), (float)sinl(a)));
      }
    L = S;
  }
  if (tw.empty()) {
    tw.push_back(make_double2(1.0, 0.0));
    twf.push_back(make_float2(1.f, 0.f));
  }
}

static void twiddles(int n, std::vector<double2>& tw, std::vector<float2>& twf) {
  tw.resize(n);
  twf.resize(n);
  for (int e = 0; e < n; ++e) {
    ld a = -2.0L * kPi * e / n;
    tw[e] = make_double2((double)cosl(a), (double)sinl(a));
    twf[e] = make_float2((float)cosl(a), (float)sinl(a));
  }
}

template <typename T>
static int upload(T** dst, const T* src, size_t n) {
  if (n == 0) return SPH_OK;
  if (cudaMalloc((void**)dst, n * sizeof(T)) != cudaSuccess) return SPH_ENOMEM;
  if (cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return SPH_ECUDA;
  return SPH_OK;
}

// the read-only device tables of a plan (shared with its clones)
static std::vector<void*> table_ptrs(const sph_plan* p) {
  return {p->P, p->dP, p->mPs, p->wfold, p->wfull, p->d_dir, p->d_z, p->kfac, p->filt, p->zinv2, p->d_ell,
          p->d_mbase, p->twz, p->twphi, p->twzf, p->twphif, p->revz, p->revphi, p->twpz, p->twpphi, p->twpzf,
          p->twpphif, p->tw4f, p->tw4d, p->tilesA, p->tilesA32, p->tilesS, p->tilesS32, p->d_bplanes, p->d_toff};
}

PlanTables::~PlanTables() {
  for (void* q : dev)
    if (q) cudaFree(q);
  for (TcSet& t : tc) {
    if (t.items) cudaFree(t.items);
    if (t.blocks) cudaFree(t.blocks);
  }
  if (binv) cudaFree(binv);
  if (d2bor) cudaFree(d2bor);
}

// Frees a plan's own buffers; its tables go with the last plan that shares
// them (a plan whose creation failed owns its tables alone).
static void plan_free(sph_plan* p) {
  for (auto e : p->ev_pool) cudaEventDestroy(e);
  mixed_free_scratch(p);
  for (void* q : {(void*)p->G, (void*)p->energy, (void*)p->spectrum, (void*)p->d_neu})
    if (q) cudaFree(q);
  if (p->bc_own) {  // boundary matrices of kinds other than the shared ones
    if (p->binv) cudaFree(p->binv);
    if (p->d2bor) cudaFree(p->d2bor);
    p->binv = p->d2bor = nullptr;
  }
  for (auto& q : p->sp)
    if (q) cudaFree(q);
  for (auto& q : p->gr)
    if (q) cudaFree(q);
  for (auto& q : p->fsp)
    if (q) cudaFree(q);
  if (!p->tables) {
    mixed_free_tables(p);
    for (void* q : table_ptrs(p))
      if (q) cudaFree(q);
    if (p->binv) cudaFree(p->binv);
    if (p->d2bor) cudaFree(p->d2bor);
  }
  delete p;
}

// hands the plan's tables to a shared owner (after a successful creation)
static void own_tables(sph_plan* p) {
  p->tables = std::make_shared<PlanTables>();
  p->tables->dev = table_ptrs(p);
  p->tables->tc[0] = p->tcAS;
  p->tables->tc[1] = p->tcAV;
  p->tables->tc[2] = p->tcSS;
  p->tables->tc[3] = p->tcSV;
}

static std::vector<LegTile> row_tiles(int lmax, int block, bool by_l, int nlat2) {
  std::vector<LegTile> t;
  for (int m = 0; m <= lmax; ++m) {
    if (by_l) {
      for (int l0 = m; l0 <= lmax; l0 += block) t.push_back({m, l0});
    } else {
      for (int i0 = 0; i0 < nlat2; i0 += block) t.push_back({m, i0});
    }
  }
  return t;
}

extern "C" int sph_plan_create(sph_plan** out, int lmax, int nlat, int nphi, int nz, int Cz, int oz,
                               double rint, double rext, const double* dir, int precision) {
  if (!out) return SPH_EINVAL;
  *out = nullptr;
  if (lmax < 0 || nlat < 2 || (nlat & 1) || nphi <= 2 * lmax || nz < 1) return SPH_EINVAL;
  if (Cz < 0 || oz < 0 || (Cz > 0 && (oz < 1 || nz - Cz < oz || !dir))) return SPH_EINVAL;
  if (precision != SPH_FP64 && precision != SPH_MIXED) return SPH_EINVAL;
  if (nz > 4096 || nphi > 8192) return SPH_EINVAL;
  if (precision == SPH_MIXED && !mixed_nphi_ok(nphi)) return SPH_EINVAL;
  sph_plan* p = new sph_plan();
  p->lmax = lmax;
  p->nlat = nlat;
  p->nlat2 = nlat / 2;
  p->ldn = (p->nlat2 + 3) & ~3;
  p->nphi = nphi;
  p->nz = nz;
  p->C = Cz;
  p->d = oz;
  p->nlm = (lmax + 1) * (lmax + 2) / 2;
  p->N = nz - Cz;
  p->nzv = nz;
  p->nlmv = p->nlm;
  p->precision = precision;
  p->rint = rint;
  p->rext = rext;
  if (fft_factor(nz, p->fz) || fft_factor(nphi, p->fphi)) {
    delete p;
    return SPH_EINVAL;
  }
  // grid (box_init, src/pseudo/pseudospec_mod.f90:174-227)
  gl_grid(nlat, p->ct, p->w);
  p->theta.resize(nlat);
  for (int i = 0; i < nlat; ++i) p->theta[i] = acos(p->ct[i]);
  p->phi.resize(nphi);
  for (int j = 0; j < nphi; ++j) p->phi[j] = 2.0 * 3.14159265358979323846 / nphi * j;
  p->dz = p->N > 1 ? (rext - rint) / (nz - Cz - 1) : 1.0;
  p->Dkz = 2.0 * 3.14159265358979323846 / (p->dz * nz);
  p->z.resize(nz);
  p->kz.resize(nz);
  for (int k = 0; k < nz; ++k) p->z[k] = rint + p->dz * k;
  // odd nz: the FFT frequencies 0..nz/2, -nz/2..-1 (the reference leaves kz(nz) unset)
  for (int k = 0; k < nz; ++k) p->kz[k] = (double)(k < (nz + 1) / 2 ? k : k - nz) * p->Dkz;
  if (nz % 2 == 0) {  // kz(nz/2+1) = -nz/2 Dkz (pseudospec_mod.f90:223-226)
    for (int k = 0; k < nz / 2; ++k) {
      p->kz[k] = (double)k * p->Dkz;
      p->kz[k + nz / 2] = (double)(k - nz / 2) * p->Dkz;
    }
  }
  p->mbase.resize(lmax + 2);
  for (int m = 0; m <= lmax + 1; ++m) p->mbase[m] = m * (2 * lmax + 3 - m) / 2;
  p->ell.resize(p->nlm);
  p->emm.resize(p->nlm);
  for (int m = 0; m <= lmax; ++m)
    for (int l = m; l <= lmax; ++l) {
      p->ell[p->mbase[m] + l - m] = l;
      p->emm[p->mbase[m] + l - m] = m;
    }
  if (Cz > 0) p->dir.assign(dir, dir + (size_t)Cz * oz);

  // Legendre tables on the northern nodes, [lm][node], built in parallel over m
  const int n2 = p->nlat2, ldn = p->ldn;
  std::vector<double> hP((size_t)p->nlm * ldn, 0.0), hdP((size_t)p->nlm * ldn, 0.0),
      hmPs((size_t)p->nlm * ldn, 0.0);
  {
    int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (int t = 0; t < nth; ++t)
      th.emplace_back([&, t]() {
        std::vector<double> cP(lmax + 1), cdP(lmax + 1), cmP(lmax + 1);
        for (int m = t; m <= lmax; m += nth)
          for (int i = 0; i < n2; ++i) {
            ld x = p->ct[i];
            ld s = sqrtl((1.0L - x) * (1.0L + x));
            legendre_column(lmax, m, x, s, cP.data(), cdP.data(), cmP.data());
            for (int l = m; l <= lmax; ++l) {
              size_t o = (size_t)(p->mbase[m] + l - m) * ldn + i;
              hP[o] = cP[l - m];
              hdP[o] = cdP[l - m];
              hmPs[o] = cmP[l - m];
            }
          }
      });
    for (auto& x : th) x.join();
  }
  std::vector<double> wf(ldn, 0.0);
  for (int i = 0; i < n2; ++i) wf[i] = p->w[i] * (2.0 * 3.14159265358979323846 / nphi);
  std::vector<double2> kf((size_t)4 * nz);
  for (int o = 1; o <= 4; ++o)
    for (int k = 0; k < nz; ++k) {
      // ip * kz**p (pseudospec_hd.f90:85,93)
      double kp = 1.0;
      for (int q = 0; q < o; ++q) kp *= p->kz[k];
      double re = (o % 4 == 0) ? 1 : (o % 4 == 2) ? -1 : 0;
      double im = (o % 4 == 1) ? 1 : (o % 4 == 3) ? -1 : 0;
      kf[(size_t)(o - 1) * nz + k] = make_double2(re * kp, im * kp);
    }
  std::vector<double> filt(nz), zinv2(nz);
  const double alpha = 16.0 * log(10.0);
  for (int k = 0; k < nz; ++k) {
    filt[k] = exp(-alpha * pow(2.0 * p->kz[k] / nz / p->Dkz, 100.0));
    zinv2[k] = 1.0 / (p->z[k] * p->z[k]);
  }
  std::vector<double2> twz, twp;
  std::vector<float2> twzf, twpf;
  twiddles(nz, twz, twzf);
  twiddles(nphi, twp, twpf);
  std::vector<int> revz = digit_reversal(p->fz), revphi = digit_reversal(p->fphi);
  std::vector<double2> tpz, tpp;
  std::vector<float2> tpzf, tppf;
  pass_twiddles(nz, tpz, tpzf);
  pass_twiddles(nphi, tpp, tppf);
  std::vector<double2> t4, t4b;
  std::vector<float2> t4f, t4fb;
  {
    const int n1 = ct::split_n1(nphi), n2 = nphi / n1;
    pass_twiddles(n1, t4, t4f);
    p->tw4off = (int)t4.size();
    pass_twiddles(n2, t4b, t4fb);
    t4.insert(t4.end(), t4b.begin(), t4b.end());
    t4f.insert(t4f.end(), t4fb.begin(), t4fb.end());
  }
  auto tA = row_tiles(lmax, 64, true, n2);
  auto tA32 = row_tiles(lmax, 32, true, n2);
  auto tS = row_tiles(lmax, 64, false, n2);
  auto tS32 = row_tiles(lmax, 32, false, n2);
  // heaviest synthesis tiles (small m: K = lmax+1-m) first


  int rc = SPH_OK;
#define UP(dst, vec)                                              \
  if (rc == SPH_OK) rc = upload(&(dst), (vec).data(), (vec).size());
#define UPLOAD_OK(dst, vec) UP(dst, vec)
  UP(p->P, hP);
  UP(p->dP, hdP);
  UP(p->mPs, hmPs);
  UP(p->wfold, wf);
  UP(p->wfull, p->w);
  UP(p->d_z, p->z);
  UP(p->kfac, kf);
  UP(p->filt, filt);
  UP(p->zinv2, zinv2);
  UP(p->d_ell, p->ell);
  UP(p->d_mbase, p->mbase);
  UP(p->twz, twz);
  UP(p->twphi, twp);
  UP(p->twzf, twzf);
  UP(p->twphif, twpf);
  UP(p->revz, revz);
  UP(p->revphi, revphi);
  UP(p->twpz, tpz);
  UP(p->twpphi, tpp);
  UP(p->twpzf, tpzf);
  UP(p->twpphif, tppf);
  UP(p->tw4f, t4f);
  UP(p->tw4d, t4);
  UP(p->tilesA, tA);
  UP(p->tilesA32, tA32);
  UP(p->tilesS, tS);
  UP(p->tilesS32, tS32);
  if (Cz > 0) UP(p->d_dir, p->dir);
  p->ntilesA = (int)tA.size();
  p->ntilesA32 = (int)tA32.size();
  p->ntilesS = (int)tS.size();
  p->ntilesS32 = (int)tS32.size();
  p->fz.tw = p->twz;
  p->fz.twf = p->twzf;
  p->fz.rev = p->revz;
  p->fz.twp = p->twpz;
  p->fz.twpf = p->twpzf;
  p->fphi.tw = p->twphi;
  p->fphi.twf = p->twphif;
  p->fphi.rev = p->revphi;
  p->fphi.twp = p->twpphi;
  p->fphi.twpf = p->twpphif;
  p->Gfield = (size_t)(lmax + 1) * 2 * nz * ldn;
  if (rc == SPH_OK && cudaMalloc((void**)&p->G, SPH_MAX_FIELDS * p->Gfield * sizeof(double2)) != cudaSuccess)
    rc = SPH_ENOMEM;
  // node columns past nlat/2 are never written and must read as zero
  if (rc == SPH_OK && cudaMemset(p->G, 0, SPH_MAX_FIELDS * p->Gfield * sizeof(double2)) != cudaSuccess)
    rc = SPH_ECUDA;
  if (rc == SPH_OK && cudaMalloc((void**)&p->energy, sizeof(double)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && precision == SPH_MIXED) rc = mixed_setup(p, hP, hdP, hmPs);
  // status word of the kernels with bounded waits (every plan: the FP64
  // forward phi transform waits on its TMA copies too)
  if (rc == SPH_OK && !p->dflag) {
    if (cudaMalloc((void**)&p->dflag, sizeof(int)) != cudaSuccess) rc = SPH_ENOMEM;
    else if (cudaMemset(p->dflag, 0, sizeof(int)) != cudaSuccess) rc = SPH_ECUDA;
  }
  if (rc == SPH_OK && precision == SPH_MIXED && Cz > 0 && oz > 0) {
    std::vector<int> bp;
    for (int k = 0; k < p->N; ++k)
      if (k < oz || k >= p->N - oz) bp.push_back(k);
    p->nbplanes = (int)bp.size();
    UPLOAD_OK(p->d_bplanes, bp);
  }
#undef UPLOAD_OK
#undef UP
  if (rc != SPH_OK) {
    plan_free(p);
    return rc;
  }
  own_tables(p);
  *out = p;
  return SPH_OK;
}

extern "C" int sph_plan_clone(const sph_plan* src, sph_plan** out) {
  if (!out) return SPH_EINVAL;
  *out = nullptr;
  if (!src || !src->tables) return SPH_EINVAL;
  sph_plan* p = new sph_plan(*src);  // sizes, host grids, table pointers; one more owner of the tables
  // its own buffers: nothing of the source's scratch, timers, slab or boundary state
  p->G = nullptr;
  for (auto& q : p->sp) q = nullptr;
  for (auto& q : p->gr) q = nullptr;
  for (auto& q : p->fsp) q = nullptr;
  p->nsp = p->ngr = 0;
  p->energy = p->spectrum = nullptr;
  p->dflag = nullptr;
  p->Tana = p->Tsyn = nullptr;
  p->d_ztitems = nullptr;
  p->nztitems = 0;
  p->contg = nullptr;
  p->phi2 = nullptr;
  p->phi2_planes = 0;
  p->ev_pool.clear();
  p->ev_class.clear();
  p->ev_used = 0;
  p->timing = 0;
  p->k0 = 0;
  p->nzv = p->nz;
  p->lm0 = 0;
  p->nlmv = p->nlm;
  p->sel_kz = nullptr;
  p->sel_n = 0;
  p->bpass = 0;
  p->bc_ready = 0;
  p->bc_own = 0;
  p->bck[0] = p->bck[1] = 0;
  p->binv = p->d2bor = nullptr;
  p->d_neu = nullptr;
  int rc = SPH_OK;
  if (!p->neu[0].empty() || !p->neu[1].empty()) {  // the Neumann reconstructors, copied
    std::vector<double> both((size_t)2 * p->d, 0.0);
    for (int o = 0; o < 2; ++o)
      if (!p->neu[o].empty()) std::copy(p->neu[o].begin(), p->neu[o].end(), both.begin() + (size_t)o * p->d);
    rc = upload(&p->d_neu, both.data(), both.size());
  }
  if (rc == SPH_OK && cudaMalloc((void**)&p->G, SPH_MAX_FIELDS * p->Gfield * sizeof(double2)) != cudaSuccess)
    rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(p->G, 0, SPH_MAX_FIELDS * p->Gfield * sizeof(double2)) != cudaSuccess)
    rc = SPH_ECUDA;
  if (rc == SPH_OK && cudaMalloc((void**)&p->energy, sizeof(double)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && p->precision == SPH_MIXED) rc = mixed_alloc_scratch(p);
  if (rc == SPH_OK && !p->dflag) {
    if (cudaMalloc((void**)&p->dflag, sizeof(int)) != cudaSuccess) rc = SPH_ENOMEM;
    else if (cudaMemset(p->dflag, 0, sizeof(int)) != cudaSuccess) rc = SPH_ECUDA;
  }
  if (rc != SPH_OK) {
    plan_free(p);  // drops its reference to the tables only
    return rc;
  }
  *out = p;
  return SPH_OK;
}

extern "C" int sph_plan_destroy(sph_plan* p) {
  if (!p) return SPH_EINVAL;
  cudaDeviceSynchronize();
  plan_free(p);
  return SPH_OK;
}

extern "C" int sph_fcgram_load_tables(const char* tdir, int C, int d, double* dir) {
  if (!tdir || !dir || C < 1 || d < 1) return SPH_EINVAL;
  std::vector<double> A((size_t)C * d), Q((size_t)d * d);
  char path[4096];
  snprintf(path, sizeof path, "%s/A%d-%d.dat", tdir, C, d);
  FILE* f = fopen(path, "rb");
  if (!f) return SPH_EIO;
  size_t got = fread(A.data(), sizeof(double), A.size(), f);
  fclose(f);
  if (got != A.size()) return SPH_EIO;
  snprintf(path, sizeof path, "%s/Q%d.dat", tdir, d);
  f = fopen(path, "rb");
  if (!f) return SPH_EIO;
  got = fread(Q.data(), sizeof(double), Q.size(), f);
  fclose(f);
  if (got != Q.size()) return SPH_EIO;
  // Q = TRANSPOSE(Q); dir = MATMUL(A, Q)   (fcgram_mod.f90:257-258)
  for (int i = 0; i < C; ++i)
    for (int j = 0; j < d; ++j) {
      double s = 0.0;
      for (int k = 0; k < d; ++k) s += A[i + (size_t)C * k] * Q[j + (size_t)d * k];
      dir[i + (size_t)C * j] = s;
    }
  return SPH_OK;
}

extern "C" int sph_fcgram_load_neumann_tables(const char* tdir, int d, int ord, double dx, double* neu) {
  if (!tdir || !neu || d < 1 || (ord != 1 && ord != 2) || !(dx > 0.0)) return SPH_EINVAL;
  std::vector<double> Q((size_t)d * d), Qn((size_t)d * d);
  char path[4096];
  snprintf(path, sizeof path, "%s/Q%d.dat", tdir, d);
  FILE* f = fopen(path, "rb");
  if (!f) return SPH_EIO;
  size_t got = fread(Q.data(), sizeof(double), Q.size(), f);
  fclose(f);
  if (got != Q.size()) return SPH_EIO;
  snprintf(path, sizeof path, "%s/Q%dn%d.dat", tdir, ord, d);
  f = fopen(path, "rb");
  if (!f) return SPH_EIO;
  double dxp = 0.0;
  got = fread(&dxp, sizeof(double), 1, f);
  got += fread(Qn.data(), sizeof(double), Qn.size(), f);
  fclose(f);
  if (got != Qn.size() + 1 || !(dxp > 0.0)) return SPH_EIO;
  // neu = MATMUL(Q(d,:), TRANSPOSE(Qn)); neu(d) *= (dx/dxp)^ord  (fcgram_mod.f90:357-363)
  for (int k = 0; k < d; ++k) {
    double acc = 0.0;
    for (int j = 0; j < d; ++j) acc += Q[(d - 1) + (size_t)d * j] * Qn[k + (size_t)d * j];
    neu[k] = acc;
  }
  neu[d - 1] *= ord == 1 ? dx / dxp : (dx / dxp) * (dx / dxp);
  return SPH_OK;
}

extern "C" int sph_plan_set_neumann(sph_plan* p, const double* neu1, const double* neu2) {
  if (!p || p->d < 1 || (!neu1 && !neu2)) return SPH_EINVAL;
  if (neu1) p->neu[0].assign(neu1, neu1 + p->d);
  if (neu2) p->neu[1].assign(neu2, neu2 + p->d);
  std::vector<double> both((size_t)2 * p->d, 0.0);
  for (int o = 0; o < 2; ++o)
    if (!p->neu[o].empty()) std::copy(p->neu[o].begin(), p->neu[o].end(), both.begin() + (size_t)o * p->d);
  if (!p->d_neu && cudaMalloc((void**)&p->d_neu, both.size() * sizeof(double)) != cudaSuccess) return SPH_ENOMEM;
  SPH_CUDA_OK(cudaMemcpy(p->d_neu, both.data(), both.size() * sizeof(double), cudaMemcpyHostToDevice));
  return SPH_OK;
}

extern "C" int sph_neumann_reconstruct(sph_plan* p, double* f, int boun, int ord, void* s) {
  if (!p || !f) return SPH_EINVAL;
  return launch_reconstruct(p, reinterpret_cast<double2*>(f), boun, ord, nullptr, (cudaStream_t)s);
}

extern "C" int sph_robin_reconstruct(sph_plan* p, double* f, int boun, const double* a, void* s) {
  if (!p || !f || !a) return SPH_EINVAL;
  return launch_reconstruct(p, reinterpret_cast<double2*>(f), boun, 1, a, (cudaStream_t)s);
}

extern "C" int sph_plan_sizes(const sph_plan* p, int* nlm, long long* ge, long long* se) {
  if (!p) return SPH_EINVAL;
  if (nlm) *nlm = p->nlm;
  if (ge) *ge = (long long)grid_elems(p);
  if (se) *se = (long long)spec_elems(p);
  return SPH_OK;
}

extern "C" int sph_grid(const sph_plan* p, double* theta, double* weights, double* phi, double* z,
                        double* kz, int* ell, int* emm) {
  if (!p) return SPH_EINVAL;
  if (theta) std::copy(p->theta.begin(), p->theta.end(), theta);
  if (weights) std::copy(p->w.begin(), p->w.end(), weights);
  if (phi) std::copy(p->phi.begin(), p->phi.end(), phi);
  if (z) std::copy(p->z.begin(), p->z.end(), z);
  if (kz) std::copy(p->kz.begin(), p->kz.end(), kz);
  if (ell) std::copy(p->ell.begin(), p->ell.end(), ell);
  if (emm) std::copy(p->emm.begin(), p->emm.end(), emm);
  return SPH_OK;
}

// ---------------------------------------------------------------- timers
int timer_start(const sph_plan* cp, int cls, cudaStream_t st) {
  sph_plan* p = const_cast<sph_plan*>(cp);
  if (!p->timing) return -1;
  int slot = p->ev_used++;
  while ((int)p->ev_pool.size() < 2 * p->ev_used) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) {
      p->ev_used--;
      return -1;
    }
    p->ev_pool.push_back(e);
  }
  if ((int)p->ev_class.size() < p->ev_used) p->ev_class.resize(p->ev_used);
  p->ev_class[slot] = cls;
  cudaEventRecord(p->ev_pool[2 * slot], st);
  return slot;
}

void timer_stop(const sph_plan* cp, int slot, cudaStream_t st) {
  if (slot < 0) return;
  sph_plan* p = const_cast<sph_plan*>(cp);
  cudaEventRecord(p->ev_pool[2 * slot + 1], st);
}

extern "C" int sph_plan_set_tiles(sph_plan* p, int rows, int ring_pairs, int z_cols) {
  if (!p) return SPH_EINVAL;
  if (rows != 0 && rows != 32 && rows != 64 && rows != 128) return SPH_EINVAL;
  if (ring_pairs != 0 && (ring_pairs != 1 && ring_pairs != 2 && ring_pairs != 4 && ring_pairs != 8))
    return SPH_EINVAL;
  if (ring_pairs && (p->nlat2 % ring_pairs != 0 || (size_t)ring_pairs * p->nphi > 8192)) return SPH_EINVAL;
  if (z_cols != 0 && (z_cols < 1 || z_cols > 64 || (z_cols & (z_cols - 1)) || z_cols * p->nz > 4096))
    return SPH_EINVAL;
  p->tile_np = ring_pairs;
  p->tile_lb = z_cols;
  if (p->precision == SPH_MIXED && rows != p->tile_nr) {
    // the scalar table tiles are rebuilt: not while clones share them
    if (p->tables && p->tables.use_count() > 1) return SPH_EINVAL;
    p->tile_nr = rows;
    const int rc = mixed_retile(p);
    if (p->tables) {
      p->tables->tc[0] = p->tcAS;
      p->tables->tc[2] = p->tcSS;
    }
    return rc;
  }
  return SPH_OK;
}

extern "C" int sph_plan_status(sph_plan* p) {
  if (!p) return SPH_EINVAL;
  SPH_CUDA_OK(cudaDeviceSynchronize());
  const int rc = mixed_status(p);
  if (rc == SPH_ETIMEDOUT) SPH_CUDA_OK(cudaMemset(p->dflag, 0, sizeof(int)));
  return rc;
}

extern "C" int sph_timer_enable(sph_plan* p, int on) {
  if (!p) return SPH_EINVAL;
  p->timing = on ? 1 : 0;
  return SPH_OK;
}

extern "C" int sph_timer_reset(sph_plan* p) {
  if (!p) return SPH_EINVAL;
  p->ev_used = 0;
  return SPH_OK;
}

extern "C" int sph_timer_read(sph_plan* p, double* ms, int* launches) {
  if (!p || !ms || !launches) return SPH_EINVAL;
  for (int c = 0; c < SPH_NTIMERS; ++c) {
    ms[c] = 0.0;
    launches[c] = 0;
  }
  for (int i = 0; i < p->ev_used; ++i) {
    if (cudaEventSynchronize(p->ev_pool[2 * i + 1]) != cudaSuccess) return SPH_ECUDA;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, p->ev_pool[2 * i], p->ev_pool[2 * i + 1]) != cudaSuccess) return SPH_ECUDA;
    ms[p->ev_class[i]] += t;
    launches[p->ev_class[i]] += 1;
  }
  return SPH_OK;
}

// ---------------------------------------------------------------- transforms
#define ST(s) ((cudaStream_t)(s))
#define RC(x)                 \
  do {                        \
    int r_ = (x);             \
    if (r_ != SPH_OK) return r_; \
  } while (0)
#define D2(x) reinterpret_cast<double2*>(x)
#define CD2(x) reinterpret_cast<const double2*>(x)

// Selects the planes that feed the FC-Gram continuation for the FP64
// launchers while it lives (mixed plans recompute them in FP64).
struct BoundaryPlanes {
  const sph_plan* p;
  explicit BoundaryPlanes(const sph_plan* p_) : p(p_) {
    p->sel_kz = p->d_bplanes;
    p->sel_n = p->nbplanes;
  }
  ~BoundaryPlanes() {
    p->sel_kz = nullptr;
    p->sel_n = 0;
  }
};

// While it lives, the angular launchers (which take their plane count from
// nz) see the caller's plane slab as the plan's planes.  The angular
// transform of a plane does not depend on the plane's index.
struct PlaneSlab {
  sph_plan* p;
  int nz0;
  explicit PlaneSlab(sph_plan* p_) : p(p_), nz0(p_->nz) { p->nz = p->nzv; }
  ~PlaneSlab() { p->nz = nz0; }
};

extern "C" int sph_plan_set_slab(sph_plan* p, int k0, int nplanes, int lm0, int nlm_local) {
  if (!p || k0 < 0 || nplanes < 1 || k0 + nplanes > p->nz || lm0 < 0 || nlm_local < 1 ||
      lm0 + nlm_local > p->nlm)
    return SPH_EINVAL;
  p->k0 = k0;
  p->nzv = nplanes;
  p->lm0 = lm0;
  p->nlmv = nlm_local;
  return SPH_OK;
}

extern "C" int sph_range(int n1, int n2, int nprocs, int irank, int* ista, int* iend) {
  if (!ista || !iend || nprocs < 1 || irank < 0 || irank >= nprocs || n2 < n1 - 1) return SPH_EINVAL;
  // range (src/sphp/sphp_sca.F90:596-626): the first mod(n, nprocs) ranks take one more
  const int n = n2 - n1 + 1, w1 = n / nprocs, w2 = n % nprocs;
  *ista = irank * w1 + n1 + std::min(irank, w2);
  *iend = *ista + w1 - 1 + (w2 > irank ? 1 : 0);
  return SPH_OK;
}

extern "C" int sph_fftp2d_real_to_complex_xy(sph_plan* p, const double* in, double* out, void* s) {
  if (!p || !in || !out) return SPH_EINVAL;
  PlaneSlab view(p);
  const double* g[1] = {in};
  if (p->precision == SPH_MIXED) {
    RC(launch_phi_fwd32(p, g, 1, ST(s)));
    RC(launch_tc_analysis(p, 0, D2(out), nullptr, ST(s)));
    if (!p->nbplanes || !p->bpass) return SPH_OK;
    BoundaryPlanes sel(p);
    RC(launch_phi_fwd(p, g, 1, ST(s)));
    return launch_leg_analysis(p, 0, D2(out), ST(s));
  }
  RC(launch_phi_fwd(p, g, 1, ST(s)));
  return launch_leg_analysis(p, 0, D2(out), ST(s));
}

extern "C" int sph_fftp2d_complex_to_real_xy(sph_plan* p, const double* in, double* out, void* s) {
  if (!p || !in || !out) return SPH_EINVAL;
  PlaneSlab view(p);
  double* g[1] = {out};
  if (p->precision == SPH_MIXED) {
    RC(launch_tc_synthesis(p, 0, CD2(in), nullptr, ST(s)));
    RC(launch_phi_inv32(p, g, 1, ST(s)));
    if (!p->nbplanes || !p->bpass) return SPH_OK;
    BoundaryPlanes sel(p);
    RC(launch_leg_synthesis(p, CD2(in), 0, ST(s)));
    return launch_phi_inv(p, g, 1, ST(s));
  }
  RC(launch_leg_synthesis(p, CD2(in), 0, ST(s)));
  return launch_phi_inv(p, g, 1, ST(s));
}

extern "C" int sph_fftp1d_real_to_complex_z(sph_plan* p, double* inout, void* s) {
  if (!p || !inout) return SPH_EINVAL;
  return launch_zfft(p, Z_FWD, CD2(inout), D2(inout), 0, ST(s));
}

extern "C" int sph_fftp1d_complex_to_real_z(sph_plan* p, double* inout, void* s) {
  if (!p || !inout) return SPH_EINVAL;
  return launch_zfft(p, Z_INV, CD2(inout), D2(inout), 0, ST(s));
}

extern "C" int sph_fftp3d_real_to_complex(sph_plan* p, const double* in, double* out, void* s) {
  if (!p || !slab_whole(p)) return SPH_EINVAL;  // the 3D transforms need the slab transpose
  if (p && in && out && p->precision == SPH_MIXED && p->C > 0 && p->contg) {
    // continue the physical planes first (FP64): the continuation then acts
    // on exact data and the angular round-off of every plane stays local
    const double* g[1] = {in};
    const double* gh[1] = {p->contg};
    RC(launch_cont_phys(p, g, 1, ST(s)));
    RC(launch_phi_fwd32(p, g, 1, ST(s), gh));
    RC(launch_tc_analysis(p, 0, D2(out), nullptr, ST(s)));
    return launch_zfft(p, Z_FWD, CD2(out), D2(out), 0, ST(s), false);
  }
  RC(sph_fftp2d_real_to_complex_xy(p, in, out, s));
  return sph_fftp1d_real_to_complex_z(p, out, s);
}

extern "C" int sph_fftp3d_complex_to_real(sph_plan* p, double* in, double* out, void* s) {
  if (!p || !slab_whole(p)) return SPH_EINVAL;
  if (in && out && zinv_tiles_ok(p)) {  // mixed: the z inverse writes the synthesis tiles (input preserved)
    RC(launch_zinv_tiles(p, CD2(in), 0, ST(s)));
    RC(launch_tc_synthesis_tiles(p, 0, ST(s)));
    double* g[1] = {out};
    return launch_phi_inv32(p, g, 1, ST(s));
  }
  RC(sph_fftp1d_complex_to_real_z(p, in, s));
  return sph_fftp2d_complex_to_real_xy(p, in, out, s);
}

extern "C" int sph_fftp2d_vec_to_qst(sph_plan* p, const double* vr, const double* vt, const double* vp,
                                     double* q, double* sO, double* t, void* s) {
  if (!p || !vr || !vt || !vp || !q || !sO || !t) return SPH_EINVAL;
  PlaneSlab view(p);
  const double* g[3] = {vr, vt, vp};
  if (p->precision == SPH_MIXED) {
    RC(launch_phi_fwd32(p, g, 3, ST(s)));
    RC(launch_tc_analysis(p, 0, D2(q), nullptr, ST(s)));
    RC(launch_tc_analysis(p, 1, D2(sO), D2(t), ST(s)));
    if (!p->nbplanes || !p->bpass) return SPH_OK;
    BoundaryPlanes sel(p);
    RC(launch_phi_fwd(p, g, 3, ST(s)));
    RC(launch_leg_analysis(p, 0, D2(q), ST(s)));
    return launch_vec_analysis(p, D2(sO), D2(t), ST(s));
  }
  RC(launch_phi_fwd(p, g, 3, ST(s)));
  RC(launch_leg_analysis(p, 0, D2(q), ST(s)));
  return launch_vec_analysis(p, D2(sO), D2(t), ST(s));
}

extern "C" int sph_fftp2d_qst_to_vec(sph_plan* p, const double* q, const double* sI, const double* t,
                                     double* vr, double* vt, double* vp, void* s) {
  if (!p || !vr || !vt || !vp || !q || !sI || !t) return SPH_EINVAL;
  PlaneSlab view(p);
  double* g[3] = {vr, vt, vp};
  if (p->precision == SPH_MIXED) {
    RC(launch_tc_synthesis(p, 0, CD2(q), nullptr, ST(s)));
    RC(launch_tc_synthesis(p, 1, CD2(sI), CD2(t), ST(s)));
    RC(launch_phi_inv32(p, g, 3, ST(s)));
    if (!p->nbplanes || !p->bpass) return SPH_OK;
    BoundaryPlanes sel(p);
    RC(launch_leg_synthesis(p, CD2(q), 0, ST(s)));
    RC(launch_vec_synthesis(p, CD2(sI), CD2(t), ST(s)));
    return launch_phi_inv(p, g, 3, ST(s));
  }
  RC(launch_leg_synthesis(p, CD2(q), 0, ST(s)));
  RC(launch_vec_synthesis(p, CD2(sI), CD2(t), ST(s)));
  return launch_phi_inv(p, g, 3, ST(s));
}

extern "C" int sph_fftp3d_vec_to_qst(sph_plan* p, const double* vr, const double* vt, const double* vp,
                                     double* q, double* sO, double* t, void* s) {
  if (!p || !vr || !vt || !vp || !q || !sO || !t || !slab_whole(p)) return SPH_EINVAL;
  if (p->precision == SPH_MIXED && p->C > 0 && p->contg) {
    const double* g[3] = {vr, vt, vp};
    const double* gh[3] = {p->contg, p->contg + (size_t)p->C * p->nphi * p->nlat,
                           p->contg + (size_t)2 * p->C * p->nphi * p->nlat};
    RC(launch_cont_phys(p, g, 3, ST(s)));
    RC(launch_phi_fwd32(p, g, 3, ST(s), gh));
    RC(launch_tc_analysis(p, 0, D2(q), nullptr, ST(s)));
    RC(launch_tc_analysis(p, 1, D2(sO), D2(t), ST(s)));
    for (double* x : {q, sO, t}) RC(launch_zfft(p, Z_FWD, CD2(x), D2(x), 0, ST(s), false));
    return SPH_OK;
  }
  RC(sph_fftp2d_vec_to_qst(p, vr, vt, vp, q, sO, t, s));
  for (double* x : {q, sO, t}) RC(sph_fftp1d_real_to_complex_z(p, x, s));
  return SPH_OK;
}

extern "C" int sph_fftp3d_qst_to_vec(sph_plan* p, double* q, double* sI, double* t, double* vr, double* vt,
                                     double* vp, void* s) {
  if (!p || !vr || !vt || !vp || !q || !sI || !t || !slab_whole(p)) return SPH_EINVAL;
  if (zinv_tiles_ok(p)) {  // mixed: the z inverses write the synthesis tiles (inputs preserved)
    RC(launch_zinv_tiles(p, CD2(q), 0, ST(s)));
    RC(launch_tc_synthesis_tiles(p, 0, ST(s)));
    RC(launch_zinv_tiles(p, CD2(sI), 0, ST(s)));
    RC(launch_zinv_tiles(p, CD2(t), 1, ST(s)));
    RC(launch_tc_synthesis_tiles(p, 1, ST(s)));
    double* g[3] = {vr, vt, vp};
    return launch_phi_inv32(p, g, 3, ST(s));
  }
  for (double* x : {q, sI, t}) RC(sph_fftp1d_complex_to_real_z(p, x, s));
  return sph_fftp2d_qst_to_vec(p, q, sI, t, vr, vt, vp, s);
}

// ---------------------------------------------------------------- operators
extern "C" int sph_derivr(sph_plan* p, const double* a, double* b, int order, char esp, void* s) {
  if (!p || !a || !b || order < 0 || order > 4) return SPH_EINVAL;
  if (esp == 'k') return launch_kmul(p, CD2(a), D2(b), order, ST(s));
  if (esp != 'r') return SPH_EINVAL;
  if (order == 0) {  // forward and back: the continuation points are recomputed
    RC(launch_zfft(p, Z_FWD, CD2(a), D2(b), 0, ST(s)));
    return launch_zfft(p, Z_INV, CD2(b), D2(b), 0, ST(s));
  }
  return launch_zfft(p, Z_DERIV, CD2(a), D2(b), order, ST(s));
}

extern "C" int sph_laplang(sph_plan* p, const double* a, double* b, void* s) {
  if (!p || !a || !b) return SPH_EINVAL;
  return launch_laplang(p, CD2(a), D2(b), ST(s));
}

extern "C" int sph_multr(sph_plan* p, const double* a, double* b, int power, void* s) {
  if (!p || !a || !b) return SPH_EINVAL;
  return launch_multr(p, CD2(a), D2(b), power, ST(s));
}

extern "C" int sph_dlr(sph_plan* p, const double* a, double* b, void* s) {
  if (!p || !a || !b) return SPH_EINVAL;
  return launch_zfft(p, Z_DLR, CD2(a), D2(b), 2, ST(s));
}

extern "C" int sph_saxpby_c(sph_plan* p, double* z, const double* x, double a, const double* y, double b,
                            void* s) {
  if (!p || !z || !x || !y) return SPH_EINVAL;
  return launch_saxpby(p, z, x, a, y, b, 2 * spec_view(p), ST(s));
}

extern "C" int sph_saxpby_r(sph_plan* p, double* z, const double* x, double a, const double* y, double b,
                            void* s) {
  if (!p || !z || !x || !y) return SPH_EINVAL;
  return launch_saxpby(p, z, x, a, y, b, grid_view(p), ST(s));
}

extern "C" int sph_fc_filter(sph_plan* p, double* a, char esp, void* s) {
  if (!p || !a) return SPH_EINVAL;
  if (esp == 'k') return launch_filter_k(p, D2(a), ST(s));
  if (esp != 'r') return SPH_EINVAL;
  return launch_zfft(p, Z_FILTER, CD2(a), D2(a), 0, ST(s));
}

extern "C" int sph_copy(sph_plan* p, const double* a, double* b, void* s) {
  if (!p || !a || !b) return SPH_EINVAL;
  SPH_CUDA_OK(cudaMemcpyAsync(b, a, spec_view(p) * sizeof(double2), cudaMemcpyDeviceToDevice, ST(s)));
  return SPH_OK;
}

extern "C" int sph_prodvec(sph_plan* p, const double* ar, const double* at, const double* ap,
                           const double* br, const double* bt, const double* bp, double* cr, double* ct,
                           double* cp, void* s) {
  if (!p || !ar || !at || !ap || !br || !bt || !bp || !cr || !ct || !cp) return SPH_EINVAL;
  const double* A[3] = {ar, at, ap};
  const double* B[3] = {br, bt, bp};
  double* Cc[3] = {cr, ct, cp};
  return launch_prodvec(p, A, B, Cc, ST(s));
}

// ---------------------------------------------------------------- boundary
// Host pieces of invDl_setup (src/boundary/boundary_mod.f90:140-241), in
// extended precision.  The reference builds the derivative matrices by
// probing its FFT derivative with unit vectors (derivr_mat,
// boundary_mod.f90:96-137) and factors B_l in FP64; both round at the
// level of the largest matrix entries (about 1e-13 of them at nz = 128),
// and B_l^-1 and the second derivative that phi = D_l W takes afterwards
// amplify that to 1e-11 (no slip) and 1e-10 (free slip) in phi.  Here the
// matrices come from a direct DFT with long double twiddles and sums, the
// LU and the solve run in long double, and only binv and the four d2 rows
// are rounded to FP64: W = binv phi is then correct to a few ulp.

// Columns of the FC-Gram radial derivatives of orders 1 and 2 applied to the
// unit vectors e_j on the N physical points: continuation (the z transform's
// summation order), forward DFT / nz, (i kz)^order, inverse DFT, real part.
static void host_derivr_matrices(const sph_plan* p, std::vector<ld>& D1, std::vector<ld>& D2) {
  const int nz = p->nz, n = p->N, C = p->C, d = p->d;
  D1.assign((size_t)n * n, 0.0L);
  D2.assign((size_t)n * n, 0.0L);
  std::vector<ld> cs((size_t)nz * nz), sn((size_t)nz * nz);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < nz; ++j) {
      const ld a = -2.0L * kPi * (ld)((long)k * j % nz) / nz;
      cs[(size_t)k * nz + j] = cosl(a);
      sn[(size_t)k * nz + j] = sinl(a);
    }
  std::vector<ld> f(nz), Fr(nz), Fi(nz), R1(nz), I1(nz), R2(nz), I2(nz);
  for (int j = 0; j < n; ++j) {
    std::fill(f.begin(), f.end(), 0.0L);
    f[j] = 1.0L;
    for (int ii = 0; ii < C; ++ii) {
      ld acc = (ld)p->dir[ii] * f[n - d] + (ld)p->dir[C - 1 - ii] * f[d - 1];
      for (int jj = 1; jj < d; ++jj)
        acc = (acc + (ld)p->dir[ii + (size_t)C * jj] * f[n - d + jj]) +
              (ld)p->dir[(C - 1 - ii) + (size_t)C * jj] * f[d - 1 - jj];
      f[n + ii] = acc;
    }
    for (int k = 0; k < nz; ++k) {
      ld sr = 0, si = 0;
      for (int q = 0; q < nz; ++q) {
        sr += cs[(size_t)k * nz + q] * f[q];
        si += sn[(size_t)k * nz + q] * f[q];
      }
      const ld re = sr / nz, im = si / nz, kz = (ld)p->kz[k];
      R1[k] = -kz * im;  // (i kz) (re + i im)
      I1[k] = kz * re;
      R2[k] = -kz * kz * re;  // (i kz)^2 (re + i im)
      I2[k] = -kz * kz * im;
    }
    for (int i = 0; i < n; ++i) {
      ld s1 = 0, s2 = 0;
      for (int k = 0; k < nz; ++k) {  // real part of the inverse DFT (sign +1)
        const ld c = cs[(size_t)k * nz + i], sv = sn[(size_t)k * nz + i];
        s1 += c * R1[k] + sv * I1[k];
        s2 += c * R2[k] + sv * I2[k];
      }
      D1[i + (size_t)n * j] = s1;
      D2[i + (size_t)n * j] = s2;
    }
  }
}

// LU with partial pivoting (DGETRF's steps), column-major, in long double
static int lu_decompose(int n, std::vector<ld>& a, std::vector<int>& piv) {
  piv.resize(n);
  for (int k = 0; k < n; ++k) {
    int pr = k;
    ld best = fabsl(a[k + (size_t)n * k]);
    for (int i = k + 1; i < n; ++i)
      if (fabsl(a[i + (size_t)n * k]) > best) {
        best = fabsl(a[i + (size_t)n * k]);
        pr = i;
      }
    piv[k] = pr;
    if (best == 0.0L) return 1;
    if (pr != k)
      for (int j = 0; j < n; ++j) std::swap(a[k + (size_t)n * j], a[pr + (size_t)n * j]);
    const ld inv = 1.0L / a[k + (size_t)n * k];
    for (int i = k + 1; i < n; ++i) a[i + (size_t)n * k] *= inv;
    for (int j = k + 1; j < n; ++j) {
      const ld f = a[k + (size_t)n * j];
      if (f != 0.0L)
        for (int i = k + 1; i < n; ++i) a[i + (size_t)n * j] -= a[i + (size_t)n * k] * f;
    }
  }
  return 0;
}

// solve with the factors (DGETRS's steps), one right-hand side
static void lu_apply(int n, const std::vector<ld>& a, const std::vector<int>& piv, ld* x) {
  for (int k = 0; k < n; ++k) std::swap(x[k], x[piv[k]]);
  for (int k = 0; k < n; ++k)
    for (int i = k + 1; i < n; ++i) x[i] -= a[i + (size_t)n * k] * x[k];
  for (int k = n - 1; k >= 0; --k) {
    x[k] /= a[k + (size_t)n * k];
    for (int i = 0; i < k; ++i) x[i] -= a[i + (size_t)n * k] * x[k];
  }
}

// binv(:, :, l) for l = 1..lmax: columns 3..N-2 of B_l^-1 (invDl_setup's M_l),
// the l spread over host threads
static int host_binv(const sph_plan* p, int kin, int kout, const std::vector<ld>& d1, const std::vector<ld>& d2,
                     std::vector<double>& binv) {
  const int n = p->N, lmax = p->lmax;
  binv.assign((size_t)std::max(lmax, 1) * n * (n - 4), 0.0);
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<int> failed(nth, 0);
  std::vector<std::thread> th;
  for (int t = 0; t < nth; ++t)
    th.emplace_back([&, t]() {
      std::vector<ld> b((size_t)n * n), esc(n), x(n);
      std::vector<int> piv;
      for (int l = 1 + t; l <= lmax; l += nth) {
        std::fill(b.begin(), b.end(), 0.0L);
        auto B = [&](int i, int j) -> ld& { return b[(i - 1) + (size_t)n * (j - 1)]; };
        auto DM1 = [&](int i, int j) { return d1[(i - 1) + (size_t)n * (j - 1)]; };
        auto DM2 = [&](int i, int j) { return d2[(i - 1) + (size_t)n * (j - 1)]; };
        B(1, 1) = 1.0L;
        // W' = 0 (noslip) or W'' - 2 W'/r = 0 (freeslip) at the inner wall
        for (int j = 1; j <= n; ++j) B(2, j) = kin ? DM2(1, j) - 2.0L / (ld)p->z[0] * DM1(1, j) : DM1(1, j);
        for (int i = 3; i <= n - 2; ++i) {
          for (int j = 1; j <= n; ++j) B(i, j) = DM2(i, j);
          const ld zi = (ld)p->z[i - 1];
          B(i, i) = B(i, i) - (ld)(l * (l + 1)) / (zi * zi);
        }
        for (int j = 1; j <= n; ++j)
          B(n - 1, j) = kout ? DM2(n, j) - 2.0L / (ld)p->z[n - 1] * DM1(n, j) : DM1(n, j);
        B(n, n) = 1.0L;
        for (int i = 1; i <= n; ++i) {  // rows scaled by their largest entry, as the reference does
          ld mx = 0.0L;
          for (int j = 1; j <= n; ++j) mx = std::max(mx, fabsl(B(i, j)));
          esc[i - 1] = mx;
          for (int j = 1; j <= n; ++j) B(i, j) /= mx;
        }
        if (lu_decompose(n, b, piv)) {
          failed[t] = 1;
          return;
        }
        double* M = &binv[(size_t)(l - 1) * n * (n - 4)];
        for (int j = 0; j < n - 4; ++j) {
          std::fill(x.begin(), x.end(), 0.0L);
          x[j + 2] = 1.0L / esc[j + 2];
          lu_apply(n, b, piv, x.data());
          for (int i = 0; i < n; ++i) M[i + (size_t)n * j] = (double)x[i];
        }
      }
    });
  for (auto& x : th) x.join();
  for (int f : failed)
    if (f) return SPH_EINVAL;
  return SPH_OK;
}

static int ensure_nl_scratch(sph_plan* p) {
  for (int i = 0; i < 12; ++i)
    if (!p->sp[i] && cudaMalloc((void**)&p->sp[i], spec_elems(p) * sizeof(double2)) != cudaSuccess)
      return SPH_ENOMEM;
  for (int i = 0; i < 9; ++i)
    if (!p->gr[i] && cudaMalloc((void**)&p->gr[i], grid_elems(p) * sizeof(double)) != cudaSuccess)
      return SPH_ENOMEM;
  p->nsp = 12;
  p->ngr = 9;
  return SPH_OK;
}

extern "C" int sph_setup_bc(sph_plan* p, const char* bcint, const char* bcext) {
  if (!p) return SPH_EINVAL;
  // v_parsebc (vboundary.f90:10-31) knows 'noslip' (0); 'freeslip' (1) is
  // added here: W = 0, W'' - 2 W'/r = 0, Z' - 2 Z/r = 0 at the wall
  auto parse = [](const char* s) {
    if (!s) return -1;
    std::string t(s);
    t.erase(0, t.find_first_not_of(" \t"));
    t.erase(t.find_last_not_of(" \t") + 1);
    for (auto& c : t) c = (char)tolower(c);
    return t == "noslip" ? 0 : t == "freeslip" ? 1 : -1;
  };
  const int kin = parse(bcint), kout = parse(bcext);
  if (kin < 0 || kout < 0) return SPH_EINVAL;
  const int n = p->N, lmax = p->lmax;
  if (p->C <= 0 || n < 6) return SPH_EINVAL;
  if ((kin == 1 || kout == 1) && (p->neu[0].empty() || !p->d_neu)) return SPH_ENOTREADY;
  const int kinds = kin + 2 * kout;
  if (p->bc_ready && p->bck[0] == kin && p->bck[1] == kout) return SPH_OK;
  if (p->bc_own) {
    if (p->binv) cudaFree(p->binv);
    if (p->d2bor) cudaFree(p->d2bor);
    p->bc_own = 0;
  }
  p->binv = p->d2bor = nullptr;
  p->bc_ready = 0;
  p->bck[0] = kin;
  p->bck[1] = kout;
  if (p->tables && p->tables->binv && p->tables->bc_kinds == kinds) {  // built for a plan sharing the tables
    p->binv = p->tables->binv;
    p->d2bor = p->tables->d2bor;
    RC(ensure_nl_scratch(p));
    p->bc_ready = 1;
    return SPH_OK;
  }
  std::vector<ld> d1, d2;
  host_derivr_matrices(p, d1, d2);
  std::vector<double> binv;
  RC(host_binv(p, kin, kout, d1, d2, binv));
  std::vector<double> d2bor((size_t)4 * n);
  for (int j = 0; j < n; ++j) {
    d2bor[0 + 4 * (size_t)j] = (double)d2[0 + (size_t)n * j];
    d2bor[1 + 4 * (size_t)j] = (double)d2[1 + (size_t)n * j];
    d2bor[2 + 4 * (size_t)j] = (double)d2[(n - 2) + (size_t)n * j];
    d2bor[3 + 4 * (size_t)j] = (double)d2[(n - 1) + (size_t)n * j];
  }
  double *db = nullptr, *dd = nullptr;
  int rc = upload(&db, binv.data(), binv.size());
  if (rc == SPH_OK) rc = upload(&dd, d2bor.data(), d2bor.size());
  if (rc != SPH_OK) {
    if (db) cudaFree(db);
    if (dd) cudaFree(dd);
    return rc;
  }
  p->binv = db;
  p->d2bor = dd;
  if (p->tables && !p->tables->binv) {  // the tables own them from now on
    p->tables->binv = db;
    p->tables->d2bor = dd;
    p->tables->bc_kinds = kinds;
  } else {
    p->bc_own = 1;  // other kinds than the shared matrices: this plan's own
  }
  RC(ensure_nl_scratch(p));
  p->bc_ready = 1;
  return SPH_OK;
}

extern "C" int sph_dirichlet(sph_plan* p, double* a, void* s) {
  if (!p || !a) return SPH_EINVAL;
  return launch_dirichlet(p, D2(a), ST(s));
}

extern "C" int sph_invDl(sph_plan* p, const double* phi, double* w, void* s) {
  if (!p || !phi || !w) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  return launch_invDl(p, CD2(phi), D2(w), ST(s));
}

extern "C" int sph_v_imposebc(sph_plan* p, double* tor, double* phi, double* pol, void* s) {
  if (!p || !tor || !phi || !pol) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  RC(launch_bc_walls(p, D2(tor), ST(s)));
  RC(launch_invDl(p, CD2(phi), D2(pol), ST(s)));
  return launch_zfft(p, Z_DLR, CD2(pol), D2(phi), 2, ST(s));
}

extern "C" int sph_v_imposebc_fast(sph_plan* p, double* tor, double* phi, double* pol, void* s) {
  if (!p || !tor || !phi || !pol) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  RC(launch_bc_walls(p, D2(tor), ST(s)));
  RC(launch_invDl(p, CD2(phi), D2(pol), ST(s)));
  return launch_bc_fast_rows(p, D2(phi), CD2(pol), ST(s));
}

// ---------------------------------------------------------------- NL + RK3
// Mixed plans: inside the NL step the planes that feed the FC-Gram
// continuation are transformed in FP64 as well, so that the radial
// derivatives of the step do not amplify their angular round-off.
struct BoundaryPass {
  const sph_plan* p;
  explicit BoundaryPass(const sph_plan* p_) : p(p_) { p->bpass = 1; }
  ~BoundaryPass() { p->bpass = 0; }
};

static int nl_rhs_impl(sph_plan* p, const double2* Z, const double2* W, const double2* F, double nu,
                       double2* rz, double2* rf, cudaStream_t st) {
  BoundaryPass bp(p);
  double2 *s0 = p->sp[0], *s1 = p->sp[1], *s2 = p->sp[2], *s3 = p->sp[3], *s4 = p->sp[4];
  double* g[9];
  for (int i = 0; i < 9; ++i) g[i] = p->gr[i];
  // u: Q = l(l+1) W/r^2, S = W'/r, T = Z/r
  RC(launch_qst_scale(p, W, s0, -2, 1, 1.0, st));
  RC(launch_zfft(p, Z_DERIV, W, s3, 1, st));
  RC(launch_qst_scale(p, s3, s1, -1, 0, 1.0, st));
  RC(launch_qst_scale(p, Z, s2, -1, 0, 1.0, st));
  RC(sph_fftp2d_qst_to_vec(p, (double*)s0, (double*)s1, (double*)s2, g[0], g[1], g[2], st));
  // curl u: Q = l(l+1) Z/r^2, S = Z'/r, T = -phi/r
  RC(launch_qst_scale(p, Z, s0, -2, 1, 1.0, st));
  RC(launch_zfft(p, Z_DERIV, Z, s3, 1, st));
  RC(launch_qst_scale(p, s3, s1, -1, 0, 1.0, st));
  RC(launch_qst_scale(p, F, s2, -1, 0, -1.0, st));
  RC(sph_fftp2d_qst_to_vec(p, (double*)s0, (double*)s1, (double*)s2, g[3], g[4], g[5], st));
  SPH_CUDA_OK(cudaMemsetAsync(p->energy, 0, sizeof(double), st));
  RC(launch_energy(p, g[0], g[1], g[2], p->energy, st));
  // N = u x curl u, back to (Q, S, T)
  const double* A[3] = {g[0], g[1], g[2]};
  const double* B[3] = {g[3], g[4], g[5]};
  double* Cc[3] = {g[6], g[7], g[8]};
  RC(launch_prodvec(p, A, B, Cc, st));
  RC(sph_fftp2d_vec_to_qst(p, g[6], g[7], g[8], (double*)s0, (double*)s1, (double*)s2, st));
  // rhs_z = r T_N + nu D_l Z
  RC(launch_multr(p, s2, s4, 1, st));
  RC(launch_zfft(p, Z_DLR, Z, s3, 2, st));
  RC(launch_saxpby(p, (double*)rz, (const double*)s4, 1.0, (const double*)s3, nu, 2 * spec_elems(p), st));
  // rhs_phi = (r S_N)' - Q_N + nu D_l phi
  RC(launch_multr(p, s1, s4, 1, st));
  RC(launch_zfft(p, Z_DERIV, s4, s3, 1, st));
  RC(launch_saxpby(p, (double*)rf, (const double*)s3, 1.0, (const double*)s0, -1.0, 2 * spec_elems(p), st));
  RC(launch_zfft(p, Z_DLR, F, s4, 2, st));
  RC(launch_saxpby(p, (double*)rf, (const double*)rf, 1.0, (const double*)s4, nu, 2 * spec_elems(p), st));
  return SPH_OK;
}

extern "C" int sph_nl_rhs(sph_plan* p, const double* Z, const double* W, const double* phi, double nu,
                          double* rhs_z, double* rhs_phi, double* energy, void* s) {
  if (!p || !Z || !W || !phi || !rhs_z || !rhs_phi || !slab_whole(p)) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  RC(nl_rhs_impl(p, CD2(Z), CD2(W), CD2(phi), nu, D2(rhs_z), D2(rhs_phi), ST(s)));
  if (energy) {
    SPH_CUDA_OK(cudaMemcpyAsync(energy, p->energy, sizeof(double), cudaMemcpyDeviceToHost, ST(s)));
    SPH_CUDA_OK(cudaStreamSynchronize(ST(s)));
  }
  return SPH_OK;
}

extern "C" int sph_rk3_step(sph_plan* p, double* Z, double* W, double* phi, double nu, double dt,
                            double* energy, void* s) {
  if (!p || !Z || !W || !phi || !slab_whole(p)) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  cudaStream_t st = ST(s);
  const size_t bytes = spec_elems(p) * sizeof(double2);
  double2 *Z0 = p->sp[5], *F0 = p->sp[6], *rz = p->sp[7], *rf = p->sp[8], *e0 = p->sp[9];
  SPH_CUDA_OK(cudaMemcpyAsync(Z0, Z, bytes, cudaMemcpyDeviceToDevice, st));
  SPH_CUDA_OK(cudaMemcpyAsync(F0, phi, bytes, cudaMemcpyDeviceToDevice, st));
  for (int o = 3; o >= 1; --o) {
    RC(nl_rhs_impl(p, CD2(Z), CD2(W), CD2(phi), nu, rz, rf, st));
    if (o == 3) SPH_CUDA_OK(cudaMemcpyAsync(e0, p->energy, sizeof(double), cudaMemcpyDeviceToDevice, st));
    RC(launch_saxpby(p, Z, (const double*)Z0, 1.0, (const double*)rz, dt / o, 2 * spec_elems(p), st));
    RC(launch_saxpby(p, phi, (const double*)F0, 1.0, (const double*)rf, dt / o, 2 * spec_elems(p), st));
    RC(sph_v_imposebc(p, Z, phi, W, st));
  }
  if (energy) {
    SPH_CUDA_OK(cudaMemcpyAsync(energy, e0, sizeof(double), cudaMemcpyDeviceToHost, st));
    SPH_CUDA_OK(cudaStreamSynchronize(st));
  }
  return SPH_OK;
}
