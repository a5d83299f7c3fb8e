// sph_oracle.cpp -- CPU restatement of REDONDITO's pseudospectral transform
// core.  TEST INFRASTRUCTURE ONLY: the oracle that the CUDA path is checked
// against, and the timed CPU baseline.  The product never links or calls it.
//
// The reference's CPU path is Fortran + SHTns + FFTW + OpenMPI + LAPACK, none
// of which can be built here, so this file restates its arithmetic:
//   * SHTns (version unpinned; orthonormal, no Condon-Shortley phase, Gauss
//     grid, theta contiguous; sphp_sca.F90:117-122) by Gauss-Legendre
//     quadrature with associated Legendre functions from the standard
//     three-term recurrence, evaluated in 80-bit long double;
//   * FFTW 3.3.11 many-DFT (sphp_sca.F90:124-127,389,525) by a mixed-radix
//     Cooley-Tukey FFT written here;
//   * LAPACK DGETRF/DGETRS (boundary_mod.f90:193,209) by partial-pivot LU;
//   * DGEMM (boundary_mod.f90:279) by plain loops.
// Every routine cites the reference lines it follows.
#include "sph_oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef std::complex<double> cplx;
typedef long double ldouble;

static const ldouble PI_L = 3.141592653589793238462643383279502884L;

// ---------------------------------------------------------------- FFT
// Mixed-radix decimation-in-time FFT, out of place, unnormalised.
// sign = -1: sum_j x_j exp(-2 pi i jk/n) (FFTW_FORWARD, sphp_mod.F90:34);
// sign = +1: FFTW_BACKWARD.
struct OFFT {
  int n = 0;
  std::vector<int> fac;
  std::vector<cplx> tw;  // tw[e] = exp(-2 pi i e / n)
  void init(int n_) {
    n = n_;
    fac.clear();
    int r = n;
    for (int p : {4, 2, 3, 5, 7}) {
      while (r % p == 0) { fac.push_back(p); r /= p; }
    }
    for (int p = 11; r > 1; p += 2) {
      while (r % p == 0) { fac.push_back(p); r /= p; }
    }
    tw.resize(n);
    for (int e = 0; e < n; ++e) {
      ldouble a = -2.0L * PI_L * (ldouble)e / (ldouble)n;
      tw[e] = cplx((double)cosl(a), (double)sinl(a));
    }
  }
  void rec(const cplx* in, long is, cplx* out, int len, int fi, int step, int sign) const {
    if (len == 1) { out[0] = in[0]; return; }
    int p = fac[fi], m = len / p;
    for (int r = 0; r < p; ++r) rec(in + r * is, is * p, out + r * m, m, fi + 1, step * p, sign);
    cplx t[64];
    std::vector<cplx> tv;
    cplx* tp = t;
    if (p > 64) { tv.resize(p); tp = tv.data(); }
    for (int k = 0; k < m; ++k) {
      for (int r = 0; r < p; ++r) {
        cplx w = tw[((long)r * k * step) % n];
        if (sign > 0) w = std::conj(w);
        tp[r] = out[r * m + k] * w;
      }
      for (int q = 0; q < p; ++q) {
        cplx s = 0;
        for (int r = 0; r < p; ++r) {
          cplx w = tw[((long)r * q * m * step) % n];
          if (sign > 0) w = std::conj(w);
          s += tp[r] * w;
        }
        out[q * m + k] = s;
      }
    }
  }
  void exec(const cplx* in, cplx* out, int sign) const { rec(in, 1, out, n, 0, 1, sign); }
};

// ---------------------------------------------------------------- plan
struct orc_plan {
  int lmax, nlat, nphi, nz, C, d, nlm, N;
  double rint, rext, dz, Dkz;
  std::vector<double> theta, ct, st, w;  // nlat
  std::vector<double> z, kz;             // nz
  std::vector<double> dir;               // C*d col-major
  std::vector<int> ell, emm, mbase;      // nlm, nlm, lmax+2
  OFFT fphi, fz;
  // Neumann reconstructors (fcgram_mod.f90:267-365): neu[0] first, neu[1]
  // second normal derivative, d values each (empty: not loaded)
  std::vector<double> neu[2];
  // boundary: kinds at the inner and outer wall (0 noslip, 1 freeslip)
  int bck[2] = {0, 0};
  int bc_ready = 0;
  std::vector<double> binv;   // N x (N-4) x lmax
  std::vector<double> d2bor;  // 4 x N (col-major: d2bor[k + 4*j])
};

static inline int LM(const orc_plan* p, int l, int m) { return p->mbase[m] + (l - m); }

static int g_threads = 0;
extern "C" void orc_set_threads(int n) { g_threads = n; }
extern "C" int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}
#define OMP_THREADS num_threads(orc_get_threads())

// Gauss-Legendre nodes and weights on [-1,1] by Newton iteration on the
// Legendre recurrence; ct is returned in decreasing order (theta from the
// north pole, as SHTns's Gauss grid, sphp_sca.F90:120-122).
static void gauss_legendre(int n, std::vector<double>& ct, std::vector<double>& w) {
  ct.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    ldouble x = cosl(PI_L * ((ldouble)i + 0.75L) / ((ldouble)n + 0.5L));
    ldouble dp = 0;
    auto eval = [&](ldouble xx, ldouble& pn, ldouble& dpn) {
      ldouble p0 = 1, p1 = xx;
      for (int k = 2; k <= n; ++k) {
        ldouble p2 = ((2 * k - 1) * xx * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      pn = p1;
      dpn = n * (xx * p1 - p0) / (xx * xx - 1);
    };
    for (int it = 0; it < 100; ++it) {
      ldouble pn;
      eval(x, pn, dp);
      ldouble dx = pn / dp;
      x -= dx;
      if (fabsl(dx) < 1e-18L * fabsl(x) + 1e-30L) break;
    }
    {
      ldouble pn;
      eval(x, pn, dp);
    }
    ldouble wi = 2.0L / ((1 - x * x) * dp * dp);
    ct[i] = (double)x;
    ct[n - 1 - i] = (double)(-x);
    w[i] = w[n - 1 - i] = (double)wi;
  }
}

// Orthonormal associated Legendre functions without the Condon-Shortley
// phase, P(l) = Pbar_lm(cos theta) for l = m..lmax, and optionally
// dP(l) = d Pbar_lm / d theta.  Y_lm = Pbar_lm e^{i m phi}, int |Y|^2 = 1.
static void plm_column(int lmax, int m, ldouble x, ldouble s, double* P, double* dP) {
  ldouble pmm = sqrtl(1.0L / (4.0L * PI_L));
  for (int k = 1; k <= m; ++k) pmm *= sqrtl((2.0L * k + 1.0L) / (2.0L * k)) * s;
  ldouble pl2 = 0, pl1 = pmm;
  std::vector<ldouble> tmp(lmax - m + 1);
  tmp[0] = pmm;
  if (m < lmax) {
    ldouble p = sqrtl(2.0L * m + 3.0L) * x * pmm;
    tmp[1] = p;
    pl2 = pmm;
    pl1 = p;
    for (int l = m + 2; l <= lmax; ++l) {
      ldouble ll = l, mm = m;
      ldouble a = sqrtl((4 * ll * ll - 1) / (ll * ll - mm * mm));
      ldouble b = sqrtl(((ll - 1) * (ll - 1) - mm * mm) / (4 * (ll - 1) * (ll - 1) - 1));
      ldouble pn = a * (x * pl1 - b * pl2);
      tmp[l - m] = pn;
      pl2 = pl1;
      pl1 = pn;
    }
  }
  for (int l = m; l <= lmax; ++l) P[l - m] = (double)tmp[l - m];
  if (dP) {
    for (int l = m; l <= lmax; ++l) {
      ldouble ll = l, mm = m;
      ldouble prev = (l > m) ? tmp[l - m - 1] : 0.0L;
      ldouble c = (l > m) ? sqrtl((2 * ll + 1) * (ll * ll - mm * mm) / (2 * ll - 1)) : 0.0L;
      dP[l - m] = (double)((ll * x * tmp[l - m] - c * prev) / s);
    }
  }
}

extern "C" orc_plan* orc_plan_create(int lmax, int nlat, int nphi, int nz, int C, int d,
                                     double rint, double rext, const double* dir) {
  if (lmax < 0 || nlat < 2 || (nlat & 1) || nphi <= 2 * lmax || nz < 1) return nullptr;
  if (C < 0 || d < 0 || (C > 0 && (d < 1 || nz - C < d || !dir))) return nullptr;
  orc_plan* p = new orc_plan();
  p->lmax = lmax; p->nlat = nlat; p->nphi = nphi; p->nz = nz; p->C = C; p->d = d;
  p->nlm = (lmax + 1) * (lmax + 2) / 2;
  p->N = nz - C;
  p->rint = rint; p->rext = rext;
  gauss_legendre(nlat, p->ct, p->w);
  p->theta.resize(nlat); p->st.resize(nlat);
  for (int i = 0; i < nlat; ++i) {
    p->theta[i] = std::acos(p->ct[i]);
    p->st[i] = std::sqrt((1.0 - p->ct[i]) * (1.0 + p->ct[i]));
  }
  // pseudospec_mod.f90:196-200, 223-227
  p->dz = (p->N > 1) ? (rext - rint) / (nz - C - 1) : 1.0;
  p->Dkz = 2.0 * M_PI / (p->dz * nz);
  p->z.resize(nz); p->kz.resize(nz);
  for (int k = 0; k < nz; ++k) p->z[k] = rint + p->dz * k;
  for (int k = 0; k < nz / 2; ++k) {
    p->kz[k] = (double)k * p->Dkz;
    p->kz[k + nz / 2] = (double)(k - nz / 2) * p->Dkz;
  }
  if (nz & 1) {  // odd nz: the reference's loop leaves kz(nz) unset; use the FFT frequency
    for (int k = 0; k < nz; ++k) p->kz[k] = (double)((k <= nz / 2) ? k : k - nz) * p->Dkz;
  }
  p->mbase.resize(lmax + 2);
  // mbase[m] = lm(m,m), so lm(l,m) = mbase[m] + (l - m)
  for (int m = 0; m <= lmax + 1; ++m) p->mbase[m] = m * (2 * lmax + 3 - m) / 2;
  p->ell.resize(p->nlm); p->emm.resize(p->nlm);
  for (int m = 0; m <= lmax; ++m)
    for (int l = m; l <= lmax; ++l) { p->ell[LM(p, l, m)] = l; p->emm[LM(p, l, m)] = m; }
  if (C > 0) p->dir.assign(dir, dir + (size_t)C * d);
  p->fphi.init(nphi);
  p->fz.init(nz);
  return p;
}

extern "C" void orc_plan_destroy(orc_plan* p) { delete p; }
extern "C" int orc_nlm(const orc_plan* p) { return p->nlm; }

extern "C" void orc_grid(const orc_plan* p, double* theta, double* ct, double* w, double* z,
                         double* kz, int* ell, int* emm) {
  if (theta) std::copy(p->theta.begin(), p->theta.end(), theta);
  if (ct) std::copy(p->ct.begin(), p->ct.end(), ct);
  if (w) std::copy(p->w.begin(), p->w.end(), w);
  if (z) std::copy(p->z.begin(), p->z.end(), z);
  if (kz) std::copy(p->kz.begin(), p->kz.end(), kz);
  if (ell) std::copy(p->ell.begin(), p->ell.end(), ell);
  if (emm) std::copy(p->emm.begin(), p->emm.end(), emm);
}

// fcgram_mod.f90:186-263 (load_dirichlet_tables): dir = A . Q^T.
extern "C" int orc_load_dirichlet_tables(const char* tdir, int C, int d, double* dir) {
  std::vector<double> A((size_t)C * d), Q((size_t)d * d);
  char path[4096];
  snprintf(path, sizeof path, "%s/A%d-%d.dat", tdir, C, d);
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  size_t got = fread(A.data(), sizeof(double), A.size(), f);
  fclose(f);
  if (got != A.size()) return 2;
  snprintf(path, sizeof path, "%s/Q%d.dat", tdir, d);
  f = fopen(path, "rb");
  if (!f) return 1;
  got = fread(Q.data(), sizeof(double), Q.size(), f);
  fclose(f);
  if (got != Q.size()) return 2;
  // dir(i,j) = sum_k A(i,k) * Q^T(k,j) = sum_k A(i,k) Q(j,k)
  for (int i = 0; i < C; ++i)
    for (int j = 0; j < d; ++j) {
      double s = 0;
      for (int k = 0; k < d; ++k) s += A[i + (size_t)C * k] * Q[j + (size_t)d * k];
      dir[i + (size_t)C * j] = s;
    }
  return 0;
}

// ---------------------------------------------------------------- phi FFTs
// F[(k*nlat + i)*(lmax+1) + m] = sum_j f(theta_i, phi_j, k) e^{-i m phi_j}
// for m <= lmax: two real rings per complex FFT.
static void phi_forward(const orc_plan* p, const double* grid, std::vector<cplx>& F) {
  const int nlat = p->nlat, nphi = p->nphi, M = p->lmax + 1, nz = p->nz;
  F.assign((size_t)nz * nlat * M, 0.0);
#pragma omp parallel OMP_THREADS
  {
    std::vector<cplx> zin(nphi), zout(nphi);
#pragma omp for schedule(static)
    for (long kp = 0; kp < (long)nz * (nlat / 2); ++kp) {
      int k = (int)(kp / (nlat / 2)), i = 2 * (int)(kp % (nlat / 2));
      const double* g = grid + (size_t)k * nphi * nlat;
      for (int j = 0; j < nphi; ++j) zin[j] = cplx(g[(size_t)j * nlat + i], g[(size_t)j * nlat + i + 1]);
      p->fphi.exec(zin.data(), zout.data(), -1);
      cplx* F0 = &F[((size_t)k * nlat + i) * M];
      cplx* F1 = &F[((size_t)k * nlat + i + 1) * M];
      for (int m = 0; m < M; ++m) {
        cplx a = zout[m], b = std::conj(zout[(nphi - m) % nphi]);
        F0[m] = 0.5 * (a + b);
        F1[m] = cplx(0, -0.5) * (a - b);
      }
    }
  }
}

// f(theta_i, phi_j, k) = Re F_0 + 2 Re sum_{m>0} F_m e^{i m phi_j}
static void phi_inverse(const orc_plan* p, const std::vector<cplx>& F, double* grid) {
  const int nlat = p->nlat, nphi = p->nphi, M = p->lmax + 1, nz = p->nz;
#pragma omp parallel OMP_THREADS
  {
    std::vector<cplx> zin(nphi), zout(nphi);
#pragma omp for schedule(static)
    for (long kp = 0; kp < (long)nz * (nlat / 2); ++kp) {
      int k = (int)(kp / (nlat / 2)), i = 2 * (int)(kp % (nlat / 2));
      const cplx* F0 = &F[((size_t)k * nlat + i) * M];
      const cplx* F1 = &F[((size_t)k * nlat + i + 1) * M];
      std::fill(zin.begin(), zin.end(), cplx(0));
      // z = x + i y with x <-> ring i, y <-> ring i+1 (Hermitian spectra)
      zin[0] = cplx(F0[0].real(), F1[0].real());
      for (int m = 1; m < M; ++m) {
        zin[m] += F0[m] + cplx(0, 1) * F1[m];
        zin[nphi - m] += std::conj(F0[m]) + cplx(0, 1) * std::conj(F1[m]);
      }
      p->fphi.exec(zin.data(), zout.data(), +1);
      double* g = grid + (size_t)k * nphi * nlat;
      for (int j = 0; j < nphi; ++j) {
        g[(size_t)j * nlat + i] = zout[j].real();
        g[(size_t)j * nlat + i + 1] = zout[j].imag();
      }
    }
  }
}

// ---------------------------------------------------------------- SHT
// sphp_sca.F90:311-313 (spat_to_SH per plane): Gauss quadrature,
// a_lm = sum_i w_i (2 pi/nphi) Pbar_lm(x_i) F_m(theta_i).
static void legendre_analysis(const orc_plan* p, const std::vector<cplx>& F, double* spec) {
  const int nlat = p->nlat, M = p->lmax + 1, nz = p->nz, lmax = p->lmax, nlm = p->nlm;
  cplx* S = reinterpret_cast<cplx*>(spec);
  for (size_t q = 0; q < (size_t)nz * nlm; ++q) S[q] = 0;
  const double sc = 2.0 * M_PI / p->nphi;
#pragma omp parallel OMP_THREADS
  {
    std::vector<double> P(M);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= lmax; ++m) {
      for (int i = 0; i < nlat / 2; ++i) {
        int im = nlat - 1 - i;
        plm_column(lmax, m, (ldouble)p->ct[i], sqrtl((1.0L - (ldouble)p->ct[i]) * (1.0L + (ldouble)p->ct[i])), P.data(), nullptr);
        double wi = p->w[i] * sc;
        for (int k = 0; k < nz; ++k) {
          cplx fe = (F[((size_t)k * nlat + i) * M + m] + F[((size_t)k * nlat + im) * M + m]) * wi;
          cplx fo = (F[((size_t)k * nlat + i) * M + m] - F[((size_t)k * nlat + im) * M + m]) * wi;
          cplx* out = S + (size_t)k * nlm + p->mbase[m];
          for (int l = m; l <= lmax; ++l) out[l - m] += P[l - m] * (((l - m) & 1) ? fo : fe);
        }
      }
    }
  }
  // m = 0 coefficients are real (prueba_sphp.f90:97)
  for (int k = 0; k < nz; ++k)
    for (int l = 0; l <= lmax; ++l) S[(size_t)k * nlm + l] = cplx(S[(size_t)k * nlm + l].real(), 0.0);
}

// sphp_sca.F90:484-486 (SH_to_spat per plane): F_m(theta_i) = sum_l a_lm Pbar_lm.
static void legendre_synthesis(const orc_plan* p, const double* spec, std::vector<cplx>& F) {
  const int nlat = p->nlat, M = p->lmax + 1, nz = p->nz, lmax = p->lmax, nlm = p->nlm;
  const cplx* S = reinterpret_cast<const cplx*>(spec);
  F.assign((size_t)nz * nlat * M, 0.0);
#pragma omp parallel OMP_THREADS
  {
    std::vector<double> P(M);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= lmax; ++m) {
      for (int i = 0; i < nlat / 2; ++i) {
        int im = nlat - 1 - i;
        plm_column(lmax, m, (ldouble)p->ct[i], sqrtl((1.0L - (ldouble)p->ct[i]) * (1.0L + (ldouble)p->ct[i])), P.data(), nullptr);
        for (int k = 0; k < nz; ++k) {
          const cplx* a = S + (size_t)k * nlm + p->mbase[m];
          cplx se = 0, so = 0;
          for (int l = m; l <= lmax; ++l) {
            cplx v = a[l - m];
            if (m == 0) v = cplx(v.real(), 0.0);
            if ((l - m) & 1) so += P[l - m] * v; else se += P[l - m] * v;
          }
          F[((size_t)k * nlat + i) * M + m] = se + so;
          F[((size_t)k * nlat + im) * M + m] = se - so;
        }
      }
    }
  }
}

extern "C" void orc_sh_analysis(const orc_plan* p, const double* grid, double* spec) {
  std::vector<cplx> F;
  phi_forward(p, grid, F);
  legendre_analysis(p, F, spec);
}

extern "C" void orc_sh_synthesis(const orc_plan* p, const double* spec, double* grid) {
  std::vector<cplx> F;
  legendre_synthesis(p, spec, F);
  phi_inverse(p, F, grid);
}

// sphp_vec.F90:88-92 (spat_to_SHqst): Q from v_r; S, T from (v_theta, v_phi):
//   S_lm = 1/(l(l+1)) sum_i W_i [Vt_m dPbar - i m Vp_m Pbar/sin]
//   T_lm = 1/(l(l+1)) sum_i W_i [-i m Vt_m Pbar/sin - Vp_m dPbar]
// (convention pinned by prueba_vec.f90:5-7: v = Q Y r + S r grad Y - T r x grad Y).
extern "C" void orc_qst_analysis(const orc_plan* p, const double* vr, const double* vt,
                                 const double* vp, double* q, double* s, double* t) {
  orc_sh_analysis(p, vr, q);
  const int nlat = p->nlat, M = p->lmax + 1, nz = p->nz, lmax = p->lmax, nlm = p->nlm;
  std::vector<cplx> Ft, Fp;
  phi_forward(p, vt, Ft);
  phi_forward(p, vp, Fp);
  cplx* S = reinterpret_cast<cplx*>(s);
  cplx* T = reinterpret_cast<cplx*>(t);
  for (size_t x = 0; x < (size_t)nz * nlm; ++x) { S[x] = 0; T[x] = 0; }
  const double sc = 2.0 * M_PI / p->nphi;
  const cplx I(0, 1);
#pragma omp parallel OMP_THREADS
  {
    std::vector<double> P(M), dP(M);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= lmax; ++m) {
      for (int i = 0; i < nlat / 2; ++i) {
        int im = nlat - 1 - i;
        ldouble x = p->ct[i], sn = sqrtl((1.0L - x) * (1.0L + x));
        plm_column(lmax, m, x, sn, P.data(), dP.data());
        double wi = p->w[i] * sc, rs = (double)(1.0L / sn);
        for (int k = 0; k < nz; ++k) {
          cplx t0 = Ft[((size_t)k * nlat + i) * M + m] * wi, t1 = Ft[((size_t)k * nlat + im) * M + m] * wi;
          cplx p0 = Fp[((size_t)k * nlat + i) * M + m] * wi, p1 = Fp[((size_t)k * nlat + im) * M + m] * wi;
          cplx* so = S + (size_t)k * nlm + p->mbase[m];
          cplx* to = T + (size_t)k * nlm + p->mbase[m];
          for (int l = (m == 0 ? 1 : m); l <= lmax; ++l) {
            double sg = ((l - m) & 1) ? -1.0 : 1.0;  // Pbar(-x) = sg Pbar(x), dPbar(pi-th) = -sg dPbar(th)
            double Pl = P[l - m] * rs * m, dPl = dP[l - m];
            cplx vt_dp = dPl * (t0 - sg * t1), vp_dp = dPl * (p0 - sg * p1);
            cplx vt_p = Pl * (t0 + sg * t1), vp_p = Pl * (p0 + sg * p1);
            so[l - m] += vt_dp - I * vp_p;
            to[l - m] += -I * vt_p - vp_dp;
          }
        }
      }
    }
  }
  for (int k = 0; k < nz; ++k) {
    for (int lm = 0; lm < nlm; ++lm) {
      int l = p->ell[lm];
      double f = l ? 1.0 / ((double)l * (l + 1)) : 0.0;
      cplx& sv = S[(size_t)k * nlm + lm];
      cplx& tv = T[(size_t)k * nlm + lm];
      sv *= f; tv *= f;
      if (p->emm[lm] == 0) { sv = cplx(sv.real(), 0); tv = cplx(tv.real(), 0); }
    }
  }
}

// sphp_vec.F90:156-160 (SHqst_to_spat):
//   Vt_m = sum_l S dPbar + i m T Pbar/sin ;  Vp_m = sum_l i m S Pbar/sin - T dPbar
extern "C" void orc_qst_synthesis(const orc_plan* p, const double* q, const double* s,
                                  const double* t, double* vr, double* vt, double* vp) {
  orc_sh_synthesis(p, q, vr);
  const int nlat = p->nlat, M = p->lmax + 1, nz = p->nz, lmax = p->lmax, nlm = p->nlm;
  const cplx* S = reinterpret_cast<const cplx*>(s);
  const cplx* T = reinterpret_cast<const cplx*>(t);
  std::vector<cplx> Ft((size_t)nz * nlat * M), Fp((size_t)nz * nlat * M);
  const cplx I(0, 1);
#pragma omp parallel OMP_THREADS
  {
    std::vector<double> P(M), dP(M);
#pragma omp for schedule(dynamic, 1)
    for (int m = 0; m <= lmax; ++m) {
      for (int i = 0; i < nlat / 2; ++i) {
        int im = nlat - 1 - i;
        ldouble x = p->ct[i], sn = sqrtl((1.0L - x) * (1.0L + x));
        plm_column(lmax, m, x, sn, P.data(), dP.data());
        double rs = (double)(1.0L / sn);
        for (int k = 0; k < nz; ++k) {
          const cplx* sa = S + (size_t)k * nlm + p->mbase[m];
          const cplx* ta = T + (size_t)k * nlm + p->mbase[m];
          // even/odd sums with respect to the mirror ring
          cplx te = 0, to_ = 0, pe = 0, po = 0;  // vt, vp: e = symmetric part, o = antisymmetric
          for (int l = m; l <= lmax; ++l) {
            cplx sv = sa[l - m], tv = ta[l - m];
            if (m == 0) { sv = cplx(sv.real(), 0); tv = cplx(tv.real(), 0); }
            if (l == 0) { sv = 0; tv = 0; }
            double Pl = P[l - m] * rs * m, dPl = dP[l - m];
            bool odd = (l - m) & 1;   // Pbar antisymmetric, dPbar symmetric
            cplx a = sv * dPl, b = I * tv * Pl;       // vt terms: dP part, P part
            cplx c = I * sv * Pl, e = -tv * dPl;      // vp terms
            if (odd) { te += a; to_ += b; pe += e; po += c; }
            else { to_ += a; te += b; po += e; pe += c; }
          }
          Ft[((size_t)k * nlat + i) * M + m] = te + to_;
          Ft[((size_t)k * nlat + im) * M + m] = te - to_;
          Fp[((size_t)k * nlat + i) * M + m] = pe + po;
          Fp[((size_t)k * nlat + im) * M + m] = pe - po;
        }
      }
    }
  }
  phi_inverse(p, Ft, vt);
  phi_inverse(p, Fp, vp);
}

// ---------------------------------------------------------------- z
// sphp_sca.F90:369-381: FC-Gram continuation of one column, in the
// reference's loop order; f has nz entries (0-based).
static void continuation(const orc_plan* p, cplx* f) {
  const int n = p->nz, C = p->C, d = p->d;
  if (C <= 0) return;
  const double* dir = p->dir.data();
  auto D = [&](int ii, int jj) { return dir[(ii - 1) + (size_t)C * (jj - 1)]; };
  auto F = [&](int k) -> cplx& { return f[k - 1]; };
  for (int ii = 1; ii <= C; ++ii) F(n - C + ii) = D(ii, 1) * F(n - C - d + 1) + D(C - ii + 1, 1) * F(d);
  for (int jj = 2; jj <= d; ++jj)
    for (int ii = 1; ii <= C; ++ii)
      F(n - C + ii) = F(n - C + ii) + D(ii, jj) * F(n - C - d + jj) + D(C - ii + 1, jj) * F(d - jj + 1);
}

// ncols columns of a (nz, ncols) array: the plan's nlm for whole fields, or
// any count for a slice of the lm columns (every column is independent)
static void z_columns(const orc_plan* p, double* spec, int ncols, int sign, bool cont, bool norm) {
  const int nz = p->nz, nlm = ncols;
  cplx* S = reinterpret_cast<cplx*>(spec);
#pragma omp parallel OMP_THREADS
  {
    std::vector<cplx> a(nz), b(nz);
#pragma omp for schedule(static)
    for (int lm = 0; lm < nlm; ++lm) {
      for (int k = 0; k < nz; ++k) a[k] = S[(size_t)k * nlm + lm];
      if (cont) continuation(p, a.data());
      p->fz.exec(a.data(), b.data(), sign);
      for (int k = 0; k < nz; ++k) S[(size_t)k * nlm + lm] = norm ? b[k] / (double)nz : b[k];
    }
  }
}

// fftp1d_real_to_complex_z: continuation, FFTW_FORWARD, /nz (sphp_sca.F90:332-397)
extern "C" void orc_z_forward(const orc_plan* p, double* spec) { z_columns(p, spec, p->nlm, -1, true, true); }
// fftp1d_complex_to_real_z: FFTW_BACKWARD, no normalisation (sphp_sca.F90:495-530)
extern "C" void orc_z_inverse(const orc_plan* p, double* spec) { z_columns(p, spec, p->nlm, +1, false, false); }
// the same on ncols columns of a (nz, ncols) array
extern "C" void orc_z_forward_cols(const orc_plan* p, double* spec, int ncols) {
  z_columns(p, spec, ncols, -1, true, true);
}
extern "C" void orc_z_inverse_cols(const orc_plan* p, double* spec, int ncols) {
  z_columns(p, spec, ncols, +1, false, false);
}

extern "C" void orc_3d_forward(const orc_plan* p, const double* grid, double* spec) {
  orc_sh_analysis(p, grid, spec);
  orc_z_forward(p, spec);
}
extern "C" void orc_3d_inverse(const orc_plan* p, const double* spec, double* grid) {
  std::vector<double> tmp(spec, spec + (size_t)2 * p->nz * p->nlm);
  orc_z_inverse(p, tmp.data());
  orc_sh_synthesis(p, tmp.data(), grid);
}

// ---------------------------------------------------------------- operators
static size_t nspec(const orc_plan* p) { return (size_t)p->nz * p->nlm; }

// derivr_k (pseudospec_hd.f90:60-98): b = (i kz)^p a, Nyquist kept.
static void derivr_k(const orc_plan* p, const cplx* a, cplx* b, int order) {
  cplx ip = 1;
  for (int q = 0; q < order; ++q) ip *= cplx(0, 1);
  const int nz = p->nz, nlm = p->nlm;
#pragma omp parallel for OMP_THREADS schedule(static)
  for (int k = 0; k < nz; ++k) {
    double kp = 1;
    for (int q = 0; q < order; ++q) kp *= p->kz[k];
    cplx f = ip * kp;
    for (int lm = 0; lm < nlm; ++lm) b[(size_t)k * nlm + lm] = f * a[(size_t)k * nlm + lm];
  }
}

// derivr (pseudospec_hd.f90:18-135); derivr_r copies a, goes to kz and back.
extern "C" int orc_derivr(const orc_plan* p, const double* a, double* b, int order, char esp) {
  const cplx* A = reinterpret_cast<const cplx*>(a);
  cplx* B = reinterpret_cast<cplx*>(b);
  if (esp == 'k') { derivr_k(p, A, B, order); return 0; }
  if (esp != 'r') return 1;
  std::vector<cplx> c1(A, A + nspec(p));
  orc_z_forward(p, reinterpret_cast<double*>(c1.data()));
  derivr_k(p, c1.data(), B, order);
  orc_z_inverse(p, b);
  return 0;
}

// laplang (pseudospec_hd.f90:138-172): b = -l(l+1) a
extern "C" void orc_laplang(const orc_plan* p, const double* a, double* b) {
  const cplx* A = reinterpret_cast<const cplx*>(a);
  cplx* B = reinterpret_cast<cplx*>(b);
  for (int k = 0; k < p->nz; ++k)
    for (int lm = 0; lm < p->nlm; ++lm) {
      int l = p->ell[lm];
      B[(size_t)k * p->nlm + lm] = (double)(-l * (l + 1)) * A[(size_t)k * p->nlm + lm];
    }
}

// multr (pseudospec_hd.f90:175-208): b = z^p a
extern "C" void orc_multr(const orc_plan* p, const double* a, double* b, int power) {
  const cplx* A = reinterpret_cast<const cplx*>(a);
  cplx* B = reinterpret_cast<cplx*>(b);
  for (int k = 0; k < p->nz; ++k) {
    // Fortran z**p with an integer p: repeated products, reciprocal for p < 0
    double zp = 1.0;
    for (int q = 0; q < std::abs(power); ++q) zp *= p->z[k];
    if (power < 0) zp = 1.0 / zp;
    for (int lm = 0; lm < p->nlm; ++lm) B[(size_t)k * p->nlm + lm] = zp * A[(size_t)k * p->nlm + lm];
  }
}

// saxpby_c (pseudospec_hd.f90:291-326): z = a x + b y
extern "C" void orc_saxpby_c(const orc_plan* p, double* z, const double* x, double a,
                             const double* y, double b) {
  for (size_t q = 0; q < 2 * nspec(p); ++q) z[q] = a * x[q] + b * y[q];
}

// saxpby_r (pseudospec_hd.f90:329-366)
extern "C" void orc_saxpby_r(const orc_plan* p, double* z, const double* x, double a,
                             const double* y, double b) {
  size_t n = (size_t)p->nz * p->nphi * p->nlat;
  for (size_t q = 0; q < n; ++q) z[q] = a * x[q] + b * y[q];
}

// dlr (pseudospec_hd.f90:254-288): D_l = d2/dr2 - l(l+1)/r^2
extern "C" void orc_dlr(const orc_plan* p, const double* a, double* b) {
  orc_derivr(p, a, b, 2, 'r');
  std::vector<double> c1(2 * nspec(p)), c2(2 * nspec(p));
  orc_laplang(p, a, c1.data());
  orc_multr(p, c1.data(), c2.data(), -2);
  orc_saxpby_c(p, b, b, 1.0, c2.data(), 1.0);
}

// fc_filter_k (pseudospec_hd.f90:407-440): a *= exp(-alpha (2 kz/(nz Dkz))^100)
static void fc_filter_k(const orc_plan* p, cplx* A) {
  const double alpha = 16.0 * std::log(10.0), pp = 50.0;
  for (int k = 0; k < p->nz; ++k) {
    double f = std::exp(-alpha * std::pow(2.0 * p->kz[k] / p->nz / p->Dkz, 2.0 * pp));
    for (int lm = 0; lm < p->nlm; ++lm) A[(size_t)k * p->nlm + lm] *= f;
  }
}

extern "C" int orc_fc_filter(const orc_plan* p, double* a, char esp) {
  cplx* A = reinterpret_cast<cplx*>(a);
  if (esp == 'k') { fc_filter_k(p, A); return 0; }
  if (esp != 'r') return 1;
  orc_z_forward(p, a);
  fc_filter_k(p, A);
  orc_z_inverse(p, a);
  return 0;
}

extern "C" void orc_copy(const orc_plan* p, const double* a, double* b) {
  std::memcpy(b, a, sizeof(double) * 2 * nspec(p));
}

// prodvec (pseudospec_hd.f90:211-251): C = A x B on the physical planes
// (k <= pkend = nz - Cz); continuation planes of C are set to zero.
extern "C" void orc_prodvec(const orc_plan* p, const double* ar, const double* at,
                            const double* ap, const double* br, const double* bt,
                            const double* bp, double* cr, double* ct, double* cp) {
  size_t plane = (size_t)p->nphi * p->nlat, nphys = plane * p->N, ntot = plane * p->nz;
  for (size_t q = 0; q < nphys; ++q) {
    double xr = ar[q], xt = at[q], xp = ap[q], yr = br[q], yt = bt[q], yp = bp[q];
    cr[q] = xt * yp - xp * yt;
    ct[q] = xp * yr - xr * yp;
    cp[q] = xr * yt - xt * yr;
  }
  for (size_t q = nphys; q < ntot; ++q) cr[q] = ct[q] = cp[q] = 0.0;
}

// ---------------------------------------------------------------- boundary
// dirichlet (boundary_mod.f90:62-93)
extern "C" void orc_dirichlet(const orc_plan* p, double* a) {
  cplx* A = reinterpret_cast<cplx*>(a);
  for (int lm = 0; lm < p->nlm; ++lm) {
    A[lm] = 0;
    A[(size_t)(p->N - 1) * p->nlm + lm] = 0;
  }
}

// derivr_mat (boundary_mod.f90:96-137): column j = derivr of e_j on the
// N physical points.  The oracle probes one column per lm slot.
extern "C" void orc_derivr_mat(const orc_plan* p, int order, double* dmat) {
  const int n = p->N, nlm = p->nlm, nz = p->nz;
  std::vector<cplx> c1((size_t)nz * nlm), c2((size_t)nz * nlm);
  for (int j0 = 0; j0 < n; j0 += nlm) {
    std::fill(c1.begin(), c1.end(), cplx(0));
    for (int lm = 0; lm < nlm; ++lm) {
      int j = j0 + lm;
      if (j < n) c1[(size_t)j * nlm + lm] = 1.0;
    }
    orc_derivr(p, reinterpret_cast<double*>(c1.data()), reinterpret_cast<double*>(c2.data()), order, 'r');
    for (int lm = 0; lm < nlm; ++lm) {
      int j = j0 + lm;
      if (j < n)
        for (int i = 0; i < n; ++i) dmat[i + (size_t)n * j] = c2[(size_t)i * nlm + lm].real();
    }
  }
}

// LU with partial pivoting (DGETRF) and solve (DGETRS), column-major.
static int lu_factor(int n, double* a, int* piv) {
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = std::fabs(a[k + (size_t)n * k]);
    for (int i = k + 1; i < n; ++i) {
      double v = std::fabs(a[i + (size_t)n * k]);
      if (v > best) { best = v; pr = i; }
    }
    piv[k] = pr;
    if (best == 0.0) return k + 1;
    if (pr != k)
      for (int j = 0; j < n; ++j) std::swap(a[k + (size_t)n * j], a[pr + (size_t)n * j]);
    double inv = 1.0 / a[k + (size_t)n * k];
    for (int i = k + 1; i < n; ++i) a[i + (size_t)n * k] *= inv;
    for (int j = k + 1; j < n; ++j) {
      double f = a[k + (size_t)n * j];
      if (f != 0.0)
        for (int i = k + 1; i < n; ++i) a[i + (size_t)n * j] -= a[i + (size_t)n * k] * f;
    }
  }
  return 0;
}

static void lu_solve(int n, const double* a, const int* piv, double* b, int nrhs) {
  for (int c = 0; c < nrhs; ++c) {
    double* x = b + (size_t)n * c;
    for (int k = 0; k < n; ++k) std::swap(x[k], x[piv[k]]);
    for (int k = 0; k < n; ++k)
      for (int i = k + 1; i < n; ++i) x[i] -= a[i + (size_t)n * k] * x[k];
    for (int k = n - 1; k >= 0; --k) {
      x[k] /= a[k + (size_t)n * k];
      for (int i = 0; i < k; ++i) x[i] -= a[i + (size_t)n * k] * x[k];
    }
  }
}

// invDl_setup (boundary_mod.f90:140-241)
// load_neumann_tables (fcgram_mod.f90:267-365): neu = Q(d,:) . Qn^T from
// Q{d}.dat and Q{ord}n{d}.dat (its first double the tables' spacing dxp),
// the last entry scaled by (dx/dxp)^ord.  0 on success.
extern "C" int orc_load_neumann_tables(const char* tdir, int d, int ord, double dx, double* neu) {
  if (ord != 1 && ord != 2) return 3;
  std::vector<double> Q((size_t)d * d), Qn((size_t)d * d);
  char path[4096];
  snprintf(path, sizeof path, "%s/Q%d.dat", tdir, d);
  FILE* f = fopen(path, "rb");
  if (!f) return 1;
  size_t got = fread(Q.data(), sizeof(double), Q.size(), f);
  fclose(f);
  if (got != Q.size()) return 2;
  snprintf(path, sizeof path, "%s/Q%dn%d.dat", tdir, ord, d);
  f = fopen(path, "rb");
  if (!f) return 1;
  double dxp = 0.0;
  got = fread(&dxp, sizeof(double), 1, f);
  got += fread(Qn.data(), sizeof(double), Qn.size(), f);
  fclose(f);
  if (got != Qn.size() + 1 || dxp <= 0.0) return 2;
  // neu(k) = sum_j Q(d, j) Qn(k, j)   (column-major Q(i,j) = Q[i-1 + d (j-1)])
  for (int k = 0; k < d; ++k) {
    double acc = 0.0;
    for (int j = 0; j < d; ++j) acc += Q[(d - 1) + (size_t)d * j] * Qn[k + (size_t)d * j];
    neu[k] = acc;
  }
  neu[d - 1] *= ord == 1 ? dx / dxp : (dx / dxp) * (dx / dxp);
  return 0;
}

extern "C" void orc_set_neumann(orc_plan* p, const double* neu1, const double* neu2) {
  if (neu1) p->neu[0].assign(neu1, neu1 + p->d);
  if (neu2) p->neu[1].assign(neu2, neu2 + p->d);
}

// The boundary value of one column from its outward normal derivative (of
// order ord) held at the boundary point and the d-1 values inside, as
// neumann_reconstruct (fcgram_mod.f90:368-520, z boundaries 5 and 6, in the
// reference's summation order); with `a`, robin_reconstruct
// (fcgram_mod.f90:523-650): f' + a f = g, g held at the boundary point.
static cplx reconstruct_one(const orc_plan* p, const cplx* f, int nlm, int boun, const double* neu, bool robin,
                            double a) {
  const int d = p->d, n = p->N;
  const int b = boun == 0 ? 0 : n - 1;
  cplx acc = neu[d - 1] * f[(size_t)b * nlm];
  for (int k = 1; k <= d - 1; ++k) {
    const int row = boun == 0 ? d - k : n - 1 - d + k;  // 0-based: point d+1-k, or N-d+k
    acc = acc + neu[k - 1] * f[(size_t)row * nlm];
  }
  if (robin) acc = acc / (a * neu[d - 1] + 1.0);
  return acc;
}

extern "C" int orc_neumann_reconstruct(const orc_plan* p, double* spec, int boun, int ord) {
  if ((boun != 0 && boun != 1) || (ord != 1 && ord != 2) || p->neu[ord - 1].empty()) return 1;
  cplx* F = reinterpret_cast<cplx*>(spec);
  const int b = boun == 0 ? 0 : p->N - 1;
  for (int lm = 0; lm < p->nlm; ++lm)
    F[(size_t)b * p->nlm + lm] = reconstruct_one(p, F + lm, p->nlm, boun, p->neu[ord - 1].data(), false, 0.0);
  return 0;
}

extern "C" int orc_robin_reconstruct(const orc_plan* p, double* spec, int boun, const double* a) {
  if ((boun != 0 && boun != 1) || p->neu[0].empty()) return 1;
  cplx* F = reinterpret_cast<cplx*>(spec);
  const int b = boun == 0 ? 0 : p->N - 1;
  for (int lm = 0; lm < p->nlm; ++lm)
    F[(size_t)b * p->nlm + lm] = reconstruct_one(p, F + lm, p->nlm, boun, p->neu[0].data(), true, a[lm]);
  return 0;
}

// Boundary kinds per wall (inner, outer): 0 noslip (v_parsebc's only type,
// vboundary.f90:10-31): Z = W = dW/dr = 0; 1 freeslip (stress-free, no
// penetration): W = 0, W'' - 2 W'/r = 0, Z' - 2 Z/r = 0 (the toroidal
// condition by robin_reconstruct, a = +2/rint inside, -2/rext outside, with
// the outward normal derivative).
extern "C" int orc_bc_setup_kinds(orc_plan* p, int kint, int kext) {
  if (kint < 0 || kint > 1 || kext < 0 || kext > 1) return 3;
  if ((kint == 1 || kext == 1) && p->neu[0].empty()) return 4;
  p->bck[0] = kint;
  p->bck[1] = kext;
  p->bc_ready = 0;
  return orc_bc_setup(p);
}

extern "C" int orc_bc_setup(orc_plan* p) {
  const int n = p->N, lmax = p->lmax;
  if (n < 6 || p->C <= 0) return 1;
  std::vector<double> d1((size_t)n * n), d2((size_t)n * n), b((size_t)n * n), esc(n);
  std::vector<int> piv(n);
  orc_derivr_mat(p, 1, d1.data());
  orc_derivr_mat(p, 2, d2.data());
  p->binv.assign((size_t)n * (n - 4) * std::max(lmax, 1), 0.0);
  auto B = [&](int i, int j) -> double& { return b[(i - 1) + (size_t)n * (j - 1)]; };
  auto D1 = [&](int i, int j) { return d1[(i - 1) + (size_t)n * (j - 1)]; };
  auto D2 = [&](int i, int j) { return d2[(i - 1) + (size_t)n * (j - 1)]; };
  for (int l = 1; l <= lmax; ++l) {
    std::fill(b.begin(), b.end(), 0.0);
    B(1, 1) = 1.0;
    // row 2: W' = 0 (noslip) or W'' - 2 W'/r = 0 (freeslip) at the inner wall
    for (int j = 1; j <= n; ++j) B(2, j) = p->bck[0] ? D2(1, j) - 2.0 / p->z[0] * D1(1, j) : D1(1, j);
    for (int i = 3; i <= n - 2; ++i) {
      for (int j = 1; j <= n; ++j) B(i, j) = D2(i, j);
      B(i, i) = B(i, i) - (double)(l * (l + 1)) / (p->z[i - 1] * p->z[i - 1]);
    }
    for (int j = 1; j <= n; ++j) B(n - 1, j) = p->bck[1] ? D2(n, j) - 2.0 / p->z[n - 1] * D1(n, j) : D1(n, j);
    B(n, n) = 1.0;
    for (int i = 1; i <= n; ++i) {
      double mx = 0;
      for (int j = 1; j <= n; ++j) mx = std::max(mx, std::fabs(B(i, j)));
      esc[i - 1] = mx;
      for (int j = 1; j <= n; ++j) B(i, j) /= mx;
    }
    if (lu_factor(n, b.data(), piv.data())) return 2;
    double* bi = &p->binv[(size_t)n * (n - 4) * (l - 1)];
    for (int j = 1; j <= n - 4; ++j) bi[(j + 2 - 1) + (size_t)n * (j - 1)] = 1.0 / esc[j + 2 - 1];
    lu_solve(n, b.data(), piv.data(), bi, n - 4);
  }
  p->d2bor.assign((size_t)4 * n, 0.0);
  for (int j = 0; j < n; ++j) {
    p->d2bor[0 + 4 * (size_t)j] = d2[0 + (size_t)n * j];
    p->d2bor[1 + 4 * (size_t)j] = d2[1 + (size_t)n * j];
    p->d2bor[2 + 4 * (size_t)j] = d2[(n - 2) + (size_t)n * j];
    p->d2bor[3 + 4 * (size_t)j] = d2[(n - 1) + (size_t)n * j];
  }
  p->bc_ready = 1;
  return 0;
}

// The boundary tables given directly (binv: N x (N-4) per l = 1..lmax;
// d2bor: 4 x N), for the wall kinds kint / kext: the operators of
// v_imposebc then run on tables built elsewhere (an extended-precision
// evaluation of invDl_setup's matrices).  0 on success.
extern "C" int orc_bc_set_tables(orc_plan* p, int kint, int kext, const double* binv, const double* d2bor) {
  if (kint < 0 || kint > 1 || kext < 0 || kext > 1 || !binv || !d2bor) return 3;
  if ((kint == 1 || kext == 1) && p->neu[0].empty()) return 4;
  const int n = p->N;
  if (n < 6 || p->C <= 0) return 1;
  p->bck[0] = kint;
  p->bck[1] = kext;
  p->binv.assign(binv, binv + (size_t)n * (n - 4) * std::max(p->lmax, 1));
  p->d2bor.assign(d2bor, d2bor + (size_t)4 * n);
  p->bc_ready = 1;
  return 0;
}

extern "C" void orc_bc_tables(const orc_plan* p, double* binv, double* d2bor) {
  if (binv) std::copy(p->binv.begin(), p->binv.end(), binv);
  if (d2bor) std::copy(p->d2bor.begin(), p->d2bor.end(), d2bor);
}

// invDl (boundary_mod.f90:244-292): W(1:N) = M_l phi(3:N-2), zero elsewhere
// and for l = 0.
extern "C" void orc_invDl(const orc_plan* p, const double* phi, double* w) {
  const int n = p->N, nlm = p->nlm;
  const cplx* F = reinterpret_cast<const cplx*>(phi);
  cplx* W = reinterpret_cast<cplx*>(w);
  for (size_t q = 0; q < nspec(p); ++q) W[q] = 0;
#pragma omp parallel for OMP_THREADS schedule(static)
  for (int lm = 0; lm < nlm; ++lm) {
    int l = p->ell[lm];
    if (l == 0) continue;
    const double* M = &p->binv[(size_t)n * (n - 4) * (l - 1)];
    for (int i = 0; i < n; ++i) {
      cplx s = 0;
      for (int j = 0; j < n - 4; ++j) s += M[i + (size_t)n * j] * F[(size_t)(j + 2) * nlm + lm];
      W[(size_t)i * nlm + lm] = s;
    }
  }
}

// v_imposebc / v_imposebc_fast (vboundary.f90:59-130)
// The toroidal condition of each wall: Z = 0 (noslip) or the Robin
// reconstruction of Z' - 2 Z/r = 0 (freeslip, g = 0).
static void toroidal_bc(const orc_plan* p, double* tor) {
  cplx* T = reinterpret_cast<cplx*>(tor);
  for (int w = 0; w < 2; ++w) {
    const int b = w == 0 ? 0 : p->N - 1;
    const double a = w == 0 ? 2.0 / p->z[0] : -2.0 / p->z[p->N - 1];
    for (int lm = 0; lm < p->nlm; ++lm) {
      T[(size_t)b * p->nlm + lm] = 0.0;
      if (p->bck[w]) T[(size_t)b * p->nlm + lm] = reconstruct_one(p, T + lm, p->nlm, w, p->neu[0].data(), true, a);
    }
  }
}

extern "C" void orc_imposebc(const orc_plan* p, double* tor, double* phi, double* pol, int fast) {
  toroidal_bc(p, tor);
  orc_invDl(p, phi, pol);
  if (!fast) { orc_dlr(p, pol, phi); return; }
  const int n = p->N, nlm = p->nlm, nz = p->nz;
  cplx* F = reinterpret_cast<cplx*>(phi);
  const cplx* W = reinterpret_cast<const cplx*>(pol);
  const int rows[4] = {1, 2, n - 1, n};
  for (int lm = 0; lm < nlm; ++lm) {
    int l = p->ell[lm];
    if (l == 0) {
      for (int k = 0; k < nz; ++k) F[(size_t)k * nlm + lm] = 0;
      continue;
    }
    for (int r = 0; r < 4; ++r) {
      int i = rows[r];
      cplx s = 0;
      for (int j = 0; j < n; ++j) s += p->d2bor[r + 4 * (size_t)j] * W[(size_t)j * nlm + lm];
      double zi = p->z[i - 1];
      F[(size_t)(i - 1) * nlm + lm] = s - (double)(l * (l + 1)) * W[(size_t)(i - 1) * nlm + lm] / (zi * zi);
    }
  }
}

// ---------------------------------------------------------------- NL + RK3
// Toroidal/poloidal velocity u = curl curl (W r^) + curl (Z r^), phi = D_l W:
//   u:     Q = l(l+1) W/r^2,  S = W'/r,  T = Z/r
//   omega: Q = l(l+1) Z/r^2,  S = Z'/r,  T = -phi/r
// N = u x omega (prodvec) -> QST analysis; projections with r.curl and
// r.curl curl:  dZ/dt = r T_N + nu D_l Z ;  dphi/dt = (r S_N)' - Q_N + nu D_l phi.
struct Fields {
  std::vector<double> a, b, c;
};

static void mul_rpow_lfac(const orc_plan* p, const double* in, double* out, int rp, int lfac, double sc) {
  const cplx* A = reinterpret_cast<const cplx*>(in);
  cplx* B = reinterpret_cast<cplx*>(out);
  for (int k = 0; k < p->nz; ++k) {
    double zp = std::pow(p->z[k], (double)rp);
    for (int lm = 0; lm < p->nlm; ++lm) {
      int l = p->ell[lm];
      double f = sc * zp * (lfac ? (double)(l * (l + 1)) : 1.0);
      B[(size_t)k * p->nlm + lm] = f * A[(size_t)k * p->nlm + lm];
    }
  }
}

static double grid_energy(const orc_plan* p, const double* ur, const double* ut, const double* up) {
  const int nlat = p->nlat, nphi = p->nphi, n = p->N;
  double e = 0;
  for (int k = 0; k < n; ++k) {
    double ck = (k == 0 || k == n - 1) ? 0.5 : 1.0;
    double rk = p->z[k];
    double sk = 0;
    for (int j = 0; j < nphi; ++j)
      for (int i = 0; i < nlat; ++i) {
        size_t q = ((size_t)k * nphi + j) * nlat + i;
        sk += p->w[i] * (ur[q] * ur[q] + ut[q] * ut[q] + up[q] * up[q]);
      }
    e += ck * rk * rk * sk;
  }
  return 0.5 * e * p->dz * 2.0 * M_PI / nphi;
}

extern "C" void orc_velocity(const orc_plan* p, const double* Z, const double* W, const double* phi,
                             double* ur, double* ut, double* up, double* wr, double* wt, double* wp) {
  const size_t ns = 2 * nspec(p);
  std::vector<double> q(ns), s(ns), t(ns), tmp(ns);
  // velocity
  mul_rpow_lfac(p, W, q.data(), -2, 1, 1.0);
  orc_derivr(p, W, tmp.data(), 1, 'r');
  mul_rpow_lfac(p, tmp.data(), s.data(), -1, 0, 1.0);
  mul_rpow_lfac(p, Z, t.data(), -1, 0, 1.0);
  orc_qst_synthesis(p, q.data(), s.data(), t.data(), ur, ut, up);
  if (!wr) return;
  // vorticity
  mul_rpow_lfac(p, Z, q.data(), -2, 1, 1.0);
  orc_derivr(p, Z, tmp.data(), 1, 'r');
  mul_rpow_lfac(p, tmp.data(), s.data(), -1, 0, 1.0);
  mul_rpow_lfac(p, phi, t.data(), -1, 0, -1.0);
  orc_qst_synthesis(p, q.data(), s.data(), t.data(), wr, wt, wp);
}

extern "C" void orc_nl_rhs(const orc_plan* p, const double* Z, const double* W, const double* phi,
                           double nu, double* rhs_z, double* rhs_phi, double* energy) {
  const size_t ns = 2 * nspec(p);
  const size_t ng = (size_t)p->nz * p->nphi * p->nlat;
  std::vector<double> u0(ng), u1(ng), u2(ng), w0(ng), w1(ng), w2(ng), n0(ng), n1(ng), n2(ng);
  orc_velocity(p, Z, W, phi, u0.data(), u1.data(), u2.data(), w0.data(), w1.data(), w2.data());
  if (energy) *energy = grid_energy(p, u0.data(), u1.data(), u2.data());
  orc_prodvec(p, u0.data(), u1.data(), u2.data(), w0.data(), w1.data(), w2.data(), n0.data(),
              n1.data(), n2.data());
  std::vector<double> qn(ns), sn(ns), tn(ns), tmp(ns), tmp2(ns);
  orc_qst_analysis(p, n0.data(), n1.data(), n2.data(), qn.data(), sn.data(), tn.data());
  // rhs_z = r T_N + nu D_l Z
  orc_multr(p, tn.data(), tmp.data(), 1);
  orc_dlr(p, Z, tmp2.data());
  orc_saxpby_c(p, rhs_z, tmp.data(), 1.0, tmp2.data(), nu);
  // rhs_phi = (r S_N)' - Q_N + nu D_l phi
  orc_multr(p, sn.data(), tmp.data(), 1);
  orc_derivr(p, tmp.data(), tmp2.data(), 1, 'r');
  orc_saxpby_c(p, rhs_phi, tmp2.data(), 1.0, qn.data(), -1.0);
  orc_dlr(p, phi, tmp.data());
  orc_saxpby_c(p, rhs_phi, rhs_phi, 1.0, tmp.data(), nu);
}

// RK3 in the GHOST/SPECTER low-storage form X = X0 + (dt/o) RHS(X), o = 3,2,1,
// with v_imposebc after every stage (vboundary.f90:61-63).
// Per-degree kinetic energy from the QST potentials of u (Q = l(l+1) W/r^2,
// S = W'/r, T = Z/r), trapezoid in r over the physical points, c_m = 1 for
// m = 0 and 2 otherwise; spec[2 l] toroidal (T), spec[2 l + 1] poloidal (Q, S).
// For m = 0 only the real parts count: the synthesis of a real field drops
// the imaginary part of m = 0 (radial derivatives give one, through the
// Nyquist wavenumber the reference keeps).  The sum is grid_energy of the
// same state.
extern "C" void orc_energy_spectrum(const orc_plan* p, const double* Z, const double* W, double* spec) {
  const int nlm = p->nlm, N = p->N;
  std::vector<double> wp(2 * nspec(p));
  orc_derivr(p, W, wp.data(), 1, 'r');
  const cplx* z = reinterpret_cast<const cplx*>(Z);
  const cplx* w = reinterpret_cast<const cplx*>(W);
  const cplx* d = reinterpret_cast<const cplx*>(wp.data());
  for (int i = 0; i < 2 * (p->lmax + 1); ++i) spec[i] = 0.0;
  for (int lm = 0; lm < nlm; ++lm) {
    const int l = p->ell[lm];
    const double cm = p->emm[lm] == 0 ? 1.0 : 2.0, L = (double)l * (l + 1);
    double st = 0.0, sp = 0.0;
    auto sq = [&](cplx v) { return p->emm[lm] == 0 ? v.real() * v.real() : std::norm(v); };
    for (int k = 0; k < N; ++k) {
      const double wk = (k == 0 || k == N - 1) ? 0.5 * p->dz : p->dz, r = p->z[k];
      const size_t q = (size_t)k * nlm + lm;
      st += wk * L * sq(z[q]);
      sp += wk * (L * L * sq(w[q]) / (r * r) + L * sq(d[q]));
    }
    spec[2 * l] += 0.5 * cm * st;
    spec[2 * l + 1] += 0.5 * cm * sp;
  }
}

extern "C" void orc_rk3_step(const orc_plan* p, double* Z, double* W, double* phi, double nu,
                             double dt, double* energy) {
  const size_t ns = 2 * nspec(p);
  std::vector<double> Z0(Z, Z + ns), F0(phi, phi + ns), rz(ns), rf(ns);
  for (int o = 3; o >= 1; --o) {
    double e;
    orc_nl_rhs(p, Z, W, phi, nu, rz.data(), rf.data(), &e);
    if (o == 3 && energy) *energy = e;
    orc_saxpby_c(p, Z, Z0.data(), 1.0, rz.data(), dt / o);
    orc_saxpby_c(p, phi, F0.data(), 1.0, rf.data(), dt / o);
    orc_imposebc(p, Z, phi, W, 0);
  }
}
