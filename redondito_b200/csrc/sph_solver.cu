// sph_solver.cu -- the run loop around the nonlinear step: namelist input,
// the grid files, per-degree energy spectra and the time loop.
//
// The reference ships the transform core without a solver; SPECTER, which it
// is converted from, drives it from a main program that reads namelists,
// writes the grids and runs the time steps with periodic diagnostics.  This
// file gives that loop to callers of the C ABI:
//   namelists  &grid lmax, nz, Cz, oz (grid_init, src/pseudo/pseudospec_mod.f90:41-69)
//              &boxparams rint, rext (box_init, pseudospec_mod.f90:151-160)
//              &run dt, step, tstep, sstep, nu, filter (the loop's own group)
//   grid files theta.txt, phi.txt, z.txt (box_init, pseudospec_mod.f90:204-220)
//   balance    balance.txt: step, time, energy (FP64)
//   spectra    lspectrum.NNNN.txt: l, toroidal and poloidal energy per degree
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "sph_internal.cuh"

namespace {

// ---------------------------------------------------------------- namelists
// A Fortran namelist group "&name key = value, key = value /": keys are
// case-insensitive, values are separated by commas, blanks or new lines,
// '!' starts a comment, the group ends at '/' (or '&end'), and reals may
// use the D exponent (0.35d0).
bool read_group(const std::string& text, const char* group, std::vector<std::pair<std::string, std::string>>& kv) {
  std::string low(text);
  for (auto& c : low) c = (char)tolower((unsigned char)c);
  // drop comments
  std::string clean;
  bool comment = false, quote = false;
  for (size_t i = 0; i < low.size(); ++i) {
    const char c = low[i];
    if (c == '\n') comment = false;
    if (c == '\'' || c == '"') quote = !quote;
    if (c == '!' && !quote) comment = true;
    clean.push_back(comment ? ' ' : c);
  }
  const std::string tag = std::string("&") + group;
  size_t pos = 0;
  for (;;) {
    pos = clean.find(tag, pos);
    if (pos == std::string::npos) return false;
    const size_t after = pos + tag.size();
    if (after >= clean.size() || isspace((unsigned char)clean[after])) break;
    pos = after;
  }
  size_t i = pos + tag.size();
  size_t end = clean.find('/', i);
  const size_t amp = clean.find("&end", i);
  if (amp != std::string::npos && (end == std::string::npos || amp < end)) end = amp;
  if (end == std::string::npos) return false;
  const std::string body = clean.substr(i, end - i);
  // key = value pairs
  size_t q = 0;
  while (q < body.size()) {
    while (q < body.size() && (isspace((unsigned char)body[q]) || body[q] == ',')) ++q;
    if (q >= body.size()) break;
    size_t k0 = q;
    while (q < body.size() && (isalnum((unsigned char)body[q]) || body[q] == '_')) ++q;
    std::string key = body.substr(k0, q - k0);
    while (q < body.size() && isspace((unsigned char)body[q])) ++q;
    if (q >= body.size() || body[q] != '=' || key.empty()) return false;
    ++q;
    while (q < body.size() && isspace((unsigned char)body[q])) ++q;
    size_t v0 = q;
    while (q < body.size() && !isspace((unsigned char)body[q]) && body[q] != ',') ++q;
    kv.emplace_back(key, body.substr(v0, q - v0));
  }
  return true;
}

bool to_double(std::string v, double* out) {
  for (auto& c : v)
    if (c == 'd') c = 'e';
  if (v == ".true." || v == "t") {
    *out = 1.0;
    return true;
  }
  if (v == ".false." || v == "f") {
    *out = 0.0;
    return true;
  }
  char* e = nullptr;
  const double x = strtod(v.c_str(), &e);
  if (e == v.c_str() || *e) return false;
  *out = x;
  return true;
}

bool to_int(const std::string& v, int* out) {
  double x;
  if (!to_double(v, &x) || x != floor(x) || fabs(x) > 2e9) return false;
  *out = (int)x;
  return true;
}

int write_column(const std::string& path, const double* x, int n) {
  FILE* f = fopen(path.c_str(), "w");
  if (!f) return SPH_EIO;
  // Fortran '(1P E23.15)': one digit before the point, 15 after, width 23
  for (int i = 0; i < n; ++i) fprintf(f, "%23.15E\n", x[i]);
  return fclose(f) == 0 ? SPH_OK : SPH_EIO;
}

// Per-degree kinetic energy of u = curl curl(W r^) + curl(Z r^) from its
// QST potentials (Q = l(l+1) W/r^2, S = W'/r, T = Z/r), integrated over the
// physical shell with the weights of the grid energy (trapezoid in r):
//   tor(l) = 1/2 sum_m c_m sum_k w_k l(l+1) |Z|^2
//   pol(l) = 1/2 sum_m c_m sum_k w_k [ (l(l+1))^2 |W|^2 / r^2 + l(l+1) |W'|^2 ]
// c_m = 1 for m = 0 and 2 otherwise (real fields); for m = 0 only the real
// parts count, as in the synthesis of a real field (a radial derivative
// gives m = 0 an imaginary part through the Nyquist wavenumber the
// reference keeps).  The sum over l is the grid energy of the same state.
// One thread per lm column; FP64 atomics into spec[l][2].
__global__ void spectrum_kernel(const double2* __restrict__ Z, const double2* __restrict__ W,
                                const double2* __restrict__ Wp, const int* __restrict__ ell,
                                const int* __restrict__ mbase, const double* __restrict__ z, int lmax, int nlm,
                                int N, double dz, double* spec) {
  for (int lm = blockIdx.x * blockDim.x + threadIdx.x; lm < nlm; lm += gridDim.x * blockDim.x) {
    const int l = ell[lm];
    int m = 0;
    while (m < lmax && mbase[m + 1] <= lm) ++m;
    const double cm = m == 0 ? 1.0 : 2.0, L = (double)l * (l + 1);
    double st = 0.0, sp = 0.0;
    for (int k = 0; k < N; ++k) {
      const double wk = (k == 0 || k == N - 1) ? 0.5 * dz : dz;
      const double2 a = Z[(size_t)k * nlm + lm], b = W[(size_t)k * nlm + lm], c = Wp[(size_t)k * nlm + lm];
      const double r = z[k], im = m == 0 ? 0.0 : 1.0;
      st += wk * L * (a.x * a.x + im * a.y * a.y);
      sp += wk * (L * L * (b.x * b.x + im * b.y * b.y) / (r * r) + L * (c.x * c.x + im * c.y * c.y));
    }
    atomicAdd(spec + 2 * l, 0.5 * cm * st);
    atomicAdd(spec + 2 * l + 1, 0.5 * cm * sp);
  }
}

}  // namespace

extern "C" int sph_read_namelist(const char* path, int* lmax, int* nz, int* Cz, int* oz, double* rint, double* rext,
                                 double* dt, int* step, int* tstep, int* sstep, double* nu, int* filter) {
  if (!path) return SPH_EINVAL;
  FILE* f = fopen(path, "rb");
  if (!f) return SPH_EIO;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  fclose(f);
  std::vector<std::pair<std::string, std::string>> g, b, r;
  if (!read_group(text, "grid", g) || !read_group(text, "boxparams", b)) return SPH_EINVAL;
  // grid_init defaults: Cz = oz = 0 when they are not in the namelist
  int vlmax = -1, vnz = -1, vCz = 0, voz = 0;
  for (auto& x : g) {
    int* dst = x.first == "lmax" ? &vlmax : x.first == "nz" ? &vnz : x.first == "cz" ? &vCz : x.first == "oz" ? &voz
                                                                                                            : nullptr;
    if (!dst || !to_int(x.second, dst)) return SPH_EINVAL;
  }
  double vri = NAN, vre = NAN;
  for (auto& x : b) {
    double* dst = x.first == "rint" ? &vri : x.first == "rext" ? &vre : nullptr;
    if (!dst || !to_double(x.second, dst)) return SPH_EINVAL;
  }
  if (vlmax < 0 || vnz < 1 || vCz < 0 || voz < 0 || !(vri == vri) || !(vre == vre)) return SPH_EINVAL;
  // the loop's own group is optional; defaults: no steps
  double vdt = 0.0, vnu = 0.0;
  int vstep = 0, vts = 1, vss = 0, vfilt = 0;
  if (read_group(text, "run", r)) {
    for (auto& x : r) {
      bool ok = false;
      if (x.first == "dt") ok = to_double(x.second, &vdt);
      else if (x.first == "nu") ok = to_double(x.second, &vnu);
      else if (x.first == "step") ok = to_int(x.second, &vstep);
      else if (x.first == "tstep") ok = to_int(x.second, &vts);
      else if (x.first == "sstep") ok = to_int(x.second, &vss);
      else if (x.first == "filter") {
        double v;
        ok = to_double(x.second, &v);
        vfilt = v != 0.0;
      }
      if (!ok) return SPH_EINVAL;
    }
  }
  if (lmax) *lmax = vlmax;
  if (nz) *nz = vnz;
  if (Cz) *Cz = vCz;
  if (oz) *oz = voz;
  if (rint) *rint = vri;
  if (rext) *rext = vre;
  if (dt) *dt = vdt;
  if (step) *step = vstep;
  if (tstep) *tstep = vts;
  if (sstep) *sstep = vss;
  if (nu) *nu = vnu;
  if (filter) *filter = vfilt;
  return SPH_OK;
}

extern "C" int sph_write_grids(const sph_plan* p, const char* dir) {
  if (!p || !dir) return SPH_EINVAL;
  const std::string d(dir);
  int rc = write_column(d + "/theta.txt", p->theta.data(), p->nlat);
  if (rc == SPH_OK) rc = write_column(d + "/phi.txt", p->phi.data(), p->nphi);
  if (rc == SPH_OK) rc = write_column(d + "/z.txt", p->z.data(), p->N);  // physical points only
  return rc;
}

extern "C" int sph_energy_spectrum(sph_plan* p, const double* Z, const double* W, double* spec, void* s) {
  if (!p || !Z || !W || !spec || !slab_whole(p) || p->N < 2) return SPH_EINVAL;
  cudaStream_t st = (cudaStream_t)s;
  int rc = SPH_OK;
  if (!p->sp[0] && (rc = (cudaMalloc((void**)&p->sp[0], spec_elems(p) * sizeof(double2)) == cudaSuccess
                              ? SPH_OK
                              : SPH_ENOMEM)) != SPH_OK)
    return rc;
  if (!p->spectrum && cudaMalloc((void**)&p->spectrum, (size_t)2 * (p->lmax + 1) * sizeof(double)) != cudaSuccess)
    return SPH_ENOMEM;
  double2* Wp = p->sp[0];
  rc = launch_zfft(p, Z_DERIV, reinterpret_cast<const double2*>(W), Wp, 1, st);
  if (rc != SPH_OK) return rc;
  SPH_CUDA_OK(cudaMemsetAsync(p->spectrum, 0, (size_t)2 * (p->lmax + 1) * sizeof(double), st));
  const int threads = 128, blocks = (p->nlm + threads - 1) / threads;
  TimedLaunch tl(p, T_OPS, st);
  spectrum_kernel<<<blocks, threads, 0, st>>>(reinterpret_cast<const double2*>(Z), reinterpret_cast<const double2*>(W),
                                              Wp, p->d_ell, p->d_mbase, p->d_z, p->lmax, p->nlm, p->N, p->dz,
                                              p->spectrum);
  SPH_LAUNCH_OK();
  SPH_CUDA_OK(cudaMemcpyAsync(spec, p->spectrum, (size_t)2 * (p->lmax + 1) * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
  SPH_CUDA_OK(cudaStreamSynchronize(st));
  return SPH_OK;
}

extern "C" int sph_run(sph_plan* p, double* Z, double* W, double* phi, double nu, double dt, int nsteps, int tstep,
                       int sstep, int filter, const char* outdir, double* energy_out, void* s) {
  if (!p || !Z || !W || !phi || nsteps < 0 || tstep < 0 || sstep < 0 || dt < 0.0) return SPH_EINVAL;
  if (!p->bc_ready) return SPH_ENOTREADY;
  FILE* bal = nullptr;
  const std::string d = outdir ? outdir : "";
  if (outdir) {
    int rc = sph_write_grids(p, outdir);
    if (rc != SPH_OK) return rc;
    bal = fopen((d + "/balance.txt").c_str(), "w");
    if (!bal) return SPH_EIO;
  }
  std::vector<double> spec((size_t)2 * (p->lmax + 1));
  int rc = SPH_OK;
  double e = 0.0;
  for (int n = 0; n <= nsteps && rc == SPH_OK; ++n) {
    // state n: its spectrum, then the step (which reports the energy of the
    // state it starts from), or at the end one right-hand side for the energy
    const bool tout = tstep > 0 && n % tstep == 0, sout = outdir && sstep > 0 && n % sstep == 0;
    if (sout) {
      rc = sph_energy_spectrum(p, Z, W, spec.data(), s);
      if (rc != SPH_OK) break;
      char name[64];
      snprintf(name, sizeof name, "/lspectrum.%04d.txt", n / sstep);
      FILE* f = fopen((d + name).c_str(), "w");
      if (!f) {
        rc = SPH_EIO;
        break;
      }
      for (int l = 0; l <= p->lmax; ++l) fprintf(f, "%6d %23.15E %23.15E\n", l, spec[2 * l], spec[2 * l + 1]);
      fclose(f);
    }
    if (n < nsteps) {
      rc = sph_rk3_step(p, Z, W, phi, nu, dt, &e, s);
      if (rc == SPH_OK && filter) {  // the exponential filter of the radial modes, then the boundary rows again
        rc = sph_fc_filter(p, Z, 'r', s);
        if (rc == SPH_OK) rc = sph_fc_filter(p, phi, 'r', s);
        if (rc == SPH_OK) rc = sph_v_imposebc(p, Z, phi, W, s);
      }
    } else if (tout || energy_out) {
      rc = sph_nl_rhs(p, Z, W, phi, nu, reinterpret_cast<double*>(p->sp[7]), reinterpret_cast<double*>(p->sp[8]),
                      &e, s);
    }
    if (rc == SPH_OK && bal && tout) fprintf(bal, "%8d %23.15E %23.15E\n", n, n * dt, e);
  }
  if (bal) fclose(bal);
  if (rc == SPH_OK && energy_out) *energy_out = e;
  return rc;
}
