// sph_batch.cu -- many independent shell problems in one CUDA graph.
//
// Each problem is a plan with 1..3 scalar fields.  One run computes, for
// every (problem, field): the inverse 3D transform of its (lm, kz) spectra
// (z transform in place, like fftp3d_complex_to_real; on mixed plans one
// kernel writes the in-place result, the synthesis tiles and the radial
// derivative below), the radial
// derivative of the radial-space spectra (derivr(., 1, 'r')), and the
// forward 3D transform of the synthesised grid back into the spectra.
//
// The Legendre contractions of all problems run as ONE grouped launch per
// direction: the persistent tensor-core kernel (mixed plans) or the FP64
// tile kernel (FP64 plans) walks the triangular m-blocks of every
// (problem, field) work set.  The forward z transforms run as one grouped
// launch per z length.  The other FFT and elementwise stages run per
// problem on parallel graph branches, so that small problems overlap.  The whole
// sequence is captured once into a CUDA graph and replayed by each run.
#include <algorithm>
#include <vector>

#include "sph_internal.cuh"

struct sph_batch {
  std::vector<sph_plan*> plans;
  std::vector<int> nf;
  int precision = SPH_FP64;
  std::vector<std::vector<double*>> spec, grid, dspec;
  GroupLaunch syn, ana;
  ZGroupLaunch zf;                         // grouped forward z transforms
  std::vector<std::pair<int, int>> zrest;  // (problem, field) pairs zf does not take
  cudaStream_t main = nullptr;
  std::vector<cudaStream_t> br;
  std::vector<cudaEvent_t> ev;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int* dflag = nullptr;
};

namespace {

constexpr int NBRANCH = 16;

void batch_free(sph_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto e : b->ev) cudaEventDestroy(e);
  for (auto s : b->br) cudaStreamDestroy(s);
  if (b->main) cudaStreamDestroy(b->main);
  group_free(&b->syn);
  group_free(&b->ana);
  zgroup_free(&b->zf);
  if (b->dflag) cudaFree(b->dflag);
  delete b;
}

#define RCB(x)                   \
  do {                           \
    int r_ = (x);                \
    if (r_ != SPH_OK) return r_; \
  } while (0)
#define D2(x) reinterpret_cast<double2*>(x)
#define CD2(x) reinterpret_cast<const double2*>(x)

// fork: every branch waits for the work recorded so far on main
int fork(sph_batch* b, int& evi) {
  SPH_CUDA_OK(cudaEventRecord(b->ev[evi], b->main));
  for (auto s : b->br) SPH_CUDA_OK(cudaStreamWaitEvent(s, b->ev[evi], 0));
  ++evi;
  return SPH_OK;
}
// join: main waits for every branch
int join(sph_batch* b, int& evi) {
  for (auto s : b->br) {
    SPH_CUDA_OK(cudaEventRecord(b->ev[evi], s));
    SPH_CUDA_OK(cudaStreamWaitEvent(b->main, b->ev[evi], 0));
    ++evi;
  }
  return SPH_OK;
}

int record(sph_batch* b) {
  const bool mixed = b->precision == SPH_MIXED;
  const int np = (int)b->plans.size();
  int evi = 0;
  // 1: z inverse (in place), radial derivative, synthesis data tiles
  RCB(fork(b, evi));
  for (int p = 0; p < np; ++p) {
    const sph_plan* P = b->plans[p];
    cudaStream_t s = b->br[p % b->br.size()];
    for (int f = 0; f < b->nf[p]; ++f) {
      if (mixed && zinv_der_ok(P)) {
        // one kernel: the z inverse in place, the synthesis tiles and the
        // radial derivative from it
        RCB(launch_zinv_tiles(P, CD2(b->spec[p][f]), f, s, D2(b->spec[p][f]), D2(b->dspec[p][f])));
      } else if (mixed && zinv_tiles_ok(P)) {
        RCB(launch_zinv_tiles(P, CD2(b->spec[p][f]), f, s, D2(b->spec[p][f])));
        RCB(launch_zfft(P, Z_DERIV, CD2(b->spec[p][f]), D2(b->dspec[p][f]), 1, s));
      } else {
        RCB(launch_zfft(P, Z_INV, CD2(b->spec[p][f]), D2(b->spec[p][f]), 0, s));
        RCB(launch_zfft(P, Z_DERIV, CD2(b->spec[p][f]), D2(b->dspec[p][f]), 1, s));
        if (mixed) RCB(launch_spec_to_tiles_field(P, CD2(b->spec[p][f]), f, s));
      }
    }
  }
  RCB(join(b, evi));
  // 2: every synthesis contraction in one grouped launch
  RCB(mixed ? tc_group_launch(b->syn, b->dflag, b->main) : leg_group_launch(b->syn, b->main));
  // 3: inverse phi transforms, then the forward ones of the new grids
  RCB(fork(b, evi));
  for (int p = 0; p < np; ++p) {
    const sph_plan* P = b->plans[p];
    cudaStream_t s = b->br[p % b->br.size()];
    double* g[SPH_MAX_FIELDS] = {nullptr, nullptr, nullptr};
    const double* gc[SPH_MAX_FIELDS] = {nullptr, nullptr, nullptr};
    for (int f = 0; f < b->nf[p]; ++f) {
      g[f] = b->grid[p][f];
      gc[f] = b->grid[p][f];
    }
    if (mixed) {
      RCB(launch_phi_inv32(P, g, b->nf[p], s));
      if (P->C > 0 && P->contg) {
        const size_t per = (size_t)P->C * P->nphi * P->nlat;
        const double* gh[SPH_MAX_FIELDS] = {P->contg, P->contg + per, P->contg + 2 * per};
        RCB(launch_cont_phys(P, gc, b->nf[p], s));
        RCB(launch_phi_fwd32(P, gc, b->nf[p], s, gh));
      } else {
        RCB(launch_phi_fwd32(P, gc, b->nf[p], s));
      }
    } else {
      RCB(launch_phi_inv(P, g, b->nf[p], s));
      RCB(launch_phi_fwd(P, gc, b->nf[p], s));
    }
  }
  RCB(join(b, evi));
  // 4: every analysis contraction in one grouped launch
  RCB(mixed ? tc_group_launch(b->ana, b->dflag, b->main) : leg_group_launch(b->ana, b->main));
  // 5: z forward (mixed: the planes past N were continued physically), one
  // grouped launch per z length; the rest per problem on the branches
  RCB(zfwd_group_launch(b->zf, b->main));
  if (!b->zrest.empty()) {
    RCB(fork(b, evi));
    for (size_t k = 0; k < b->zrest.size(); ++k) {
      const int p = b->zrest[k].first, f = b->zrest[k].second;
      const sph_plan* P = b->plans[p];
      const bool cont = !(mixed && P->C > 0 && P->contg);
      RCB(launch_zfft(P, Z_FWD, CD2(b->spec[p][f]), D2(b->spec[p][f]), 0, b->br[k % b->br.size()], cont));
    }
    RCB(join(b, evi));
  }
  return SPH_OK;
}

}  // namespace

extern "C" int sph_batch_create(sph_batch** out, int nprob, sph_plan* const* plans, const int* nfields,
                                double* const* spec, double* const* grid, double* const* dspec) {
  if (!out || nprob < 1 || !plans || !nfields || !spec || !grid || !dspec) return SPH_EINVAL;
  *out = nullptr;
  sph_batch* b = new sph_batch();
  b->precision = plans[0] ? plans[0]->precision : SPH_FP64;
  int k = 0;
  for (int p = 0; p < nprob; ++p) {
    if (!plans[p] || plans[p]->precision != b->precision || nfields[p] < 1 || nfields[p] > SPH_MAX_FIELDS ||
        plans[p]->timing || !slab_whole(plans[p])) {
      delete b;
      return SPH_EINVAL;
    }
    // a plan's per-field scratch (folded coefficients, synthesis tiles,
    // continued planes) serves one problem: two problems on one plan would
    // race on it from their graph branches
    for (int q = 0; q < p; ++q)
      if (plans[q] == plans[p]) {
        delete b;
        return SPH_EINVAL;
      }
    b->plans.push_back(plans[p]);
    b->nf.push_back(nfields[p]);
    b->spec.emplace_back();
    b->grid.emplace_back();
    b->dspec.emplace_back();
    for (int f = 0; f < nfields[p]; ++f, ++k) {
      if (!spec[k] || !grid[k] || !dspec[k]) {
        delete b;
        return SPH_EINVAL;
      }
      b->spec[p].push_back(spec[k]);
      b->grid[p].push_back(grid[k]);
      b->dspec[p].push_back(dspec[k]);
    }
  }
  std::vector<GroupJob> jobs;
  for (int p = 0; p < nprob; ++p)
    for (int f = 0; f < b->nf[p]; ++f) jobs.push_back({b->plans[p], f, D2(b->spec[p][f])});
  const bool mixed = b->precision == SPH_MIXED;
  int rc = mixed ? tc_group_prepare(false, jobs, plans[0]->nsm, &b->syn) : leg_group_prepare(false, jobs, &b->syn);
  if (rc == SPH_OK)
    rc = mixed ? tc_group_prepare(true, jobs, plans[0]->nsm, &b->ana) : leg_group_prepare(true, jobs, &b->ana);
  if (rc == SPH_OK) {
    std::vector<ZJob> zj;
    std::vector<std::pair<int, int>> pf;
    for (int p = 0; p < nprob; ++p)
      for (int f = 0; f < b->nf[p]; ++f) {
        const sph_plan* P = b->plans[p];
        zj.push_back({P, D2(b->spec[p][f]), !(mixed && P->C > 0 && P->contg)});
        pf.push_back({p, f});
      }
    std::vector<int> rest;
    rc = zfwd_group_prepare(zj, &b->zf, &rest);
    for (int k : rest) b->zrest.push_back(pf[k]);
  }
  if (rc == SPH_OK && cudaMalloc((void**)&b->dflag, sizeof(int)) != cudaSuccess) rc = SPH_ENOMEM;
  if (rc == SPH_OK && cudaMemset(b->dflag, 0, sizeof(int)) != cudaSuccess) rc = SPH_ECUDA;
  if (rc == SPH_OK && cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) != cudaSuccess) rc = SPH_ECUDA;
  const int nb = std::min(nprob, NBRANCH);
  for (int i = 0; i < nb && rc == SPH_OK; ++i) {
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) rc = SPH_ECUDA;
    else b->br.push_back(s);
  }
  for (int i = 0; i < 3 + 3 * nb && rc == SPH_OK; ++i) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) rc = SPH_ECUDA;
    else b->ev.push_back(e);
  }
  if (rc == SPH_OK) {
    if (cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      rc = SPH_ECUDA;
    } else {
      rc = record(b);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(b->main, &g);
      if (rc == SPH_OK && e != cudaSuccess) rc = SPH_ECUDA;
      b->graph = g;
      if (rc == SPH_OK && cudaGraphInstantiate(&b->exec, b->graph, 0) != cudaSuccess) rc = SPH_ECUDA;
    }
  }
  if (rc != SPH_OK) {
    cudaGetLastError();
    batch_free(b);
    return rc;
  }
  *out = b;
  return SPH_OK;
}

extern "C" int sph_batch_run(sph_batch* b, void* stream) {
  if (!b || !b->exec) return SPH_EINVAL;
  SPH_CUDA_OK(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return SPH_OK;
}

extern "C" int sph_batch_status(sph_batch* b) {
  if (!b) return SPH_EINVAL;
  SPH_CUDA_OK(cudaDeviceSynchronize());
  int f = 0;
  SPH_CUDA_OK(cudaMemcpy(&f, b->dflag, sizeof(int), cudaMemcpyDeviceToHost));
  if (f) SPH_CUDA_OK(cudaMemset(b->dflag, 0, sizeof(int)));
  return f ? SPH_ETIMEDOUT : SPH_OK;
}

extern "C" int sph_batch_destroy(sph_batch* b) {
  if (!b) return SPH_EINVAL;
  cudaDeviceSynchronize();
  batch_free(b);
  return SPH_OK;
}
