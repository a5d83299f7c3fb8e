/*
 * sph_b200.h -- C ABI of the B200 (sm_100a) pseudospectral transform core.
 *
 * Drop-in for the device branch (`IF (gdev_active)`) of REDONDITO's sphp-gpu
 * transforms and of its pseudospectral/boundary operators.  A Fortran
 * ISO_C_BINDING shim keeps the reference's subroutine signatures and calls
 * these functions with device addresses (the `use_device_addr` pattern of
 * src/sphp-gpu/sphp_sca.F90:83-87).
 *
 * Conventions
 *  - Every pointer named grid/in/out/a/b/... is a DEVICE pointer.
 *  - Physical fields: double (nz planes) x (nphi) x (nlat), theta fastest,
 *    i.e. Fortran REAL(8) f(nlat,nphi,nz) with one MPI rank (ksta=1, kend=nz).
 *  - Spectral fields: interleaved complex double (re,im), lm fastest,
 *    i.e. Fortran COMPLEX(8) f(nlm,nz) with lmsta=1, lmend=nlm; lm in SHTns
 *    m-major order, lm(l,m) = m*(2*lmax+1-m)/2 + l (0-based).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls are
 *    stream-ordered and return once the work is enqueued; the Fortran shim
 *    synchronises to keep the reference's blocking semantics.
 *  - One plan per host thread: a plan's scratch is not re-entrant, like the
 *    reference's shared gcarr1-3 buffers (src/sphp-gpu/sphp_mod.F90:56-77).
 *  - Every function returns SPH_OK (0) or an SPH_E* code; the reference
 *    prints and STOPs instead (the shim maps a non-zero code to that).
 */
#ifndef SPH_B200_H
#define SPH_B200_H
#ifdef __cplusplus
extern "C" {
#endif

enum {
  SPH_OK = 0,
  SPH_EINVAL = 1,    /* bad size, pointer or argument */
  SPH_ENOMEM = 2,    /* device or host allocation failed */
  SPH_ECUDA = 3,     /* a CUDA call or launch failed */
  SPH_ENOTREADY = 4, /* boundary tables not set up (sph_setup_bc) */
  SPH_EIO = 5,       /* FC-Gram table file missing or short */
  SPH_ETIMEDOUT = 6  /* a bounded device wait gave up */
};

enum { SPH_FP64 = 0, SPH_MIXED = 1 };

typedef struct sph_plan sph_plan;

/* ---------------------------------------------------------------- plans */

/* Replaces fcgram_create_plan (src/sphp/fcgram_mod.f90:49-150) together with
 * fftp3d_create_plan (src/sphp-gpu/sphp_sca.F90:478-625), grid_init and
 * box_init (src/pseudo/pseudospec_mod.f90:41-69,126-236).
 *   lmax         : triangular truncation (mmax = lmax, mres = 1)
 *   nlat, nphi   : Gauss grid (nlat even, nphi > 2*lmax)
 *   nz           : radial points including the Cz continuation points
 *   Cz, oz       : FC-Gram continuation and matching points (0,0 = periodic)
 *   rint, rext   : shell radii; z(k) = rint + k*dz, dz = (rext-rint)/(nz-Cz-1)
 *   dir          : host pointer, Cz x oz column-major continuation operator
 *                  dir = A.Q^T (see sph_fcgram_load_tables); NULL if Cz == 0
 *   precision    : SPH_FP64, or SPH_MIXED: Legendre contractions on the
 *                  tensor cores (tcgen05, fp32 accumulation in TMEM) with
 *                  every operand split into three bf16 pieces
 *                  (hi + mid + lo, 8 significant bits each) and the six
 *                  piece products of order <= 2 kept (about 24 bits); the
 *                  hi*hi products and the five smaller ones accumulate
 *                  separately and are added in FP64.  phi FFTs in fp32
 *                  with twiddles derived in FP64 (relative L2 error
 *                  ~1e-7 per transform, <= 4e-7 at lmax 511); z
 *                  transforms, the FC-Gram continuation and operators
 *                  stay FP64.  SPH_MIXED needs nphi = 3*2^a,
 *                  12 <= nphi <= 6144.
 * Allocates the plan's device tables and scratch with cudaMalloc on the
 * current device. */
int sph_plan_create(sph_plan** plan, int lmax, int nlat, int nphi, int nz, int Cz, int oz,
                    double rint, double rext, const double* dir, int precision);

/* fcgram_destroy_plan (src/sphp/fcgram_mod.f90:153-182).  A plan's tables
 * outlive it while clones share them. */
int sph_plan_destroy(sph_plan* plan);

/* A second plan of the same sizes and precision (no reference counterpart:
 * a reference plan owns everything).  It shares src's read-only device
 * tables -- the Legendre tables, FFT twiddles, work lists, the tensor-core
 * table tiles and, once either plan has called sph_setup_bc, the boundary
 * matrices -- and allocates only its own scratch, so it costs a fraction of
 * sph_plan_create's memory and none of its host table work.  The two plans
 * may run concurrently on different streams (each has its own scratch).
 * The tables are freed with the last plan that shares them.  sph_setup_bc
 * on the clone is still required before boundary and NL calls (cheap when
 * the tables hold the matrices).  sph_plan_set_tiles cannot change the MMA
 * rows of a plan whose tables are shared (SPH_EINVAL). */
int sph_plan_clone(const sph_plan* src, sph_plan** plan);

/* load_dirichlet_tables (src/sphp/fcgram_mod.f90:186-263): reads
 * tdir/A{C}-{d}.dat and tdir/Q{d}.dat (raw column-major float64) and writes
 * dir = A.Q^T (C x d, column-major) to the host array dir. */
int sph_fcgram_load_tables(const char* tdir, int C, int d, double* dir);

/* load_neumann_tables (src/sphp/fcgram_mod.f90:267-365): reads tdir/Q{d}.dat
 * and tdir/Q{ord}n{d}.dat (its first double the tables' grid spacing dxp,
 * then d x d column-major) and writes to the host array neu (d values) the
 * reconstructor neu = Q(d,:).Qn^T, its last entry scaled by (dx/dxp)^ord:
 * the boundary value from the ord-th (1 or 2) outward normal derivative and
 * the d-1 values inside.  dx: the radial grid step of the plan it serves. */
int sph_fcgram_load_neumann_tables(const char* tdir, int d, int ord, double dx, double* neu);

/* The plan's Neumann reconstructors (host arrays of oz values; either may be
 * NULL to keep the current one), needed by sph_neumann_reconstruct,
 * sph_robin_reconstruct and the freeslip boundary kind. */
int sph_plan_set_neumann(sph_plan* plan, const double* neu1, const double* neu2);

/* Sizes of a plan: nlm, and the element counts of one physical field
 * (nlat*nphi*nz doubles) and one spectral field (nlm*nz complex). */
int sph_plan_sizes(const sph_plan* plan, int* nlm, long long* grid_elems, long long* spec_elems);

/* box_init outputs (pseudospec_mod.f90:174-227), host arrays (any may be NULL):
 * theta(nlat), Gauss weights(nlat), phi(nphi), z(nz), kz(nz), ell(nlm), emm(nlm). */
int sph_grid(const sph_plan* plan, double* theta, double* weights, double* phi, double* z,
             double* kz, int* ell, int* emm);

/* The caller's slab: the bounds the reference keeps in module mpivars
 * (ksta, kend, lmsta, lmend; src/sphp/sphp_mod.F90:68-79), computed there
 * by range (src/sphp/sphp_sca.F90:596-626) for each MPI rank; here 0-based:
 * planes [k0, k0 + nplanes) and lm columns [lm0, lm0 + nlm_local).  After
 * this call, on this plan:
 *   - the 2D transforms (sph_fftp2d_*) take physical arrays of nplanes
 *     planes, (nlat, nphi, nplanes), and spectral arrays (nlm, nplanes):
 *     the reference's per-rank in(nlat,nphi,ksta:kend) and carr1(nlm,ksta:kend)
 *     before its slab transpose (fftp3d_redist_k_to_lm, which a multi-rank
 *     caller keeps doing itself), src/sphp-gpu/sphp_sca.F90:771-853;
 *   - the z transforms, the operators and the boundary take (nlm_local, nz)
 *     arrays, the reference's (lmsta:lmend, nz) (sphp_sca.F90:332-397,
 *     pseudospec_hd.f90, boundary_mod.f90); prodvec and saxpby_r take the
 *     nplanes planes (only planes k0 + k < nz - Cz are physical);
 *   - the 3D transforms, the NL step, RK3 and batches need the whole field
 *     (they would need the slab transpose) and return SPH_EINVAL otherwise.
 * sph_plan_set_slab(p, 0, nz, 0, nlm) restores the whole field (the
 * default).  Results on a slab equal the whole-field results restricted to
 * it.  SPH_EINVAL for an empty or out-of-range slab. */
int sph_plan_set_slab(sph_plan* plan, int k0, int nplanes, int lm0, int nlm_local);

/* range (src/sphp/sphp_sca.F90:596-626): the part [ista, iend] (inclusive)
 * of [n1, n2] that rank irank of nprocs owns; the first mod(n, nprocs)
 * ranks take one element more. */
int sph_range(int n1, int n2, int nprocs, int irank, int* ista, int* iend);

/* ---------------------------------------------------------------- transforms */

/* fftp2d_real_to_complex_xy (src/sphp-gpu/sphp_sca.F90:771-853): per-plane
 * spherical-harmonic analysis of all nz planes, in (nlat,nphi,nz) -> out
 * (nlm,nz).  The input is preserved (the reference destroys it). */
int sph_fftp2d_real_to_complex_xy(sph_plan* plan, const double* in, double* out, void* stream);

/* fftp2d_complex_to_real_xy (src/sphp-gpu/sphp_sca.F90:984-1065): per-plane
 * synthesis, in (nlm,nz) preserved -> out (nlat,nphi,nz). */
int sph_fftp2d_complex_to_real_xy(sph_plan* plan, const double* in, double* out, void* stream);

/* fftp1d_real_to_complex_z (src/sphp-gpu/sphp_sca.F90:856-945 device
 * branch; CPU arithmetic src/sphp/sphp_sca.F90:332-397): FC-Gram
 * continuation, forward DFT along z (sign -1), divide by nz.  In place. */
int sph_fftp1d_real_to_complex_z(sph_plan* plan, double* inout, void* stream);

/* fftp1d_complex_to_real_z (src/sphp-gpu/sphp_sca.F90:1068-1114; CPU
 * src/sphp/sphp_sca.F90:495-530): inverse DFT along z (sign +1), no scaling.
 * In place. */
int sph_fftp1d_complex_to_real_z(sph_plan* plan, double* inout, void* stream);

/* fftp3d_real_to_complex (src/sphp-gpu/sphp_sca.F90:735-768): 2D analysis +
 * z forward.  in preserved. */
int sph_fftp3d_real_to_complex(sph_plan* plan, const double* in, double* out, void* stream);

/* fftp3d_complex_to_real (src/sphp-gpu/sphp_sca.F90:948-981): z inverse +
 * 2D synthesis.  in may be destroyed, as in the reference: FP64 plans
 * transform it in place in z; SPH_MIXED plans (nz of 16, 32, 48, 64, 96,
 * 128, 192, 256 or 512) write the z inverse straight into the synthesis
 * tiles and leave it unchanged. */
int sph_fftp3d_complex_to_real(sph_plan* plan, double* in, double* out, void* stream);

/* fftp2d_vec_to_qst (src/sphp-gpu/sphp_vec.F90:128-218): (v_r,v_th,v_ph) ->
 * (Q,S,T) with v = Q Y r + S r grad Y - T r x grad Y.  Inputs preserved. */
int sph_fftp2d_vec_to_qst(sph_plan* plan, const double* vr, const double* vt, const double* vp,
                          double* q, double* s, double* t, void* stream);

/* fftp2d_qst_to_vec (src/sphp-gpu/sphp_vec.F90:221-309). Inputs preserved. */
int sph_fftp2d_qst_to_vec(sph_plan* plan, const double* q, const double* s, const double* t,
                          double* vr, double* vt, double* vp, void* stream);

/* 3D vector transforms (no reference counterpart: the reference composes
 * them in its nonlinear-term code as fftp2d_vec_to_qst followed by
 * fftp1d_real_to_complex_z on q, s and t, and fftp1d_complex_to_real_z on
 * q, s, t followed by fftp2d_qst_to_vec; these entry points compute exactly
 * those compositions).  sph_fftp3d_qst_to_vec may destroy q, s, t the way
 * sph_fftp3d_complex_to_real may destroy its input.  On SPH_MIXED plans with FC-Gram
 * continuation the forward one continues the physical planes in FP64 before
 * the angular analysis, which keeps the continuation from amplifying the
 * angular round-off (the same holds for sph_fftp3d_real_to_complex). */
int sph_fftp3d_vec_to_qst(sph_plan* plan, const double* vr, const double* vt, const double* vp, double* q,
                          double* s, double* t, void* stream);
int sph_fftp3d_qst_to_vec(sph_plan* plan, double* q, double* s, double* t, double* vr, double* vt, double* vp,
                          void* stream);

/* ---------------------------------------------------------------- operators
 * src/pseudo/pseudospec_hd.f90.  Spectral arrays are (nlm,nz) complex. */

/* derivr (pseudospec_hd.f90:18-135): b = d^p a / dr^p; esp 'r' (a,b in
 * (lm,r): continuation + forward + (i kz)^p + inverse, one kernel) or 'k'
 * (a,b in (lm,kz): b = (i kz)^p a, Nyquist kept). a is preserved. */
int sph_derivr(sph_plan* plan, const double* a, double* b, int p, char esp, void* stream);
/* No counterpart in the reference.  The same radial derivative as
 * sph_derivr(a, b, p, 'r') for a caller that has no plan and cannot
 * allocate device memory: for example a host whose device memory belongs
 * to another allocator (an OpenMP-offload runtime mapping every array, as
 * the reference's gdevice layer does, or a pool that already holds the
 * HBM), where a plan's cudaMalloc'd tables are not an option.  The tables
 * the kernel reads (twiddles, digit-reversal order, (i kz)^p, the FC-Gram
 * operator dir, host Cz x oz column-major) are rebuilt on every call in
 * one file-scope device array of 224 KiB, which every GPU that loads this
 * library holds until the process exits; nothing in it needs to start at
 * zero.  Limits: nz <= 4096, Cz*oz <= 2048, 1 <= p <= 4 (SPH_EINVAL
 * beyond).  Grid as in sph_plan_create (z(k) = rint + k dz,
 * dz = (rext-rint)/(nz-Cz-1)).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  All calls share the one array, so calls
 * that overlap on the GPU (other streams, other host threads) race.
 * Calls no cudaMalloc/cudaFree and allocates no host memory. */
int sph_derivr_noalloc(const double* a, double* b, int nlm, int nz, int Cz, int oz, double rint,
                       double rext, const double* dir, int p, void* stream);
/* laplang (pseudospec_hd.f90:138-172): b = -l(l+1) a */
int sph_laplang(sph_plan* plan, const double* a, double* b, void* stream);
/* multr (pseudospec_hd.f90:175-208): b = z^p a */
int sph_multr(sph_plan* plan, const double* a, double* b, int p, void* stream);
/* dlr (pseudospec_hd.f90:254-288): b = d2a/dr2 - l(l+1) a / r^2 (one kernel) */
int sph_dlr(sph_plan* plan, const double* a, double* b, void* stream);
/* saxpby_c (pseudospec_hd.f90:291-326): z = a x + b y (z may alias x or y) */
int sph_saxpby_c(sph_plan* plan, double* z, const double* x, double a, const double* y, double b,
                 void* stream);
/* saxpby_r (pseudospec_hd.f90:329-366): the same on physical fields */
int sph_saxpby_r(sph_plan* plan, double* z, const double* x, double a, const double* y, double b,
                 void* stream);
/* fc_filter (pseudospec_hd.f90:369-467): a *= exp(-16 ln10 (2kz/(nz Dkz))^100), in place */
int sph_fc_filter(sph_plan* plan, double* a, char esp, void* stream);
/* copy (pseudospec_hd.f90:470-497): b = a */
int sph_copy(sph_plan* plan, const double* a, double* b, void* stream);
/* prodvec (pseudospec_hd.f90:211-251): C = A x B on the physical planes
 * k < nz - Cz; the continuation planes of C are set to zero. */
int sph_prodvec(sph_plan* plan, const double* ar, const double* at, const double* ap,
                const double* br, const double* bt, const double* bp, double* cr, double* ct,
                double* cp, void* stream);

/* ---------------------------------------------------------------- boundary
 * src/boundary/boundary_mod.f90, src/boundary/vboundary.f90 */

/* setup_bc / v_setup / invDl_setup (boundary_mod.f90:35-59,140-241;
 * vboundary.f90:34-56): the kinds of the inner (bcint) and outer (bcext)
 * wall, parsed like v_parsebc (vboundary.f90:10-31):
 *   "noslip"   (the reference's only kind)  W = dW/dr = Z = 0;
 *   "freeslip" (no reference counterpart; stress-free, no penetration)
 *              W = 0, W'' - 2 W'/r = 0, Z' - 2 Z/r = 0, the last by the
 *              Robin reconstruction (needs sph_plan_set_neumann, else
 *              SPH_ENOTREADY).
 * Builds the FC-Gram derivative matrices (a direct DFT), the row-scaled LU
 * per l and the solve on the host in long double (rows 2 and N-1 of B_l by
 * the kind of their wall), and uploads M_l (N x (N-4) per l, rounded to
 * FP64) and the d2/dr2 border rows; a clone whose source built them for the
 * same kinds shares them. */
int sph_setup_bc(sph_plan* plan, const char* bcint, const char* bcext);
/* neumann_reconstruct (src/sphp/fcgram_mod.f90:368-520, the z boundaries)
 * on spectral (nlm, nz) f: boun 0 = inner wall (z index 0), 1 = outer wall
 * (index nz - Cz - 1); on input the wall row holds the ord-th outward normal
 * derivative g, on output the reconstructed value; other rows unchanged. */
int sph_neumann_reconstruct(sph_plan* plan, double* f, int boun, int ord, void* stream);
/* robin_reconstruct (fcgram_mod.f90:523-650): f' + a f = g at the wall, g in
 * the wall row on input; a: DEVICE array of nlm real coefficients (one per
 * lm column, the reference's a over the other coordinates). */
int sph_robin_reconstruct(sph_plan* plan, double* f, int boun, const double* a, void* stream);
/* dirichlet (boundary_mod.f90:62-93): a(lm,1) = a(lm,N) = 0 */
int sph_dirichlet(sph_plan* plan, double* a, void* stream);
/* invDl (boundary_mod.f90:244-292): W = M_l phi(3:N-2), batched FP64 GEMM on
 * the device; l = 0 and the continuation points are zero. */
int sph_invDl(sph_plan* plan, const double* phi, double* w, void* stream);
/* v_imposebc (vboundary.f90:59-87): dirichlet(tor) (freeslip walls: the
 * Robin reconstruction of Z' - 2Z/r = 0 instead), pol = invDl(phi),
 * phi = D_l pol */
int sph_v_imposebc(sph_plan* plan, double* tor, double* phi, double* pol, void* stream);
/* v_imposebc_fast (vboundary.f90:90-130): phi recomputed at rows 1,2,N-1,N only */
int sph_v_imposebc_fast(sph_plan* plan, double* tor, double* phi, double* pol, void* stream);

/* ---------------------------------------------------------------- NL + RK3
 * Composed from the reference's building blocks (the reference has no
 * driver; vboundary.f90:61-63 says the BCs close every RK stage).
 * State (Z, W, phi) in (lm,r), phi = D_l W.  u = curl curl(W r^) + curl(Z r^).
 *   rhs_z   = r T_N + nu D_l Z
 *   rhs_phi = d(r S_N)/dr - Q_N + nu D_l phi,    N = u x curl u
 * energy (host double, may be NULL) = 0.5 * int |u|^2 dV over the physical
 * shell (trapezoid in r, Gauss in theta), accumulated in FP64.  Needs
 * sph_setup_bc. */
int sph_nl_rhs(sph_plan* plan, const double* Z, const double* W, const double* phi, double nu,
               double* rhs_z, double* rhs_phi, double* energy, void* stream);
/* One RK3 step, X = X0 + (dt/o) RHS(X) for o = 3,2,1 with v_imposebc after
 * each stage; Z, W, phi updated in place.  energy of the initial state. */
int sph_rk3_step(sph_plan* plan, double* Z, double* W, double* phi, double nu, double dt,
                 double* energy, void* stream);

/* ---------------------------------------------------------------- run loop
 * The time loop around the NL step, with the input and outputs of the
 * SPECTER-style main program the reference's transforms come from (the
 * reference ships the transform core without a solver). */

/* Reads a namelist file: &grid lmax, nz, Cz, oz (grid_init,
 * src/pseudo/pseudospec_mod.f90:41-69; Cz = oz = 0 when absent) and
 * &boxparams rint, rext (box_init, pseudospec_mod.f90:151-160), both
 * required; and the optional &run group of this loop (no reference
 * counterpart): dt, step (number of steps), tstep (steps between balance
 * lines), sstep (steps between spectra), nu, filter (apply fc_filter after
 * every step); defaults 0, 0, 1, 0, 0, false.  Keys are case-insensitive,
 * reals may use the D exponent, '!' starts a comment.  Any output pointer
 * may be NULL.  SPH_EIO: the file cannot be read; SPH_EINVAL: a required
 * group or key is missing, a key is unknown or a value malformed. */
int sph_read_namelist(const char* path, int* lmax, int* nz, int* Cz, int* oz, double* rint, double* rext,
                      double* dt, int* step, int* tstep, int* sstep, double* nu, int* filter);
/* box_init's grid files (pseudospec_mod.f90:204-220) in directory dir:
 * theta.txt (nlat values), phi.txt (nphi) and z.txt (the nz - Cz physical
 * points), one value per line in Fortran's 1PE23.15 format. */
int sph_write_grids(const sph_plan* plan, const char* dir);
/* Kinetic energy per degree of the state (Z, W) (no reference counterpart;
 * SPECTER writes such spectra): host spec[2l] toroidal (from Z), spec[2l+1]
 * poloidal (from W and dW/dr), l = 0..lmax, trapezoid in r over the
 * physical points like the energy of sph_nl_rhs, which their sum equals.
 * Synchronises the stream.  Needs the whole field. */
int sph_energy_spectrum(sph_plan* plan, const double* Z, const double* W, double* spec, void* stream);
/* The time loop: nsteps steps of sph_rk3_step on (Z, W, phi), each followed,
 * if filter, by fc_filter(., 'r') of Z and phi and v_imposebc.  With outdir
 * (may be NULL) it writes the grid files there, balance.txt (one line
 * "step time energy" for every tstep-th state, 0 = none) and
 * lspectrum.NNNN.txt (l, toroidal, poloidal energy of every sstep-th state,
 * NNNN = step / sstep, 0 = none).  energy_out (may be NULL): the energy of
 * the final state.  Needs sph_setup_bc. */
int sph_run(sph_plan* plan, double* Z, double* W, double* phi, double nu, double dt, int nsteps, int tstep,
            int sstep, int filter, const char* outdir, double* energy_out, void* stream);

/* ---------------------------------------------------------------- single precision
 * The arrays of a GSINGLE_PRECISION build of the reference
 * (src/sphp/fprecision_mod.F90:13-18: REAL(KIND=GP), COMPLEX(KIND=GP) with
 * GP = 4): each routine below is its FP64 counterpart above with float
 * arrays (grids: float[nz][nphi][nlat]; spectra: float pairs [nz][nlm]), on
 * an SPH_MIXED plan over whole fields (SPH_EINVAL otherwise).  The mixed
 * engine reads and writes the float grids in its phi FFTs and the float
 * spectra in its z transforms directly, and the pointwise operators read and
 * write float arrays (computing in FP64); results agree with the FP64 path to
 * the mixed form's accuracy and float rounding.  The inverse transforms
 * preserve their input. */
int sph_fftp2d_real_to_complex_xy_f32(sph_plan* plan, const float* in, float* out, void* stream);
int sph_fftp2d_complex_to_real_xy_f32(sph_plan* plan, const float* in, float* out, void* stream);
int sph_fftp1d_real_to_complex_z_f32(sph_plan* plan, float* inout, void* stream);
int sph_fftp1d_complex_to_real_z_f32(sph_plan* plan, float* inout, void* stream);
int sph_fftp3d_real_to_complex_f32(sph_plan* plan, const float* in, float* out, void* stream);
int sph_fftp3d_complex_to_real_f32(sph_plan* plan, const float* in, float* out, void* stream);
int sph_fftp2d_vec_to_qst_f32(sph_plan* plan, const float* vr, const float* vt, const float* vp, float* q,
                              float* s, float* t, void* stream);
int sph_fftp2d_qst_to_vec_f32(sph_plan* plan, const float* q, const float* s, const float* t, float* vr,
                              float* vt, float* vp, void* stream);
int sph_fftp3d_vec_to_qst_f32(sph_plan* plan, const float* vr, const float* vt, const float* vp, float* q,
                              float* s, float* t, void* stream);
int sph_fftp3d_qst_to_vec_f32(sph_plan* plan, const float* q, const float* s, const float* t, float* vr,
                              float* vt, float* vp, void* stream);
int sph_derivr_f32(sph_plan* plan, const float* a, float* b, int p, char esp, void* stream);
int sph_dlr_f32(sph_plan* plan, const float* a, float* b, void* stream);
int sph_fc_filter_f32(sph_plan* plan, float* a, char esp, void* stream);
int sph_laplang_f32(sph_plan* plan, const float* a, float* b, void* stream);
int sph_multr_f32(sph_plan* plan, const float* a, float* b, int p, void* stream);
int sph_saxpby_c_f32(sph_plan* plan, float* z, const float* x, double a, const float* y, double b, void* stream);
int sph_saxpby_r_f32(sph_plan* plan, float* z, const float* x, double a, const float* y, double b, void* stream);
int sph_copy_f32(sph_plan* plan, const float* a, float* b, void* stream);
int sph_prodvec_f32(sph_plan* plan, const float* ar, const float* at, const float* ap, const float* br,
                    const float* bt, const float* bp, float* cr, float* ct, float* cp, void* stream);
int sph_dirichlet_f32(sph_plan* plan, float* a, void* stream);
/* the boundary solve and the NL step on FP64 copies of the float spectra in
 * the plan's scratch (needs sph_setup_bc like their FP64 counterparts) */
int sph_invDl_f32(sph_plan* plan, const float* phi, float* w, void* stream);
int sph_v_imposebc_f32(sph_plan* plan, float* tor, float* phi, float* pol, void* stream);
int sph_v_imposebc_fast_f32(sph_plan* plan, float* tor, float* phi, float* pol, void* stream);
int sph_nl_rhs_f32(sph_plan* plan, const float* Z, const float* W, const float* phi, double nu, float* rhs_z,
                   float* rhs_phi, double* energy, void* stream);
int sph_rk3_step_f32(sph_plan* plan, float* Z, float* W, float* phi, double nu, double dt, double* energy,
                     void* stream);

/* ---------------------------------------------------------------- timers
 * The reference accumulates wall time per stage in gtimer handles
 * (src/sphp/sphp_mod.F90:36-41: comtime, ffttime, conttime, tottime;
 * src/utils/gtimer_mod.f90).  Here each kernel launch of a plan can be
 * bracketed by CUDA events on its own stream, accumulated per kernel class:
 *   0 phi FFT forward   1 phi FFT inverse   2 Legendre analysis
 *   3 Legendre synthesis 4 vector analysis  5 vector synthesis
 *   6 z transforms      7 pointwise/boundary operators
 * sph_timer_read synchronises the recorded events and returns, per class,
 * the summed milliseconds and the number of launches since the last reset. */
#define SPH_NTIMERS 8
int sph_timer_enable(sph_plan* plan, int on);
int sph_timer_reset(sph_plan* plan);
int sph_timer_read(sph_plan* plan, double* ms, int* launches);

/* Tile shapes of a plan (no reference counterpart; chosen per problem size
 * by redondito_b200/autotune.py).  rows: MMA rows per scalar Legendre work
 * item of an SPH_MIXED plan (32, 64 or 128; rebuilds its tensor-core tables,
 * ignored by FP64 plans); ring_pairs: Gauss ring pairs per CTA of the phi
 * transforms (1, 2, 4, 8, dividing nlat/2, ring_pairs*nphi <= 8192);
 * z_cols: lm columns per CTA of the z transforms (a power of two <= 64,
 * z_cols*nz <= 4096; nz 16, 32, 48, 64, 96, 128, 192 and 256 keep their
 * fixed width, the one their two-step kernel is compiled for).  0 selects
 * the built-in choice.  Results do not
 * depend on the tile shapes beyond round-off.  Synchronises the device. */
int sph_plan_set_tiles(sph_plan* plan, int rows, int ring_pairs, int z_cols);

/* Device status of a plan (no reference counterpart: the reference's
 * kernels have no bounded waits).  The kernels that wait on asynchronous
 * copies (the tensor-core kernels and fp32 phi transforms of an SPH_MIXED
 * plan, the forward phi transform of either form) bound every wait on a
 * shared-memory barrier; one that gives up records it in the plan.  Synchronises the device, then returns
 * SPH_ETIMEDOUT if any wait gave up since the plan was created (the
 * outputs of those calls are invalid) and clears the record, else SPH_OK. */
int sph_plan_status(sph_plan* plan);

/* ---------------------------------------------------------------- batches
 * Many independent shell problems in one CUDA graph (no reference
 * counterpart: the reference runs one problem per set of MPI ranks).
 * Problem p is a plan (all of the same precision, timers off) with
 * nfields[p] = 1..3 scalar fields; the per-field device arrays are given in
 * (problem, field) order: spec (nlm x nz complex, (lm, kz) spectra), grid
 * (nlat x nphi x nz) and dspec (nlm x nz complex).  sph_batch_run computes
 * for every field
 *   spec  -> z inverse in place (fftp1d_complex_to_real_z),
 *   dspec  = derivr(spec, 1, 'r')  (radial derivative, radial space),
 *   grid   = angular synthesis of spec (spec, grid: fftp3d_complex_to_real),
 *   spec   = fftp3d_real_to_complex(grid),
 * with the Legendre contractions of all problems in one grouped launch per
 * direction and the rest on parallel graph branches.  The graph is built
 * once by sph_batch_create (the arrays and plans must outlive the batch);
 * a plan's scratch is used by its batch, so every problem needs a plan of
 * its own (the same plan twice is SPH_EINVAL), and no other work may run on
 * the batch's plans concurrently.  sph_batch_status synchronises the device and
 * returns SPH_ETIMEDOUT if a bounded device wait of the batch gave up. */
typedef struct sph_batch sph_batch;
int sph_batch_create(sph_batch** batch, int nprob, sph_plan* const* plans, const int* nfields,
                     double* const* spec, double* const* grid, double* const* dspec);
int sph_batch_run(sph_batch* batch, void* stream);
int sph_batch_status(sph_batch* batch);
int sph_batch_destroy(sph_batch* batch);

#ifdef __cplusplus
}
#endif
#endif
