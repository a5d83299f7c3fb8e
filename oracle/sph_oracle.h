/*
 * sph_oracle.h -- CPU restatement of REDONDITO's pseudospectral transform
 * core, used ONLY as the test oracle and as the timed CPU baseline.
 *
 * TEST INFRASTRUCTURE: nothing in the product (redondito_b200/) links,
 * loads or calls this library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / reference arm use it, as the checker.
 *
 * Layouts (the reference's explicit-shape Fortran arrays, 0-based here):
 *   grid : double [nz][nphi][nlat]      REAL(GP) (nlat,nphi,nz), theta fastest
 *   spec : double2 [nz][nlm] as double  COMPLEX(GP) (nlm,nz), lm fastest,
 *          lm(l,m) = m*(2*lmax+1-m)/2 + l  (SHTns m-major order)
 * Complex values are interleaved (re, im) doubles.
 */
#ifndef SPH_ORACLE_H
#define SPH_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_plan orc_plan;

/* Plan: grid_init/box_init (src/pseudo/pseudospec_mod.f90:41-69,126-236) +
 * fcgram_create_plan (src/sphp/fcgram_mod.f90:49-150).  dir is the C x d
 * continuation operator, Fortran column-major (dir(ii,jj) = dir[ii-1 + C*(jj-1)]);
 * it may be NULL when C == 0 (periodic z).  Returns NULL on bad sizes. */
orc_plan* orc_plan_create(int lmax, int nlat, int nphi, int nz, int C, int d,
                          double rint, double rext, const double* dir);
void orc_plan_destroy(orc_plan* p);
int orc_nlm(const orc_plan* p);
void orc_set_threads(int n);
int orc_get_threads(void);

/* theta (nlat, north pole first), cos(theta), Gauss weights (nlat),
 * z (nz, continuation points included), kz (nz), ell/emm (nlm). */
void orc_grid(const orc_plan* p, double* theta, double* ct, double* w,
              double* z, double* kz, int* ell, int* emm);

/* fcgram_mod.f90:186-263: read A{C}-{d}.dat and Q{d}.dat from tdir and
 * form dir = A . Q^T (C x d, column-major).  0 on success. */
int orc_load_dirichlet_tables(const char* tdir, int C, int d, double* dir);

/* 2D transforms, plane by plane (sphp_sca.F90:273-329, 436-492). */
void orc_sh_analysis(const orc_plan* p, const double* grid, double* spec);
void orc_sh_synthesis(const orc_plan* p, const double* spec, double* grid);
/* Vector QST (sphp_vec.F90:49-165). */
void orc_qst_analysis(const orc_plan* p, const double* vr, const double* vt,
                      const double* vp, double* q, double* s, double* t);
void orc_qst_synthesis(const orc_plan* p, const double* q, const double* s,
                       const double* t, double* vr, double* vt, double* vp);

/* z transforms on spec (nz x nlm), in place (sphp_sca.F90:332-397, 495-530). */
void orc_z_forward(const orc_plan* p, double* spec);
void orc_z_inverse(const orc_plan* p, double* spec);
/* The same on ncols lm columns of a (nz, ncols) array (a slice of a field). */
void orc_z_forward_cols(const orc_plan* p, double* spec, int ncols);
void orc_z_inverse_cols(const orc_plan* p, double* spec, int ncols);
/* 3D = 2D + z (sphp_sca.F90:237-270, 400-433). */
void orc_3d_forward(const orc_plan* p, const double* grid, double* spec);
void orc_3d_inverse(const orc_plan* p, const double* spec, double* grid);

/* Operators (src/pseudo/pseudospec_hd.f90). esp = 'r' or 'k'. */
int orc_derivr(const orc_plan* p, const double* a, double* b, int order, char esp);
void orc_laplang(const orc_plan* p, const double* a, double* b);
void orc_multr(const orc_plan* p, const double* a, double* b, int power);
void orc_dlr(const orc_plan* p, const double* a, double* b);
void orc_saxpby_c(const orc_plan* p, double* z, const double* x, double a,
                  const double* y, double b);
void orc_saxpby_r(const orc_plan* p, double* z, const double* x, double a,
                  const double* y, double b);
int orc_fc_filter(const orc_plan* p, double* a, char esp);
void orc_copy(const orc_plan* p, const double* a, double* b);
void orc_prodvec(const orc_plan* p, const double* ar, const double* at,
                 const double* ap, const double* br, const double* bt,
                 const double* bp, double* cr, double* ct, double* cp);

/* Boundary (src/boundary/boundary_mod.f90, vboundary.f90). */
int orc_bc_setup(orc_plan* p);
/* load_neumann_tables (src/sphp/fcgram_mod.f90:267-365): neu (d values) for
 * the reconstruction from the ord-th normal derivative, dx the grid step.
 * 0 on success. */
int orc_load_neumann_tables(const char* tdir, int d, int ord, double dx, double* neu);
void orc_set_neumann(orc_plan* p, const double* neu1, const double* neu2);
/* neumann_reconstruct / robin_reconstruct (fcgram_mod.f90:368-650) on the
 * z boundaries of spec (nz x nlm): boun 0 inner (z index 0), 1 outer (N-1);
 * the boundary row holds g on input, the reconstructed value on output;
 * a: nlm Robin coefficients.  0 on success. */
int orc_neumann_reconstruct(const orc_plan* p, double* spec, int boun, int ord);
int orc_robin_reconstruct(const orc_plan* p, double* spec, int boun, const double* a);
/* Boundary kinds (inner, outer): 0 noslip, 1 freeslip; then bc_setup. */
int orc_bc_setup_kinds(orc_plan* p, int kint, int kext);
void orc_dirichlet(const orc_plan* p, double* a);
void orc_derivr_mat(const orc_plan* p, int order, double* d /* N x N col-major */);
void orc_invDl(const orc_plan* p, const double* phi, double* w);
void orc_imposebc(const orc_plan* p, double* tor, double* phi, double* pol, int fast);
/* binv (N x (N-4) x lmax, column-major per l) and d2bor (4 x N). */
void orc_bc_tables(const orc_plan* p, double* binv, double* d2bor);
int orc_bc_set_tables(orc_plan* p, int kint, int kext, const double* binv, const double* d2bor);

/* Nonlinear term and RK3 (composed from the reference's building blocks):
 * state = (Z, W, phi) spectra (nz x nlm each), phi = D_l W.
 * rhs_z, rhs_phi: the nonlinear + viscous right-hand sides.
 * energy: FP64 0.5 * integral |u|^2 over the physical shell. */
void orc_nl_rhs(const orc_plan* p, const double* Z, const double* W,
                const double* phi, double nu, double* rhs_z, double* rhs_phi,
                double* energy);
void orc_rk3_step(const orc_plan* p, double* Z, double* W, double* phi,
                  double nu, double dt, double* energy);
/* Per-degree kinetic energy of the state: spec[2l] toroidal, spec[2l+1]
 * poloidal, l = 0..lmax; the sum is the grid energy of nl_rhs. */
void orc_energy_spectrum(const orc_plan* p, const double* Z, const double* W, double* spec);
/* Velocity (and vorticity) on the grid from (Z, W, phi): 3 grids each. */
void orc_velocity(const orc_plan* p, const double* Z, const double* W,
                  const double* phi, double* ur, double* ut, double* up,
                  double* wr, double* wt, double* wp);

#ifdef __cplusplus
}
#endif
#endif
