/* Test infrastructure: CPU oracle for the vlp4d semi-Lagrangian step.
 *
 * A plain-C restatement of the reference's single-process vlp4d algorithm
 * (yasahi-hpc/P3-miniapps, miniapps/vlp4d/openmp).  It is the checker for
 * the CUDA library, never part of it: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it.  Its results are pinned against
 * the reference's own OpenMP build (oracle/_ref, see oracle/ref_driver.cpp)
 * and against the committed fixtures in tests/golden/.
 *
 * Arrays are FP64, layout_left: f(ix, iy, ivx, ivy) lives at
 * ix + nx*(iy + ny*(ivx + nvx*ivy)); 2D fields (ix, iy) at ix + nx*iy.
 */
#ifndef VLP4D_ORACLE_H
#define VLP4D_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n[4];         /* nx, ny, nvx, nvy */
  double minp[4];   /* minPhy_ */
  double maxp[4];   /* maxPhy_ */
  double dx[4];     /* (max - min) / n */
  double dt;
  int idcase;       /* selects the field_poisson branch (2, 6, 10, 20, other) */
} orc_domain;

/* Initial conditions.  10/20/2/5 are the reference's testcases; the others
 * are the perturbed-Maxwellian families the benchmark configurations use. */
enum {
  ORC_IC_CYL02 = 2,
  ORC_IC_CYL05 = 5,
  ORC_IC_SLD10 = 10,          /* (1+a cos(kx x) cos(ky y)) M(vx) M(vy), a=0.05, k=0.5 */
  ORC_IC_TSI20 = 20,
  ORC_IC_TSI20_MPI = 21,      /* vlp4d_mpi's case 20 (miniapps/vlp4d_mpi/openmp/Init.cpp:249-277) */
  ORC_IC_LANDAU_SUM = 110,    /* (1+a cos(k x)+a cos(k y)) M(vx) M(vy) */
  ORC_IC_TWO_STREAM = 120     /* (1+a cos(k x)+a cos(k y)) 0.5[M(vx-u)+M(vx+u)] M(vy) */
};

void orc_domain_init(orc_domain *d, const int n[4], const double minp[4], const double maxp[4],
                     double dt, int idcase);
void orc_lag_basis5(double px, double coef[6]);

void orc_advect_x(const orc_domain *d, const double *fn, double *fnp1, double dt);
void orc_advect_y(const orc_domain *d, const double *fn, double *fnp1, double dt);
void orc_advect_vx(const orc_domain *d, const double *fn, double *fnp1, const double *ex, double dt);
void orc_advect_vy(const orc_domain *d, const double *fn, double *fnp1, const double *ey, double dt);

void orc_field_rho(const orc_domain *d, const double *fn, double *rho);
/* rho is overwritten with phi, as in the reference. */
void orc_field_poisson(const orc_domain *d, double *rho, double *ex, double *ey);
void orc_diags(const orc_domain *d, const double *rho, const double *ex, const double *ey,
               double *nrj, double *mass);
/* The vlp4d_mpi diagnostics (miniapps/vlp4d_mpi/thrust/Diags.cpp:17-92). */
void orc_diags_mpi(const orc_domain *d, const double *ex, const double *ey, double *nrjx, double *nrjy);
double orc_l2norm(const orc_domain *d, const double *f);

/* rfft2 / irfft2 of a (nx1, nx2) layout_left real array; `hat` is
 * (nx1/2+1, nx2) complex, interleaved (re, im). */
void orc_rfft2(int nx1, int nx2, const double *in, double *hat);
void orc_irfft2(int nx1, int nx2, const double *hat, double *out);

/* One Strang step; fn holds the state before and after, fnp1 is scratch.
 * nrj/mass receive the mid-step diagnostic. */
void orc_step(const orc_domain *d, double *fn, double *fnp1, double *rho, double *ex, double *ey,
              double *nrj, double *mass);
/* The initial field solve + diagnostic, then nsteps steps.
 * nrj/mass hold nsteps+1 entries. */
void orc_run(const orc_domain *d, double *fn, double *fnp1, double *rho, double *ex, double *ey,
             int nsteps, double *nrj, double *mass);

void orc_init_case(const orc_domain *d, double *f, int ic, double amp, double k, double u);

/* The vlp4d_mpi step for one process (vlp4d_mpi_oracle.c).  Halo arrays:
 * extents n[d] + 6, first index -3, layout_left; orcm_size() doubles. */
size_t orcm_size(const orc_domain *d);
void orcm_get_interior(const orc_domain *d, const double *fh, double *f);
void orcm_set_interior(const orc_domain *d, double *fh, const double *f);
void orcm_halo_fill(const orc_domain *d, double *f);
void orcm_spline_xy(const orc_domain *d, double *f);
void orcm_spline_vxvy(const orc_domain *d, double *f);
int orcm_advect_2d(const orc_domain *d, double *f, double *tmp, double dt);
int orcm_advect_4d(const orc_domain *d, const double *ex, const double *ey, double *fn, double *tmp);
void orcm_field_rho(const orc_domain *d, const double *f, double *rho);
double orcm_l2norm(const orc_domain *d, const double *f);
void orcm_start(const orc_domain *d, const double *fn, double *rho, double *ex, double *ey, double out[5]);
int orcm_step(const orc_domain *d, double *fn, double *fnp1, double *tmp, double *rho, double *ex, double *ey,
              double half[4], double out[5]);
void orcm_init_case(const orc_domain *d, double *fh, int ic);

/* FP64 discrete adjoint of the restated step (vlp4d_adjoint.c).  The
 * objective is J(f) = dx*dy * sum (Ex^2 + Ey^2), E solved from f. */
void orc_lag_basis5_deriv(double px, double dcoef[6]);
void orc_advect_x_T(const orc_domain *d, const double *lam_out, double *lam_in, double dt);
void orc_advect_y_T(const orc_domain *d, const double *lam_out, double *lam_in, double dt);
void orc_advect_vx_T(const orc_domain *d, const double *lam_out, const double *f_in, const double *ex,
                     double dt, double *lam_in, double *gex);
void orc_advect_vy_T(const orc_domain *d, const double *lam_out, const double *f_in, const double *ey,
                     double dt, double *lam_in, double *gey);
void orc_field_poisson_T(const orc_domain *d, const double *gex, const double *gey, double *lam_rho);
void orc_energy_grad(const orc_domain *d, const double *f, double *J, double *lam);
void orc_step_adjoint(const orc_domain *d, const double *f_state, const double *lam_next, double *lam_out);
void orc_adjoint_run(const orc_domain *d, const double *f0, int nsteps, double *J, double *grad);

#ifdef __cplusplus
}
#endif

#endif
