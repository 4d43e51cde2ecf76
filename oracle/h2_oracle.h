/*
 * h2_oracle.h -- declarations of the CPU restatement (test infrastructure only).
 * See h2_oracle.c for the reference citations of every function.
 */
#ifndef H2_ORACLE_H
#define H2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* BoundaryType, src/common.jl:20-24 */
enum { H2O_ISOTHERMAL = 0, H2O_HEAT_FLUX = 1, H2O_CONVECTION = 2 };
/* smoother symbols, src/NonUniform.jl:36-41 */
enum { H2O_SMOOTHER_NONE = 0, H2O_SMOOTHER_GS = 1 };
/* reduction order */
enum { H2O_RED_SEQ = 0, H2O_RED_OMP = 1, H2O_RED_NONE = 2 };

/* BoundaryCondition, src/boundary_conditions.jl:15-21 */
typedef struct {
  int type;
  double temperature;
  double heat_flux;
  double htc;
  double ambient;
} h2o_bc;

/* Grid description shared by the operator functions. */
typedef struct {
  int MX, MY, MZ;
  double dx, dy, dt;
  const double *ZC; /* MZ */
  const double *dZ; /* MZ */
  const double *HC; /* 6: [x-, x+, y-, y+, z-, z+] */
  int is_steady;
} h2o_grid;

/* WorkBuffers, src/common.jl:49-65 (same 15 arrays, same roles) */
typedef struct {
  double *theta, *b, *mask, *rho, *lam, *cp;
  double *p, *p_, *r, *r0, *q, *s, *s_, *t_;
  double *hsrc;
} h2o_wk;

int h2o_has_openmp(void);
void h2o_set_threads(int nthreads);
int h2o_genz(int nk, double *Z, double *ZC, double *dZ);
double h2o_pitch(int n);
int h2o_fill_id(int MX, int MY, int MZ, double dx, double dy, const double *Z, uint8_t *ID, int nthreads);
void h2o_set_properties(size_t n, const uint8_t *ID, double *lam, double *rho, double *cp);
void h2o_apply_bc(int MX, int MY, int MZ, const h2o_bc *bc, double *th, double *lam, double *rho, double *cp,
                  double *mask);
void h2o_set_bc_coef(const h2o_bc *bc, double *HC);
void h2o_heat_src(int MX, int MY, int MZ, const uint8_t *ID, double *hsrc);
void h2o_calrhs(const h2o_grid *G, const h2o_bc *bc, double *b, const double *th, const double *rho,
                const double *cp, const double *hsrc);
double h2o_fdot1(const h2o_grid *G, const double *x, int red_mode);
double h2o_fdot2(const h2o_grid *G, const double *x, const double *y, int red_mode);
double h2o_calcrk(const h2o_grid *G, double *r, const double *th, const double *b, const double *lam,
                  const double *m, const double *rho, const double *cp, int red_mode);
void h2o_calcax(const h2o_grid *G, double *ax, const double *x, const double *lam, const double *m,
                const double *rho, const double *cp);
double h2o_rbsor_core(const h2o_grid *G, double *th, const double *lam, const double *b, const double *m,
                      const double *rho, const double *cp, double omega, int color, int red_mode);
double h2o_rbsor(const h2o_grid *G, double *th, const double *lam, const double *b, const double *m,
                 const double *rho, const double *cp, double omega, int red_mode);
void h2o_preconditioner(const h2o_grid *G, double *xx, const double *bb, const double *lam, const double *m,
                        const double *rho, const double *cp, int smoother);
void h2o_bicg1(const h2o_grid *G, double *p, const double *r, const double *q, double beta, double omg);
void h2o_triad(const h2o_grid *G, double *z, const double *x, const double *y, double a);
void h2o_bicg2(const h2o_grid *G, double *z, const double *x, const double *y, double a, double b);
int h2o_pbicgstab(const h2o_grid *G, h2o_wk *wk, double tol, int maxItr, int smoother, int verbose, int red_mode,
                  int nthreads, int *itr_out, double *res0_out, double *hist);
int h2o_cg(const h2o_grid *G, h2o_wk *wk, double tol, int maxItr, int smoother, int verbose, int red_mode,
           int nthreads, int *itr_out, double *res0_out, double *hist);
double h2o_res_sor(const h2o_grid *G, const double *th, const double *lam, const double *b, const double *m,
                   const double *rho, const double *cp, double omega);
int h2o_solve_sor(const h2o_grid *G, h2o_wk *wk, double omega, double tol, int maxItr, int red_mode, int nthreads,
                  double *res0_out, double *hist);

#ifdef __cplusplus
}
#endif
#endif
