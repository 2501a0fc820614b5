/* Step functions of the channel-flow DNS with the reference's names,
 * signatures and field layout, computed on the GPU (libchanfast_steps.so).
 *
 * Fields are host arrays in the reference's padded layout: a flat double
 * array of n0*n1*n2 values, n0 = local_nx + 2*nghost_x, n1 = local_ny +
 * 2*nghost_y, n2 = nz + 2*nghost_z, index (i*n1 + j)*n2 + k with k
 * (wall-normal) fastest (d3tensor.c:9-42).  Spectra are z-pencils
 * cout[local_nx][local_ny][n2] of complex values stored as double[2]
 * (re, im), binary compatible with fftw_complex.  Each call copies the arrays
 * it reads to the current CUDA device, computes there and copies back the
 * arrays it writes; results equal the reference CPU code bit for bit.
 *
 * The module functions keep the reference's state rules: diffuseu_*, diffusew_*
 * and pressure_* functions of one order run only after the matching
 * *_initialize{2,4}.  Where the reference aborts through check() (check.h:8-12),
 * these functions record a status instead and return; cf_steps_status() and
 * cf_steps_message() report the last call's outcome. */
#ifndef CHANFAST_STEPS_H
#define CHANFAST_STEPS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary-condition types (diffuseu.h:1-2, diffusew.h:1). */
#define DIRICHU (0)
#define NEUMANU (1)
#define DIRICHW (20)

/* Outcome of the last step-function call (no counterpart in the reference,
 * which aborts instead). */
#define CF_STEPS_OK 0
#define CF_STEPS_EINVAL (-1)  /* size or boundary-condition type out of range */
#define CF_STEPS_EORDER (-2)  /* module not initialised for this order */
#define CF_STEPS_EPIVOT (-3)  /* zero pivot in a band solve */
#define CF_STEPS_ECUDA (-4)   /* CUDA runtime error (no device, out of memory) */
int cf_steps_status(void);
const char *cf_steps_message(void);

/* ---- rk3.h:1-4, fourth.h:1-4: the coefficients as data symbols. */
extern const double rk3_alp[];
extern const double rk3_bet[];
extern const double rk3_gam[];
extern const double rk3_zet[];
extern double a1;
extern double a2;
extern double b1;
extern double b2;

/* ---- tridag.h, heptdag.h: one band system (tridag.c:4-26, heptdag.c:5-61). */
void tridag(double a[], double b[], double c[], double r[], double u[], int n);
void heptdag(double a[], double b[], double c[], double d[], double e[], double f[], double g[], double h[],
             double x[], int n);

/* ---- advect.h:1-77 (advect.c). massflux*4 also rewrite the wall ghosts of
 * u, v, w in place, as the reference does (advect.c:100-131). */
void massfluxx2(double u[], double v[], double w[], double muphx[], double mvphx[], double mwphx[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void massfluxy2(double u[], double v[], double w[], double muphy[], double mvphy[], double mwphy[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void massfluxz2(double u[], double v[], double w[], double muphz[], double mvphz[], double mwphz[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void massfluxx4(double u[], double v[], double w[], double muphx[], double mvphx[], double mwphx[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void massfluxy4(double u[], double v[], double w[], double muphy[], double mvphy[], double mwphy[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void massfluxz4(double u[], double v[], double w[], double muphz[], double mvphz[], double mwphz[],
                int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);
void advectu2(double u[], double muphx[], double mvphx[], double mwphx[], double fu[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void advectv2(double v[], double muphy[], double mvphy[], double mwphy[], double fv[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void advectw2(double w[], double muphz[], double mvphz[], double mwphz[], double fw[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void advectu4(double u[], double muphx[], double mvphx[], double mwphx[], double fu[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void advectv4(double v[], double muphy[], double mvphy[], double mwphy[], double fv[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void advectw4(double w[], double muphz[], double mvphz[], double mwphz[], double fw[], int local_nx,
              int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);

/* ---- scalar.h:1-24 (scalar.c). */
void add_buoyancy2(double c[], double fu[], double fv[], double fw[], double betg_x, double betg_y,
                   double betg_z, int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z);
void add_buoyancy4(double c[], double fu[], double fv[], double fw[], double betg_x, double betg_y,
                   double betg_z, int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z);
void advect_scalar(double mucphx[], double mvcphy[], double mwcphz[], double fc[], int local_nx, int local_ny,
                   int nz, int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void flux_quick(double u[], double v[], double w[], double c[], double mucphx[], double mvcphy[],
                double mwcphz[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                double dx, double dy, double dz[]);

/* ---- pressure.h:1-49 (pressure.c). divergence4 extrapolates w into its
 * outer ghost faces in place (pressure.c:80-97). */
void divergence2(double u[], double v[], double w[], double d[], int local_nx, int local_ny, int nz,
                 int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void divergence4(double u[], double v[], double w[], double d[], int local_nx, int local_ny, int nz,
                 int nghost_x, int nghost_y, int nghost_z, double dx, double dy, double dz[]);
void project2(double u[], double v[], double w[], double p[], int local_nx, int local_ny, int nz, int nghost_x,
              int nghost_y, int nghost_z, double dx, double dy, double dz[], double dt);
void project4(double u[], double v[], double w[], double p[], int local_nx, int local_ny, int nz, int nghost_x,
              int nghost_y, int nghost_z, double dx, double dy, double dz[], double dt);
void pressure_laplacian2(double p[], double l[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y,
                         int nghost_z, double dx, double dy, double dz[], double dt);
void pressure_laplacian4(double p[], double l[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y,
                         int nghost_z, double dx, double dy, double dz[], double dt);
void pressure_poisson2(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                       int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double dt);
void pressure_poisson4(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                       int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double dt);
void pressure_initialize2(int nz, int nghost_z);
void pressure_initialize4(int nz, int nghost_z);
void pressure_finalize2(void);
void pressure_finalize4(void);

/* ---- diffuseu.h:1-86 (diffuseu.c): cell-centred fields u, v, c. */
void apply_bc_u2(double u[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                 double xu[], double yu[], double dz[], double (*bc_bot)(double, double),
                 double (*bc_top)(double, double), int bctype_bot, int bctype_top);
void apply_bc_u4(double u[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                 double xu[], double yu[], double dz[], double (*bc_bot)(double, double),
                 double (*bc_top)(double, double), int bctype_bot, int bctype_top);
void helmholtz1d_operator_u2(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                             int nghost_y, int nghost_z, double dz[], double nudt);
void helmholtz1d_operator_u4(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                             int nghost_y, int nghost_z, double dz[], double nudt);
void solve_helmholtz1d_u2(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                          int nghost_y, int nghost_z, double dz[], double nudt, double avg_bot, double avg_top,
                          int bctype_bot, int bctype_top);
void solve_helmholtz1d_u4(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                          int nghost_y, int nghost_z, double dz[], double nudt, double avg_bot, double avg_top,
                          int bctype_bot, int bctype_top);
void add_laplacexy_operator_u2(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                               int nghost_y, int nghost_z, double dx, double dy, double nu);
void add_laplacexy_operator_u4(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                               int nghost_y, int nghost_z, double dx, double dy, double nu);
void helmholtz_operator_u2(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                           int nghost_y, int nghost_z, double dx, double dy, double dz[], double nudt);
void helmholtz_operator_u4(double u[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                           int nghost_y, int nghost_z, double dx, double dy, double dz[], double nudt);
void solve_helmholtz_u2(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                        int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double nudt,
                        double avg_bot, double avg_top, int bctype_bot, int bctype_top);
void solve_helmholtz_u4(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                        int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double nudt,
                        double avg_bot, double avg_top, int bctype_bot, int bctype_top);
void diffuseu_initialize2(int nz, int nghost_z);
void diffuseu_initialize4(int nz, int nghost_z);
void diffuseu_finalize2(void);
void diffuseu_finalize4(void);

/* ---- diffusew.h:1-85 (diffusew.c): the face field w. */
void apply_bc_w2(double w[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                 double xw[], double yw[], double dz[], double (*bc_bot)(double, double),
                 double (*bc_top)(double, double), int bctype_bot, int bctype_top);
void apply_bc_w4(double w[], int local_nx, int local_ny, int nz, int nghost_x, int nghost_y, int nghost_z,
                 double xw[], double yw[], double dz[], double (*bc_bot)(double, double),
                 double (*bc_top)(double, double), int bctype_bot, int bctype_top);
void helmholtz1d_operator_w2(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                             int nghost_y, int nghost_z, double dz[], double nudt);
void helmholtz1d_operator_w4(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                             int nghost_y, int nghost_z, double dz[], double nudt);
void solve_helmholtz1d_w2(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                          int nghost_y, int nghost_z, double dz[], double nudt, double avg_bot, double avg_top,
                          int bctype_bot, int bctype_top);
void solve_helmholtz1d_w4(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                          int nghost_y, int nghost_z, double dz[], double nudt, double avg_bot, double avg_top,
                          int bctype_bot, int bctype_top);
void add_laplacexy_operator_w2(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                               int nghost_y, int nghost_z, double dx, double dy, double nu);
void add_laplacexy_operator_w4(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                               int nghost_y, int nghost_z, double dx, double dy, double nu);
void helmholtz_operator_w2(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                           int nghost_y, int nghost_z, double dx, double dy, double dz[], double nudt);
void helmholtz_operator_w4(double w[], double h[], int local_nx, int local_ny, int nz, int nghost_x,
                           int nghost_y, int nghost_z, double dx, double dy, double dz[], double nudt);
void solve_helmholtz_w2(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                        int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double nudt,
                        double avg_bot, double avg_top, int bctype_bot, int bctype_top);
void solve_helmholtz_w4(double (*cout)[2], int nx, int local_nx, int local_x_start, int ny, int local_ny,
                        int local_y_start, int nz, int nghost_z, double dx, double dy, double dz[], double nudt,
                        double avg_bot, double avg_top, int bctype_bot, int bctype_top);
void diffusew_initialize2(int nz, int nghost_z);
void diffusew_initialize4(int nz, int nghost_z);
void diffusew_finalize2(void);
void diffusew_finalize4(void);

#ifdef __cplusplus
}
#endif

#endif /* CHANFAST_STEPS_H */
