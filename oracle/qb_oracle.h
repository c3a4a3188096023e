/* qb_oracle.h — ORACLE / TEST INFRASTRUCTURE ONLY: CPU restatement of the
 * upstream collision + transport step with run-time grid size N.  See
 * qb_oracle.c for conventions.  Only tests/, the smoke check and bench.py's
 * CPU-baseline leg use it. */
#ifndef QB_ORACLE_H
#define QB_ORACLE_H

typedef struct {
	int N, J, M;
	double L, R;
	int n1, n2, n3, n4;          /* term counts: J*J, J, J*M, J */
	double *i1r1, *i1r2;         /* FourierI1 tables */
	double *i2r1, *i2r2;         /* FourierI2 */
	double *i3r1, *i3r2;         /* FourierI3 (psiR1 complex) */
	double *i4r1, *i4r2;         /* FourierI4 */
} orc_quad;

void orc_fft2d(double *a, int n0, int n1, int sign);
void orc_zero_pad(int N, const double *f, double *ret);
void orc_extract(int N, const double *f, double *ret);

void orc_fourier_i1(int N, int J, double L, double R, double *psiR1, double *psiR2);
void orc_fourier_i2(int N, int J, double L, double R, double *psiR1, double *psiR2);
void orc_lgwt(int M, double a, double b, double *x, double *w);
void orc_fourier_i3(int N, int J, double L, double R, int M, double *psiR1, double *psiR2);
void orc_fourier_i4(int N, int J, double L, double R, double *psiR1, double *psiR2);

void orc_i1(int N, const double *f, const double *g, const double *h, int num, const double *psiR1, const double *psiR2, double *out);
void orc_i2(int N, const double *f, const double *g, const double *h, int num, const double *psiR1, const double *psiR2, double *out);
void orc_i3(int N, const double *f, const double *g, const double *h, int num, const double *psiR1, const double *psiR2, double *out);

orc_quad *orc_quad_create(int N, int J, int M, double L, double R);
void orc_quad_free(orc_quad *q);

void orc_cc(const orc_quad *q, const double *W, double *Cc);
void orc_cd(const orc_quad *q, const double *W, double *Cd);
void orc_magnetic_rotation(int N, const double *W, const double B[3], double *CB);
void orc_collision_step(const orc_quad *q, const double *W, double dt, const double B[3], double *Wnext);
void orc_collision_step_rk4(const orc_quad *q, const double *W, double dt, const double B[3], double *Wnext);

void orc_to_fourier(int N, int ncells, const double *Wv, double *Wf);
void orc_from_fourier(int N, int ncells, const double *Wf, double *Wv);

void orc_slope_periodic(double h, double dt, double A, int N, const double *Un, double *Un1);
void orc_slope_dirichlet(double h, double dt, double A, int N, const double *Un, double *Un1);
double orc_flux_right(int m, const double *A, const double *U);
double orc_flux_left(int m, const double *A, const double *U);
void orc_slope_maxwell(double h, double dt, int m, const double *A, int N, double lambda, double fluxL, double fluxR,
                       const double *UmaxwL, const double *UmaxwR, const double *Un, double *Un1);

void orc_inhom_step(const orc_quad *q, int bc, int numVol, const double *W, double h, double dt, const double *Bext, double *Wnext);
void orc_inhom_step_maxwell(const orc_quad *q, int numVol, const double *W, double h, double dt, double lambda,
                            const double *WMaxwL, const double *WMaxwR, const double *Bext, double *Wnext);
void orc_simulation_homogeneous(const orc_quad *q, const double *W0, double dt, int numsteps, const double B[3], double *Wevolv);

#endif
