/*
 * ORACLE -- test infrastructure, never part of the product path.
 *
 * A plain-C CPU restatement of the reference's RK3 substep (OpenTBL,
 * guillemborrell/OpenTBL): rhsp.F90, boun.f90, pois.f90, genflu.F90
 * (NEWGENFLU branch), lip.f90, ffts.f90 and the REAL4 rounding semantics of
 * change.f90, with global (single-domain) semantics: the MPI halo exchanges
 * and transposes of the reference become plain indexing, and the reduction
 * results are the same sums/maxima taken over the whole box. Each function
 * cites the reference file:line it follows.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use this
 * library, and only as the checker / the timed CPU port.
 *
 * PARITY UNPINNED: the reference ships no tests, golden vectors or stored
 * outputs, and cannot be built here (Fortran + MPI + FFTW + HDF5 absent). The
 * restatement is checked by known-answer tests instead (transforms against
 * numpy/scipy, compact operators against polynomial exactness, projection to
 * zero divergence, integral quantities against an independent Python
 * restatement).
 */
#ifndef OTBL_ORACLE_H
#define OTBL_ORACLE_H

#include "../include/otbl.h"
#include "../include/otbl_layout.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_fft orc_fft;
orc_fft *orc_fft_create(int n);
void orc_fft_destroy(orc_fft *p);
void orc_fft_exec(const orc_fft *p, const double *in, double *out, int sign);
void orc_c2r_line(const orc_fft *h, int nz, int nz2, const double *fou,
                  double *phys, double *work);
void orc_r2c_line(const orc_fft *h, int nz, int nz2, const double *phys,
                  double *fou, double *work);
void orc_dct_line(const orc_fft *p, int n, double *c, int iopt, double *work);

/* the reference's coefficient set-up (coeft.f90 coef, bl_1.F90 wavenumbers
 * and inlet_retheta, boun.f90 magicnumber) into the packed buffer of
 * otbl_layout.h, computed by the oracle's own code (orc_coef.c) */
int orc_coef_compute(const otbl_config *cfg, const double *y, const double *u0,
                     double *coef);

typedef struct orc_box orc_box;

orc_box *orc_create(const otbl_config *cfg, const double *coef);
void orc_destroy(orc_box *b);
void orc_set_threads(int n);
int orc_get_threads(void);

/* state arrays in the reference layout (otbl_layout.h) */
double *orc_field(orc_box *b, int id);
void orc_set_inflow(orc_box *b, const double *u0, const double *v0,
                    const double *um, const otbl_inflow *st);
void orc_get_inflow(orc_box *b, double *um, otbl_inflow *st);

int orc_rhsp(orc_box *b, int m, int setstep);
/* ener(1:15) as rhsp leaves it (rhsp.F90:116,487) */
void orc_get_energies(orc_box *b, double *ener);
void orc_outflow_correction(orc_box *b);
void orc_pois(orc_box *b, int m);
int orc_substep(orc_box *b, int m, int setstep);
int orc_advance(orc_box *b, int nsteps);
void orc_boun(orc_box *b);
void orc_genflu(orc_box *b);

/* divergence of pois.f90:41-54 into div (v-type layout; rows 1..ny-1 of
 * planes 2..nx are written, the rest set to 0) */
void orc_divergence(orc_box *b, double *div);

/* one-point statistics (orc_stats.c): statsp (stotf.F90:51-291) with the
 * x pre-pass of rhsp (rhsp.F90:70-92) on the box's current state, added to
 * acc (OTBL_NSTATS arrays (ny, nx), the order of OTBL_ST_*); and its
 * compact operators on one line/column (op 0 interpx_new, 1 diffx, 2
 * interpy_new for u, 3 for p, 4 diffy) */
void orc_statsp(orc_box *b, double *acc);
void orc_stats_operator(orc_box *b, int op, const double *in, double *out);

/* operator-level entry points (lip.f90 / ffts.f90 / change.f90) */
void orc_interpxx(orc_box *b, const double *gen, double *geni, int which,
                  int nlin);
void orc_difvisxx(orc_box *b, const double *upen_int, const double *upencil,
                  double *result, int which, int nlin);
void orc_interpyy(orc_box *b, const double *gen, double *geni, int which,
                  int dim, int m);
void orc_differzy(orc_box *b, const double *geni, double *result, int which);
void orc_vistyy(orc_box *b, const double *u, double *result, int which);
void orc_implzy(orc_box *b, double *u, const double *res, int which,
                double var1);
void orc_fourxz(orc_box *b, double *fou, double *phys, int iopt, int nlines);
void orc_cosftx(orc_box *b, double *c, int nlines, int iopt);
void orc_chp2x(orc_box *b, double *pen, const double *plan, int jee);
void orc_chx2p(orc_box *b, const double *pen, double *plan, int jee);

#ifdef __cplusplus
}
#endif
#endif
