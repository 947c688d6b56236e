/*
 * oracle.h -- ORACLE / TEST INFRASTRUCTURE ONLY (see cpsd_oracle.c).
 *
 * Entry points of the project's plain-C restatement of the reference's
 * steepest-descent path.  Layouts are the reference's: complex arrays are the
 * half box ((nfft/2+1) x nfft x nfft complex = n2ft3d doubles per band),
 * real-space arrays the padded (nfft+2) x nfft x nfft box.
 */
#ifndef CPSD_ORACLE_H
#define CPSD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ccpsdv3/gcdotc.c:16-29, gsdot.c:16-28, gssum.c:30-41 */
double oracle_gcdotc(int nfft, const double *a, const double *b);
double oracle_gsdot(int nfft, const double *a, const double *b);
double oracle_gssum(int nfft, const double *x);

/* ccpsdv3/strfac.c:10-77 and :93-123 */
void oracle_phafac(int nfft, const double *unitg, int nion, const double *r1,
                   double *ex1, double *ex2, double *ex3);
void oracle_strfac(int nfft, const double *ex1, const double *ex2,
                   const double *ex3, double *exi);

/* ccpsdv3/dirac_exchange.c:64-126 followed by vosko.c:99-167 */
void oracle_xc(int ispin, int n2ft3d, const double *dn, double *xcp, double *xce);

/* fftpack3d/fftpack3d.f:22-96 and :107-196 (defined in fft3d.c) */
void cr_fft3b_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r,
               int *nx, int *ny, int *nz, double *tmp, int *ntmp);
void rc_fft3f_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r,
               int *nx, int *ny, int *nz, double *tmp, int *ntmp);

/*
 * ccpsdv3/cpsd.c:33-698 with the reference's argument list minus cpsdwork
 * (the restatement allocates its own scratch).  *lagrange_fail receives the
 * number of steps whose Lagrange iteration stopped without converging (the
 * reference prints "ierr=10" for those, cpsd.c:477).  Returns 0, or -1 when
 * scratch cannot be allocated.
 */
int oracle_cpsd(int inner, int move, int nion, int ispin, const int *ne,
                int nfft, int nfft3d, int n2ft3d, const double *unitg,
                double omega, double dt, double fmass, const int *katm,
                const double *amass, const double *zv, int nsh,
                const double *rcell, double cewald, double rcut,
                const int *masker, const double *G, const double *tg,
                const double *vc, const double *vg, const int *lmmax,
                const double *vnlnrm, const double *vl, const double *vnl,
                double *r1, double *r2, double *fion, double *c1, double *c2,
                double *cpsi, double *dn, double *hml, double *lmd, double *E,
                double *deltae, double *deltac, double *deltar,
                int *lagrange_fail);

/*
 * Band-parallel form of the same step (move = 0), the decomposition a
 * multi-GPU run of one cell uses: this rank transforms, densifies and steps
 * only bands [lo, hi); allreduce_sum adds the spin densities of all ranks in
 * place (after the density, cpsd.c:185-194), allgather_rows gives every rank
 * the rows of buf that each rank owns (its [lo, hi), row doubles each) after
 * the steepest-descent update (cpsd.c:399-400), for c2 and for cpsi.  The
 * overlaps, the Lagrange iteration, the constraint and the energies then run
 * on the full arrays on every rank.  Returns -2 for a bad range.
 */
typedef struct {
    int lo, hi;
    void (*allreduce_sum)(double *buf, long n, void *user);
    void (*allgather_rows)(double *buf, long row, void *user);
    void *user;
} oracle_bands;

int oracle_cpsd_bands(int inner, int nion, int ispin, const int *ne,
                      int nfft, int nfft3d, int n2ft3d, const double *unitg,
                      double omega, double dt, double fmass, const int *katm,
                      const double *amass, const double *zv, int nsh,
                      const double *rcell, double cewald, double rcut,
                      const int *masker, const double *G, const double *tg,
                      const double *vc, const double *vg, const int *lmmax,
                      const double *vnlnrm, const double *vl, const double *vnl,
                      double *r1, double *r2, double *fion, double *c1, double *c2,
                      double *cpsi, double *dn, double *hml, double *lmd, double *E,
                      double *deltae, double *deltac, double *deltar,
                      int *lagrange_fail, const oracle_bands *bp);

#ifdef __cplusplus
}
#endif
#endif
