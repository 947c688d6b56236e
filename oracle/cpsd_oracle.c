/*
 * cpsd_oracle.c -- ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * The project's plain-C restatement of the reference's steepest-descent
 * electronic minimisation, ccpsdv3/cpsd.c:33-698 (Simple-CPSD), written for
 * checking the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it; the product never does.  It works in the
 * reference's own layouts (full half box per band, padded real box) and
 * restates each step in the reference's order so that results agree with the
 * reference build (oracle/_ref) to rounding.  Every block cites the reference
 * lines it follows.  No BLAS: dot products, axpys and the small matrix
 * products are plain loops in the reference's summation order where that
 * order is defined by a loop (BLAS-internal orders are not reproduced; they
 * differ by rounding only).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---------------------------------------------------------------- Γ dots */

/* plain strided dot, the role of ddot_ in the reference */
static double dot_strided(long n, const double *x, long incx, const double *y, long incy)
{
    double s = 0.0;
    for (long i = 0; i < n; ++i) s += x[i * incx] * y[i * incy];
    return s;
}

/* gcdotc.c:16-29: <a|b> over the half box, kx=0 plane counted once */
double oracle_gcdotc(int nfft, const double *a, const double *b)
{
    long n2 = (long)nfft * nfft;
    long n3 = (long)(nfft + 2) * nfft * nfft;
    return 2.0 * dot_strided(n3, a, 1, b, 1) - dot_strided(n2, a, nfft + 2, b, nfft + 2) -
           dot_strided(n2, a + 1, nfft + 2, b + 1, nfft + 2);
}

/* gsdot.c:16-28: the same weighting for real arrays of nfft3d entries */
double oracle_gsdot(int nfft, const double *a, const double *b)
{
    long nh = nfft / 2 + 1;
    long n2 = (long)nfft * nfft;
    long n3 = nh * nfft * nfft;
    return 2.0 * dot_strided(n3, a, 1, b, 1) - dot_strided(n2, a, nh, b, nh);
}

/* gssum.c:19-41 */
double oracle_gssum(int nfft, const double *x)
{
    long nh = nfft / 2 + 1;
    long n2 = (long)nfft * nfft;
    long n3 = nh * nfft * nfft;
    double s1 = 0.0, s2 = 0.0;
    for (long i = 0; i < n3; ++i) s1 += x[i];
    for (long i = 0; i < n2; ++i) s2 += x[i * nh];
    return 2.0 * s1 - s2;
}

/* ------------------------------------------------------ structure factors */

/* strfac.c:10-77: per-ion 1-D phase tables e^{-i k (b_d . r + pi)} */
void oracle_phafac(int nfft, const double *unitg, int nion, const double *r1,
                   double *ex1, double *ex2, double *ex3)
{
    const double pi = 4.0 * atan(1.0);
    int nh = nfft / 2;
    for (int ii = 0; ii < nion; ++ii) {
        const double *r = r1 + 3 * ii;
        double sw[3];
        for (int d = 0; d < 3; ++d)
            sw[d] = unitg[3 * d] * r[0] + unitg[3 * d + 1] * r[1] + unitg[3 * d + 2] * r[2] + pi;
        double *t[3] = {ex1 + (long)ii * (nfft + 2), ex2 + (long)ii * 2 * nfft,
                        ex3 + (long)ii * 2 * nfft};
        for (int d = 0; d < 3; ++d) {
            double cr = cos(sw[d]), ci = -sin(sw[d]);
            double *e = t[d];
            e[0] = 1.0;
            e[1] = 0.0;
            for (int k = 1; k <= nh; ++k) {
                double pr = e[2 * (k - 1)], pim = e[2 * (k - 1) + 1];
                e[2 * k] = pr * cr - pim * ci;
                e[2 * k + 1] = pr * ci + pim * cr;
                if (d > 0) { /* negative k mirrored as the conjugate: strfac.c:45-55 */
                    e[2 * (nfft - k)] = e[2 * k];
                    e[2 * (nfft - k) + 1] = -e[2 * k + 1];
                }
            }
            e[nfft] = 0.0; /* Nyquist entry zeroed: strfac.c:69-74 */
            e[nfft + 1] = 0.0;
        }
    }
}

/* strfac.c:93-123: exi(G) = ex1[kx] (ex2[ky] ex3[kz]) over the half box */
void oracle_strfac(int nfft, const double *ex1, const double *ex2, const double *ex3, double *exi)
{
    int nh = nfft / 2;
    long kk = 0;
    for (int k = 0; k < nfft; ++k)
        for (int j = 0; j < nfft; ++j) {
            double tr = ex2[2 * j] * ex3[2 * k] - ex2[2 * j + 1] * ex3[2 * k + 1];
            double ti = ex2[2 * j] * ex3[2 * k + 1] + ex2[2 * j + 1] * ex3[2 * k];
            for (int i = 0; i <= nh; ++i) {
                exi[kk] = ex1[2 * i] * tr - ex1[2 * i + 1] * ti;
                exi[kk + 1] = ex1[2 * i + 1] * tr + ex1[2 * i] * ti;
                kk += 2;
            }
        }
}

/* ----------------------------------------------------------- LDA xc */

/* Dirac exchange, dirac_exchange.c:14-126 (alpha = 2/3).  The spin-polarised
 * branch keeps the reference's xi = (rho[0]-rho[1])/n (dirac_exchange.c:101). */
static void dirac_exchange(int ispin, int n2ft3d, const double *rho, double *vx, double *ex)
{
    const double alpha = 0.6666666666666666667;
    const double onethird = 0.33333333333333333333;
    const double fourthird = 1.33333333333333333333;
    const double two_to_onethird = 1.25992104989487319067;
    const double A = 0.25992104989487319067;
    const double pi = 3.14159265358979311600;
    if (ispin == 1) {
        for (int i = 0; i < n2ft3d; ++i) {
            double n = rho[i] + rho[i];
            double n13 = pow(3.0 * n / pi, onethird);
            ex[i] = -(9.0 / 8.0) * alpha * n13;
            vx[i] = -(3.0 / 2.0) * alpha * n13;
        }
        return;
    }
    for (int i = 0; i < n2ft3d; ++i) {
        double n = rho[i] + rho[i + n2ft3d];
        double n13 = pow(3.0 * n / pi, onethird);
        double xi = (n > 0.0) ? (rho[0] - rho[1]) / n : 1.0;
        double ex_p = -(9.0 / 8.0) * alpha * n13;
        double ux_p = -(3.0 / 2.0) * alpha * n13;
        double ex_f = two_to_onethird * ex_p;
        double ux_f = fourthird * ex_f;
        double f = (pow(1.0 + xi, fourthird) + pow(1.0 - xi, fourthird) - 2.0) / (2.0 * A);
        double df = fourthird * (pow(1.0 + xi, onethird) - pow(1.0 - xi, onethird)) / (2.0 * A);
        ex[i] = ex_p + f * (ex_f - ex_p);
        vx[i] = ux_p + f * (ux_f - ux_p) + (+1.0 - xi) * (df * (ex_f - ex_p));
        vx[i + n2ft3d] = ux_p + f * (ux_f - ux_p) + (-1.0 - xi) * (df * (ex_f - ex_p));
    }
}

/* Vosko-Wilk-Nusair correlation, vosko.c:99-167, accumulated into xcp/xce.
 * The parameter table is the reference's, digit for digit (vosko.c:22-52),
 * because energies are compared at 1e-9 Ha. */
static void vosko(int ispin, int n2ft3d, const double *dn, double *xcp, double *xce)
{
    const double bp = 3.727440e+00, bf = 7.060420e+00;
    const double cp = 1.293520e+01, cf = 1.805780e+01;
    const double cp1 = 3.109070e-02, cf1 = 1.554530e-02;
    const double cp2 = 9.690228e-04, cf2 = 2.247860e-03;
    const double cp3 = 1.049800e-01, cf3 = 3.250000e-01;
    const double cp4 = 3.878329e-02, cf4 = 5.249122e-02;
    const double cp5 = 3.075995e+00, cf5 = 2.365463e+00;
    const double cp6 = 1.863720e+00, cf6 = 3.530210e+00;
    const double dp1 = 6.218140e-02, df1 = 3.109060e-02;
    const double dp2 = 1.938045e-03, df2 = 4.495720e-03;
    const double dp4 = -3.205972e-02, df4 = -1.779316e-02;
    const double dp5 = -1.192972e-01, df5 = -1.241661e-01;
    const double dp6 = 1.863720e+00, df6 = 3.530210e+00;
    const double dp7 = 9.461748e+00, df7 = 5.595417e+00;
    const double small_number = 1.0e-30;
    const double onesixth = 0.166666666666667;
    const double onethird = 0.333333333333333;
    const double fourthird = 1.333333333333333;
    const double A = 0.259921049894873;
    const double rs_scale = 0.620350490899400;
    for (int i = 0; i < n2ft3d; ++i) {
        double nup = dn[i] + small_number;
        double ndown = dn[i + (ispin - 1) * n2ft3d] + small_number;
        double n = nup + ndown;
        double rs = rs_scale / pow(n, onethird);
        double xi = (nup - ndown) / n;
        double x = sqrt(rs);
        double xxp = rs + bp * x + cp;
        double dxxp = 2.0 * x + bp;
        double ec_p = cp1 * log(rs / xxp) + cp2 * log((x + cp3) * (x + cp3) / xxp) +
                      cp4 * atan(cp5 / (x + cp6));
        double uc_p = ec_p - onesixth * x * (dp1 / x + dp2 / (x + cp3) + dp4 * dxxp / xxp +
                                             dp5 / ((x + dp6) * (x + dp6) + dp7));
        double xxf = rs + bf * x + cf;
        double dxxf = 2.0 * x + bf;
        double ec_f = cf1 * log(rs / xxf) + cf2 * log((x + cf3) * (x + cf3) / xxf) +
                      cf4 * atan(cf5 / (x + cf6));
        double uc_f = ec_f - onesixth * x * (df1 / x + df2 / (x + cf3) + df4 * dxxf / xxf +
                                             df5 / ((x + df6) * (x + df6) + df7));
        double f = (pow(1.0 + xi, fourthird) + pow(1.0 - xi, fourthird) - 2.0) / (2.0 * A);
        double df = fourthird * (pow(1.0 + xi, onethird) - pow(1.0 - xi, onethird)) / (2.0 * A);
        xce[i] += ec_p + f * (ec_f - ec_p);
        xcp[i] += uc_p + f * (uc_f - uc_p) + (+1.0 - xi) * (df * (ec_f - ec_p));
        if (ispin == 2)
            xcp[i + n2ft3d] += uc_p + f * (uc_f - uc_p) + (-1.0 - xi) * (df * (ec_f - ec_p));
    }
}

/* cpsd.c:370-371 */
void oracle_xc(int ispin, int n2ft3d, const double *dn, double *xcp, double *xce)
{
    dirac_exchange(ispin, n2ft3d, dn, xcp, xce);
    vosko(ispin, n2ft3d, dn, xcp, xce);
}

/* ---------------------------------------------------------- small helpers */

/* column-major C = alpha*A*B + beta*C, all n x n with leading dimension n */
static void small_gemm(int n, double alpha, const double *A, const double *B, double beta, double *C)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int l = 0; l < n; ++l) s += A[i + (long)l * n] * B[l + (long)j * n];
            C[i + (long)j * n] = alpha * s + (beta == 0.0 ? 0.0 : beta * C[i + (long)j * n]);
        }
}

/* Fortran idamax (1-based index of the first max |x|), cpsd.c:471 */
static int idamax1(int n, const double *x)
{
    int imax = 0;
    double m = fabs(x[0]);
    for (int i = 1; i < n; ++i)
        if (fabs(x[i]) > m) {
            m = fabs(x[i]);
            imax = i;
        }
    return imax + 1;
}

/* erfc approximation (Abramowitz & Stegun 7.1.28), cpsd.c:11-17 */
static double erfc_as(double w)
{
    const double B1 = 0.0705230784, B2 = 0.0422820123, B3 = 0.0092705272;
    const double B4 = 0.0001520143, B5 = 0.0002765672, B6 = 0.0000430638;
    double aa = 1.0 + w * (B1 + w * (B2 + w * (B3 + w * (B4 + w * (B5 + w * B6)))));
    double e = 1.0 / (aa * aa * aa * aa);
    return e * e * e * e;
}

/* -------------------------------------------------------------- the loop */

static int cpsd_impl(int inner, int move, int nion, int ispin, const int *ne,
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
                     int *lagrange_fail, const oracle_bands *bp)
{
    const double CERFC = 1.128379167;
    const int nbands = ne[0] + ne[1];
    const long nn = (long)n2ft3d * nbands;
    const double scal1 = 1.0 / ((double)nfft * nfft * nfft);
    const double scal2 = 1.0 / omega;
    const double dv = omega * scal1;
    const double dte = dt / sqrt(fmass); /* cpsd.c:114 */
    int n1[2] = {0, ne[0]}, n2[2] = {ne[0] - 1, ne[0] + ne[1] - 1};
    /* band-parallel: this rank transforms and steps bands [blo, bhi) only */
    const int blo = bp ? bp->lo : 0, bhi = bp ? bp->hi : nbands;
    if (bp && (move || blo < 0 || bhi > nbands || blo > bhi)) return -2;
    int inc2c = nfft / 2 + 1, inc3c = (nfft / 2 + 1) * nfft, inc2r = nfft + 2,
        inc3r = (nfft + 2) * nfft, naux = 0;
    int nf = nfft;
    long ne02 = (long)ne[0] * ne[0];

    /* scratch, the same pieces as cpsd.c:147-165 (the Lagrange matrices stay
     * contiguous in that order: the convergence test reads past st1) */
    double *dng = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *vall = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *vtmp = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *s = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *exi = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *xcp = (double *)calloc((size_t)ispin * n2ft3d, sizeof(double));
    double *xce = (double *)calloc((size_t)n2ft3d, sizeof(double));
    double *ex1 = (double *)calloc((size_t)nion * (nfft + 2), sizeof(double));
    double *ex2 = (double *)calloc((size_t)nion * 2 * nfft, sizeof(double));
    double *ex3 = (double *)calloc((size_t)nion * 2 * nfft, sizeof(double));
    double *lag = (double *)calloc((size_t)(7 * ne02 + 1), sizeof(double));
    double *dti = (double *)calloc((size_t)(nion > 0 ? nion : 1), sizeof(double));
    if (!dng || !vall || !vtmp || !s || !exi || !xcp || !xce || !ex1 || !ex2 || !ex3 || !lag || !dti) {
        free(dng); free(vall); free(vtmp); free(s); free(exi); free(xcp); free(xce);
        free(ex1); free(ex2); free(ex3); free(lag); free(dti);
        return -1;
    }
    double *s11 = lag, *s12 = lag + ne02, *s21 = lag + 2 * ne02, *s22 = lag + 3 * ne02;
    double *st1 = lag + 4 * ne02, *sa1 = lag + 5 * ne02, *sa0 = lag + 6 * ne02;
    if (move)
        for (int ii = 0; ii < nion; ++ii) dti[ii] = dt / sqrt(amass[katm[ii]]); /* cpsd.c:116-122 */
    if (lagrange_fail) *lagrange_fail = 0;

    for (int itime = 0; itime < inner; ++itime) {
        /* cpsd.c:173-174 */
        memcpy(c1, c2, sizeof(double) * (size_t)nn);
        memcpy(r1, r2, sizeof(double) * 3 * (size_t)nion);

        /* psi(G) -> psi(r), cpsd.c:177-181 */
        memcpy(cpsi, c1, sizeof(double) * (size_t)nn);
        for (int i = blo; i < bhi; ++i)
            cr_fft3b_(cpsi + (long)i * n2ft3d, &inc2c, &inc3c, &inc2r, &inc3r, &nf, &nf, &nf, NULL, &naux);

        /* spin densities, cpsd.c:185-194 */
        memset(dn, 0, sizeof(double) * (size_t)ispin * n2ft3d);
        for (int ms = 0; ms < ispin; ++ms) {
            double *d = dn + (long)ms * n2ft3d;
            for (int i = n1[ms]; i <= n2[ms]; ++i) {
                if (i < blo || i >= bhi) continue;
                const double *p = cpsi + (long)i * n2ft3d;
                for (long k = 0; k < n2ft3d; ++k) d[k] += scal2 * (p[k] * p[k]);
            }
            for (long l = 0; l < (long)nfft * nfft; ++l) {
                d[l * inc2r + nfft] = 0.0;
                d[l * inc2r + nfft + 1] = 0.0;
            }
        }
        /* band-parallel: the spin densities summed over the ranks */
        if (bp) bp->allreduce_sum(dn, (long)ispin * n2ft3d, bp->user);

        /* rho(G), cpsd.c:198-205 */
        for (long k = 0; k < n2ft3d; ++k) dng[k] = (dn[k] + dn[k + (long)(ispin - 1) * n2ft3d]) * scal1;
        rc_fft3f_(dng, &inc2c, &inc3c, &inc2r, &inc3r, &nf, &nf, &nf, NULL, &naux);
        for (long k = 0; k < n2ft3d; ++k) dng[k] *= masker[k];

        /* ionic phase factors, cpsd.c:208 */
        oracle_phafac(nfft, unitg, nion, r1, ex1, ex2, ex3);

        /* kinetic, cpsd.c:212-221 */
        for (int i = blo; i < bhi; ++i) {
            const double *a = c1 + (long)i * n2ft3d;
            double *b = c2 + (long)i * n2ft3d;
            for (long k = 0; k < nfft3d; ++k) {
                b[2 * k] = -tg[k] * a[2 * k];
                b[2 * k + 1] = -tg[k] * a[2 * k + 1];
            }
        }

        /* local and nonlocal pseudopotentials, cpsd.c:224-307 */
        memset(s, 0, sizeof(double) * (size_t)n2ft3d);
        memset(vall, 0, sizeof(double) * (size_t)n2ft3d);
        for (int ii = 0; ii < nion; ++ii) {
            int ia = katm[ii];
            oracle_strfac(nfft, ex1 + (long)ii * (nfft + 2), ex2 + (long)ii * 2 * nfft,
                          ex3 + (long)ii * 2 * nfft, exi);
            for (long k = 0; k < n2ft3d; ++k) exi[k] *= masker[k];
            for (long k = 0; k < n2ft3d; ++k) s[k] += zv[ia] * exi[k];
            const double *rex = vl + (long)ia * nfft3d;
            for (long k = 0; k < nfft3d; ++k) {
                vtmp[2 * k] = exi[2 * k] * rex[k];
                vtmp[2 * k + 1] = exi[2 * k + 1] * rex[k];
                vall[2 * k] += vtmp[2 * k];
                vall[2 * k + 1] += vtmp[2 * k + 1];
            }
            if (move) { /* local force, cpsd.c:246-257 */
                for (long k = 0; k < nfft3d; ++k)
                    xce[k] = dng[2 * k + 1] * vtmp[2 * k] - dng[2 * k] * vtmp[2 * k + 1];
                for (int d = 0; d < 3; ++d) fion[3 * ii + d] = oracle_gsdot(nfft, G + (long)d * nfft3d, xce);
            }
            for (int l = 0; l < lmmax[ia]; ++l) {
                const double *w = vnl + (long)ia * 9 * nfft3d + (long)l * nfft3d;
                if (l == 0 || l >= 4) { /* s or d: cpsd.c:265-274 */
                    for (long k = 0; k < nfft3d; ++k) {
                        vtmp[2 * k] = exi[2 * k] * w[k];
                        vtmp[2 * k + 1] = exi[2 * k + 1] * w[k];
                    }
                } else { /* p: multiplied by i, cpsd.c:277-286 */
                    for (long k = 0; k < nfft3d; ++k) {
                        vtmp[2 * k] = -exi[2 * k + 1] * w[k];
                        vtmp[2 * k + 1] = exi[2 * k] * w[k];
                    }
                }
                for (int i = blo; i < bhi; ++i) { /* cpsd.c:287-305 */
                    const double *a = c1 + (long)i * n2ft3d;
                    double *b = c2 + (long)i * n2ft3d;
                    double sw1 = -oracle_gcdotc(nfft, vtmp, a) * scal2 / vnlnrm[ia * 9 + l];
                    for (long k = 0; k < n2ft3d; ++k) b[k] += sw1 * vtmp[k];
                    if (move) {
                        for (long k = 0; k < nfft3d; ++k)
                            xce[k] = a[2 * k + 1] * vtmp[2 * k] - a[2 * k] * vtmp[2 * k + 1];
                        if (ispin == 1) sw1 *= 2;
                        for (int d = 0; d < 3; ++d)
                            fion[3 * ii + d] -= 2 * sw1 * oracle_gsdot(nfft, G + (long)d * nfft3d, xce);
                    }
                }
            }
        }

        /* Ewald forces, cpsd.c:310-364 */
        if (move) {
            for (int ii = 0; ii < nion; ++ii) {
                int ia = katm[ii];
                oracle_strfac(nfft, ex1 + (long)ii * (nfft + 2), ex2 + (long)ii * 2 * nfft,
                              ex3 + (long)ii * 2 * nfft, exi);
                for (long k = 0; k < n2ft3d; ++k) exi[k] *= masker[k];
                for (long k = 0; k < nfft3d; ++k)
                    vtmp[k] = (exi[2 * k] * s[2 * k + 1] - exi[2 * k + 1] * s[2 * k]) * vg[k];
                for (int d = 0; d < 3; ++d)
                    fion[3 * ii + d] += oracle_gsdot(nfft, G + (long)d * nfft3d, vtmp) * zv[ia] * scal2;
                for (int jj = ii + 1; jj < nion; ++jj) {
                    double dx = r1[3 * ii] - r1[3 * jj];
                    double dy = r1[3 * ii + 1] - r1[3 * jj + 1];
                    double dz = r1[3 * ii + 2] - r1[3 * jj + 2];
                    double zz = zv[katm[ii]] * zv[katm[jj]];
                    double sw1 = 0.0, sw2 = 0.0, sw3 = 0.0;
                    for (int l = 0; l < nsh; ++l) {
                        double x = rcell[l] + dx, y = rcell[l + nsh] + dy, z = rcell[l + 2 * nsh] + dz;
                        double r = sqrt(x * x + y * y + z * z);
                        double w = r / rcut;
                        double adiff = zz * (erfc_as(w) + CERFC * w * exp(-w * w)) / (r * r * r);
                        sw1 += x * adiff;
                        sw2 += y * adiff;
                        sw3 += z * adiff;
                    }
                    fion[3 * ii] += sw1;
                    fion[3 * ii + 1] += sw2;
                    fion[3 * ii + 2] += sw3;
                    fion[3 * jj] -= sw1;
                    fion[3 * jj + 1] -= sw2;
                    fion[3 * jj + 2] -= sw3;
                }
            }
        }

        /* xc potential, cpsd.c:370-371 */
        oracle_xc(ispin, n2ft3d, dn, xcp, xce);

        /* local + Hartree potential to real space, cpsd.c:373-382 */
        for (long k = 0; k < nfft3d; ++k) {
            vtmp[2 * k] = vall[2 * k] * scal2 + dng[2 * k] * vc[k];
            vtmp[2 * k + 1] = vall[2 * k + 1] * scal2 + dng[2 * k + 1] * vc[k];
        }
        cr_fft3b_(vtmp, &inc2c, &inc3c, &inc2r, &inc3r, &nf, &nf, &nf, NULL, &naux);

        /* V psi back to G and -H psi, cpsd.c:384-396 */
        for (int ms = 0; ms < ispin; ++ms)
            for (int i = n1[ms]; i <= n2[ms]; ++i) {
                if (i < blo || i >= bhi) continue;
                double *p = cpsi + (long)i * n2ft3d;
                const double *x = xcp + (long)ms * n2ft3d;
                for (long k = 0; k < n2ft3d; ++k) p[k] *= (vtmp[k] + x[k]);
                rc_fft3f_(p, &inc2c, &inc3c, &inc2r, &inc3r, &nf, &nf, &nf, NULL, &naux);
                const double *b = c2 + (long)i * n2ft3d;
                for (long k = 0; k < n2ft3d; ++k) p[k] = -scal1 * p[k] * masker[k] + b[k];
            }

        /* steepest descent, cpsd.c:399-411 */
        for (long k = (long)blo * n2ft3d; k < (long)bhi * n2ft3d; ++k) c2[k] = c1[k] + dte * cpsi[k];
        /* band-parallel: every rank's new orbitals (and -H psi) to every rank */
        if (bp) {
            bp->allgather_rows(c2, n2ft3d, bp->user);
            bp->allgather_rows(cpsi, n2ft3d, bp->user);
        }
        if (move)
            for (int ii = 0; ii < nion; ++ii)
                for (int d = 0; d < 3; ++d) r2[3 * ii + d] = r1[3 * ii + d] + dti[ii] * fion[3 * ii + d];

        /* Lagrange multipliers, cpsd.c:415-479 */
        for (int ms = 0; ms < ispin; ++ms) {
            int m = ne[ms];
            long kk = (long)m * m;
            const double *C1 = c1 + (long)ms * ne[0] * n2ft3d;
            const double *C2 = c2 + (long)ms * ne[0] * n2ft3d;
            for (int i = 0; i < m; ++i) {
                const double *c1i = C1 + (long)i * n2ft3d, *c2i = C2 + (long)i * n2ft3d;
                s22[i + i * m] = (1.0 - oracle_gcdotc(nfft, c2i, c2i)) * 0.5 / dte;
                s21[i + i * m] = (1.0 - oracle_gcdotc(nfft, c2i, c1i)) * 0.5;
                s12[i + i * m] = s21[i + i * m];
                s11[i + i * m] = -oracle_gcdotc(nfft, c1i, c1i) * 0.5 * dte;
                for (int j = i + 1; j < m; ++j) {
                    const double *c1j = C1 + (long)j * n2ft3d, *c2j = C2 + (long)j * n2ft3d;
                    s22[i + j * m] = -oracle_gcdotc(nfft, c2i, c2j) * 0.5 / dte;
                    s21[i + j * m] = -oracle_gcdotc(nfft, c2i, c1j) * 0.5;
                    s12[i + j * m] = -oracle_gcdotc(nfft, c1i, c2j) * 0.5;
                    s11[i + j * m] = -oracle_gcdotc(nfft, c1i, c1j) * 0.5 * dte;
                    s22[j + i * m] = s22[i + j * m];
                    s21[j + i * m] = s21[i + j * m];
                    s12[j + i * m] = s12[i + j * m];
                    s11[j + i * m] = s11[i + j * m];
                }
            }
            int iter = 0, done = 0;
            double adiff = 0.0;
            memcpy(sa0, s22, sizeof(double) * (size_t)kk);
            while (!done && (iter++) < 30) {
                memcpy(sa1, s22, sizeof(double) * (size_t)kk);
                small_gemm(m, 1.0, s21, sa0, 1.0, sa1);
                small_gemm(m, 1.0, sa0, s12, 1.0, sa1);
                small_gemm(m, 1.0, s11, sa0, 0.0, st1);
                small_gemm(m, 1.0, sa0, st1, 1.0, sa1);
                for (long k = 0; k < kk; ++k) st1[k] = sa1[k] - sa0[k];
                /* the reference indexes st1 with idamax's 1-based result
                 * (cpsd.c:471), i.e. the element after the largest one */
                adiff = fabs(st1[idamax1((int)kk, st1)]);
                if (adiff < 1e-15)
                    done = 1;
                else
                    memcpy(sa0, sa1, sizeof(double) * (size_t)kk);
            }
            if (!done && lagrange_fail) ++*lagrange_fail;
            memcpy(lmd + (long)ms * ne02, sa1, sizeof(double) * (size_t)kk);
        }

        /* constraint correction c2 += dte * C1 * lmd, cpsd.c:482-488 */
        for (int ms = 0; ms < ispin; ++ms) {
            int m = ne[ms];
            const double *C1 = c1 + (long)ms * ne[0] * n2ft3d;
            double *C2 = c2 + (long)ms * ne[0] * n2ft3d;
            const double *X = lmd + (long)ms * ne02;
            for (int j = 0; j < m; ++j)
                for (long k = 0; k < n2ft3d; ++k) {
                    double acc = 0.0;
                    for (int l = 0; l < m; ++l) acc += C1[k + (long)l * n2ft3d] * X[l + (long)j * m];
                    C2[k + (long)j * n2ft3d] += dte * acc;
                }
        }
    }

    /* ---- energies on c1 and cpsi of the last step, cpsd.c:494-646 ---- */
    double eorbit = 0.0;
    for (int ms = 0; ms < ispin; ++ms) {
        int m = ne[ms];
        const double *C1 = c1 + (long)ms * ne[0] * n2ft3d;
        const double *CP = cpsi + (long)ms * ne[0] * n2ft3d;
        double *H = hml + (long)ms * ne02;
        for (int i = 0; i < m; ++i) {
            H[i + i * m] = -oracle_gcdotc(nfft, C1 + (long)i * n2ft3d, CP + (long)i * n2ft3d);
            eorbit += hml[i + i * m]; /* cpsd.c:507 reads hml, not qex */
            for (int j = i + 1; j < m; ++j) {
                H[i + j * m] = -oracle_gcdotc(nfft, C1 + (long)i * n2ft3d, CP + (long)j * n2ft3d);
                H[j + i * m] = hml[i + j * m]; /* cpsd.c:511 reads hml, not qex */
            }
        }
    }
    if (ispin == 1) eorbit *= 2;

    /* Ewald, cpsd.c:520-545 */
    for (long k = 0; k < nfft3d; ++k) vtmp[k] = (s[2 * k] * s[2 * k] + s[2 * k + 1] * s[2 * k + 1]) * vg[k];
    double eion = oracle_gssum(nfft, vtmp) * 0.5 * scal2 + cewald;
    for (int ii = 0; ii < nion; ++ii)
        for (int jj = ii + 1; jj < nion; ++jj) {
            double dx = r1[3 * ii] - r1[3 * jj];
            double dy = r1[1 + 3 * ii] - r1[1 + 3 * jj];
            double dz = r1[2 + 3 * ii] - r1[2 + 3 * jj];
            double zz = zv[katm[ii]] * zv[katm[jj]];
            for (int l = 0; l < nsh; ++l) {
                double x = rcell[l] + dx, y = rcell[l + nsh] + dy, z = rcell[l + 2 * nsh] + dz;
                double r = sqrt(x * x + y * y + z * z);
                eion += zz * erfc_as(r / rcut) / r;
            }
        }

    /* Hartree, cpsd.c:548-554 */
    for (long k = 0; k < nfft3d; ++k)
        vtmp[k] = (dng[2 * k] * dng[2 * k] + dng[2 * k + 1] * dng[2 * k + 1]) * vc[k];
    double ehartr = oracle_gssum(nfft, vtmp) * omega * 0.5;

    /* xc, cpsd.c:557-570 */
    double exc = dot_strided(n2ft3d, dn, 1, xce, 1);
    double pxc = dot_strided(n2ft3d, dn, 1, xcp, 1);
    if (ispin == 1) {
        exc += exc;
        pxc += pxc;
    } else {
        exc += dot_strided(n2ft3d, dn + n2ft3d, 1, xce, 1);
        pxc += dot_strided(n2ft3d, dn + n2ft3d, 1, xcp + n2ft3d, 1);
    }
    exc *= dv;
    pxc *= dv;

    /* kinetic, cpsd.c:574-587 */
    double eke = 0.0;
    for (int i = 0; i < nbands; ++i) {
        const double *a = c1 + (long)i * n2ft3d;
        for (long k = 0; k < nfft3d; ++k) {
            vtmp[2 * k] = a[2 * k] * tg[k];
            vtmp[2 * k + 1] = a[2 * k + 1] * tg[k];
        }
        eke += oracle_gcdotc(nfft, a, vtmp);
    }
    if (ispin == 1) eke = 2 * eke;

    /* local, cpsd.c:590 */
    double elocal = oracle_gcdotc(nfft, vall, dng);

    /* nonlocal, cpsd.c:593-634 */
    double enlocal = 0.0;
    for (int ii = 0; ii < nion; ++ii) {
        int ia = katm[ii];
        oracle_strfac(nfft, ex1 + (long)ii * (nfft + 2), ex2 + (long)ii * 2 * nfft,
                      ex3 + (long)ii * 2 * nfft, exi);
        for (long k = 0; k < n2ft3d; ++k) exi[k] *= masker[k];
        for (int l = 0; l < lmmax[ia]; ++l) {
            const double *w = vnl + (long)ia * 9 * nfft3d + (long)l * nfft3d;
            if (l == 0 || l >= 4) {
                for (long k = 0; k < nfft3d; ++k) {
                    vtmp[2 * k] = exi[2 * k] * w[k];
                    vtmp[2 * k + 1] = exi[2 * k + 1] * w[k];
                }
            } else {
                for (long k = 0; k < nfft3d; ++k) {
                    vtmp[2 * k] = -exi[2 * k + 1] * w[k];
                    vtmp[2 * k + 1] = exi[2 * k] * w[k];
                }
            }
            for (int i = 0; i < nbands; ++i) {
                double sw1 = oracle_gcdotc(nfft, vtmp, c1 + (long)i * n2ft3d);
                enlocal += sw1 * sw1 * scal2 / vnlnrm[ia * 9 + l];
            }
        }
    }
    if (ispin == 1) enlocal = 2 * enlocal;

    /* cpsd.c:637-647 */
    double eold = E[0];
    E[0] = eorbit + eion + exc - ehartr - pxc;
    E[1] = eorbit;
    E[2] = ehartr;
    E[3] = exc;
    E[4] = eion;
    E[5] = eke;
    E[6] = elocal;
    E[7] = enlocal;
    E[8] = 2.0 * ehartr;
    E[9] = pxc;

    /* convergence measures, cpsd.c:649-672 (cpsi leaves holding c2 - c1) */
    *deltae = (E[0] - eold) / (dt * inner);
    for (long k = 0; k < nn; ++k) cpsi[k] = c2[k] - c1[k];
    *deltac = 0.0;
    for (int i = 0; i < nbands; ++i) {
        double a = oracle_gcdotc(nfft, cpsi + (long)i * n2ft3d, cpsi + (long)i * n2ft3d);
        if (a > *deltac) *deltac = a;
    }
    *deltac /= dte;
    *deltar = 0.0;
    if (move)
        for (int ii = 0; ii < nion; ++ii) {
            double a = sqrt(fion[3 * ii] * fion[3 * ii] + fion[3 * ii + 1] * fion[3 * ii + 1] +
                            fion[3 * ii + 2] * fion[3 * ii + 2]);
            if (a > *deltar) *deltar = a;
        }

    free(dng); free(vall); free(vtmp); free(s); free(exi); free(xcp); free(xce);
    free(ex1); free(ex2); free(ex3); free(lag); free(dti);
    return 0;
}

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
                int *lagrange_fail)
{
    return cpsd_impl(inner, move, nion, ispin, ne, nfft, nfft3d, n2ft3d, unitg, omega, dt, fmass, katm, amass,
                     zv, nsh, rcell, cewald, rcut, masker, G, tg, vc, vg, lmmax, vnlnrm, vl, vnl, r1, r2, fion,
                     c1, c2, cpsi, dn, hml, lmd, E, deltae, deltac, deltar, lagrange_fail, NULL);
}

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
                      int *lagrange_fail, const oracle_bands *bp)
{
    if (!bp || !bp->allreduce_sum || !bp->allgather_rows) return -2;
    return cpsd_impl(inner, 0, nion, ispin, ne, nfft, nfft3d, n2ft3d, unitg, omega, dt, fmass, katm, amass,
                     zv, nsh, rcell, cewald, rcut, masker, G, tg, vc, vg, lmmax, vnlnrm, vl, vnl, r1, r2, fion,
                     c1, c2, cpsi, dn, hml, lmd, E, deltae, deltac, deltar, lagrange_fail, bp);
}
