/*
 * fft3d.c -- ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing on the product path
 * links, loads or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg use it, as the oracle.
 *
 * C restatement of the reference's 3-D FFT wrapper and of the 1-D FFTPACK
 * transforms underneath it.  The reference's versions are Fortran 77 and no
 * Fortran compiler exists here, so this is the only non-reference code in the
 * reference build under oracle/_ref (it provides cr_fft3b_ / rc_fft3f_ there).
 *
 *   cr_fft3b_  <- fftpack3d/fftpack3d.f:22-96   (complex -> real, inverse)
 *   rc_fft3f_  <- fftpack3d/fftpack3d.f:107-196 (real -> complex, forward)
 *
 * 1-D semantics follow netlib FFTPACK (fftpack/fftdoc, dcfftb.f, dcfftf.f,
 * drfftb.f, drfftf.f): complex backward = sum_k c_k e^{+2 pi i jk/n}, complex
 * forward = sum_j c_j e^{-2 pi i jk/n}, real forward/backward in the
 * (r0, re1, im1, ..., r_{n/2}) half-complex format, all unnormalised.  The
 * arithmetic is a mixed-radix Cooley-Tukey recursion (radices 2,3,4,5 and a
 * generic odd radix); results differ from FFTPACK's only by rounding.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* twiddle table W[j] = exp(sign * 2 pi i j / n), j < n, interleaved re/im */
static void make_twiddles(int n, int sign, double *w)
{
    for (int j = 0; j < n; ++j) {
        /* reduce the angle exactly: j/n in [0,1) */
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)j / (long double)n;
        w[2 * j] = (double)cosl(a);
        w[2 * j + 1] = (double)(sign * sinl(a));
    }
}

static int smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/*
 * Out-of-place recursive DFT: y[k] = sum_j x[j*xs] W_n^{jk}, k < n, where
 * W_n^m = W[(m * wstep) mod nfull] and W is the table for length nfull.
 * x and y are complex interleaved; xs is the input stride in complex units.
 */
static void cdft_rec(int n, const double *x, int xs, double *y,
                     const double *W, int nfull, int wstep)
{
    if (n == 1) {
        y[0] = x[0];
        y[1] = x[1];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    for (int r = 0; r < p; ++r)
        cdft_rec(m, x + 2 * r * xs, xs * p, y + 2 * r * m, W, nfull, wstep * p);
    /* combine: X[k + m q] = sum_r W_n^{r (k + m q)} Y_r[k] */
    double tre[64], tim[64];
    double *bre = tre, *bim = tim;
    double *heap = NULL;
    if (p > 64) {
        heap = (double *)malloc(sizeof(double) * 2 * (size_t)p);
        bre = heap;
        bim = heap + p;
    }
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) {
            int widx = (int)(((long)r * k * wstep) % nfull);
            double wr = W[2 * widx], wi = W[2 * widx + 1];
            double yr = y[2 * (r * m + k)], yi = y[2 * (r * m + k) + 1];
            bre[r] = yr * wr - yi * wi;
            bim[r] = yr * wi + yi * wr;
        }
        if (p == 2) {
            y[2 * k] = bre[0] + bre[1];
            y[2 * k + 1] = bim[0] + bim[1];
            y[2 * (k + m)] = bre[0] - bre[1];
            y[2 * (k + m) + 1] = bim[0] - bim[1];
        } else if (p == 4) {
            /* W_4 = W_n^{n/4}: +-i depending on the table's sign */
            int w1 = (int)(((long)m * wstep) % nfull);
            double s = W[2 * w1 + 1]; /* +1 or -1: imaginary part of W_4 */
            double a0r = bre[0] + bre[2], a0i = bim[0] + bim[2];
            double a1r = bre[0] - bre[2], a1i = bim[0] - bim[2];
            double a2r = bre[1] + bre[3], a2i = bim[1] + bim[3];
            double a3r = bre[1] - bre[3], a3i = bim[1] - bim[3];
            /* i*s*(a3) */
            double b3r = -s * a3i, b3i = s * a3r;
            y[2 * k] = a0r + a2r;
            y[2 * k + 1] = a0i + a2i;
            y[2 * (k + m)] = a1r + b3r;
            y[2 * (k + m) + 1] = a1i + b3i;
            y[2 * (k + 2 * m)] = a0r - a2r;
            y[2 * (k + 2 * m) + 1] = a0i - a2i;
            y[2 * (k + 3 * m)] = a1r - b3r;
            y[2 * (k + 3 * m) + 1] = a1i - b3i;
        } else {
            for (int q = 0; q < p; ++q) {
                double sr = 0.0, si = 0.0;
                for (int r = 0; r < p; ++r) {
                    int widx = (int)(((long)((r * q) % p) * m * wstep) % nfull);
                    double wr = W[2 * widx], wi = W[2 * widx + 1];
                    sr += bre[r] * wr - bim[r] * wi;
                    si += bre[r] * wi + bim[r] * wr;
                }
                y[2 * (k + m * q)] = sr;
                y[2 * (k + m * q) + 1] = si;
            }
        }
    }
    free(heap);
}

/* complex 1-D transform of a contiguous line, in place, with the twiddle
 * table W of its length and direction (made once per pass, as the wrapper
 * calls dcffti once per pass: fftpack3d.f:50,66,170,185) */
static void cfft1d(int n, double *line, double *work, const double *W)
{
    memcpy(work, line, sizeof(double) * 2 * (size_t)n);
    cdft_rec(n, work, 1, line, W, n, 1);
}

/*
 * Real forward transform (drfftf semantics, n even): x[0..n-1] ->
 * X[k] = sum_j x_j e^{-2 pi i jk/n}, k = 0..n/2, written as n/2+1 complex
 * values into out (2*(n/2+1) doubles).  Uses the half-length complex packing
 * z_j = x_{2j} + i x_{2j+1}.
 */
static void rfft_fwd(int n, const double *x, double *out, double *work,
                     const double *W, const double *Wn)
{
    int h = n / 2;
    double *z = work;          /* h complex */
    double *Z = work + 2 * h;  /* h complex */
    for (int j = 0; j < h; ++j) {
        z[2 * j] = x[2 * j];
        z[2 * j + 1] = x[2 * j + 1];
    }
    cdft_rec(h, z, 1, Z, W, h, 1);
    for (int k = 0; k <= h; ++k) {
        int kk = k % h;
        int km = (h - k) % h;
        double zr = Z[2 * kk], zi = Z[2 * kk + 1];
        double cr = Z[2 * km], ci = -Z[2 * km + 1]; /* conj(Z_{h-k}) */
        double er = 0.5 * (zr + cr), ei = 0.5 * (zi + ci);
        /* O = (Z - conj)/(2i) = -i (Z - conj)/2 */
        double dr = 0.5 * (zr - cr), di = 0.5 * (zi - ci);
        double or_ = di, oi = -dr;
        int wi_ = k % n;
        double wr = Wn[2 * wi_], wim = Wn[2 * wi_ + 1];
        double tr = wr * or_ - wim * oi, ti = wr * oi + wim * or_;
        out[2 * k] = er + tr;
        out[2 * k + 1] = ei + ti;
    }
    out[1] = 0.0;          /* rc_fft3f: tmp(2) = 0 (fftpack3d.f:160) */
    out[2 * h + 1] = 0.0;  /* rc_fft3f: tmp(nx+2) = 0 (fftpack3d.f:161) */
}

/*
 * Real backward transform (drfftb semantics, n even): X[0..n/2] (complex,
 * the imaginary parts of X_0 and X_{n/2} are ignored) ->
 * x_j = sum_{k<n} X_k e^{+2 pi i jk/n} with X_{n-k} = conj(X_k).
 */
static void rfft_bwd(int n, const double *X, double *x, double *work,
                     const double *W, const double *Wn)
{
    int h = n / 2;
    double *Z = work;
    double *z = work + 2 * h;
    /* Wn holds e^{+2 pi i k/n} = W^{-k} */
    for (int k = 0; k < h; ++k) {
        double xr = X[2 * k], xi = X[2 * k + 1];
        double yr = X[2 * (h - k)], yi = -X[2 * (h - k) + 1]; /* conj(X_{h-k}) = X_{k+h} */
        if (k == 0) {
            xi = 0.0;
            yi = 0.0;
        }
        double er = xr + yr, ei = xi + yi;
        double dr = xr - yr, di = xi - yi;
        double wr = Wn[2 * k], wim = Wn[2 * k + 1];
        double or_ = dr * wr - di * wim, oi = dr * wim + di * wr;
        /* Z = E + i O */
        Z[2 * k] = er - oi;
        Z[2 * k + 1] = ei + or_;
    }
    cdft_rec(h, Z, 1, z, W, h, 1);
    for (int j = 0; j < h; ++j) {
        x[2 * j] = z[2 * j];
        x[2 * j + 1] = z[2 * j + 1];
    }
}

/* zcopy-style strided gather/scatter of complex values (stride in complex units) */
static void zgather(int n, const double *a, int inc, double *line)
{
    for (int j = 0; j < n; ++j) {
        line[2 * j] = a[2 * (size_t)j * inc];
        line[2 * j + 1] = a[2 * (size_t)j * inc + 1];
    }
}
static void zscatter(int n, const double *line, double *a, int inc)
{
    for (int j = 0; j < n; ++j) {
        a[2 * (size_t)j * inc] = line[2 * j];
        a[2 * (size_t)j * inc + 1] = line[2 * j + 1];
    }
}

struct fftws {
    double *line, *work, *W, *Wn, *out;
};
static int ws_alloc(struct fftws *w, int nmax)
{
    w->out = (double *)malloc(sizeof(double) * (size_t)(2 * nmax + 4));
    w->line = (double *)malloc(sizeof(double) * (size_t)(2 * nmax + 4));
    w->work = (double *)malloc(sizeof(double) * (size_t)(4 * nmax + 8));
    w->W = (double *)malloc(sizeof(double) * (size_t)(2 * nmax + 4));
    w->Wn = (double *)malloc(sizeof(double) * (size_t)(2 * nmax + 4));
    return w->out && w->line && w->work && w->W && w->Wn;
}
static void ws_free(struct fftws *w)
{
    free(w->out);
    free(w->line);
    free(w->work);
    free(w->W);
    free(w->Wn);
}

/*
 * cr_fft3b: A(kx,ky,kz) -> A(x,y,z), fftpack3d.f:22-96.  Fortran ABI (all by
 * reference).  tmp/ntmp is the caller's scratch; this restatement allocates
 * its own and leaves tmp untouched.
 */
void cr_fft3b_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r,
               int *nx, int *ny, int *nz, double *tmp, int *ntmp)
{
    (void)tmp;
    (void)ntmp;
    int NX = *nx, NY = *ny, NZ = *nz;
    int i2c = *inc2c, i3c = *inc3c, i2r = *inc2r, i3r = *inc3r;
    int nmax = NX > NY ? NX : NY;
    if (NZ > nmax) nmax = NZ;
    struct fftws w;
    if (!ws_alloc(&w, nmax + 2)) {
        ws_free(&w);
        return;
    }
    /* kz lines: fftpack3d.f:50-58 */
    make_twiddles(NZ, +1, w.W);
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX / 2 + 1; ++i) {
            double *a = A + 2 * i + (size_t)j * i2r;
            zgather(NZ, a, i3c, w.line);
            cfft1d(NZ, w.line, w.work, w.W);
            zscatter(NZ, w.line, a, i3c);
        }
    /* ky lines: fftpack3d.f:66-74 */
    make_twiddles(NY, +1, w.W);
    for (int k = 0; k < NZ; ++k)
        for (int i = 0; i < NX / 2 + 1; ++i) {
            double *a = A + 2 * i + (size_t)k * i3r;
            zgather(NY, a, i2c, w.line);
            cfft1d(NY, w.line, w.work, w.W);
            zscatter(NY, w.line, a, i2c);
        }
    /* kx lines, complex -> real: fftpack3d.f:81-94 */
    make_twiddles(NX / 2, +1, w.W);
    make_twiddles(NX, +1, w.Wn);
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j) {
            double *a = A + (size_t)j * i2r + (size_t)k * i3r;
            memcpy(w.line, a, sizeof(double) * (size_t)(NX + 2));
            rfft_bwd(NX, w.line, w.out, w.work, w.W, w.Wn);
            memcpy(a, w.out, sizeof(double) * (size_t)NX);
            a[NX] = 0.0;     /* fftpack3d.f:90 */
            a[NX + 1] = 0.0; /* fftpack3d.f:91 */
        }
    ws_free(&w);
}

/* rc_fft3f: A(x,y,z) -> A(kx,ky,kz), fftpack3d.f:107-196 */
void rc_fft3f_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r,
               int *nx, int *ny, int *nz, double *tmp, int *ntmp)
{
    (void)tmp;
    (void)ntmp;
    int NX = *nx, NY = *ny, NZ = *nz;
    int i2c = *inc2c, i3c = *inc3c, i2r = *inc2r, i3r = *inc3r;
    int nmax = NX > NY ? NX : NY;
    if (NZ > nmax) nmax = NZ;
    struct fftws w;
    if (!ws_alloc(&w, nmax + 2)) {
        ws_free(&w);
        return;
    }
    /* x lines, real -> complex with Im(kx=0)=Im(kx=n/2)=0: fftpack3d.f:151-164 */
    make_twiddles(NX / 2, -1, w.W);
    make_twiddles(NX, -1, w.Wn);
    for (int k = 0; k < NZ; ++k)
        for (int j = 0; j < NY; ++j) {
            double *a = A + (size_t)j * i2r + (size_t)k * i3r;
            rfft_fwd(NX, a, w.out, w.work, w.W, w.Wn);
            memcpy(a, w.out, sizeof(double) * (size_t)(NX + 2));
        }
    /* ky lines, forward: fftpack3d.f:170-178 */
    make_twiddles(NY, -1, w.W);
    for (int k = 0; k < NZ; ++k)
        for (int i = 0; i < NX / 2 + 1; ++i) {
            double *a = A + 2 * i + (size_t)k * i3r;
            zgather(NY, a, i2c, w.line);
            cfft1d(NY, w.line, w.work, w.W);
            zscatter(NY, w.line, a, i2c);
        }
    /* kz lines, forward: fftpack3d.f:185-193 */
    make_twiddles(NZ, -1, w.W);
    for (int j = 0; j < NY; ++j)
        for (int i = 0; i < NX / 2 + 1; ++i) {
            double *a = A + 2 * i + (size_t)j * i2r;
            zgather(NZ, a, i3c, w.line);
            cfft1d(NZ, w.line, w.work, w.W);
            zscatter(NZ, w.line, a, i3c);
        }
    ws_free(&w);
}
