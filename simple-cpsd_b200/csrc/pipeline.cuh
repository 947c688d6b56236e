// pipeline.cuh -- the input pipeline's device work: Kleinman-Bylander
// pseudopotential tables on the half-box G grid from tabulated radial data
// (ckbppv3/dkbppv3.c, kbpp()).
//
// For every G != 0, with q = |G|, x_i = q rho_i and simp() =
// h/3 (2 sum_even f + 4 sum_odd f - f_0 - f_{n-1}) (dkbppv3.c simp):
//   s      f_i = sin(x) wp_0 vp_0                          vnl_0    = sqrt(4 pi) S / q
//   p      f_i = (sin(x)/x - cos(x)) wp_1 vp_1, f_0 = 0      vnl_1..3 = sqrt(12 pi) S / q * (gx, gy, gz)/q
//   d      f_i = (3 (sin(x)/x - cos(x))/x - sin(x)) wp_2 vp_2, f_0 = 0
//                                                           vnl_4..8 = sqrt(60 pi) S / q * the five real d harmonics
//   local  f_i = rho_i vp_lmax sin(x)                       vl = 4 pi S / q - 4 pi zv cos(q rho_{n-1}) / q^2
// vp_l (l < lmax) is already vp_l - vp_lmax, as kbpp() makes it first.
// G = 0: vl = 4 pi simp(vp_lmax rho^2) + 2 pi zv rho_{n-1}^2, vnl_0 =
// sqrt(4 pi) simp(rho wp_0 vp_0), the other channels 0.
//
// One thread per G point; the radial tables sit in shared memory and all
// lanes read the same entry at once (broadcast).  Even and odd terms are
// summed apart and combined as simp() combines them.
#pragma once

#include "common.cuh"

constexpr int kKbppThreads = 128;
constexpr int kKbppMaxRho = 4095;  // radial points held in shared memory (6 tables, <= 192 KB)

struct KbppArgs {
    int nfft3d, nrho, lmax;
    double drho, zv;
    const double *rho;  // [nrho]
    const double *vp;   // [(lmax+1) * nrho], nonlocal channels already minus the local one
    const double *wp;   // [(lmax+1) * nrho]
    const double *G;    // [3 * nfft3d]
    double *vl;         // [nfft3d]
    double *vnl;        // [lmax^2 * nfft3d]
};

// simp() of ckbppv3/dkbppv3.c on one table (a thread's sequential sum)
CPSD_D double kb_simp(int n, const double *f, double h)
{
    double s2 = 0.0, s4 = 0.0;
    for (int i = 0; i < n; i += 2) s2 += f[i];
    for (int i = 1; i < n; i += 2) s4 += f[i];
    return (2.0 * s2 + 4.0 * s4 - f[0] - f[n - 1]) * (h / 3.0);
}

__global__ void __launch_bounds__(kKbppThreads) kbpp_kernel(KbppArgs a)
{
    extern __shared__ double kb_sm[];
    const int n = a.nrho, lmax = a.lmax;
    double *r = kb_sm;         // rho
    double *wv0 = r + n;       // wp_0 vp_0
    double *wv1 = wv0 + n;     // wp_1 vp_1
    double *wv2 = wv1 + n;     // wp_2 vp_2
    double *rv = wv2 + n;      // rho vp_lmax
    double *tmp = rv + n;      // G = 0 integrands (block 0)
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        r[i] = a.rho[i];
        wv0[i] = (lmax > 0) ? a.wp[i] * a.vp[i] : 0.0;
        wv1[i] = (lmax > 1) ? a.wp[i + n] * a.vp[i + n] : 0.0;
        wv2[i] = (lmax > 2) ? a.wp[i + 2 * n] * a.vp[i + 2 * n] : 0.0;
        rv[i] = a.rho[i] * a.vp[i + lmax * n];
    }
    __syncthreads();
    const long N = a.nfft3d;
    const double pi = 3.14159265358979323846, fourpi = 4.0 * pi;
    const double p0 = sqrt(fourpi), p1 = sqrt(3.0 * fourpi), p2 = sqrt(15.0 * fourpi);
    const double h3 = a.drho / 3.0;
    if (blockIdx.x == 0) {  // G = 0 (dkbppv3.c: the terms after the G loop)
        for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = a.vp[i + lmax * n] * (r[i] * r[i]);
        __syncthreads();
        double vl0 = 0.0;
        if (threadIdx.x == 0) vl0 = fourpi * kb_simp(n, tmp, a.drho) + 2.0 * pi * a.zv * r[n - 1] * r[n - 1];
        __syncthreads();
        if (lmax > 0)
            for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = r[i] * a.wp[i] * a.vp[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            a.vl[0] = vl0;
            if (lmax > 0) a.vnl[0] = p0 * kb_simp(n, tmp, a.drho);
            for (int l = 1; l < lmax * lmax; ++l) a.vnl[(long)l * N] = 0.0;
        }
    }
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < N; k += (long)gridDim.x * blockDim.x) {
        if (k == 0) continue;
        double gx = a.G[k], gy = a.G[k + N], gz = a.G[k + 2 * N];
        const double q = sqrt(gx * gx + gy * gy + gz * gz);
        gx /= q;
        gy /= q;
        gz /= q;
        // even / odd partial sums per channel (s, p, d, local); first and
        // last terms for simp()
        double se = 0.0, so = 0.0, pe = 0.0, po = 0.0, de = 0.0, dd = 0.0, le = 0.0, lo = 0.0;
        double fs0 = 0.0, fl0 = 0.0, fsn = 0.0, fpn = 0.0, fdn = 0.0, fln = 0.0, csn = 0.0;
        auto term = [&](int i, double &sacc, double &pacc, double &dacc, double &lacc) {
            const double x = q * r[i];
            double sn, cs;
            sincos(x, &sn, &cs);
            const double fs = sn * wv0[i];
            const double fl = rv[i] * sn;
            double fp = 0.0, fd = 0.0;
            if (i > 0 && lmax > 1) {
                const double t = sn / x - cs;
                fp = t * wv1[i];
                if (lmax > 2) fd = (3.0 * t / x - sn) * wv2[i];
            }
            sacc += fs;
            pacc += fp;
            dacc += fd;
            lacc += fl;
            fsn = fs;
            fpn = fp;
            fdn = fd;
            fln = fl;
            csn = cs;
        };
        term(0, se, pe, de, le);
        fs0 = fsn;
        fl0 = fln;
        int i = 1;
        for (; i + 1 < n; i += 2) {
            term(i, so, po, dd, lo);
            term(i + 1, se, pe, de, le);
        }
        if (i < n) term(i, so, po, dd, lo);
        const double sd[2] = {de, dd}, sp[2] = {pe, po}, ss[2] = {se, so}, sl[2] = {le, lo};
        if (lmax > 2) {
            const double S = (2.0 * sd[0] + 4.0 * sd[1] - 0.0 - fdn) * h3;
            const double d = p2 * S / q;
            a.vnl[k + 4 * N] = d * (3.0 * gz * gz - 1.0) / (2.0 * sqrt(3.0));
            a.vnl[k + 5 * N] = d * gx * gy;
            a.vnl[k + 6 * N] = d * gy * gz;
            a.vnl[k + 7 * N] = d * gz * gx;
            a.vnl[k + 8 * N] = d * (gx * gx - gy * gy) / 2.0;
        }
        if (lmax > 1) {
            const double S = (2.0 * sp[0] + 4.0 * sp[1] - 0.0 - fpn) * h3;
            const double p = p1 * S / q;
            a.vnl[k + 1 * N] = p * gx;
            a.vnl[k + 2 * N] = p * gy;
            a.vnl[k + 3 * N] = p * gz;
        }
        if (lmax > 0) {
            const double S = (2.0 * ss[0] + 4.0 * ss[1] - fs0 - fsn) * h3;
            a.vnl[k] = p0 * S / q;
        }
        const double S = (2.0 * sl[0] + 4.0 * sl[1] - fl0 - fln) * h3;
        a.vl[k] = S * fourpi / q - a.zv * fourpi * csn / (q * q);
    }
}

// Shared memory of kbpp_kernel for n radial points.
inline size_t kbpp_smem_bytes(int n) { return sizeof(double) * 6 * (size_t)n; }
