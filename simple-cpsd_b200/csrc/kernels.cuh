// kernels.cuh -- pointwise, reduction, GEMM and Lagrange kernels of one SD step.
//
// Every routine cites the reference lines (ccpsdv3/, Simple-CPSD) whose
// arithmetic it carries.  Complex arrays are cx<double>; packed arrays run
// over the cutoff sphere (see fft.cuh), real grids over n^3 points.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace cg = cooperative_groups;

// ------------------------------------------------------------ reductions
template <int NT>
CPSD_D double block_sum(double v, double *sh)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < NT / 32; ++i) r += sh[i];
    return r;  // valid in thread 0
}

// ------------------------------------------------------------ phase factors
// ccpsdv3/strfac.c:10-77: ex_d[k] = e^{-i k (b_d . r + pi)} by recurrence,
// negative k mirrored as conjugates (ex2, ex3), Nyquist entry zeroed.
// ex1: [nion][nh], ex2/ex3: [nion][n]
__global__ void phase_tables_kernel(int nion, int n, const double *__restrict__ unitg,
                                    const double *__restrict__ r1, cx<double> *ex1,
                                    cx<double> *ex2, cx<double> *ex3)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= 3 * nion) return;
    const int ii = id / 3, d = id % 3;
    const double pi = 3.14159265358979323846;  // 4 atan(1), strfac's pi argument
    const double sw = unitg[3 * d] * r1[3 * ii] + unitg[3 * d + 1] * r1[3 * ii + 1] +
                      unitg[3 * d + 2] * r1[3 * ii + 2] + pi;
    const double cr = cos(sw), ci = -sin(sw);
    const int h = n / 2;
    cx<double> *e = (d == 0) ? ex1 + (long)ii * (h + 1) : ((d == 1) ? ex2 : ex3) + (long)ii * n;
    e[0] = cx<double>{1.0, 0.0};
    cx<double> p{1.0, 0.0};
    for (int k = 1; k <= h; ++k) {
        cx<double> q{p.x * cr - p.y * ci, p.x * ci + p.y * cr};
        e[k] = q;
        if (d > 0) e[n - k] = cx<double>{q.x, -q.y};
        p = q;
    }
    e[h] = cx<double>{0.0, 0.0};
}

// exi(G) = ex1[i] (ex2[j] ex3[k]) in the reference's multiplication order, strfac.c:112-115
CPSD_D cx<double> strfac_point(cx<double> e1, cx<double> e2, cx<double> e3)
{
    double tr = e2.x * e3.x - e2.y * e3.y;
    double ti = e2.x * e3.y + e2.y * e3.x;
    return cx<double>{e1.x * tr - e1.y * ti, e1.y * tr + e1.x * ti};
}

// ------------------------------------------------------------ local psp, projectors
// ccpsdv3/cpsd.c:224-245 (s, vall), :260-286 (projectors), :373-379 (V(G))
struct VlocArgs {
    int npw, npw_pad, n, nh, nion;
    const int *pt_i, *pt_j, *pt_k;
    const int *katm;
    const double *zv;
    const cx<double> *ex1, *ex2, *ex3;
    const double *vl;   // [nkatm][npw]
    const double *vnl;  // [nkatm][9][npw]
    const int *lmmax;   // [nkatm]
    const int *proj_off;  // [nion] first projector row of each ion
    cx<double> *s, *vall;
    cx<double> *proj;   // [nproj][npw_pad]
};

__global__ void vloc_proj_kernel(VlocArgs a)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.npw_pad) return;
    if (p >= a.npw) {  // keep the GEMM padding at zero
        for (int ii = 0; ii < a.nion; ++ii) {
            const int nl = a.lmmax[a.katm[ii]];
            for (int l = 0; l < nl; ++l) a.proj[(long)(a.proj_off[ii] + l) * a.npw_pad + p] = cx<double>{0, 0};
        }
        return;
    }
    const int i = a.pt_i[p], j = a.pt_j[p], k = a.pt_k[p];
    cx<double> s{0, 0}, vall{0, 0};
    for (int ii = 0; ii < a.nion; ++ii) {
        const int ia = a.katm[ii];
        cx<double> exi = strfac_point(a.ex1[(long)ii * a.nh + i], a.ex2[(long)ii * a.n + j],
                                      a.ex3[(long)ii * a.n + k]);
        const double z = a.zv[ia];
        s.x += z * exi.x;
        s.y += z * exi.y;
        const double v = a.vl[(long)ia * a.npw + p];
        vall.x += exi.x * v;
        vall.y += exi.y * v;
        const int nl = a.lmmax[ia];
        for (int l = 0; l < nl; ++l) {
            const double w = a.vnl[((long)ia * 9 + l) * a.npw + p];
            cx<double> chi = (l == 0 || l >= 4) ? cx<double>{exi.x * w, exi.y * w}
                                                : cx<double>{-exi.y * w, exi.x * w};
            a.proj[(long)(a.proj_off[ii] + l) * a.npw_pad + p] = chi;
        }
    }
    a.s[p] = s;
    a.vall[p] = vall;
}

// V(G) = vall / omega + dng vc (cpsd.c:373-379), once the density is known
__global__ void vg_kernel(int npw, const cx<double> *__restrict__ vall, const cx<double> *__restrict__ dng,
                          const double *__restrict__ vc, double scal2, cx<double> *__restrict__ Vg)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npw) return;
    const cx<double> v = vall[p], d = dng[p];
    const double k = vc[p];
    Vg[p] = cx<double>{v.x * scal2 + d.x * k, v.y * scal2 + d.y * k};
}

// ------------------------------------------------------------ ion forces
// move = 1 (cpsd.c:246-257, 291-304, 310-364).  All Gamma-point sums use the
// weight w (1 on kx = 0, 2 elsewhere: gsdot of ccpsdv3/gsdot.c) over the
// sphere; G_d is the d-th Cartesian component of G per sphere point.
constexpr int kForceChunks = 16;  // point chunks of the local + k-space Ewald sums

struct ForceArgs {
    int npw, n, nh, nion;
    const int *pt_i, *pt_j, *pt_k, *katm;
    const cx<double> *ex1, *ex2, *ex3;  // phase tables of r1
    const double *w, *G;                // G: [3][npw]
    const double *vl, *vg, *zv;
    const cx<double> *dng, *s;
    double scal2;
    double *fpart;  // [chunk][ion][3]
};

// Local force (cpsd.c:246-257: sum_G G_d (Im dng Re exi - Re dng Im exi) vl)
// and k-space Ewald force (cpsd.c:318-328: sum_G G_d (exi x s) vg zv scal2)
// of ion blockIdx.y over point chunk blockIdx.x, fixed-order block sums.
__global__ void __launch_bounds__(256) force_local_ewald_kernel(ForceArgs a)
{
    __shared__ double sh[32];
    const int ii = blockIdx.y, ch = blockIdx.x;
    const int per = (a.npw + kForceChunks - 1) / kForceChunks;
    const int p0 = ch * per, p1 = min(a.npw, p0 + per);
    const int ia = a.katm[ii];
    const double zs = a.zv[ia] * a.scal2;
    double f[3] = {0.0, 0.0, 0.0};
    for (int p = p0 + threadIdx.x; p < p1; p += 256) {
        const cx<double> e = strfac_point(a.ex1[(long)ii * a.nh + a.pt_i[p]], a.ex2[(long)ii * a.n + a.pt_j[p]],
                                          a.ex3[(long)ii * a.n + a.pt_k[p]]);
        const cx<double> d = a.dng[p], sp = a.s[p];
        const double vl = a.vl[(long)ia * a.npw + p];
        const double loc = vl * (d.y * e.x - d.x * e.y);
        const double ewk = (e.x * sp.y - e.y * sp.x) * a.vg[p] * zs;
        const double t = a.w[p] * (loc + ewk);
        for (int k = 0; k < 3; ++k) f[k] += t * a.G[(long)k * a.npw + p];
    }
    for (int k = 0; k < 3; ++k) {
        const double v = block_sum<256>(f[k], sh);
        if (threadIdx.x == 0) a.fpart[((long)ch * a.nion + ii) * 3 + k] = v;
    }
}

// Nonlocal force per projector P (cpsd.c:291-304): with Y_P = sum_b sw1(P, b)
// c1_b, fnl[P][d] = sum_G w G_d Im(conj(chi_P) Y_P).
__global__ void __launch_bounds__(256) force_nonlocal_kernel(int npw, long ld, const double *__restrict__ w,
                                                             const double *__restrict__ G,
                                                             const cx<double> *__restrict__ proj,
                                                             const cx<double> *__restrict__ Y,
                                                             double *__restrict__ fnl)
{
    __shared__ double sh[32];
    const int P = blockIdx.x;
    const cx<double> *chi = proj + (long)P * ld, *y = Y + (long)P * ld;
    double f[3] = {0.0, 0.0, 0.0};
    for (int p = threadIdx.x; p < npw; p += 256) {
        const cx<double> c = chi[p], v = y[p];
        const double t = w[p] * (c.x * v.y - c.y * v.x);
        for (int k = 0; k < 3; ++k) f[k] += t * G[(long)k * npw + p];
    }
    for (int k = 0; k < 3; ++k) {
        const double v = block_sum<256>(f[k], sh);
        if (threadIdx.x == 0) fnl[3 * P + k] = v;
    }
}

// Real-space Ewald force of each pair ii < jj (cpsd.c:331-362), summed over
// the image cells: ewp[pair][3], pair = ii (2 nion - ii - 1) / 2 + jj - ii - 1.
__global__ void __launch_bounds__(256) force_ewald_pairs_kernel(int nion, int nsh, const double *__restrict__ r1,
                                                                const double *__restrict__ rcell,
                                                                const double *__restrict__ zv,
                                                                const int *__restrict__ katm, double rcut,
                                                                double *__restrict__ ewp)
{
    const double B1 = 0.0705230784, B2 = 0.0422820123, B3 = 0.0092705272;
    const double B4 = 0.0001520143, B5 = 0.0002765672, B6 = 0.0000430638;
    const double CERFC = 1.128379167;  // 2 / sqrt(pi), as cpsd.c rounds it
    const int ii = blockIdx.x;
    const long off = (long)ii * (2L * nion - ii - 1) / 2;
    for (int jj = ii + 1 + threadIdx.x; jj < nion; jj += 256) {
        const double dx = r1[3 * ii] - r1[3 * jj];
        const double dy = r1[3 * ii + 1] - r1[3 * jj + 1];
        const double dz = r1[3 * ii + 2] - r1[3 * jj + 2];
        const double zz = zv[katm[ii]] * zv[katm[jj]];
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int l = 0; l < nsh; ++l) {
            const double x = rcell[l] + dx, y = rcell[l + nsh] + dy, z = rcell[l + 2 * nsh] + dz;
            const double r = sqrt(x * x + y * y + z * z);
            const double wr = r / rcut;
            double aa = (1.0 + wr * (B1 + wr * (B2 + wr * (B3 + wr * (B4 + wr * (B5 + wr * B6))))));
            aa *= aa * aa * aa;
            const double erfc = 1.0 / (aa * aa * aa * aa);
            const double ad = zz * (erfc + CERFC * wr * exp(-wr * wr)) / (r * r * r);
            s1 += x * ad;
            s2 += y * ad;
            s3 += z * ad;
        }
        const long pr = off + (jj - ii - 1);
        ewp[3 * pr] = s1;
        ewp[3 * pr + 1] = s2;
        ewp[3 * pr + 2] = s3;
    }
}

// fion = local + k-space Ewald - nonlocal + real-space Ewald, and the ion SD
// step r2 = r1 + dti fion (cpsd.c:401-411); one thread per ion, fixed order.
__global__ void force_total_kernel(int nion, double nl_factor, const int *__restrict__ proj_off,
                                   const int *__restrict__ lmmax, const int *__restrict__ katm,
                                   const double *__restrict__ fpart, const double *__restrict__ fnl,
                                   const double *__restrict__ ewp, const double *__restrict__ dti,
                                   const double *__restrict__ r1, double *__restrict__ fion,
                                   double *__restrict__ r2)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x;
    if (ii >= nion) return;
    double f[3] = {0.0, 0.0, 0.0};
    for (int ch = 0; ch < kForceChunks; ++ch)
        for (int k = 0; k < 3; ++k) f[k] += fpart[((long)ch * nion + ii) * 3 + k];
    const int nl = lmmax[katm[ii]];
    for (int l = 0; l < nl; ++l)
        for (int k = 0; k < 3; ++k) f[k] -= nl_factor * fnl[3 * (proj_off[ii] + l) + k];
    for (int a = 0; a < ii; ++a) {  // pairs (a, ii) enter with a minus sign (cpsd.c:359-361)
        const long pr = (long)a * (2L * nion - a - 1) / 2 + (ii - a - 1);
        for (int k = 0; k < 3; ++k) f[k] -= ewp[3 * pr + k];
    }
    const long off = (long)ii * (2L * nion - ii - 1) / 2;
    for (int b = ii + 1; b < nion; ++b)  // pairs (ii, b): plus (cpsd.c:356-358)
        for (int k = 0; k < 3; ++k) f[k] += ewp[3 * (off + b - ii - 1) + k];
    for (int k = 0; k < 3; ++k) {
        fion[3 * ii + k] = f[k];
        r2[3 * ii + k] = r1[3 * ii + k] + dti[ii] * f[k];
    }
}

// coefficients of the KB back-projection, ccpsdv3/cpsd.c:289:
// coefT[b][P] = -beta[P][b] * scal2 / vnlnrm[P]
// (and, for the nonlocal force, the same in [P][b] order when coefP is given)
__global__ void kb_coef_kernel(int nproj, int nb, const double *__restrict__ beta,
                               const double *__restrict__ vnlnrm_p, double scal2,
                               double *__restrict__ coefT, double *__restrict__ coefP)
{
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nproj * nb) return;
    const int P = id / nb, b = id % nb;
    const double v = -beta[id] * scal2 / vnlnrm_p[P];
    coefT[(long)b * nproj + P] = v;
    if (coefP) coefP[id] = v;
}

// ------------------------------------------------------------ density + xc
// dn_ms = scal2 * sum_b psi_b^2 (cpsd.c:185-194); Dirac exchange then Vosko
// correlation (dirac_exchange.c:64-126, vosko.c:99-167); the forward-FFT
// input (dn_0 + dn_{ispin-1}) * scal1 (cpsd.c:198-199).
struct XcArgs {
    long n3;
    int ispin;
    int nchunk0, nchunk1;  // chunks of spin 0, then of spin 1
    const double *part;    // [nchunk][n3]
    double scal1, scal2;
    double *dn, *xcp, *xce, *rfwd;
};

CPSD_D void dirac_vosko(int ispin, double nup_in, double ndn_in, double rho0, double rho1,
                        double &vx0, double &vx1, double &ex)
{
    // --- Dirac exchange, alpha = 2/3 (dirac_exchange.c:14-24, 84-122)
    const double alpha = 0.6666666666666666667;
    const double onethird_d = 0.33333333333333333333;
    const double fourthird_d = 1.33333333333333333333;
    const double two_to_onethird_d = 1.25992104989487319067;
    const double A_d = 0.25992104989487319067;
    const double pi_d = 3.14159265358979311600;
    // cube roots of the (non-negative) density by cbrt: the reference's
    // pow(x, 1/3) to within an ulp
    if (ispin == 1) {
        const double n = nup_in + nup_in;
        const double n13 = cbrt(3.0 * n / pi_d);
        ex = -(9.0 / 8.0) * alpha * n13;
        vx0 = -(3.0 / 2.0) * alpha * n13;
        vx1 = vx0;
    } else {
        const double n = nup_in + ndn_in;
        const double n13 = cbrt(3.0 * n / pi_d);
        // the reference's xi here uses the first two density values (dirac_exchange.c:101)
        const double xi = (n > 0.0) ? (rho0 - rho1) / n : 1.0;
        const double ex_p = -(9.0 / 8.0) * alpha * n13;
        const double ux_p = -(3.0 / 2.0) * alpha * n13;
        const double ex_f = two_to_onethird_d * ex_p;
        const double ux_f = fourthird_d * ex_f;
        const double f = (pow(1.0 + xi, fourthird_d) + pow(1.0 - xi, fourthird_d) - 2.0) / (2.0 * A_d);
        const double df = fourthird_d * (pow(1.0 + xi, onethird_d) - pow(1.0 - xi, onethird_d)) / (2.0 * A_d);
        ex = ex_p + f * (ex_f - ex_p);
        vx0 = ux_p + f * (ux_f - ux_p) + (+1.0 - xi) * (df * (ex_f - ex_p));
        vx1 = ux_p + f * (ux_f - ux_p) + (-1.0 - xi) * (df * (ex_f - ex_p));
    }
    // --- Vosko-Wilk-Nusair, the reference's parameter table (vosko.c:22-57)
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
    const double nup = nup_in + small_number;
    const double ndown = ((ispin == 1) ? nup_in : ndn_in) + small_number;
    const double n = nup + ndown;
    const double rs = rs_scale / cbrt(n);
    const double xi = (nup - ndown) / n;
    const double x = sqrt(rs);
    const double xxp = rs + bp * x + cp;
    const double dxxp = 2.0 * x + bp;
    const double ec_p = cp1 * log(rs / xxp) + cp2 * log((x + cp3) * (x + cp3) / xxp) + cp4 * atan(cp5 / (x + cp6));
    const double uc_p = ec_p - onesixth * x * (dp1 / x + dp2 / (x + cp3) + dp4 * dxxp / xxp +
                                               dp5 / ((x + dp6) * (x + dp6) + dp7));
    if (ispin == 1) {
        // closed shell: nup == ndown, so xi = 0 and f = df = 0 exactly; the
        // reference's sums reduce to the paramagnetic terms bit for bit
        ex += ec_p;
        vx0 += uc_p;
        return;
    }
    const double xxf = rs + bf * x + cf;
    const double dxxf = 2.0 * x + bf;
    const double ec_f = cf1 * log(rs / xxf) + cf2 * log((x + cf3) * (x + cf3) / xxf) + cf4 * atan(cf5 / (x + cf6));
    const double uc_f = ec_f - onesixth * x * (df1 / x + df2 / (x + cf3) + df4 * dxxf / xxf +
                                               df5 / ((x + df6) * (x + df6) + df7));
    const double f = (pow(1.0 + xi, fourthird) + pow(1.0 - xi, fourthird) - 2.0) / (2.0 * A);
    const double df = fourthird * (pow(1.0 + xi, onethird) - pow(1.0 - xi, onethird)) / (2.0 * A);
    ex += ec_p + f * (ec_f - ec_p);
    vx0 += uc_p + f * (uc_f - uc_p) + (+1.0 - xi) * (df * (ec_f - ec_p));
    if (ispin == 2) vx1 += uc_p + f * (uc_f - uc_p) + (-1.0 - xi) * (df * (ec_f - ec_p));
}

__global__ void density_xc_kernel(XcArgs a)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n3) return;
    double d[2] = {0.0, 0.0}, r0 = 0.0, r1 = 0.0;
    for (int c = 0; c < a.nchunk0; ++c) {
        d[0] += a.part[(long)c * a.n3 + r];
        if (a.ispin == 2) {
            r0 += a.part[(long)c * a.n3 + 0];
            r1 += a.part[(long)c * a.n3 + 1];
        }
    }
    for (int c = a.nchunk0; c < a.nchunk0 + a.nchunk1; ++c) d[1] += a.part[(long)c * a.n3 + r];
    d[0] *= a.scal2;
    d[1] *= a.scal2;
    r0 *= a.scal2;
    r1 *= a.scal2;
    double vx0, vx1, ex;
    dirac_vosko(a.ispin, d[0], d[1], r0, r1, vx0, vx1, ex);
    a.dn[r] = d[0];
    a.xcp[r] = vx0;
    a.xce[r] = ex;
    if (a.ispin == 2) {
        a.dn[a.n3 + r] = d[1];
        a.xcp[a.n3 + r] = vx1;
    }
    a.rfwd[r] = (d[0] + d[a.ispin - 1]) * a.scal1;
}

// Band-parallel steps split density_xc_kernel at the exchange: this rank's
// chunk sums (its bands only) -> dn_part, summed over the ranks into dn,
// then the xc potential from dn.  The arithmetic per point is that of
// density_xc_kernel, so one rank owning every band gets the same bits.
__global__ void density_sum_kernel(XcArgs a, double *dn_part)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n3) return;
    double d0 = 0.0, d1 = 0.0;
    for (int c = 0; c < a.nchunk0; ++c) d0 += a.part[(long)c * a.n3 + r];
    for (int c = a.nchunk0; c < a.nchunk0 + a.nchunk1; ++c) d1 += a.part[(long)c * a.n3 + r];
    dn_part[r] = d0 * a.scal2;
    if (a.ispin == 2) dn_part[a.n3 + r] = d1 * a.scal2;
}

__global__ void xc_from_density_kernel(XcArgs a)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.n3) return;
    const double d0 = a.dn[r], d1 = (a.ispin == 2) ? a.dn[a.n3 + r] : 0.0;
    // the reference's xi of the spin-polarised exchange reads the first two
    // spin-0 density values (dirac_exchange.c:101)
    const double r0 = (a.ispin == 2) ? a.dn[0] : 0.0, r1 = (a.ispin == 2) ? a.dn[1] : 0.0;
    double vx0, vx1, ex;
    dirac_vosko(a.ispin, d0, d1, r0, r1, vx0, vx1, ex);
    a.xcp[r] = vx0;
    a.xce[r] = ex;
    if (a.ispin == 2) a.xcp[a.n3 + r] = vx1;
    a.rfwd[r] = (d0 + (a.ispin == 2 ? d1 : d0)) * a.scal1;
}

// dn = sum over the parts in their order (the ranks' spin densities of a
// band-parallel step on one device)
constexpr int kMaxGroupRanks = 8;
struct PartSum {
    const double *part[kMaxGroupRanks];
    int nparts;
};
__global__ void sum_parts_kernel(PartSum p, long n, double *out)
{
    const long r = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    double acc = p.part[0][r];
    for (int q = 1; q < p.nparts; ++q) acc += p.part[q][r];
    out[r] = acc;
}

// ------------------------------------------------------------ FP64 GEMMs
// part[prod][split][i][j] = sum_{k in chunk} w(k) A_prod[i*lda+k] B_prod[j*ldb+k];
// K counts reals, the weight is per complex pair (w[k/2]): the Gamma-point
// dot of ccpsdv3/gcdotc.c as a matrix product.  Up to kTnMaxProd products of
// the same shape share one launch (blockIdx.z = prod * splits + split).
constexpr int kTnMaxProd = 4;

struct TnBatch {
    const double *A[kTnMaxProd];
    const double *B[kTnMaxProd];
    double *C[kTnMaxProd];
    int nprod, splits;
};

// C_prod[i*ldc+j] = alpha * sum_s part[prod][s][i][j] (+ beta C): one warp
// per output, lanes stride over the splits, then a fixed xor butterfly, so
// the order of the additions (and the bits of the result) never changes.
__global__ void splitk_reduce_kernel(int M, int N, long ldc, const double *__restrict__ part, double alpha,
                                     double beta, const __grid_constant__ TnBatch bt)
{
    const long wid = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long MN = (long)M * N;
    if (wid >= MN * bt.nprod) return;  // whole warps leave together
    const int prod = (int)(wid / MN);
    const long e = wid % MN;
    const double *p = part + (long)prod * bt.splits * MN + e;
    double s = 0.0;
    for (int q = lane; q < bt.splits; q += 32) s += p[(long)q * MN];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const int i = (int)(e / N), j = (int)(e % N);
        double *c = bt.C[prod] + (long)i * ldc + j;
        *c = alpha * s + (beta == 0.0 ? 0.0 : beta * *c);
    }
}

// ------------------------------------------------------------ FP64 tensor-core GEMMs
// Two products on the FP64 tensor cores (mma.sync m8n8k4 f64: exact FP64
// products, FP64 sums): the split-K weighted TN partials above and the
// back-projection NN product (the reference's dgemm('N','N') on
// column-major psi blocks, cpsd.c:483-488).  A CTA of four warps owns a 64x64 output
// tile, each warp a 32x32 quadrant of 4x4 fragments of 8x8.  A shared tile
// holds 16 values of the contraction index per row; MMA step s (0..3) feeds
// fragment k-slot q with tile column 4q+s, so one lane's four values for a
// tile are a contiguous 32-byte run (two 16-byte loads).  The next tile is
// fetched into registers while the current one is multiplied: two shared
// buffers, one barrier per tile.  Row strides keep every shared access free
// of bank conflicts: kDmS = 18 puts consecutive rows 9 16-byte units apart,
// kDmSB = 65 (NN B tile, [l][k]) staggers the four k-slots by one bank.
constexpr int kDmT = 64, kDmK = 16, kDmThreads = 128, kDmS = 18, kDmSB = 65;

CPSD_D void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// part[prod][split][i][j] as above; grid (M tiles, N tiles, nprod * splits).
__global__ void __launch_bounds__(kDmThreads, 4)
gemm_tn_dmma_kernel(int M, int N, int K, long lda, long ldb, const double *__restrict__ w, int kchunk,
                    const __grid_constant__ TnBatch bt, double *__restrict__ part)
{
    __shared__ __align__(16) double As[2][kDmT * kDmS], Bs[2][kDmT * kDmS];
    const int prod = blockIdx.z / bt.splits, split = blockIdx.z % bt.splits;
    const double *__restrict__ A = bt.A[prod];
    const double *__restrict__ B = bt.B[prod];
    const int i0 = blockIdx.x * kDmT, j0 = blockIdx.y * kDmT;
    const int k0 = split * kchunk, k1 = min(K, k0 + kchunk);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32, fr = lane >> 2, fq = lane & 3;
    double ra[4][2], rb[4][2];
    // loader: pass q moves reals (2p, 2p+1) of tile row e>>3, e = tid + 128q, p = e&7
    auto fetch = [&](int kk) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + kDmThreads * q, row = e >> 3, k = kk + 2 * (e & 7);
            const int i = i0 + row, j = j0 + row;
            const double wk = (w != nullptr && k < k1) ? w[k >> 1] : 1.0;  // k even: one weight per pair
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const bool ok = k + h < k1;
                ra[q][h] = (ok && i < M) ? A[(long)i * lda + k + h] * wk : 0.0;
                rb[q][h] = (ok && j < N) ? B[(long)j * ldb + k + h] : 0.0;
            }
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + kDmThreads * q, off = (e >> 3) * kDmS + 2 * (e & 7);
            *reinterpret_cast<double2 *>(&As[buf][off]) = make_double2(ra[q][0], ra[q][1]);
            *reinterpret_cast<double2 *>(&Bs[buf][off]) = make_double2(rb[q][0], rb[q][1]);
        }
    };
    double acc[4][4][2] = {};
    int buf = 0;
    if (k0 < k1) {
        fetch(k0);
        stash(0);
    }
    __syncthreads();
    for (int kk = k0; kk < k1; kk += kDmK) {
        const bool more = kk + kDmK < k1;
        if (more) fetch(kk + kDmK);
        // two halves of two k-steps each: one 16-byte fragment load per
        // operand row per half keeps the fragments in 32 registers
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            double2 a[4], b[4];
#pragma unroll
            for (int f = 0; f < 4; ++f) {
                a[f] = *reinterpret_cast<const double2 *>(As[buf] + (wr + 8 * f + fr) * kDmS + 4 * fq + 2 * hh);
                b[f] = *reinterpret_cast<const double2 *>(Bs[buf] + (wc + 8 * f + fr) * kDmS + 4 * fq + 2 * hh);
            }
#pragma unroll
            for (int fi = 0; fi < 4; ++fi)
#pragma unroll
                for (int fj = 0; fj < 4; ++fj) dmma(acc[fi][fj][0], acc[fi][fj][1], a[fi].x, b[fj].x);
#pragma unroll
            for (int fi = 0; fi < 4; ++fi)
#pragma unroll
                for (int fj = 0; fj < 4; ++fj) dmma(acc[fi][fj][0], acc[fi][fj][1], a[fi].y, b[fj].y);
        }
        if (more) stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
    double *out = part + ((long)prod * bt.splits + split) * M * N;
#pragma unroll
    for (int fi = 0; fi < 4; ++fi) {
        const int i = i0 + wr + 8 * fi + fr;
        if (i >= M) continue;
#pragma unroll
        for (int fj = 0; fj < 4; ++fj)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = j0 + wc + 8 * fj + 2 * fq + h;
                if (j < N) out[(long)i * N + j] = acc[fi][fj][h];
            }
    }
}

// Out[j*ldo+k] = beta*Out + alpha * sum_l
// Mat[l + j*ldm] * B[l*ldb + k]; grid x over 64-wide k tiles, y over j tiles.
__global__ void __launch_bounds__(kDmThreads, 4)
gemm_nn_dmma_kernel(int NJ, int K, int L, double alpha, const double *__restrict__ Mat, long ldm,
                    const double *__restrict__ B, long ldb, double beta, double *__restrict__ Out, long ldo)
{
    __shared__ __align__(16) double Ms[2][kDmT * kDmS], Bs[2][kDmK * kDmSB];
    const int k0 = blockIdx.x * kDmT, j0 = blockIdx.y * kDmT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32, fr = lane >> 2, fq = lane & 3;
    double rm[4][2], rb[8];
    auto fetch = [&](int l0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {  // Mat: tile row j = e>>3, l pair (2p, 2p+1)
            const int e = tid + kDmThreads * q, j = j0 + (e >> 3), l = l0 + 2 * (e & 7);
#pragma unroll
            for (int h = 0; h < 2; ++h) rm[q][h] = (j < NJ && l + h < L) ? Mat[(long)j * ldm + l + h] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {  // B: tile row l = e>>6, column k = e&63
            const int e = tid + kDmThreads * q, l = l0 + (e >> 6), k = k0 + (e & 63);
            rb[q] = (l < L && k < K) ? B[(long)l * ldb + k] : 0.0;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + kDmThreads * q;
            *reinterpret_cast<double2 *>(&Ms[buf][(e >> 3) * kDmS + 2 * (e & 7)]) = make_double2(rm[q][0], rm[q][1]);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = tid + kDmThreads * q;
            Bs[buf][(e >> 6) * kDmSB + (e & 63)] = rb[q];
        }
    };
    double acc[4][4][2] = {};
    int buf = 0;
    if (L > 0) {
        fetch(0);
        stash(0);
    }
    __syncthreads();
    for (int l0 = 0; l0 < L; l0 += kDmK) {
        const bool more = l0 + kDmK < L;
        if (more) fetch(l0 + kDmK);
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {  // two k-steps per half, as in the TN kernel
            double2 a[4];
#pragma unroll
            for (int f = 0; f < 4; ++f)
                a[f] = *reinterpret_cast<const double2 *>(Ms[buf] + (wr + 8 * f + fr) * kDmS + 4 * fq + 2 * hh);
#pragma unroll
            for (int s2 = 0; s2 < 2; ++s2) {
                const double *bs = Bs[buf] + (4 * fq + 2 * hh + s2) * kDmSB + wc + fr;
                double b[4];
#pragma unroll
                for (int fj = 0; fj < 4; ++fj) b[fj] = bs[8 * fj];
#pragma unroll
                for (int fi = 0; fi < 4; ++fi)
#pragma unroll
                    for (int fj = 0; fj < 4; ++fj)
                        dmma(acc[fi][fj][0], acc[fi][fj][1], s2 ? a[fi].y : a[fi].x, b[fj]);
            }
        }
        if (more) stash(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int fi = 0; fi < 4; ++fi) {
        const int j = j0 + wr + 8 * fi + fr;
        if (j >= NJ) continue;
#pragma unroll
        for (int fj = 0; fj < 4; ++fj)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = k0 + wc + 8 * fj + 2 * fq + h;
                if (k < K) {
                    double *o = Out + (long)j * ldo + k;
                    *o = alpha * acc[fi][fj][h] + (beta == 0.0 ? 0.0 : beta * *o);
                }
            }
    }
}

// ------------------------------------------------------------ Lagrange multipliers
// ccpsdv3/cpsd.c:415-479.  One cluster of kLagCluster CTAs per launch; CTA r
// owns a contiguous range of columns.  Overlaps come in row-major from the
// GEMMs: M22[i][j] = <c2_i|c2_j>, M21[i][j] = <c2_i|c1_j>, M11[i][j] = <c1_i|c1_j>.
constexpr int kLagCluster = 8;
constexpr int kLagThreads = 256;

struct LagArgs {
    int ispin, ne0, ne1;
    double dte;
    const double *M22[2], *M21[2], *M11[2];
    double *s11, *s12, *s21, *s22, *st1, *X0, *X1;  // ne0^2 each, column-major
    double *lmd;                                     // [ms*ne0^2 + i + j*m]
    double *red;                                     // [cluster CTAs][2]
    int *fail;                                       // steps whose iteration did not converge
    int lb;                                          // l-chunk of the cluster kernel's row tiles
};

// Cluster of kLagClusterMax (or kLagCluster where 16 cannot be scheduled)
// CTAs; CTA r owns a block of columns.  Thread layout: row i = tid % RT
// (RT = min(m, 256)) and a block of this CTA's columns.  Per iteration the
// rows of s21, s11 and X stream through shared memory in chunks of LB
// columns l; the CTA's columns of X, s12 and st1 stay in shared memory.
constexpr int kLagClusterMax = 16;
constexpr int kLagCols = 16;

CPSD_HD size_t lagrange_cluster_smem(int m, int cl, int lb)
{
    const int per = (m + cl - 1) / cl;
    return sizeof(double) * (3 * (size_t)m * per + 3 * (size_t)m * lb);
}

// widest l-chunk (32, 16, 8 or 4) whose tiles fit in `limit` bytes; 0 if none
inline int lagrange_lb(int m, int cl, size_t limit)
{
    for (int lb = 32; lb >= 4; lb /= 2)
        if (lagrange_cluster_smem(m, cl, lb) <= limit) return lb;
    return 0;
}

__global__ void __launch_bounds__(kLagThreads) lagrange_kernel(LagArgs a)
{
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int ncta = (int)cl.num_blocks();
    const int tid = threadIdx.x;
    extern __shared__ double lsm[];
    __shared__ double shv[kLagThreads / 32];
    __shared__ int shi[kLagThreads / 32];
    const long ne02 = (long)a.ne0 * a.ne0;
    for (int ms = 0; ms < a.ispin; ++ms) {
        const int m = ms ? a.ne1 : a.ne0;
        const long kk = (long)m * m;
        if (m == 0) continue;
        const double *M22 = a.M22[ms], *M21 = a.M21[ms], *M11 = a.M11[ms];
        const double dte = a.dte;
        // s matrices, cpsd.c:420-437 (upper triangles mirrored as the reference does)
        for (long e = (long)rank * kLagThreads + tid; e < kk; e += (long)ncta * kLagThreads) {
            const int i = (int)(e % m), j = (int)(e / m);
            double v22, v21, v12, v11;
            if (i == j) {
                v22 = (1.0 - M22[(long)i * m + i]) * 0.5 / dte;
                v21 = (1.0 - M21[(long)i * m + i]) * 0.5;
                v12 = v21;
                v11 = -M11[(long)i * m + i] * 0.5 * dte;
            } else {
                const int lo = i < j ? i : j, hi = i < j ? j : i;
                v22 = -M22[(long)lo * m + hi] * 0.5 / dte;
                v21 = -M21[(long)lo * m + hi] * 0.5;   // <c2_lo|c1_hi>
                v12 = -M21[(long)hi * m + lo] * 0.5;   // <c1_lo|c2_hi>
                v11 = -M11[(long)lo * m + hi] * 0.5 * dte;
            }
            a.s22[e] = v22;
            a.s21[e] = v21;
            a.s12[e] = v12;
            a.s11[e] = v11;
            a.X0[e] = v22;  // sa0 = s22, cpsd.c:441
        }
        cl.sync();
        const int per = (m + ncta - 1) / ncta;  // columns per CTA
        const int jb = rank * per, je = min(m, jb + per);
        const int ncl = max(0, je - jb);
        const int RT = min(m, kLagThreads);
        const int nsub = kLagThreads / RT;
        const int csub = (ncl + nsub - 1) / max(nsub, 1);  // columns per thread
        const int i = tid % RT, sub = tid / RT;
        const int j0 = sub * csub;
        const bool active = (sub < nsub) && (i < m);
        const int LB = a.lb;
        double *Xs = lsm, *S12s = lsm + (long)m * per, *ST = lsm + 2L * m * per;
        double *T21 = lsm + 3L * m * per, *T11 = T21 + (long)m * LB, *TX = T11 + (long)m * LB;
        for (int e = tid; e < m * ncl; e += kLagThreads) {
            const int l = e % m, jl = e / m;
            S12s[jl * m + l] = a.s12[l + (long)(jb + jl) * m];
        }
        double *cur = a.X0, *nxt = a.X1;
        bool done = false;
        int iter = 0;
        while (!done && iter < 30) {
            ++iter;
            for (int e = tid; e < m * ncl; e += kLagThreads) {
                const int l = e % m, jl = e / m;
                Xs[jl * m + l] = cur[l + (long)(jb + jl) * m];
            }
            // sa1 = s22 + s21 sa0 + sa0 s12 ; st1 = s11 sa0   (cpsd.c:444-462);
            // the partial sa1 waits in nxt for the second product
            for (int cb = 0; cb < csub; cb += kLagCols) {
                double t1[kLagCols], t2[kLagCols], t3[kLagCols];
#pragma unroll
                for (int q = 0; q < kLagCols; ++q) t1[q] = t2[q] = t3[q] = 0.0;
                for (int l0 = 0; l0 < m; l0 += LB) {
                    const int lw = min(LB, m - l0);
                    __syncthreads();  // previous tile consumed (and Xs written)
                    for (int e = tid; e < m * lw; e += kLagThreads) {
                        const int ii = e % m, ll = e / m;
                        const long g = ii + (long)(l0 + ll) * m;
                        T21[ll * m + ii] = a.s21[g];
                        T11[ll * m + ii] = a.s11[g];
                        TX[ll * m + ii] = cur[g];
                    }
                    __syncthreads();
                    if (active) {
                        for (int ll = 0; ll < lw; ++ll) {
                            const int l = l0 + ll;
                            const double a21 = T21[ll * m + i], a11 = T11[ll * m + i], xil = TX[ll * m + i];
#pragma unroll
                            for (int q = 0; q < kLagCols; ++q) {
                                const int jl = j0 + cb + q;
                                if (cb + q < csub && jl < ncl) {
                                    const double xlj = Xs[jl * m + l];
                                    t1[q] = fma(a21, xlj, t1[q]);
                                    t2[q] = fma(xil, S12s[jl * m + l], t2[q]);
                                    t3[q] = fma(a11, xlj, t3[q]);
                                }
                            }
                        }
                    }
                }
                if (active) {
#pragma unroll
                    for (int q = 0; q < kLagCols; ++q) {
                        const int jl = j0 + cb + q;
                        if (cb + q < csub && jl < ncl) {
                            const int j = jb + jl;
                            nxt[i + (long)j * m] = t2[q] + (t1[q] + a.s22[i + (long)j * m]);
                            ST[jl * m + i] = t3[q];
                        }
                    }
                }
            }
            // sa1 += sa0 st1 (cpsd.c:463-468); st1 = sa1 - sa0 (:469-470)
            double bestv = -1.0;
            int besti = 0x7fffffff;
            for (int cb = 0; cb < csub; cb += kLagCols) {
                double t4[kLagCols];
#pragma unroll
                for (int q = 0; q < kLagCols; ++q) t4[q] = 0.0;
                for (int l0 = 0; l0 < m; l0 += LB) {
                    const int lw = min(LB, m - l0);
                    __syncthreads();
                    for (int e = tid; e < m * lw; e += kLagThreads) {
                        const int ii = e % m, ll = e / m;
                        TX[ll * m + ii] = cur[ii + (long)(l0 + ll) * m];
                    }
                    __syncthreads();
                    if (active) {
                        for (int ll = 0; ll < lw; ++ll) {
                            const int l = l0 + ll;
                            const double xil = TX[ll * m + i];
#pragma unroll
                            for (int q = 0; q < kLagCols; ++q) {
                                const int jl = j0 + cb + q;
                                if (cb + q < csub && jl < ncl) t4[q] = fma(xil, ST[jl * m + l], t4[q]);
                            }
                        }
                    }
                }
                if (active) {
#pragma unroll
                    for (int q = 0; q < kLagCols; ++q) {
                        const int jl = j0 + cb + q;
                        if (cb + q < csub && jl < ncl) {
                            const long f = i + (long)(jb + jl) * m;
                            const double sa1 = t4[q] + nxt[f];
                            nxt[f] = sa1;
                            const double d = sa1 - cur[f];
                            a.st1[f] = d;
                            const double ad = fabs(d);
                            if (ad > bestv || (ad == bestv && f < besti)) {
                                bestv = ad;
                                besti = (int)f;
                            }
                        }
                    }
                }
            }
            // block argmax (first index of the largest |st1|, as idamax)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, bestv, o);
                int oi = __shfl_xor_sync(0xffffffffu, besti, o);
                if (ov > bestv || (ov == bestv && oi < besti)) {
                    bestv = ov;
                    besti = oi;
                }
            }
            if ((tid & 31) == 0) {
                shv[tid >> 5] = bestv;
                shi[tid >> 5] = besti;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < kLagThreads / 32; ++w)
                    if (shv[w] > bestv || (shv[w] == bestv && shi[w] < besti)) {
                        bestv = shv[w];
                        besti = shi[w];
                    }
                a.red[2 * rank] = bestv;
                a.red[2 * rank + 1] = (double)besti;
            }
            cl.sync();
            // every CTA reduces the cluster's candidates in the same order
            double gv = -1.0;
            long gi = 0x7fffffff;
            for (int r = 0; r < ncta; ++r) {
                const double v = a.red[2 * r];
                const long ix = (long)a.red[2 * r + 1];
                if (v > gv || (v == gv && ix < gi)) {
                    gv = v;
                    gi = ix;
                }
            }
            // idamax returns an index in 1..kk even when every entry is NaN
            // (then no comparison succeeds and it returns 1); the sentinel
            // must never reach the read below
            if (gi < 0 || gi >= kk) gi = 0;
            // the reference reads st1 at idamax's 1-based result (cpsd.c:471):
            // the element after the largest; past the end of st1 lies sa1
            const long nx = gi + 1;
            const double adiff = fabs(nx < ne02 ? a.st1[nx] : nxt[nx - ne02]);
            done = adiff < 1e-15;
            cl.sync();
            if (!done) {
                double *t = cur;
                cur = nxt;
                nxt = t;
            }
        }
        if (!done && rank == 0 && tid == 0) atomicAdd(a.fail, 1);
        // lmd = sa1, cpsd.c:478 (after 30 unconverged iterations sa1 was swapped into cur)
        const double *fin = done ? nxt : cur;
        for (int e = tid; e < m * ncl; e += kLagThreads) {
            const int ii = e % m, j = jb + e / m;
            a.lmd[ms * ne02 + ii + (long)j * m] = fin[ii + (long)j * m];
        }
        cl.sync();
    }
}

// Small systems (ne0 <= kLagSmallMax): the same iteration in one CTA with
// every matrix in shared memory; block barriers instead of cluster barriers.
constexpr int kLagSmallMax = 32;

// Smem layout of lagrange_small_kernel: seven matrices padded to mp = m
// rounded up to 8, leading dimension mp + 4 (fragment loads of lanes
// 4r + k hit 16 different banks), then the unpadded differences.
CPSD_HD int lag_small_mp(int m) { return (m + 7) / 8 * 8; }
CPSD_HD int lag_small_ld(int m) { return lag_small_mp(m) + 4; }
inline size_t lag_small_smem_bytes(int ne0)
{
    return sizeof(double) * ((size_t)7 * lag_small_mp(ne0) * lag_small_ld(ne0) + (size_t)ne0 * ne0);
}

// One 8 x 8 tile of P = A B (column-major, leading dimension ld, inner
// dimension kd, a multiple of 4) on the FP64 tensor cores: a lane's
// fragment d[0..1] holds P(i0 + lane/4, j0 + 2 (lane%4) + e).
CPSD_D void lag_tile_mma(const double *A, const double *B, int ld, int kd, int i0, int j0, int lane,
                         double (&d)[2])
{
    const int r = lane >> 2, q = lane & 3;
    d[0] = d[1] = 0.0;
    for (int k0 = 0; k0 < kd; k0 += 4) dmma(d[0], d[1], A[(i0 + r) + (k0 + q) * ld], B[(k0 + q) + (j0 + r) * ld]);
}

// cpsd.c:420-479 for m <= kLagSmallMax bands: one CTA; the four m x m
// products of an iteration on the FP64 tensor cores (mma.sync m8n8k4),
// 8 x 8 tiles spread over the warps; two barriers per iteration.
__global__ void __launch_bounds__(kLagThreads) lagrange_small_kernel(LagArgs a)
{
    constexpr int NW = kLagThreads / 32;
    constexpr int TMAX = (kLagSmallMax / 8) * (kLagSmallMax / 8);  // tiles of the largest matrix
    constexpr int TPW = (TMAX + NW - 1) / NW;                      // tiles per warp
    extern __shared__ double lag_sm[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long ne02 = (long)a.ne0 * a.ne0;
    // the layout is sized for ne0 (ne1 <= ne0 reuses it)
    const int LD = lag_small_ld(a.ne0), SZ = lag_small_mp(a.ne0) * LD;
    double *s11 = lag_sm, *s12 = lag_sm + SZ, *s21 = lag_sm + 2 * SZ, *s22 = lag_sm + 3 * SZ;
    double *st1 = lag_sm + 4 * SZ;
    double *X[2] = {lag_sm + 5 * SZ, lag_sm + 6 * SZ};
    // sa1 - sa0 of each iteration (cpsd.c:469) at the reference's unpadded
    // index i + j m: what the reference keeps in st1 for its convergence
    // read; entries past m^2 keep the last ones written, as st1's do there
    double *dif = lag_sm + 7 * SZ;
    __shared__ double shv[NW];
    __shared__ int shi[NW];
    for (int ms = 0; ms < a.ispin; ++ms) {
        const int m = ms ? a.ne1 : a.ne0;
        const long kk = (long)m * m;
        if (m == 0) continue;
        const int mp = lag_small_mp(m), ld = lag_small_ld(m), nt = (mp / 8) * (mp / 8);
        const double *M22 = a.M22[ms], *M21 = a.M21[ms], *M11 = a.M11[ms];
        const double dte = a.dte;
        for (int e = tid; e < mp * ld; e += kLagThreads) {  // cpsd.c:420-437, zero padding
            const int i = e % ld, j = e / ld;
            double v22 = 0.0, v21 = 0.0, v12 = 0.0, v11 = 0.0;
            if (i < m && j < m) {
                if (i == j) {
                    v22 = (1.0 - M22[i * m + i]) * 0.5 / dte;
                    v21 = (1.0 - M21[i * m + i]) * 0.5;
                    v12 = v21;
                    v11 = -M11[i * m + i] * 0.5 * dte;
                } else {
                    const int lo = i < j ? i : j, hi = i < j ? j : i;
                    v22 = -M22[lo * m + hi] * 0.5 / dte;
                    v21 = -M21[lo * m + hi] * 0.5;
                    v12 = -M21[hi * m + lo] * 0.5;
                    v11 = -M11[lo * m + hi] * 0.5 * dte;
                }
            }
            s22[e] = v22;
            s21[e] = v21;
            s12[e] = v12;
            s11[e] = v11;
            X[0][e] = v22;
            X[1][e] = 0.0;
            st1[e] = 0.0;
        }
        __syncthreads();
        int cur = 0, iter = 0;
        bool done = false;
        while (!done && iter < 30) {
            ++iter;
            const double *c = X[cur];
            double *nx = X[cur ^ 1];
            double part[TPW][2];
            // X S12 + (S21 X + S22) and st1 = S11 X (cpsd.c:444-462)
#pragma unroll
            for (int u = 0; u < TPW; ++u) {
                const int t = warp + u * NW;
                if (t >= nt) break;
                const int i0 = (t % (mp / 8)) * 8, j0 = (t / (mp / 8)) * 8;
                double t1[2], t2[2], t3[2];
                lag_tile_mma(s21, c, ld, mp, i0, j0, lane, t1);
                lag_tile_mma(c, s12, ld, mp, i0, j0, lane, t2);
                lag_tile_mma(s11, c, ld, mp, i0, j0, lane, t3);
                const int i = i0 + (lane >> 2), j = j0 + 2 * (lane & 3);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    part[u][h] = t2[h] + (t1[h] + s22[i + (j + h) * ld]);
                    st1[i + (j + h) * ld] = t3[h];
                }
            }
            __syncthreads();
            // sa1 = that + X st1, the differences and their largest entry (cpsd.c:463-470)
            double bestv = -1.0;
            int besti = 0x7fffffff;
#pragma unroll
            for (int u = 0; u < TPW; ++u) {
                const int t = warp + u * NW;
                if (t >= nt) break;
                const int i0 = (t % (mp / 8)) * 8, j0 = (t / (mp / 8)) * 8;
                double t4[2];
                lag_tile_mma(c, st1, ld, mp, i0, j0, lane, t4);
                const int i = i0 + (lane >> 2), j = j0 + 2 * (lane & 3);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int o = i + (j + h) * ld;
                    const double v = t4[h] + part[u][h];
                    nx[o] = v;
                    if (i < m && j + h < m) {
                        const double d = v - c[o];
                        const int e = i + (j + h) * m;
                        dif[e] = d;
                        const double ad = fabs(d);
                        if (ad > bestv || (ad == bestv && e < besti)) {
                            bestv = ad;
                            besti = e;
                        }
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, bestv, o);
                int oi = __shfl_xor_sync(0xffffffffu, besti, o);
                if (ov > bestv || (ov == bestv && oi < besti)) {
                    bestv = ov;
                    besti = oi;
                }
            }
            if (lane == 0) {
                shv[warp] = bestv;
                shi[warp] = besti;
            }
            __syncthreads();
            // every thread combines the warp maxima in the same order and
            // takes the same decision: no third barrier for a broadcast
            bestv = shv[0];
            besti = shi[0];
#pragma unroll
            for (int w = 1; w < NW; ++w)
                if (shv[w] > bestv || (shv[w] == bestv && shi[w] < besti)) {
                    bestv = shv[w];
                    besti = shi[w];
                }
            // idamax returns an index in 1..kk even when every entry is
            // NaN: the sentinel must never reach the read below
            if (besti < 0 || (long)besti >= kk) besti = 0;
            // idamax's 1-based index used as 0-based (cpsd.c:471); past st1 lies
            // sa1, whose first entry is element (0, 0)
            const long nxi = (long)besti + 1;
            const double adiff = fabs(nxi < ne02 ? dif[nxi] : nx[nxi - ne02]);
            done = adiff < 1e-15;
            if (!done) cur ^= 1;
            // the next iteration writes st1, shv and shi only after its first barrier
        }
        if (!done && tid == 0) atomicAdd(a.fail, 1);
        // converged: sa1 is the buffer just written; stopped at 30: it was swapped into cur
        const double *fin = done ? X[cur ^ 1] : X[cur];
        for (long e = tid; e < kk; e += kLagThreads) a.lmd[ms * ne02 + e] = fin[(e % m) + (e / m) * ld];
        __syncthreads();
    }
}

// ------------------------------------------------- Lagrange, 2-D tiles
// lagrange_tile_kernel: the same fixed point as lagrange_kernel (cpsd.c:
// 439-478, including the idamax read and the 30-iteration limit) for up to
// 128 bands per spin, on a cluster of 4 x 4 CTAs.  CTA (p, q) owns the tile
// rows I_p x columns J_q (T = ceil(m / 4) of each) of sa0, sa1 and st1, and
// keeps its constant panels s21[I_p, :], s11[I_p, :], s12[:, J_q] and
// s22[I_p, J_q] in shared memory for all iterations.  Per iteration:
//   phase 1: gather sa0[I_p, :] and sa0[:, J_q] from the tiles of its row and
//            column (distributed shared memory), t = s22 + s21 sa0 + sa0 s12,
//            st1 = s11 sa0 on its tile;               cluster barrier;
//   phase 2: gather st1[:, J_q], sa1 = t + sa0 st1, st1 = sa1 - sa0, the
//            tile's argmax of |st1|;                  cluster barrier;
// then every CTA reduces the 16 candidates in rank order and reads the
// element after the maximum, as the reference does.  sa1 goes into the
// other half of a double-buffered tile, so the two barriers are all an
// iteration needs.
constexpr int kLagTileGrid = 4;  // 4 x 4 CTAs
constexpr int kLagTileMax = 128;

CPSD_HD size_t lagrange_tile_smem(int m)
{
    const size_t T = (size_t)(m + kLagTileGrid - 1) / kLagTileGrid;
    // S21r, S11r, S12c, Xr, Xc, STc: m*T each; S22t, STt: T*T; Xt: 2*T*T; slots
    return sizeof(double) * (6 * (size_t)m * T + 4 * T * T + 2 * kLagTileGrid * kLagTileGrid);
}

__global__ void __launch_bounds__(kLagThreads) lagrange_tile_kernel(LagArgs a)
{
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int p = rank / kLagTileGrid, q = rank % kLagTileGrid;
    const int tid = threadIdx.x;
    extern __shared__ double tsm[];
    const long ne02 = (long)a.ne0 * a.ne0;
    const int T = (a.ne0 + kLagTileGrid - 1) / kLagTileGrid;  // tile edge (sized for the larger spin)
    double *S21r = tsm, *S11r = S21r + (long)a.ne0 * T, *S12c = S11r + (long)a.ne0 * T;
    double *Xr = S12c + (long)a.ne0 * T, *Xc = Xr + (long)a.ne0 * T, *STc = Xc + (long)a.ne0 * T;
    double *S22t = STc + (long)a.ne0 * T, *STt = S22t + T * T, *Xt = STt + T * T;  // Xt: two halves
    double *slot = Xt + 2 * T * T;                                                 // [rank][2]
    for (int ms = 0; ms < a.ispin; ++ms) {
        const int m = ms ? a.ne1 : a.ne0;
        const long kk = (long)m * m;
        if (m == 0) continue;
        const int t = (m + kLagTileGrid - 1) / kLagTileGrid;  // this spin's tile edge
        const int i0 = p * t, j0 = q * t;
        const int nr = max(0, min(m, i0 + t) - i0), nc = max(0, min(m, j0 + t) - j0);
        const double *M22 = a.M22[ms], *M21 = a.M21[ms], *M11 = a.M11[ms];
        const double dte = a.dte;
        // s matrices, cpsd.c:420-437 (upper triangles mirrored as the reference does)
        for (long e = (long)rank * kLagThreads + tid; e < kk; e += (long)kLagTileGrid * kLagTileGrid * kLagThreads) {
            const int i = (int)(e % m), j = (int)(e / m);
            double v22, v21, v12, v11;
            if (i == j) {
                v22 = (1.0 - M22[(long)i * m + i]) * 0.5 / dte;
                v21 = (1.0 - M21[(long)i * m + i]) * 0.5;
                v12 = v21;
                v11 = -M11[(long)i * m + i] * 0.5 * dte;
            } else {
                const int lo = i < j ? i : j, hi = i < j ? j : i;
                v22 = -M22[(long)lo * m + hi] * 0.5 / dte;
                v21 = -M21[(long)lo * m + hi] * 0.5;   // <c2_lo|c1_hi>
                v12 = -M21[(long)hi * m + lo] * 0.5;   // <c1_lo|c2_hi>
                v11 = -M11[(long)lo * m + hi] * 0.5 * dte;
            }
            a.s22[e] = v22;
            a.s21[e] = v21;
            a.s12[e] = v12;
            a.s11[e] = v11;
        }
        cl.sync();
        // constant panels; sa0 = s22 (cpsd.c:441) into the first half of Xt
        for (int e = tid; e < m * t; e += kLagThreads) {
            const int l = e / t, ii = e % t;
            S21r[l * t + ii] = ii < nr ? a.s21[(i0 + ii) + (long)l * m] : 0.0;
            S11r[l * t + ii] = ii < nr ? a.s11[(i0 + ii) + (long)l * m] : 0.0;
            const int jj = e % t;
            S12c[l * t + jj] = jj < nc ? a.s12[l + (long)(j0 + jj) * m] : 0.0;
        }
        for (int e = tid; e < t * t; e += kLagThreads) {
            const int jj = e / t, ii = e % t;
            const double v = (ii < nr && jj < nc) ? a.s22[(i0 + ii) + (long)(j0 + jj) * m] : 0.0;
            S22t[jj * t + ii] = v;
            Xt[jj * t + ii] = v;
        }
        // thread -> one row ii of the tile and 4 of its columns
        const int ii = tid % 32, jq = (tid / 32) * 4;
        const bool rowok = ii < nr;
        int half = 0;  // which half of Xt holds sa0
        bool done = false;
        int iter = 0;
        cl.sync();  // every tile's sa0 is in place (later: ordered by the candidates' barrier)
        while (!done && iter < 30) {
            ++iter;
            // gather sa0[I_p, :] (Xr, [l][ii]) and sa0[:, J_q] (Xc, [l][jj])
            for (int g = 0; g < kLagTileGrid; ++g) {
                const double *rowt = cl.map_shared_rank(Xt + half * t * t, p * kLagTileGrid + g);
                const double *colt = cl.map_shared_rank(Xt + half * t * t, g * kLagTileGrid + q);
                for (int e = tid; e < t * t; e += kLagThreads) {
                    const int c = e / t, r = e % t;  // tile element (r, c), stored [c][r]
                    const int lr = g * t + c, lc = g * t + r;
                    if (lr < m) Xr[lr * t + r] = rowt[e];
                    if (lc < m) Xc[lc * t + c] = colt[e];
                }
            }
            __syncthreads();
            // t = s22 + s21 sa0 + sa0 s12 ; st1 = s11 sa0   (cpsd.c:444-462)
            double t1[4], t2[4], st[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) t1[k] = t2[k] = st[k] = 0.0;
            if (rowok)
                for (int l = 0; l < m; ++l) {
                    const double a21 = S21r[l * t + ii], a11 = S11r[l * t + ii], xil = Xr[l * t + ii];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const double xlj = Xc[l * t + jq + k];
                        t1[k] = fma(a21, xlj, t1[k]);
                        t2[k] = fma(xil, S12c[l * t + jq + k], t2[k]);
                        st[k] = fma(a11, xlj, st[k]);
                    }
                }
            // (rows ii >= t are not in the tile: their slots belong to the next column)
            if (ii < t) {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (jq + k < t) STt[(jq + k) * t + ii] = st[k];
            }
            cl.sync();  // every tile's st1 = s11 sa0 is in place
            for (int g = 0; g < kLagTileGrid; ++g) {
                const double *stt = cl.map_shared_rank(STt, g * kLagTileGrid + q);
                for (int e = tid; e < t * t; e += kLagThreads) {
                    const int c = e / t, r = e % t;
                    const int lc = g * t + r;
                    if (lc < m) STc[lc * t + c] = stt[e];
                }
            }
            __syncthreads();
            // sa1 += sa0 st1 (cpsd.c:463-468); st1 = sa1 - sa0 (:469-470)
            double s2[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) s2[k] = 0.0;
            if (rowok)
                for (int l = 0; l < m; ++l) {
                    const double xil = Xr[l * t + ii];
#pragma unroll
                    for (int k = 0; k < 4; ++k) s2[k] = fma(xil, STc[l * t + jq + k], s2[k]);
                }
            double bestv = -1.0;
            long besti = 0x7fffffff;
            double *nxt = Xt + (half ^ 1) * t * t;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int jj = jq + k;
                if (rowok && jj < nc) {
                    // sa1 = s22, += s21 sa0, += sa0 s12, += sa0 st1: the
                    // order of lagrange_kernel
                    const double sa1 = s2[k] + (t2[k] + (t1[k] + S22t[jj * t + ii]));
                    const long f = (i0 + ii) + (long)(j0 + jj) * m;
                    nxt[jj * t + ii] = sa1;
                    a.X1[f] = sa1;
                    const double d = sa1 - Xt[half * t * t + jj * t + ii];
                    a.st1[f] = d;
                    const double ad = fabs(d);
                    if (ad > bestv || (ad == bestv && f < besti)) {
                        bestv = ad;
                        besti = f;
                    }
                }
            }
            // tile argmax (first column-major index of the largest |st1|, as idamax)
            __shared__ double shv[kLagThreads / 32];
            __shared__ long shi[kLagThreads / 32];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, bestv, o);
                const long oi = __shfl_xor_sync(0xffffffffu, besti, o);
                if (ov > bestv || (ov == bestv && oi < besti)) {
                    bestv = ov;
                    besti = oi;
                }
            }
            if ((tid & 31) == 0) {
                shv[tid >> 5] = bestv;
                shi[tid >> 5] = besti;
            }
            __syncthreads();
            if (tid == 0) {
                for (int w = 1; w < kLagThreads / 32; ++w)
                    if (shv[w] > bestv || (shv[w] == bestv && shi[w] < besti)) {
                        bestv = shv[w];
                        besti = shi[w];
                    }
                slot[2 * rank] = bestv;
                slot[2 * rank + 1] = (double)besti;
            }
            cl.sync();  // every tile's candidate, st1 and sa1 are in place
            double gv = -1.0;
            long gi = 0x7fffffff;
            for (int r = 0; r < kLagTileGrid * kLagTileGrid; ++r) {
                const double *sl = cl.map_shared_rank(slot, r);
                const double v = sl[0];
                const long ix = (long)sl[1];
                if (v > gv || (v == gv && ix < gi)) {
                    gv = v;
                    gi = ix;
                }
            }
            // idamax returns an index in 1..kk even when every entry is NaN
            if (gi < 0 || gi >= kk) gi = 0;
            // the reference reads st1 at idamax's 1-based result (cpsd.c:471):
            // the element after the largest; past the end of st1 lies sa1
            const long nx = gi + 1;
            const double adiff = fabs(nx < ne02 ? a.st1[nx] : a.X1[nx - ne02]);
            done = adiff < 1e-15;
            half ^= 1;  // sa1 becomes sa0 (when done, it is the result)
        }
        if (!done && rank == 0 && tid == 0) atomicAdd(a.fail, 1);
        // lmd = the last sa1 (cpsd.c:478)
        const double *fin = Xt + half * t * t;
        for (int e = tid; e < t * t; e += kLagThreads) {
            const int jj = e / t, r = e % t;
            if (r < nr && jj < nc) a.lmd[ms * ne02 + (i0 + r) + (long)(j0 + jj) * m] = fin[e];
        }
        cl.sync();  // the slots and tiles are reused by the next spin
    }
}

// ------------------------------------------------------------ energies
// per-block partial sums over packed points of the three single-field terms
// (cpsd.c:520-526 k-space Ewald, :548-554 Hartree, :590 local)
__global__ void packed_terms_kernel(int npw, const double *__restrict__ w, const cx<double> *__restrict__ s,
                                    const double *__restrict__ vg, const cx<double> *__restrict__ dng,
                                    const double *__restrict__ vc, const cx<double> *__restrict__ vall,
                                    double *part)
{
    __shared__ double sh[32];
    double e0 = 0, e1 = 0, e2 = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npw; p += gridDim.x * blockDim.x) {
        const double ww = w[p];
        const cx<double> sv = s[p], d = dng[p], va = vall[p];
        e0 += ww * (sv.x * sv.x + sv.y * sv.y) * vg[p];
        e1 += ww * (d.x * d.x + d.y * d.y) * vc[p];
        e2 += ww * (va.x * d.x + va.y * d.y);
    }
    double r0 = block_sum<256>(e0, sh);
    double r1 = block_sum<256>(e1, sh);
    double r2 = block_sum<256>(e2, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = r0;
        part[gridDim.x + blockIdx.x] = r1;
        part[2 * gridDim.x + blockIdx.x] = r2;
    }
}

// per band: eke_b = sum w tg |c1|^2 (cpsd.c:574-586), dc_b = sum w |c2-c1|^2 (:650-659)
__global__ void band_terms_kernel(int npw, long ldc, const double *__restrict__ w,
                                  const double *__restrict__ tg, const cx<double> *__restrict__ c1,
                                  const cx<double> *__restrict__ c2, double *part /* [2][nb][blocks] */)
{
    __shared__ double sh[32];
    const int b = blockIdx.y;
    const cx<double> *a = c1 + (long)b * ldc, *c = c2 + (long)b * ldc;
    double ek = 0, dc = 0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npw; p += gridDim.x * blockDim.x) {
        const double ww = w[p];
        const cx<double> x = a[p], y = c[p];
        ek += ww * tg[p] * (x.x * x.x + x.y * x.y);
        const double dx = y.x - x.x, dy = y.y - x.y;
        dc += ww * (dx * dx + dy * dy);
    }
    double r0 = block_sum<256>(ek, sh);
    double r1 = block_sum<256>(dc, sh);
    if (threadIdx.x == 0) {
        part[(long)b * gridDim.x + blockIdx.x] = r0;
        part[((long)gridDim.y + b) * gridDim.x + blockIdx.x] = r1;
    }
}

// exc, pxc partial sums over the real grid (cpsd.c:557-570)
__global__ void grid_terms_kernel(long n3, int ispin, const double *__restrict__ dn,
                                  const double *__restrict__ xce, const double *__restrict__ xcp,
                                  double *part)
{
    __shared__ double sh[32];
    double ex = 0, px = 0;
    for (long r = (long)blockIdx.x * blockDim.x + threadIdx.x; r < n3; r += (long)gridDim.x * blockDim.x) {
        const double d0 = dn[r];
        ex += d0 * xce[r];
        px += d0 * xcp[r];
        if (ispin == 2) {
            const double d1 = dn[n3 + r];
            ex += d1 * xce[r];
            px += d1 * xcp[n3 + r];
        }
    }
    double r0 = block_sum<256>(ex, sh);
    double r1 = block_sum<256>(px, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = r0;
        part[gridDim.x + blockIdx.x] = r1;
    }
}

// hml from M[i][j] = <c1_i|cpsi_j> (row-major per spin), with the reference's
// mirroring and eorbit reads (cpsd.c:497-515); one thread.
struct FinalArgs {
    int ispin, ne0, ne1, nion, nsh, nproj, nb, inner;
    int pblocks, bblocks, gblocks;
    const double *ppart, *bpart, *gpart;
    const double *Mh[2];
    double *hml;
    const double *beta, *vnlnrm_p;
    const double *ewald_part;  // real-space Ewald sum per ion (ewald_real_kernel)
    double scal2, omega, dv, cewald, rcut, dt, dte;
    double *E;  // in: E[0] previous energy; out: E[0..9], E[10] deltae, E[11] deltac
};

// Real-space Ewald sum, cpsd.c:527-545 (A&S 7.1.28 erfc, cpsd.c:11-17): block
// ii sums the pairs (ii, jj > ii) over the nsh image cells, one (pair, image)
// term per thread, and writes a fixed-order block sum to part[ii].
__global__ void __launch_bounds__(256) ewald_real_kernel(int nion, int nsh, const double *__restrict__ r1,
                                                         const double *__restrict__ rcell,
                                                         const double *__restrict__ zv,
                                                         const int *__restrict__ katm, double rcut,
                                                         double *__restrict__ part)
{
    __shared__ double sh[32];
    const double B1 = 0.0705230784, B2 = 0.0422820123, B3 = 0.0092705272;
    const double B4 = 0.0001520143, B5 = 0.0002765672, B6 = 0.0000430638;
    const int ii = blockIdx.x;
    const long cnt = (long)(nion - 1 - ii) * nsh;
    double ew = 0.0;
    for (long e = threadIdx.x; e < cnt; e += 256) {
        const int jj = ii + 1 + (int)(e / nsh);
        const int l = (int)(e % nsh);
        const double dx = r1[3 * ii] - r1[3 * jj];
        const double dy = r1[1 + 3 * ii] - r1[1 + 3 * jj];
        const double dz = r1[2 + 3 * ii] - r1[2 + 3 * jj];
        const double zz = zv[katm[ii]] * zv[katm[jj]];
        const double x = rcell[l] + dx, y = rcell[l + nsh] + dy, z = rcell[l + 2 * nsh] + dz;
        const double r = sqrt(x * x + y * y + z * z);
        const double w = r / rcut;
        const double aa = (1.0 + w * (B1 + w * (B2 + w * (B3 + w * (B4 + w * (B5 + w * B6))))));
        const double erfc = 1.0 / (aa * aa * aa * aa);
        ew += zz * (erfc * erfc * erfc * erfc) / r;
    }
    const double t = block_sum<256>(ew, sh);
    if (threadIdx.x == 0) part[ii] = t;
}

// One block of kFinalThreads: every sum is a fixed-order block reduction, so
// the energies are bitwise reproducible run to run.
constexpr int kFinalThreads = 256;

__global__ void __launch_bounds__(kFinalThreads) final_energy_kernel(FinalArgs a)
{
    __shared__ double sh[32];
    const int tid = threadIdx.x;
    const long ne02 = (long)a.ne0 * a.ne0;
    // hml (cpsd.c:497-513): the upper triangle is -<c1_i|cpsi_j>, mirrored; the
    // mirror and eorbit read hml at the spin-0 offset for both spins
    double eo = 0.0;
    for (int ms = 0; ms < a.ispin; ++ms) {
        const int m = ms ? a.ne1 : a.ne0;
        double *H = a.hml + ms * ne02;
        const double *M = a.Mh[ms];
        for (int e = tid; e < m * m; e += kFinalThreads) {
            const int i = e % m, j = e / m;
            if (i <= j) H[i + j * m] = -M[(long)i * m + j];
        }
        __syncthreads();
        for (int e = tid; e < m * m; e += kFinalThreads) {
            const int i = e % m, j = e / m;
            if (i < j) H[j + i * m] = a.hml[i + j * m];
        }
        for (int i = tid; i < m; i += kFinalThreads) eo += a.hml[i + i * m];
        __syncthreads();
    }
    double eorbit = block_sum<kFinalThreads>(eo, sh);
    // single-field packed terms
    double t[3];
    for (int q = 0; q < 3; ++q) {
        double v = 0.0;
        for (int k = tid; k < a.pblocks; k += kFinalThreads) v += a.ppart[q * a.pblocks + k];
        t[q] = block_sum<kFinalThreads>(v, sh);
    }
    // real-space Ewald: per-ion partials of ewald_real_kernel, summed in ion order
    double eion_real = 0.0;
    if (tid == 0)
        for (int ii = 0; ii < a.nion; ++ii) eion_real += a.ewald_part[ii];
    // xc
    double ex = 0.0, px = 0.0;
    for (int k = tid; k < a.gblocks; k += kFinalThreads) {
        ex += a.gpart[k];
        px += a.gpart[a.gblocks + k];
    }
    double exc = block_sum<kFinalThreads>(ex, sh);
    double pxc = block_sum<kFinalThreads>(px, sh);
    // kinetic and deltac per band
    double ek = 0.0, dcmax = 0.0;
    for (int b = tid; b < a.nb; b += kFinalThreads) {
        double s1 = 0.0, s2 = 0.0;
        for (int k = 0; k < a.bblocks; ++k) {
            s1 += a.bpart[(long)b * a.bblocks + k];
            s2 += a.bpart[((long)a.nb + b) * a.bblocks + k];
        }
        ek += s1;
        dcmax = fmax(dcmax, s2);
    }
    double eke = block_sum<kFinalThreads>(ek, sh);
    // max over threads (order-independent)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dcmax = fmax(dcmax, __shfl_xor_sync(0xffffffffu, dcmax, o));
    __syncthreads();
    if ((tid & 31) == 0) sh[tid >> 5] = dcmax;
    __syncthreads();
    double dc = 0.0;
    if (tid == 0)
        for (int i = 0; i < kFinalThreads / 32; ++i) dc = fmax(dc, sh[i]);
    __syncthreads();
    // nonlocal energy from the last step's projections, cpsd.c:593-634
    double en = 0.0;
    for (long e = tid; e < (long)a.nproj * a.nb; e += kFinalThreads) {
        const double sw = a.beta[e];
        en += sw * sw * a.scal2 / a.vnlnrm_p[e / a.nb];
    }
    double enl = block_sum<kFinalThreads>(en, sh);
    if (tid != 0) return;
    if (a.ispin == 1) eorbit *= 2;
    const double eion = t[0] * 0.5 * a.scal2 + a.cewald + eion_real;
    const double ehartr = t[1] * a.omega * 0.5;
    const double elocal = t[2];
    if (a.ispin == 1) {
        exc += exc;
        pxc += pxc;
    }
    exc *= a.dv;
    pxc *= a.dv;
    if (a.ispin == 1) eke = 2 * eke;
    if (a.ispin == 1) enl = 2 * enl;
    const double eold = a.E[0];
    a.E[0] = eorbit + eion + exc - ehartr - pxc;
    a.E[1] = eorbit;
    a.E[2] = ehartr;
    a.E[3] = exc;
    a.E[4] = eion;
    a.E[5] = eke;
    a.E[6] = elocal;
    a.E[7] = enl;
    a.E[8] = 2.0 * ehartr;
    a.E[9] = pxc;
    a.E[10] = (a.E[0] - eold) / (a.dt * a.inner);
    a.E[11] = dc / a.dte;
}

// ------------------------------------------------------------ epilogue eigenpairs
// ccpsdv3/main.c:470-481: per spin, dsyev('V','U') of hml, then eigsrt
// (ccpsdv3/eigsrt.c:9-36: selection sort into descending order, ties to the
// later index, eigenvector columns moved with their values).  Here: cyclic
// Jacobi, rounds of the round-robin pair order (n/2 disjoint pairs per
// round, n padded to even with an idle index), so one round's rotations run
// in parallel: rows of A, then columns of A and V.  Rotation and thresholds
// follow the classical scheme (Rutishauser; as in Numerical Recipes
// "jacobi"): t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)), theta =
// (a_qq - a_pp) / (2 a_pq); in the first sweeps only |a_pq| above 0.2 S / n^2
// (S = sum of |a_ij|, i < j) rotate; from the fifth sweep on an a_pq that
// no longer changes a_pp or a_qq (|a_pp| + 100 |a_pq| == |a_pp|, the same
// for a_qq) is set to zero.  The sweeps end when S is zero.  One CTA per
// spin; A and V (column-major, ld n) live in global memory (L2).
constexpr int kEigThreads = 1024, kEigMaxSweeps = 60;

struct EigArgs {
    const double *hml;   // per spin ms at hml + ms*ne0*ne0, column-major, ld ne[ms]; upper triangle read
    int ne[2], ne0;
    double *A, *V;       // workspace: per spin ne0*ne0 each
    double *eig;         // eig[ms*ne0 + i], descending
    double *vec;         // eigenvectors in hml's layout, columns in eig's order
    int *sweeps;         // per spin: sweeps run (kEigMaxSweeps + 1: not converged)
};

__global__ void __launch_bounds__(kEigThreads) jacobi_eig_kernel(EigArgs a)
{
    __shared__ double rc[128], rs[128], rapp[128], raqq[128], rt[128], red[32];
    __shared__ int rp[128], rq[128], perm[256];
    __shared__ double sum_off;
    const int ms = blockIdx.x, n = a.ne[ms], tid = threadIdx.x;
    if (n <= 0) return;
    const long off = (long)ms * a.ne0 * a.ne0;
    const double *H = a.hml + off;
    double *A = a.A + off, *V = a.V + off;
    for (long e = tid; e < (long)n * n; e += kEigThreads) {
        const int i = (int)(e % n), j = (int)(e / n);
        A[e] = (i <= j) ? H[i + (long)j * n] : H[j + (long)i * n];
        V[e] = (i == j) ? 1.0 : 0.0;
    }
    __syncthreads();
    const int np = n + (n & 1), half = np / 2, m1 = np - 1;
    int sweep = 1;
    for (; sweep <= kEigMaxSweeps; ++sweep) {
        // S = sum_{i<j} |a_ij|
        double v = 0.0;
        for (long e = tid; e < (long)n * n; e += kEigThreads) {
            const int i = (int)(e % n), j = (int)(e / n);
            if (i < j) v += fabs(A[e]);
        }
        v = block_sum<kEigThreads>(v, red);
        if (tid == 0) sum_off = v;
        __syncthreads();
        const double S = sum_off;
        if (S == 0.0) break;
        const double tresh = (sweep < 4) ? 0.2 * S / ((double)n * n) : 0.0;
        for (int r = 0; r < m1; ++r) {
            if (tid < half) {
                int p, q;
                if (tid == 0) {
                    p = 0;
                    q = 1 + r;
                } else {
                    p = 1 + (r + tid) % m1;
                    q = 1 + (r - tid + m1) % m1;
                }
                if (p > q) {
                    const int x = p;
                    p = q;
                    q = x;
                }
                double c = 1.0, s = 0.0, t = 0.0;
                bool rot = false;
                if (q < n) {
                    const double app = A[p + (long)p * n], aqq = A[q + (long)q * n], apq = A[p + (long)q * n];
                    const double g = 100.0 * fabs(apq);
                    if (sweep > 4 && fabs(app) + g == fabs(app) && fabs(aqq) + g == fabs(aqq)) {
                        A[p + (long)q * n] = 0.0;
                        A[q + (long)p * n] = 0.0;
                    } else if (fabs(apq) > tresh && apq != 0.0) {
                        const double h = aqq - app;
                        if (fabs(h) + g == fabs(h)) {
                            t = apq / h;
                        } else {
                            const double theta = 0.5 * h / apq;
                            t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
                            if (theta < 0.0) t = -t;
                        }
                        c = 1.0 / sqrt(1.0 + t * t);
                        s = t * c;
                        rot = true;
                        rapp[tid] = app;
                        raqq[tid] = aqq;
                        rt[tid] = t * apq;
                    }
                }
                rp[tid] = rot ? p : -1;
                rq[tid] = q;
                rc[tid] = c;
                rs[tid] = s;
            }
            __syncthreads();
            // rows p, q of A: A <- P^T A
            for (long e = tid; e < (long)half * n; e += kEigThreads) {
                const int k = (int)(e / n), j = (int)(e % n), p = rp[k];
                if (p < 0) continue;
                const int q = rq[k];
                const double c = rc[k], s = rs[k];
                const double ap = A[p + (long)j * n], aq = A[q + (long)j * n];
                A[p + (long)j * n] = c * ap - s * aq;
                A[q + (long)j * n] = s * ap + c * aq;
            }
            __syncthreads();
            // columns p, q of A and V: A <- A P, V <- V P
            for (long e = tid; e < (long)half * n; e += kEigThreads) {
                const int k = (int)(e / n), i = (int)(e % n), p = rp[k];
                if (p < 0) continue;
                const int q = rq[k];
                const double c = rc[k], s = rs[k];
                double *cp = A + (long)p * n, *cq = A + (long)q * n;
                double x = cp[i], y = cq[i];
                cp[i] = c * x - s * y;
                cq[i] = s * x + c * y;
                cp = V + (long)p * n;
                cq = V + (long)q * n;
                x = cp[i];
                y = cq[i];
                cp[i] = c * x - s * y;
                cq[i] = s * x + c * y;
            }
            __syncthreads();
            // the rotated 2 x 2 blocks (touched by their own rotation only):
            // a_pp - t a_pq, a_qq + t a_pq and exact zeros off the diagonal
            if (tid < half && rp[tid] >= 0) {
                const int p = rp[tid], q = rq[tid];
                A[p + (long)p * n] = rapp[tid] - rt[tid];
                A[q + (long)q * n] = raqq[tid] + rt[tid];
                A[p + (long)q * n] = 0.0;
                A[q + (long)p * n] = 0.0;
            }
            __syncthreads();
        }
        // restore exact symmetry from the upper triangle
        for (long e = tid; e < (long)n * n; e += kEigThreads) {
            const int i = (int)(e % n), j = (int)(e / n);
            if (i > j) A[e] = A[j + (long)i * n];
        }
        __syncthreads();
    }
    // eigsrt: descending selection sort, ties to the later index
    if (tid == 0) {
        for (int i = 0; i < n; ++i) perm[i] = i;
        for (int i = 0; i < n - 1; ++i) {
            int k = i;
            double p = A[perm[i] + (long)perm[i] * n];
            for (int j = i + 1; j < n; ++j) {
                const double d = A[perm[j] + (long)perm[j] * n];
                if (d >= p) {
                    k = j;
                    p = d;
                }
            }
            if (k != i) {
                const int x = perm[i];
                perm[i] = perm[k];
                perm[k] = x;
            }
        }
        a.sweeps[ms] = sweep;
    }
    __syncthreads();
    for (int i = tid; i < n; i += kEigThreads) a.eig[(long)ms * a.ne0 + i] = A[perm[i] + (long)perm[i] * n];
    for (long e = tid; e < (long)n * n; e += kEigThreads) {
        const int i = (int)(e % n), j = (int)(e / n);
        a.vec[off + i + (long)j * n] = V[i + (long)perm[j] * n];
    }
}
