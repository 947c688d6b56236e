// capi.cu -- the reference-facing entry points of include/cpsd_b200.h:
// cpsd() / cpsd_gpu_cpsd() (ccpsdv3/cpsd.c:33-71), the Fortran-ABI
// cr_fft3b_ / rc_fft3f_ (fftpack3d/fftpack3d.f:22-196), the input pipeline
// (kbpp() of ckbppv3/dkbppv3.c, cmakepsi/dmakepsi.c) and the epilogue's
// ELCOUT / IONOUT writers (ccpsdv3/main.c:537-566).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "cpsd_b200.h"
#include "fft.cuh"
#include "dropin.h"
#include "host_pool.h"
#include "pipeline.cuh"

namespace {

std::mutex g_mu;
cpsd_gpu_ctx *g_ctx = nullptr;
struct Signature {
    int nfft = 0, ispin = 0, ne0 = 0, ne1 = 0, nion = 0, nkatm = 0, nsh = 0, device = -1;
    std::vector<int> masker1;
    std::vector<int> masker;  // as passed (every value twice, main.c:189-195)
    bool same_shape(const Signature &o) const
    {
        return nfft == o.nfft && ispin == o.ispin && ne0 == o.ne0 && ne1 == o.ne1 && nion == o.nion &&
               nkatm == o.nkatm && nsh == o.nsh && device == o.device;
    }
    // the caller's mask against the context's, compared in slices on the
    // host threads (it is read every call: 2 nfft3d ints)
    bool same_mask(const int *m, int nfft3d) const
    {
        const size_t n = (size_t)2 * nfft3d;
        if (masker.size() != n) return false;
        constexpr int kSlices = 32;
        std::atomic<int> diff{0};
        cpsd_host::Pool::get().run(kSlices, [&](int t) {
            const size_t a = n * t / kSlices, b = n * (t + 1) / kSlices;
            if (memcmp(m + a, masker.data() + a, sizeof(int) * (b - a))) diff = 1;
        });
        return diff.load() == 0;
    }
};
Signature g_sig;


}  // namespace

extern "C" int cpsd_gpu_cpsd(const int inner, const int move, const int nion, const int ispin, const int *ne,
                             const int nfft, const int nfft3d, const int n2ft3d, const double *unitg,
                             const double omega, const double dt, const double fmass, const int *katm,
                             const double *amass, const double *zv, const int nsh, const double *rcell,
                             const double cewald, const double rcut, const int *masker, const double *G,
                             const double *tg, const double *vc, const double *vg, const int *lmmax,
                             const double *vnlnrm, const double *vl, const double *vnl, double *r1, double *r2,
                             double *fion, double *c1, double *c2, double *cpsi, double *dn, double *hml,
                             double *lmd, double *E, double *deltae, double *deltac, double *deltar)
{
    if (!ne || !unitg || !masker || !c2 || !E) return CPSD_ERR_ARG;
    const int nh = nfft / 2 + 1;
    if (nfft <= 0 || nfft3d != nh * nfft * nfft || n2ft3d != (nfft + 2) * nfft * nfft) return CPSD_ERR_ARG;
    int nkatm = 1;
    for (int ii = 0; ii < nion; ++ii) nkatm = std::max(nkatm, katm[ii] + 1);
    Signature sig;
    sig.nfft = nfft;
    sig.ispin = ispin;
    sig.ne0 = ne[0];
    sig.ne1 = ispin == 2 ? ne[1] : 0;
    sig.nion = nion;
    sig.nkatm = nkatm;
    sig.nsh = nsh;
    cudaGetDevice(&sig.device);

    std::lock_guard<std::mutex> lk(g_mu);
    if (g_ctx && sig.same_shape(g_sig)) {
        // a driver's loop passes the same mask and tables every call
        // (main.c:422-426): run on the context's, and check them on host
        // threads beside the steps; a mismatch discards the run and takes
        // the full path below
        int rc = cpsd_gpu_set_scalars(g_ctx, unitg, omega, dt, fmass, cewald, rcut);
        if (rc) return rc;
        const DropinCheck check{masker, g_sig.masker.data(), g_sig.masker.size(),
                                TableArgs{katm, amass, zv, rcell, G, tg, vc, vg, lmmax, vnlnrm, vl, vnl}};
        rc = cpsd_dropin_state_run_fetch(g_ctx, r2, inner, move, E, deltae, deltac, deltar, c1, c2, cpsi, dn, hml,
                                         lmd, r1, r2, fion, &check);
        if (rc != kDropinRedo) return rc;
    }
    if (!g_ctx || !sig.same_shape(g_sig) || !g_sig.same_mask(masker, nfft3d)) {
        sig.masker1.resize(nfft3d);
        for (int k = 0; k < nfft3d; ++k) sig.masker1[k] = masker[2 * k];
        sig.masker.assign(masker, masker + (size_t)2 * nfft3d);
        if (g_ctx) cpsd_gpu_destroy(g_ctx);
        g_ctx = nullptr;
        cpsd_gpu_params p{};
        p.nfft = nfft;
        p.ispin = ispin;
        p.ne[0] = sig.ne0;
        p.ne[1] = sig.ne1;
        p.nion = nion;
        p.nkatm = nkatm;
        p.nsh = nsh;
        p.precision = CPSD_PREC_FP64;
        p.device = sig.device;
        memcpy(p.unitg, unitg, sizeof(p.unitg));
        p.omega = omega;
        p.dt = dt;
        p.fmass = fmass;
        p.cewald = cewald;
        p.rcut = rcut;
        int rc = cpsd_gpu_create(&p, sig.masker1.data(), &g_ctx);
        if (rc) return rc;
        g_sig = sig;
    }
    // per-call scalars (the reference passes them every call)
    cpsd_gpu_ctx *c = g_ctx;
    int rc = cpsd_gpu_set_scalars(c, unitg, omega, dt, fmass, cewald, rcut);
    if (rc) return rc;
    rc = cpsd_gpu_set_tables(c, katm, amass, zv, rcell, G, tg, vc, vg, lmmax, vnlnrm, vl, vnl);
    if (rc) return rc;
    return cpsd_dropin_state_run_fetch(c, r2, inner, move, E, deltae, deltac, deltar, c1, c2, cpsi, dn, hml, lmd,
                                       r1, r2, fion, nullptr);
}

extern "C" cpsd_gpu_ctx *cpsd_gpu_dropin_context(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_ctx;
}

extern "C" void cpsd(const int inner, const int move, const int nion, const int ispin, const int *ne,
                     const int nfft, const int nfft3d, const int n2ft3d, const double *unitg, const double omega,
                     const double dt, const double fmass, const int *katm, const double *amass, const double *zv,
                     const int nsh, const double *rcell, const double cewald, const double rcut,
                     const int *masker, const double *G, const double *tg, const double *vc, const double *vg,
                     int *lmmax, double *vnlnrm, double *vl, double *vnl, double *r1, double *r2, double *fion,
                     double *c1, double *c2, double *cpsi, double *dn, double *hml, double *lmd,
                     double *cpsdwork, double *E, double *deltae, double *deltac, double *deltar)
{
    (void)cpsdwork;
    const int rc = cpsd_gpu_cpsd(inner, move, nion, ispin, ne, nfft, nfft3d, n2ft3d, unitg, omega, dt, fmass,
                                 katm, amass, zv, nsh, rcell, cewald, rcut, masker, G, tg, vc, vg, lmmax, vnlnrm,
                                 vl, vnl, r1, r2, fion, c1, c2, cpsi, dn, hml, lmd, E, deltae, deltac, deltar);
    if (rc == CPSD_WARN_LAGRANGE)
        printf("ierr=10\n");  // the reference's message for the same condition (cpsd.c:477)
    else if (rc != CPSD_OK)
        printf("cpsd (B200): error %d: %s\n", rc, cpsd_gpu_strerror(rc));
}

// ====================================================================== input pipeline
namespace {

// simp() of ckbppv3/dkbppv3.c, in its order of operations
double host_simp(int n, const double *y, double h)
{
    double s2 = 0.0, s4 = 0.0;
    for (int i = 0; i < n; i += 2) s2 += y[i];
    for (int i = 1; i < n; i += 2) s4 += y[i];
    double s = 2.0 * s2 + 4.0 * s4 - y[0] - y[n - 1];
    return s * (h / 3.0);
}

struct DevBuf {
    double *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
};

}  // namespace

extern "C" int cpsd_gpu_kbpp(double zv, int lmax, int nrho, double drho, const double *rho, double *vp,
                             const double *wp, int nfft3d, const double *G, double *vl, double *vnl,
                             double *vnlnrm)
{
    if (lmax < 0 || lmax > 3 || nrho < 2 || nrho > kKbppMaxRho || nfft3d < 1 || !rho || !vp || !wp || !G ||
        !vl || (lmax > 0 && (!vnl || !vnlnrm)))
        return CPSD_ERR_ARG;
    const long N = nfft3d, n = nrho, lmmax = (long)lmax * lmax;
    // kbpp(): nonlocal channels relative to the local one, then their norms
    for (int l = 0; l < lmax; ++l)
        for (long i = 0; i < n; ++i) vp[i + l * n] -= vp[i + lmax * n];
    std::vector<double> f(n);
    for (int l = 0; l < lmax; ++l) {
        for (long i = 0; i < n; ++i) f[i] = vp[i + l * n] * wp[i + l * n] * wp[i + l * n];
        const double a = host_simp(nrho, f.data(), drho);
        for (int i = l * l; i < (l + 1) * (l + 1); ++i) vnlnrm[i] = a;
    }
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return CPSD_ERR_CUDA;
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    DevBuf dr, dvp, dwp, dG, dvl, dvnl;
    const size_t tab = sizeof(double) * (lmax + 1) * n;
    if (cudaMalloc(&dr.p, sizeof(double) * n) != cudaSuccess || cudaMalloc(&dvp.p, tab) != cudaSuccess ||
        cudaMalloc(&dwp.p, tab) != cudaSuccess || cudaMalloc(&dG.p, sizeof(double) * 3 * N) != cudaSuccess ||
        cudaMalloc(&dvl.p, sizeof(double) * N) != cudaSuccess ||
        (lmmax > 0 && cudaMalloc(&dvnl.p, sizeof(double) * lmmax * N) != cudaSuccess))
        return CPSD_ERR_CUDA;
    if (cudaMemcpyAsync(dr.p, rho, sizeof(double) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dvp.p, vp, tab, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dwp.p, wp, tab, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(dG.p, G, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s) != cudaSuccess)
        return CPSD_ERR_CUDA;
    const size_t smem = kbpp_smem_bytes(nrho);
    if (cudaFuncSetAttribute(kbpp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return CPSD_ERR_CUDA;
    KbppArgs a{};
    a.nfft3d = nfft3d;
    a.nrho = nrho;
    a.lmax = lmax;
    a.drho = drho;
    a.zv = zv;
    a.rho = dr.p;
    a.vp = dvp.p;
    a.wp = dwp.p;
    a.G = dG.p;
    a.vl = dvl.p;
    a.vnl = dvnl.p;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return CPSD_ERR_CUDA;
    const long blocks = std::max<long>(1, std::min<long>((N + kKbppThreads - 1) / kKbppThreads, (long)sms * 16));
    kbpp_kernel<<<(unsigned)blocks, kKbppThreads, smem, s>>>(a);
    if (cudaGetLastError() != cudaSuccess) return CPSD_ERR_CUDA;
    if (cudaMemcpyAsync(vl, dvl.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        (lmmax > 0 &&
         cudaMemcpyAsync(vnl, dvnl.p, sizeof(double) * lmmax * N, cudaMemcpyDeviceToHost, s) != cudaSuccess))
        return CPSD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CPSD_ERR_CUDA;
    return CPSD_OK;
}

extern "C" int cpsd_makepsi(int nfft, int ispin, const int *ne, const int *waves, double *psi)
{
    if (nfft < 2 || (nfft & 1) || (ispin != 1 && ispin != 2) || !ne || !waves || !psi || ne[0] < 0 ||
        ne[1] < 0 || (ispin == 2 && ne[1] > ne[0]))
        return CPSD_ERR_ARG;
    const int nh = nfft / 2 + 1;
    const long nfft3 = (long)(nfft + 2) * nfft * nfft;
    // PSI0.DAT rows "i j k l" (cmakepsi/dmakepsi.c:93-107): G index and the
    // coefficient: l < 0 -> i/sqrt(2), l == 0 -> 1, l > 0 -> 1/sqrt(2)
    const double scale = 1.0 / sqrt(2.0);
    for (int n = 0; n < ne[0]; ++n) {
        const int i = waves[4 * n], j = waves[4 * n + 1], k = waves[4 * n + 2];
        if (i < 0 || i >= nh || j <= -nfft || j >= nfft || k <= -nfft || k >= nfft) return CPSD_ERR_ARG;
    }
    double *band = psi;
    for (int ms = 0; ms < ispin; ++ms)
        for (int n = 0; n < (ms ? ne[1] : ne[0]); ++n) {  // spin 1 reuses the first ne[1] rows (dmakepsi.c:117)
            const int *w = waves + 4 * n;
            const int k1 = w[0], k2 = (w[1] + nfft) % nfft, k3 = (w[2] + nfft) % nfft, l = w[3];
            const double re = l < 0 ? 0.0 : (l == 0 ? 1.0 : scale), im = l < 0 ? scale : 0.0;
            memset(band, 0, sizeof(double) * nfft3);
            long idx = 2L * (k1 + (long)k2 * nh + (long)k3 * nh * nfft);
            band[idx] = re;
            band[idx + 1] = im;
            if (k1 == 0) {  // the Hermitian partner on the kx = 0 plane
                const int kk2 = (nfft - k2) % nfft, kk3 = (nfft - k3) % nfft;
                idx = 2L * (k1 + (long)kk2 * nh + (long)kk3 * nh * nfft);
                band[idx] = re;
                band[idx + 1] = -im;
            }
            band += nfft3;
        }
    return CPSD_OK;
}

// ====================================================================== epilogue files
extern "C" int cpsd_write_elcout(const char *path, int icube, int nfft, double unit, int ispin, const int *ne,
                                 const double *c1)
{
    if (!path || !ne || !c1 || nfft <= 0 || ne[0] < 0 || ne[1] < 0) return CPSD_ERR_ARG;
    FILE *fp = fopen(path, "wb");
    if (!fp) return CPSD_ERR_IO;
    const size_t nn = (size_t)(ne[0] + ne[1]) * (size_t)(nfft + 2) * nfft * nfft;
    bool ok = fwrite(&icube, sizeof(int), 1, fp) == 1 && fwrite(&nfft, sizeof(int), 1, fp) == 1 &&
              fwrite(&unit, sizeof(double), 1, fp) == 1 && fwrite(&ispin, sizeof(int), 1, fp) == 1 &&
              fwrite(ne, sizeof(int), 2, fp) == 2 && fwrite(c1, sizeof(double), nn, fp) == nn;
    ok = (fclose(fp) == 0) && ok;
    return ok ? CPSD_OK : CPSD_ERR_IO;
}

extern "C" int cpsd_write_ionout(const char *path, int nkatm, const char *const *fname, const int *lmax, int nion,
                                 const int *katm, const double *r2)
{
    if (!path || nkatm < 0 || nion < 0 || (nkatm > 0 && (!fname || !lmax)) || (nion > 0 && (!katm || !r2)))
        return CPSD_ERR_ARG;
    FILE *fp = fopen(path, "w");
    if (!fp) return CPSD_ERR_IO;
    bool ok = fprintf(fp, "%d\n", nkatm) > 0;
    for (int ia = 0; ia < nkatm && ok; ++ia) ok = fprintf(fp, "'%s ' %d\n", fname[ia], lmax[ia]) > 0;
    ok = ok && fprintf(fp, "%d\n", nion) > 0;
    for (int ii = 0; ii < nion && ok; ++ii) {
        ok = fprintf(fp, "%d ", katm[ii] + 1) > 0;
        for (int d = 0; d < 3 && ok; ++d) ok = fprintf(fp, "%lf ", r2[3 * ii + d]) > 0;
        for (int d = 0; d < 3 && ok; ++d) ok = fprintf(fp, "%lf ", 0.0) > 0;
        ok = ok && fprintf(fp, "\n") > 0;
    }
    ok = (fclose(fp) == 0) && ok;
    return ok ? CPSD_OK : CPSD_ERR_IO;
}

// ====================================================================== 3-D FFT drop-ins
namespace {

// unpadded real grid from the reference's (n+2)-padded x lines
__global__ void unpad_real_kernel(int n, const double *__restrict__ src, double *__restrict__ dst)
{
    const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long n3 = (long)n * n * n;
    if (id >= n3) return;
    const int x = (int)(id % n);
    const long yz = id / n;
    dst[id] = src[yz * (n + 2) + x];
}

__global__ void copy_pad_kernel(int n, const double *__restrict__ src, double *__restrict__ dst)
{
    const long n2r = (long)(n + 2) * n * n;
    const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n2r) return;
    const int x = (int)(id % (n + 2));
    const long yz = id / (n + 2);
    dst[id] = (x < n) ? src[yz * n + x] : 0.0;
}

// half box -> packed (full geometry: every point), and back
__global__ void perm_kernel(long count, const int *__restrict__ idx, const cx<double> *__restrict__ src,
                            cx<double> *__restrict__ dst, int to_packed)
{
    const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= count) return;
    if (to_packed)
        dst[p] = src[idx[p]];
    else
        dst[idx[p]] = src[p];
}

struct FftCtx {
    int n = 0, device = -1;
    long nfft3d = 0, n2ft3d = 0, n3 = 0;
    cudaStream_t st = nullptr;
    double *buf = nullptr, *grid = nullptr;
    cx<double> *packed = nullptr;
    void *Taux = nullptr;
    int *pt_idx = nullptr, *col_i = nullptr, *col_j = nullptr, *col_ptr = nullptr, *pt_k = nullptr,
        *colidx = nullptr;
    Geom g{};
    std::vector<void *> allocs;
    ~FftCtx()
    {
        for (void *p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }
};

thread_local int t_fft_status = CPSD_OK;
std::mutex f_mu;
std::unique_ptr<FftCtx> f_ctx;

}  // namespace

// engine.cu provides the transform instantiations through this factory
int cpsd_fft_run_full(int n, int dir, const Geom &g, double *grid, cx<double> *packed, void *Taux,
                      cudaStream_t st, int init_kx, int *ok);

namespace {

template <typename X>
int dalloc(FftCtx &f, X **p, size_t count)
{
    void *q = nullptr;
    if (cudaMalloc(&q, count * sizeof(X)) != cudaSuccess) return CPSD_ERR_CUDA;
    f.allocs.push_back(q);
    *p = (X *)q;
    return CPSD_OK;
}

int fft_setup(int n)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CPSD_ERR_CUDA;
    if (f_ctx && f_ctx->n == n && f_ctx->device == dev) return CPSD_OK;
    f_ctx.reset();
    std::unique_ptr<FftCtx> f(new FftCtx());
    f->n = n;
    f->device = dev;
    const int nh = n / 2 + 1;
    f->nfft3d = (long)nh * n * n;
    f->n2ft3d = 2 * f->nfft3d;
    f->n3 = (long)n * n * n;
    if (cudaStreamCreateWithFlags(&f->st, cudaStreamNonBlocking) != cudaSuccess) return CPSD_ERR_CUDA;
    // full geometry: columns (kx, ky) for every kx <= n/2, every kz
    std::vector<int> col_i, col_j, col_ptr{0}, pt_k, pt_idx, colidx((size_t)nh * n);
    for (int i = 0; i < nh; ++i)
        for (int j = 0; j < n; ++j) {
            colidx[(size_t)i * n + j] = (int)col_i.size();
            col_i.push_back(i);
            col_j.push_back(j);
            for (int k = 0; k < n; ++k) {
                pt_k.push_back(k);
                pt_idx.push_back(i + j * nh + k * nh * n);
            }
            col_ptr.push_back((int)pt_k.size());
        }
    auto up = [&](int **d, const std::vector<int> &v) -> int {
        if (dalloc(*f, d, v.size())) return CPSD_ERR_CUDA;
        return cudaMemcpy(*d, v.data(), v.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess
                   ? CPSD_OK
                   : CPSD_ERR_CUDA;
    };
    if (up(&f->col_i, col_i) || up(&f->col_j, col_j) || up(&f->col_ptr, col_ptr) || up(&f->pt_k, pt_k) ||
        up(&f->pt_idx, pt_idx) || up(&f->colidx, colidx))
        return CPSD_ERR_CUDA;
    if (dalloc(*f, &f->buf, f->n2ft3d) || dalloc(*f, &f->grid, f->n3) || dalloc(*f, &f->packed, f->nfft3d))
        return CPSD_ERR_CUDA;
    unsigned char *t = nullptr;
    if (dalloc(*f, &t, sizeof(cx<double>) * (size_t)n * nh * n)) return CPSD_ERR_CUDA;
    f->Taux = t;
    f->g.n = n;
    f->g.nh = nh;
    f->g.KX = nh;
    f->g.ncol = (int)col_i.size();
    f->g.npw = (int)pt_k.size();
    f->g.npw_pad = f->g.npw;
    f->g.col_i = f->col_i;
    f->g.col_j = f->col_j;
    f->g.col_ptr = f->col_ptr;
    f->g.pt_k = f->pt_k;
    f->g.colidx = f->colidx;
    f_ctx = std::move(f);
    return CPSD_OK;
}

int fft_call(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r, int *nx, int *ny, int *nz, int dir)
{
    if (!A || !nx || !ny || !nz || !inc2c || !inc3c || !inc2r || !inc3r) return CPSD_ERR_ARG;
    const int n = *nx;
    if (*ny != n || *nz != n) return CPSD_ERR_ARG;
    const int nh = n / 2 + 1;
    if (*inc2c != nh || *inc3c != nh * n || *inc2r != n + 2 || *inc3r != (n + 2) * n) return CPSD_ERR_ARG;
    std::lock_guard<std::mutex> lk(f_mu);
    int rc = fft_setup(n);
    if (rc) return rc;
    FftCtx &f = *f_ctx;
    cudaStream_t s = f.st;
    const size_t bytes = sizeof(double) * f.n2ft3d;
    if (cudaMemcpyAsync(f.buf, A, bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) return CPSD_ERR_CUDA;
    const unsigned gb = (unsigned)((f.nfft3d + 255) / 256);
    int ok = 0;
    if (dir > 0) {  // cr_fft3b: half box -> real
        perm_kernel<<<gb, 256, 0, s>>>(f.nfft3d, f.pt_idx, (const cx<double> *)f.buf, f.packed, 1);
        rc = cpsd_fft_run_full(n, +1, f.g, f.grid, f.packed, f.Taux, s, nh, &ok);
        if (rc) return rc;
        copy_pad_kernel<<<(unsigned)((f.n2ft3d + 255) / 256), 256, 0, s>>>(n, f.grid, f.buf);
    } else {  // rc_fft3f: real -> half box
        unpad_real_kernel<<<(unsigned)((f.n3 + 255) / 256), 256, 0, s>>>(n, f.buf, f.grid);
        rc = cpsd_fft_run_full(n, -1, f.g, f.grid, f.packed, f.Taux, s, nh, &ok);
        if (rc) return rc;
        perm_kernel<<<gb, 256, 0, s>>>(f.nfft3d, f.pt_idx, f.packed, (cx<double> *)f.buf, 0);
    }
    if (cudaGetLastError() != cudaSuccess) return CPSD_ERR_CUDA;
    if (cudaMemcpyAsync(A, f.buf, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return CPSD_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CPSD_ERR_CUDA;
    return ok ? CPSD_OK : CPSD_ERR_GRID;
}

}  // namespace

extern "C" void cr_fft3b_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r, int *nx, int *ny, int *nz,
                          double *tmp, int *ntmp)
{
    (void)tmp;
    (void)ntmp;
    t_fft_status = fft_call(A, inc2c, inc3c, inc2r, inc3r, nx, ny, nz, +1);
    if (t_fft_status == CPSD_ERR_CUDA) (void)cudaGetLastError();  // leave no stale error behind
    if (t_fft_status) printf("cr_fft3b (B200): error %d: %s\n", t_fft_status, cpsd_gpu_strerror(t_fft_status));
}

extern "C" void rc_fft3f_(double *A, int *inc2c, int *inc3c, int *inc2r, int *inc3r, int *nx, int *ny, int *nz,
                          double *tmp, int *ntmp)
{
    (void)tmp;
    (void)ntmp;
    t_fft_status = fft_call(A, inc2c, inc3c, inc2r, inc3r, nx, ny, nz, -1);
    if (t_fft_status == CPSD_ERR_CUDA) (void)cudaGetLastError();  // leave no stale error behind
    if (t_fft_status) printf("rc_fft3f (B200): error %d: %s\n", t_fft_status, cpsd_gpu_strerror(t_fft_status));
}

extern "C" int cpsd_gpu_fft_status(void) { return t_fft_status; }
