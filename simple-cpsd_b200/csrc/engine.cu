// engine.cu -- context, geometry, step orchestration and the C ABI of
// include/cpsd_b200.h.  One context = one cell resident on one GPU; every SD
// step is a fixed sequence of kernel launches on the context's stream.
#include <cuda_runtime.h>

#if defined(__x86_64__)
#include <emmintrin.h>
#endif

#include <algorithm>
#include <atomic>
#include <map>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "cpsd_b200.h"
#include "fft.cuh"
#include "dropin.h"
#include "host_pool.h"
#include "kernels.cuh"
#include "mlp.cuh"
#include "tc_gemm.cuh"

namespace {

// On failure: remember the error for cpsd_gpu_strerror and clear the
// runtime's last-error slot so that a caller's next CUDA call does not trip
// over it.
#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) {                                   \
            last_cuda_error() = e_;                                \
            (void)cudaGetLastError();                              \
            return CPSD_ERR_CUDA;                                  \
        }                                                          \
    } while (0)

cudaError_t &last_cuda_error()
{
    static thread_local cudaError_t e = cudaSuccess;
    return e;
}

inline long cdiv(long a, long b) { return (a + b - 1) / b; }

constexpr int kTuneMaxCtas = 8;  // largest split-K target (CTAs per SM) a tuning may set
// trust region of the guarded learned step (cpsd_gpu_run_guarded): the bound
// on log K shrinks after a rejected block and grows after an accepted one
// (steady state near one rejected block in eight)
constexpr double kCapShrink = 0.7, kCapGrow = 0.1;

// Streaming multiprocessors of the current device (148 on a B200), looked up
// once per device.
int device_sms()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) return 148;
    cache[dev].store(v, std::memory_order_relaxed);
    return v;
}

// Allow a kernel the device's opt-in shared memory minus its static part.
template <typename K>
cudaError_t allow_max_smem(K kernel, int optin)
{
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                optin - (int)fa.sharedSizeBytes);
}

// ------------------------------------------------------------ geometry
struct HostGeom {
    int n = 0, nh = 0, KX = 0, ncol = 0, npw = 0, npw_pad = 0;
    std::vector<int> col_i, col_j, col_ptr, pt_k, pt_i, pt_j, pt_idx, colidx, inv_idx;
    // the sphere points in ascending full-box index (pt_idx[pt_ord[q]] grows
    // with q): host loops over the reference's grids walk them in memory
    // order instead of one column (stride nh*n) at a time
    std::vector<int> pt_ord;
    std::vector<int> yrun;  // 3 per line kx < KX (see Geom::yrun), empty if some line is not two runs
    std::vector<double> w;
};

// Columns (kx, ky) holding mask points, ordered kx then ky; points ordered by
// column then kz.  full=true takes every half-box point (no pruning).
HostGeom build_geom(int n, const int *masker1, bool full)
{
    HostGeom h;
    h.n = n;
    h.nh = n / 2 + 1;
    const long nfft3d = (long)h.nh * n * n;
    h.inv_idx.assign(nfft3d, -1);
    h.col_ptr.push_back(0);
    for (int i = 0; i < h.nh; ++i)
        for (int j = 0; j < n; ++j) {
            int cnt = 0;
            for (int k = 0; k < n; ++k) {
                const long idx = i + (long)j * h.nh + (long)k * h.nh * n;
                if (full || masker1[idx]) {
                    h.inv_idx[idx] = (int)h.pt_k.size();
                    h.pt_k.push_back(k);
                    h.pt_i.push_back(i);
                    h.pt_j.push_back(j);
                    h.pt_idx.push_back((int)idx);
                    h.w.push_back(i == 0 ? 1.0 : 2.0);
                    ++cnt;
                }
            }
            if (cnt) {
                h.col_i.push_back(i);
                h.col_j.push_back(j);
                h.col_ptr.push_back((int)h.pt_k.size());
                h.KX = std::max(h.KX, i + 1);
            }
        }
    h.ncol = (int)h.col_i.size();
    h.npw = (int)h.pt_k.size();
    h.pt_ord.reserve(h.npw);
    for (long idx = 0; idx < nfft3d; ++idx)
        if (h.inv_idx[idx] >= 0) h.pt_ord.push_back(h.inv_idx[idx]);
    h.npw_pad = (int)cdiv(std::max(h.npw, 1), 32) * 32;
    h.w.resize(h.npw_pad, 0.0);
    h.colidx.assign((size_t)std::max(h.KX, 1) * n, -1);
    for (int c = 0; c < h.ncol; ++c) h.colidx[(size_t)h.col_i[c] * n + h.col_j[c]] = c;
    // The columns of one line kx are usually y in [0, a) and [b, n) (the
    // sphere's |ky| range): then a line's column of y is arithmetic.
    h.yrun.assign((size_t)3 * std::max(h.KX, 1), 0);
    for (int i = 0; i < h.KX; ++i) {
        const int *row = h.colidx.data() + (size_t)i * n;
        int a = 0;
        while (a < n && row[a] >= 0) ++a;
        int b = n;
        while (b > a && row[b - 1] >= 0) --b;
        bool ok = true;
        for (int j = a; j < b && ok; ++j) ok = row[j] < 0;
        const int first = (a > 0) ? row[0] : (b < n ? row[b] : 0);
        for (int j = 0; j < n && ok; ++j) {
            const int want = j < a ? first + j : (j >= b ? first + a + (j - b) : -1);
            ok = row[j] == want;
        }
        if (!ok) {
            h.yrun.clear();
            break;
        }
        h.yrun[3 * i] = first;
        h.yrun[3 * i + 1] = a;
        h.yrun[3 * i + 2] = b;
    }
    return h;
}

// ------------------------------------------------------------ device memory
struct DevArena {
    std::vector<void *> ptrs;
    ~DevArena() { release(); }
    void release()
    {
        for (void *p : ptrs) cudaFree(p);
        ptrs.clear();
    }
    template <typename X>
    cudaError_t alloc(X **p, size_t count)
    {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(X));
        if (e != cudaSuccess) return e;
        ptrs.push_back(q);
        *p = static_cast<X *>(q);
        // Zero-filled before the caller sees it: the fill runs on the legacy
        // stream, which the contexts' non-blocking streams do not wait for,
        // so an asynchronous copy into the buffer on a context stream could
        // otherwise be overwritten by the fill (a chunk table written right
        // after its allocation read back as zeros).
        e = cudaMemsetAsync(q, 0, std::max<size_t>(count, 1) * sizeof(X), 0);
        if (e != cudaSuccess) return e;
        return cudaStreamSynchronize(0);
    }
};

template <typename X>
cudaError_t upload(DevArena &ar, X **d, const std::vector<X> &h)
{
    cudaError_t e = ar.alloc(d, h.size());
    if (e != cudaSuccess) return e;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpy(*d, h.data(), h.size() * sizeof(X), cudaMemcpyHostToDevice);
}

// ------------------------------------------------------------ transform engines
struct FftOps {
    virtual ~FftOps() = default;
    virtual size_t elem() const = 0;
    virtual int init(DevArena &ar, int KX, int ncol) = 0;
    virtual void inv_z(const Geom &g, const cx<double> *psi, long ldp, void *Tb, int nb, cudaStream_t s) = 0;
    virtual void fwd_z_store(const Geom &g, const void *Tb, cx<double> *out, long ldo, double scale,
                             int nb, cudaStream_t s) = 0;
    virtual void fwd_z_sd(const Geom &g, const void *Tb, const ZEpilogue &e, int nb, cudaStream_t s) = 0;
    virtual void plane(int mode, const Geom &g, void *Tb, const PlaneArgs &a, int nchunks, cudaStream_t s) = 0;
    virtual int plane_ctas_per_sm(int mode) const = 0;  // resident CTAs of a plane pass
    virtual int plane_ctas_per_plane(int mode) const = 0;  // CTAs sharing one z plane (row split)
    // occupancy builds of a plane pass (1 or 2) and the one that runs
    virtual int plane_variants(int mode) const = 0;
    virtual int plane_variant(int mode) const = 0;
    virtual void set_plane_variant(int mode, int v) = 0;
};

template <typename T, int NF>
struct FftOpsT final : FftOps {
    Twiddles<T> tw{};
    int KX = 0;
    size_t zsmem = 0;
    size_t psmem[4] = {0, 0, 0, 0};
    size_t psmem_split = 0;  // the row-split density build (no staged columns)
    bool hi_fits[4] = {false, false, false, false};  // the high-occupancy build's CTAs fit an SM
    int occ[4] = {0, 0, 0, 0};                       // plane build that runs, per mode

    size_t elem() const override { return sizeof(cx<T>); }

    static cx<T> turn(int m, int N, int sign)  // e^{sign 2 pi i m / N}
    {
        long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)N;
        return cx<T>{(T)cosl(a), (T)(sign * sinl(a))};
    }
    // count values e^{sign 2 pi i m / N}, m < count, at v[at..]
    static void fill(std::vector<cx<T>> &v, int at, int N, int sign, int count)
    {
        for (int m = 0; m < count; ++m) v[at + m] = turn(m, N, sign);
    }
    // line_fft's table of Line<N>: v[at + q*P + t] = W_N^{t q}
    template <int N>
    static void fill_line(std::vector<cx<T>> &v, int at, int sign)
    {
        using L = Line<N>;
        for (int q = 0; q < L::Q; ++q)
            for (int t = 0; t < L::P; ++t) v[at + q * L::P + t] = turn(t * q, N, sign);
    }
    // line_fft_dif's table of Line<N>: v[at + t*Q + q] = W_N^{q t}
    template <int N>
    static void fill_dif(std::vector<cx<T>> &v, int at, int sign)
    {
        using L = Line<N>;
        for (int t = 0; t < L::P; ++t)
            for (int q = 0; q < L::Q; ++q) v[at + t * L::Q + q] = turn(q * t, N, sign);
    }

    int init(DevArena &ar, int kx, int ncol) override
    {
        KX = kx;
        constexpr int H = NF / 2;
        using TL = TwLayout<NF>;
        std::vector<cx<T>> tab(TL::total);
        fill_line<NF>(tab, TL::n_inv, +1);
        fill_line<NF>(tab, TL::n_fwd, -1);
        fill_line<H>(tab, TL::h_inv, +1);
        fill_line<H>(tab, TL::h_fwd, -1);
        fill_dif<H>(tab, TL::h_fwd_dif, -1);
        fill(tab, TL::r_inv, NF, +1, H + 1);
        fill(tab, TL::r_fwd, NF, -1, H + 1);
        cx<T> *d = nullptr;
        CK(upload(ar, &d, tab));
        tw = Twiddles<T>::template at<NF>(d);

        zsmem = z_smem_bytes<T, NF>();
        int dev = 0, optin = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        CK(cudaFuncSetAttribute(inv_z_kernel<T, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem));
        CK(cudaFuncSetAttribute(fwd_z_kernel<T, NF, ZEPI_STORE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem));
        CK(cudaFuncSetAttribute(fwd_z_kernel<T, NF, ZEPI_SD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zsmem));
        for (int m = 0; m < 4; ++m) psmem[m] = plane_smem_bytes<T, NF>(m, KX, ncol);
        psmem_split = plane_smem_bytes<T, NF>(PM_DENSITY, KX, 0);
        for (int m = 0; m < 4; ++m)
            if ((int)psmem[m] > optin) psmem[m] = 0;  // mode unavailable for this sphere
        // The limit is a per-kernel (process-wide) attribute shared by every
        // context on the device: set it to the device maximum, launch with
        // what this sphere needs.
        CK(allow_plane<PM_DENSITY>(optin));
        CK(allow_plane<PM_APPLYV>(optin));
        CK(allow_plane<PM_INVREAL>(optin));
        CK(allow_plane<PM_FWDREAL>(optin));
        // the high-occupancy build needs its CTAs' shared memory (plus the
        // per-CTA reserve) to fit an SM; it starts as the default where it
        // does, except where its register cap is known to spill (FP64 lines
        // of 32 values and more per lane); a tuner may switch per mode
        int sm_bytes = 0, reserve = 0;
        CK(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        CK(cudaDeviceGetAttribute(&reserve, cudaDevAttrReservedSharedMemoryPerBlock, dev));
        const bool has_two[4] = {plane_has_two_cta_build<NF, PM_DENSITY>(), plane_has_two_cta_build<NF, PM_APPLYV>(),
                                 plane_has_two_cta_build<NF, PM_INVREAL>(), plane_has_two_cta_build<NF, PM_FWDREAL>()};
        for (int m = 0; m < 4; ++m) {
            const size_t hi = (m == PM_DENSITY && plane_row_split<NF, PM_DENSITY, 2>() > 1) ? psmem_split : psmem[m];
            hi_fits[m] = has_two[m] && psmem[m] != 0 && 2 * (hi + (size_t)reserve) <= (size_t)sm_bytes;
            occ[m] = hi_fits[m] ? 1 : 0;
        }
        // the row-split density build at NF >= 128 redoes each plane's y
        // lines in two CTAs: measured slower than the whole-plane build, so
        // it is only a candidate of the tuner
        if (plane_row_split<NF, PM_DENSITY, 2>() > 1) occ[PM_DENSITY] = 0;
        return CPSD_OK;
    }

    template <int MODE>
    cudaError_t allow_plane(int optin)
    {
        cudaError_t e = allow_max_smem(plane_kernel<T, NF, MODE, 1>, optin);
        if constexpr (plane_has_two_cta_build<NF, MODE>())
            if (e == cudaSuccess) e = allow_max_smem(plane_kernel<T, NF, MODE, 2>, optin);
        return e;
    }

    // occ 1: the two-CTA build (128 registers a thread), occ 0: one CTA per SM
    template <int MODE>
    void launch_plane(dim3 grid, int nt, const Geom &g, void *Tb, const PlaneArgs &a, cudaStream_t s)
    {
        if constexpr (plane_has_two_cta_build<NF, MODE>())
            if (occ[MODE]) {
                dim3 g2 = grid;
                g2.z = plane_row_split<NF, MODE, 2>();  // the density pass's row halves
                const size_t sm = (g2.z > 1) ? psmem_split : psmem[MODE];
                plane_kernel<T, NF, MODE, 2><<<g2, nt, sm, s>>>(g, (cx<T> *)Tb, a, tw);
                return;
            }
        plane_kernel<T, NF, MODE, 1><<<grid, nt, psmem[MODE], s>>>(g, (cx<T> *)Tb, a, tw);
    }

    void inv_z(const Geom &g, const cx<double> *psi, long ldp, void *Tb, int nb, cudaStream_t s) override
    {
        constexpr int CPB = kThreads / Line<NF>::P;
        dim3 grid((unsigned)cdiv(g.ncol, CPB), (unsigned)nb);
        inv_z_kernel<T, NF><<<grid, kThreads, zsmem, s>>>(g, psi, ldp, (cx<T> *)Tb, tw);
    }
    void fwd_z_store(const Geom &g, const void *Tb, cx<double> *out, long ldo, double scale, int nb,
                     cudaStream_t s) override
    {
        constexpr int CPB = kThreads / Line<NF>::P;
        ZEpilogue e{};
        e.out = out;
        e.ldo = ldo;
        e.scale = scale;
        dim3 grid((unsigned)cdiv(g.ncol, CPB), (unsigned)nb);
        fwd_z_kernel<T, NF, ZEPI_STORE><<<grid, kThreads, zsmem, s>>>(g, (const cx<T> *)Tb, e, tw);
    }
    void fwd_z_sd(const Geom &g, const void *Tb, const ZEpilogue &e, int nb, cudaStream_t s) override
    {
        constexpr int CPB = kThreads / Line<NF>::P;
        dim3 grid((unsigned)cdiv(g.ncol, CPB), (unsigned)nb);
        fwd_z_kernel<T, NF, ZEPI_SD><<<grid, kThreads, zsmem, s>>>(g, (const cx<T> *)Tb, e, tw);
    }
    void plane(int mode, const Geom &g, void *Tb, const PlaneArgs &a, int nchunks, cudaStream_t s) override
    {
        // a CTA takes plane_bands_per_cta chunks (one band each for V psi)
        dim3 grid(NF, (unsigned)cdiv(nchunks, plane_bands_per_cta(NF, mode)));
        PlaneArgs pa = a;
        pa.nchunks = nchunks;
        const int nt = plane_threads<T, NF>(mode);
        switch (mode) {
        case PM_DENSITY: launch_plane<PM_DENSITY>(grid, nt, g, Tb, pa, s); break;
        case PM_APPLYV: launch_plane<PM_APPLYV>(grid, nt, g, Tb, pa, s); break;
        case PM_INVREAL: launch_plane<PM_INVREAL>(grid, nt, g, Tb, pa, s); break;
        default: launch_plane<PM_FWDREAL>(grid, nt, g, Tb, pa, s); break;
        }
    }
    bool mode_ok(int mode) const { return psmem[mode] != 0; }
    int plane_ctas_per_sm(int mode) const override { return occ[mode & 3] ? 2 : 1; }
    int plane_ctas_per_plane(int mode) const override
    {
        return (mode == PM_DENSITY && occ[PM_DENSITY]) ? plane_row_split<NF, PM_DENSITY, 2>() : 1;
    }
    int plane_variants(int mode) const override { return hi_fits[mode & 3] ? 2 : 1; }
    int plane_variant(int mode) const override { return occ[mode & 3]; }
    void set_plane_variant(int mode, int v) override
    {
        if (mode >= 0 && mode < 4) occ[mode] = (v && hi_fits[mode]) ? 1 : 0;
    }
};

bool grid_supported(int n)
{
    return n == 16 || n == 24 || n == 32 || n == 48 || n == 64 || n == 128;
}

template <typename T>
std::unique_ptr<FftOps> make_fft_t(int n)
{
    switch (n) {
    case 16: return std::unique_ptr<FftOps>(new FftOpsT<T, 16>());
    case 24: return std::unique_ptr<FftOps>(new FftOpsT<T, 24>());
    case 32: return std::unique_ptr<FftOps>(new FftOpsT<T, 32>());
    case 48: return std::unique_ptr<FftOps>(new FftOpsT<T, 48>());
    case 64: return std::unique_ptr<FftOps>(new FftOpsT<T, 64>());
    case 128: return std::unique_ptr<FftOps>(new FftOpsT<T, 128>());
    default: return nullptr;
    }
}

// FP64 transforms for the parity path; FP32 transforms for the mixed path
// (orbitals, potentials, densities and every reduction stay FP64).
std::unique_ptr<FftOps> make_fft(int n, int precision = CPSD_PREC_FP64)
{
    return precision == CPSD_PREC_MIXED ? make_fft_t<float>(n) : make_fft_t<double>(n);
}

template <typename T>
size_t plane_need_t(int n, int mode, int KX, int ncol)
{
    switch (n) {
    case 16: return plane_smem_bytes<T, 16>(mode, KX, ncol);
    case 24: return plane_smem_bytes<T, 24>(mode, KX, ncol);
    case 32: return plane_smem_bytes<T, 32>(mode, KX, ncol);
    case 48: return plane_smem_bytes<T, 48>(mode, KX, ncol);
    case 64: return plane_smem_bytes<T, 64>(mode, KX, ncol);
    default: return plane_smem_bytes<T, 128>(mode, KX, ncol);
    }
}

size_t plane_need(int n, int mode, int KX, int ncol, int precision = CPSD_PREC_FP64)
{
    return precision == CPSD_PREC_MIXED ? plane_need_t<float>(n, mode, KX, ncol) : plane_need_t<double>(n, mode, KX, ncol);
}

}  // namespace

// ------------------------------------------------------------ network object
struct cpsd_mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    DevArena ar;
    float *p = nullptr, *m1 = nullptr, *m2 = nullptr, *g = nullptr;
    __nv_bfloat16 *wq = nullptr;
    long adam_t = 0;
    // training buffers, grown on demand
    int cap = 0;
    float *X = nullptr, *T = nullptr, *y = nullptr, *H = nullptr, *D = nullptr, *dy = nullptr, *lp = nullptr;
};

// ------------------------------------------------------------ context
struct cpsd_gpu_ctx {
    cpsd_gpu_params prm{};
    int n = 0, nh = 0, nb = 0, ne0 = 0, ne1 = 0, nion = 0, nkatm = 0, nsh = 0, ispin = 1;
    int sms = 148;  // streaming multiprocessors of the context's device
    long nfft3d = 0, n2ft3d = 0, n3 = 0;
    double scal1 = 0, scal2 = 0, dv = 0, dte = 0;
    cudaStream_t st = nullptr;
    DevArena ar;
    HostGeom hg;
    Geom g{};
    FftOps *fft = nullptr;                 // the active transform engine
    std::unique_ptr<FftOps> fft64, fft32;  // FP64 (parity) and FP32 (mixed) engines
    int precision = CPSD_PREC_FP64;
    int gemm_mode = CPSD_GEMM_FP64;  // TN products of the mixed path (CPSD_GEMM_*)
    int npw = 0, npw_pad = 0, nproj = 0;
    long ldc = 0;  // complex stride between bands
    int nchunk0 = 0, nchunk1 = 0;
    int gemm_splits_cap = 0;
    size_t gemm_ws_elems = 0;
    int launches_per_step = 0;
    int lag_fail_total = 0;
    long long nlaunch = 0, h2d = 0, d2h = 0;  // kernel launches and host<->device bytes so far
    bool use_graph = true;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};  // one captured SD step per ping-pong parity
    int graph_launches = 0;
    // several SD steps captured as one graph (the steps of a cpsd() call),
    // per (steps, parity); a few kept
    struct MultiGraph {
        int steps, par, launches;
        cudaGraphExec_t exec;
    };
    std::vector<MultiGraph> mgraphs;
    // second stream of a step: structure factors, projectors and the kinetic +
    // nonlocal part of -H psi run beside the density -> potential chain
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_sf = nullptr, ev_side = nullptr;
    // early fetch (the drop-in): once the steps are done, c1, c2 and the
    // density go to the pinned staging on the side stream while the
    // energies run; get_state_host then only waits for ev_fetch
    bool early_fetch = false, fetched = false;
    cudaEvent_t ev_steps = nullptr, ev_fetch = nullptr;
    // the density of a call's last step is final once its density pass has
    // run: ev_dn is recorded there (in the last step of each captured graph)
    // so that its copy to the host can start during the rest of the step
    cudaEvent_t ev_dn = nullptr;
    bool rec_dn = false;
    cudaStream_t cs = nullptr;  // the stream the GEMM helpers launch on
    bool lag_tile = false;  // 4 x 4 tiled solver (<= 128 bands, 16-CTA clusters schedulable)
    bool lag_tile_ok = false;  // the tiled solver can run on this device for these bands
    // tuning (cpsd_gpu_set_tuning / cpsd_gpu_autotune): split-K target of the
    // TN products, density chunk capacity and the model's chunk counts
    int tn_ctas = 2;
    int dens_cap = 0;
    int dens_model[2] = {0, 0};
    // band-parallel SD (cpsd_gpu_set_band_range): this context transforms and
    // steps bands [bp_lo, bp_hi); dn_part holds its spin densities before the
    // caller sums them over the ranks; its density chunks in chunk_bp
    bool bp = false;
    int bp_lo = 0, bp_hi = 0;
    double *dn_part = nullptr;
    int *chunk_bp = nullptr;
    int nchunk_bp[2] = {0, 0};
    int lag_cluster = 8;  // CTAs per cluster of the Lagrange solver (16 where schedulable)
    int lag_lb = 0;       // its row-tile width
    // learned preconditioner (optional): shells, stats, features, outputs
    cpsd_mlp *mlp = nullptr;
    int *shell = nullptr, *dstep = nullptr;
    float *pcap = nullptr;  // [lo, hi] range of the learned log step scale
    cx<double> *saved = nullptr;  // cpsd_gpu_save_orbitals copy (with the step counters)
    int *saved_step = nullptr;
    long long saved_steps_run = 0;
    double *epart = nullptr;  // real-space Ewald sum per ion
    cx<double> *pR = nullptr;  // residual of -H psi outside the occupied subspace
    // ion motion (move = 1)
    bool motion_ok = false;  // G vectors and masses given by cpsd_gpu_set_tables
    int move = 0;            // the step graphs hold the force kernels
    std::vector<double> amass_h;
    double *Gv = nullptr, *dti = nullptr, *fpart = nullptr, *fnl = nullptr, *ewp = nullptr, *coefP = nullptr;
    cx<double> *Ynl = nullptr;
    double *pM = nullptr;      // <cpsi_b|c1_a> per spin
    double *pstats = nullptr, tmax = 0.0;
    long long steps_run = 0;  // SD steps taken by this context
    float *py = nullptr;
    // optional phase timing: events recorded between the phases of a step
    // (captured into the step graphs), read back by cpsd_gpu_phase_times()
    bool phase_timing = false;
    cudaEvent_t pev[16] = {};
    bool tables_ok = false, state_ok = false, ran = false;

    // device
    int *pt_i = nullptr, *pt_j = nullptr, *pt_k = nullptr, *pt_idx = nullptr, *inv_idx = nullptr;
    int *col_i = nullptr, *col_j = nullptr, *col_ptr = nullptr, *colidx = nullptr, *yrun = nullptr;
    double *w = nullptr, *tg = nullptr, *vc = nullptr, *vg = nullptr, *vl = nullptr, *vnl = nullptr;
    double *zv = nullptr, *rcell = nullptr, *unitg = nullptr, *vnlnrm_p = nullptr;
    int *katm = nullptr, *lmmax = nullptr, *proj_off = nullptr;
    cx<double> *cbuf[2] = {nullptr, nullptr};
    int cur = 0;
    cx<double> *cpsi = nullptr;
    double *r1 = nullptr, *r2 = nullptr, *fion = nullptr;
    void *Tb = nullptr, *Taux = nullptr;
    double *rho_part = nullptr, *dn = nullptr, *xcp = nullptr, *xce = nullptr, *rfwd = nullptr, *Vr = nullptr;
    cx<double> *dng = nullptr, *vall = nullptr, *sfac = nullptr, *Vg = nullptr, *proj = nullptr;
    cx<double> *ex1 = nullptr, *ex2 = nullptr, *ex3 = nullptr;
    double *beta = nullptr, *coefT = nullptr, *Mov = nullptr, *gws = nullptr, *lag = nullptr;
    double *lmd = nullptr, *hml = nullptr, *Edev = nullptr, *red = nullptr;
    int *chunk_dens = nullptr, *chunk_band = nullptr, *flags = nullptr;
    // epilogue (allocated on first use): Jacobi workspace, eigenpairs, overlaps
    double *eigA = nullptr, *eigV = nullptr, *eigD = nullptr, *eigVec = nullptr, *ortho = nullptr;
    int *eig_sweeps = nullptr;
    // pinned host staging of two packed band sets (nb x ldc each): the sphere
    // is all that crosses PCIe for the host-layout orbitals
    struct Pinned {
        cx<double> *p = nullptr;
        ~Pinned()
        {
            if (p) cudaFreeHost(p);
        }
    } hstage;
    Pinned tstage;  // packed tables of cpsd_gpu_set_tables
    size_t tstage_bytes = 0;
    std::vector<char> tables_last;  // the staged bytes of the last upload (a repeat is not sent again)
    Pinned dstage;  // the density (ispin * n^3) on its way to the padded host layout
    int pblocks = 0, bblocks = 0, gblocks = 0;
    double *ppart = nullptr, *bpart = nullptr, *gpart = nullptr;
};

namespace {

// Band ranges of the density pass: n0 chunks of spin 0's ne0 bands, then
// n1 chunks of spin 1's (starts, ends appended: n0 + n1 + 1 entries).
std::vector<int> density_chunk_table(int ne0, int n0, int ne1, int n1)
{
    std::vector<int> b0;
    for (int q = 0; q <= n0; ++q) b0.push_back((int)((long)ne0 * q / n0));
    for (int q = 1; q <= n1; ++q) b0.push_back(ne0 + (int)((long)ne1 * q / n1));
    return b0;
}

// Split-K plan of a batch of weighted TN products: about two CTAs per SM
// (sms: the device's SM count), each split at least 64 reals, partials
// within ws_elems.
struct TnPlan {
    long splits;
    int kchunk;
};

TnPlan tn_plan(int M, int N, int K, int nprod, bool tc, size_t ws_elems, int sms, int ctas_per_sm = 2)
{
    const int tm = tc ? kTcM : kDmT, tn = tc ? kTcN : kDmT, bk = tc ? kTcBK : kDmK;
    const long tiles = cdiv(M, tm) * cdiv(N, tn) * nprod;
    long splits = std::max<long>(1, cdiv((long)ctas_per_sm * sms, tiles));
    splits = std::min<long>(splits, std::max<long>(1, K / 64));
    while ((size_t)splits * M * N * nprod > ws_elems && splits > 1) --splits;
    const int kchunk = (int)(cdiv(cdiv(K, splits), bk) * bk);
    return TnPlan{cdiv(K, kchunk), kchunk};
}

// C_q = alpha A_q' W B_q (+ beta C_q), q < nprod: split-K partial products
// (FP64 tensor cores, or 3xTF32 on tcgen05 when tc) and a fixed-order FP64
// reduction.  Returns the number of launches.
int launch_tn(int M, int N, int K, int nprod, const double *const *A, long lda, const double *const *B, long ldb,
              const double *w, double alpha, double beta, double *const *C, long ldc, bool tc, double *ws,
              size_t ws_elems, int *err, cudaStream_t s, int ctas_per_sm = 2)
{
    const TnPlan pl = tn_plan(M, N, K, nprod, tc, ws_elems, device_sms(), ctas_per_sm);
    TnBatch bt{};
    for (int q = 0; q < nprod; ++q) {
        bt.A[q] = A[q];
        bt.B[q] = B[q];
        bt.C[q] = C[q];
    }
    bt.nprod = nprod;
    bt.splits = (int)pl.splits;
    if (tc) {
        dim3 grid((unsigned)cdiv(M, kTcM), (unsigned)cdiv(N, kTcN), (unsigned)(pl.splits * nprod));
        tc_gemm_tn_kernel<<<grid, kTcThreads, kTcSmem, s>>>(M, N, K, lda, ldb, w, pl.kchunk, bt, ws, err);
    } else {
        dim3 grid((unsigned)cdiv(M, kDmT), (unsigned)cdiv(N, kDmT), (unsigned)(pl.splits * nprod));
        gemm_tn_dmma_kernel<<<grid, kDmThreads, 0, s>>>(M, N, K, lda, ldb, w, pl.kchunk, bt, ws);
    }
    splitk_reduce_kernel<<<(unsigned)cdiv((long)M * N * nprod * 32, 256), 256, 0, s>>>(M, N, ldc, ws, alpha, beta,
                                                                                       bt);
    return 2;
}

// Which products may run on the tensor cores (bits of CPSD_GEMM_*):
// TN_PROJECTOR: the KB projector coefficients and back-projection, and the
// learned step's residual (errors there stay inside the occupied subspace,
// which the constraint rotates away); TN_OVERLAPS: the Lagrange overlaps and
// the constraint correction c2 += dte C1 lmd.
enum { TN_PROJECTOR = 1, TN_OVERLAPS = 2 };

// Batched weighted TN products of a context; `which` names the product so
// that the tensor-core variant runs where the context runs mixed precision
// and its GEMM mode includes that product.
int gemm_tn_batch(cpsd_gpu_ctx *c, int M, int N, int K, int nprod, const double *const *A, long lda,
                  const double *const *B, long ldb, const double *w, double alpha, double beta,
                  double *const *C, long ldc, int which = 0)
{
    if (M <= 0 || N <= 0 || nprod <= 0) return CPSD_OK;
    if (nprod > kTnMaxProd) return CPSD_ERR_ARG;
    const bool tc = (c->gemm_mode & which) != 0 && c->precision == CPSD_PREC_MIXED;
    c->nlaunch += launch_tn(M, N, K, nprod, A, lda, B, ldb, w, alpha, beta, C, ldc, tc, c->gws, c->gemm_ws_elems,
                            c->flags + 2, c->cs, c->tn_ctas);
    return CPSD_OK;
}

int gemm_tn(cpsd_gpu_ctx *c, int M, int N, int K, const double *A, long lda, const double *B, long ldb,
            const double *w, double alpha, double beta, double *C, long ldc, int which = 0)
{
    return gemm_tn_batch(c, M, N, K, 1, &A, lda, &B, ldb, w, alpha, beta, &C, ldc, which);
}

// The three overlaps C2'WC2, C2'WC1, C1'WC1 of one spin: one fused
// tensor-core pass (tc_overlaps3_kernel) where the context runs its overlaps
// on the tensor cores, the spin has at most 128 bands and the operands are
// 16-byte aligned for cp.async; otherwise the batched TN products.
int overlaps3(cpsd_gpu_ctx *c, int m, int K, long ld, const double *C2, const double *C1, double *const *Cs)
{
    const double *As[3] = {C2, C2, C1}, *Bs[3] = {C2, C1, C1};
    const bool tc = (c->gemm_mode & TN_OVERLAPS) != 0 && c->precision == CPSD_PREC_MIXED;
    const bool fits = m > 0 && m <= kTcM && (ld % 2) == 0 && K % 2 == 0 && ((uintptr_t)C1 % 16) == 0 &&
                      ((uintptr_t)C2 % 16) == 0;
    if (!tc || !fits) return gemm_tn_batch(c, m, m, K, 3, As, ld, Bs, ld, c->w, 1.0, 0.0, Cs, m, TN_OVERLAPS);
    const long mm = (long)m * m;
    long splits = std::min<long>(c->sms, std::max<long>(1, K / 64));
    while ((size_t)splits * 3 * mm > c->gemm_ws_elems && splits > 1) --splits;
    const int kchunk = (int)(cdiv(cdiv(K, splits), kOvBK) * kOvBK);
    splits = cdiv(K, kchunk);
    tc_overlaps3_kernel<<<(unsigned)splits, kTcThreads, kOvSmem, c->cs>>>(m, K, ld, C2, C1, c->w, kchunk,
                                                                         (int)splits, c->gws, c->flags + 2);
    TnBatch bt{};
    for (int q = 0; q < 3; ++q) {
        bt.A[q] = As[q];
        bt.B[q] = Bs[q];
        bt.C[q] = Cs[q];
    }
    bt.nprod = 3;
    bt.splits = (int)splits;
    splitk_reduce_kernel<<<(unsigned)cdiv(mm * 3 * 32, 256), 256, 0, c->cs>>>(m, m, m, c->gws, 1.0, 0.0, bt);
    c->nlaunch += 2;
    return CPSD_OK;
}

// Out = beta Out + alpha Mat B (K the long grid dimension); `which` names the
// product as for gemm_tn_batch, so the tensor-core variant runs where the
// context runs mixed precision and its GEMM mode includes it.
void gemm_nn(cpsd_gpu_ctx *c, int NJ, int K, int L, double alpha, const double *Mat, long ldm,
             const double *B, long ldb, double beta, double *Out, long ldo, int which = 0)
{
    if (NJ <= 0 || L <= 0) return;
    if ((c->gemm_mode & which) != 0 && c->precision == CPSD_PREC_MIXED) {
        dim3 grid((unsigned)cdiv(K, kTcN), (unsigned)cdiv(NJ, kTcM));
        tc_gemm_nn_kernel<<<grid, kTcThreads, kTcSmem, c->cs>>>(NJ, K, L, alpha, Mat, ldm, B, ldb, beta, Out, ldo,
                                                                c->flags + 2);
    } else {
        dim3 grid((unsigned)cdiv(K, kDmT), (unsigned)cdiv(NJ, kDmT));
        gemm_nn_dmma_kernel<<<grid, kDmThreads, 0, c->cs>>>(NJ, K, L, alpha, Mat, ldm, B, ldb, beta, Out, ldo);
    }
    c->nlaunch += 1;
}

const double *Mblk(cpsd_gpu_ctx *c, int ms, int which)
{
    // 4 overlap blocks per spin: 0 M22, 1 M21, 2 M11, 3 hml source
    return c->Mov + ((long)ms * 4 + which) * (long)c->ne0 * c->ne0;
}

const char *const kPhaseNames[] = {
    "inv_z_bands", "density_plane", "density_xc", "rho_fft",     "vloc_proj",  "potential_fft",
    "kinetic_nonlocal", "applyv_plane", "fwd_z_sd", "overlaps", "lagrange", "constraint",
};
constexpr int kNumPhases = (int)(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]));

inline void mark(cpsd_gpu_ctx *c, int i)
{
    // External: during stream capture the record becomes an event node of the graph
    if (c->phase_timing) cudaEventRecordWithFlags(c->pev[i], c->st, cudaEventRecordExternal);
}

// Side-stream work of a step (or in order on `side` = the main stream):
// phase factors, local psp and projectors (cpsd.c:208, 224-286) ...
void issue_sf(cpsd_gpu_ctx *c, cudaStream_t side)
{
    if (c->nion > 0) {
        phase_tables_kernel<<<(unsigned)cdiv(3 * c->nion, 128), 128, 0, side>>>(c->nion, c->n, c->unitg, c->r1,
                                                                             c->ex1, c->ex2, c->ex3);
        c->nlaunch += 1;
    }
    VlocArgs va{};
    va.npw = c->npw;
    va.npw_pad = c->npw_pad;
    va.n = c->n;
    va.nh = c->nh;
    va.nion = c->nion;
    va.pt_i = c->pt_i;
    va.pt_j = c->pt_j;
    va.pt_k = c->pt_k;
    va.katm = c->katm;
    va.zv = c->zv;
    va.ex1 = c->ex1;
    va.ex2 = c->ex2;
    va.ex3 = c->ex3;
    va.vl = c->vl;
    va.vnl = c->vnl;
    va.lmmax = c->lmmax;
    va.proj_off = c->proj_off;
    va.s = c->sfac;
    va.vall = c->vall;
    va.proj = c->proj;
    vloc_proj_kernel<<<(unsigned)cdiv(c->npw_pad, 128), 128, 0, side>>>(va); c->nlaunch += 1;
}

// ... and the kinetic + nonlocal part of -H psi into c2 (cpsd.c:212-221,
// 287-290) for the bands [lo, lo + nbl) this context steps
int issue_knl(cpsd_gpu_ctx *c, cudaStream_t side, const cx<double> *c1, cx<double> *c2, int lo, int nbl)
{
    cudaStream_t s = c->st;
    const int K = 2 * c->npw_pad;
    const long ldr = 2L * c->npw_pad;
    const cx<double> *c1l = c1 + (long)lo * c->ldc;
    cx<double> *c2l = c2 + (long)lo * c->ldc;
    c->cs = side;
    if (c->nproj > 0) {
        int rc = gemm_tn(c, c->nproj, nbl, K, (const double *)c->proj, ldr, (const double *)c1l, ldr, c->w, 1.0,
                         0.0, c->beta + lo, c->nb, TN_PROJECTOR);
        if (rc) {
            c->cs = s;
            return rc;
        }
        kb_coef_kernel<<<(unsigned)cdiv((long)c->nproj * c->nb, 256), 256, 0, side>>>(
            c->nproj, c->nb, c->beta, c->vnlnrm_p, c->scal2, c->coefT, c->move ? c->coefP : nullptr);
        c->nlaunch += 1;
        // the nonlocal part alone; the SD epilogue adds the kinetic term
        gemm_nn(c, nbl, K, c->nproj, 1.0, c->coefT + (long)lo * c->nproj, c->nproj, (const double *)c->proj, ldr,
                0.0, (double *)c2l, ldr, TN_PROJECTOR);
        if (c->move) {  // nonlocal force: Y_P = sum_b sw1(P, b) c1_b, then sum_G G Im(conj(chi_P) Y_P)
            gemm_nn(c, c->nproj, K, c->nb, 1.0, c->coefP, c->nb, (const double *)c1, ldr, 0.0, (double *)c->Ynl,
                    ldr);
            force_nonlocal_kernel<<<c->nproj, 256, 0, side>>>(c->npw, c->ldc, c->w, c->Gv, c->proj, c->Ynl,
                                                             c->fnl);
            c->nlaunch += 1;
        }
    }
    c->cs = s;
    return CPSD_OK;
}

// One SD step in three phases.  A context that steps every band runs them
// back to back (one_step); a band-parallel context (c->bp) steps only its
// bands [bp_lo, bp_hi) in phases 0 and 1, and its caller exchanges between
// them: after phase 0 the spin densities of all ranks are summed into dn
// (dn_part holds this rank's), after phase 1 every rank's new orbitals and
// -H psi rows reach every rank.  Phase 2 (overlaps, Lagrange, constraint)
// then runs on all bands everywhere.
int step_phase(cpsd_gpu_ctx *c, int phase)
{
    cudaStream_t s = c->st;
    cx<double> *c1 = c->cbuf[c->cur], *c2 = c->cbuf[c->cur ^ 1];
    const int K = 2 * c->npw_pad;
    const long ldr = 2L * c->npw_pad;
    const int lo = c->bp ? c->bp_lo : 0, nbl = c->bp ? c->bp_hi - c->bp_lo : c->nb;
    // The structure factors, projectors and the kinetic + nonlocal part of
    // -H psi need only c1 and the ions: they run on a second stream beside
    // the density -> potential -> V psi chain, joined before the SD update.
    // With phase timing on, everything stays on one stream so the phases add up.
    const bool fork = !c->phase_timing;
    cudaStream_t side = fork ? c->st2 : s;
    if (phase == 0) {
        CK(cudaMemcpyAsync(c->r1, c->r2, sizeof(double) * 3 * c->nion, cudaMemcpyDeviceToDevice, s));  // cpsd.c:174
        if (fork) {
            CK(cudaEventRecord(c->ev_fork, s));
            CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
            issue_sf(c, side);
            CK(cudaEventRecord(c->ev_sf, c->st2));
            int rc = issue_knl(c, side, c1, c2, lo, nbl);
            if (rc) return rc;
            CK(cudaEventRecord(c->ev_side, c->st2));
        }

        mark(c, 0);
        // psi(G) -> psi(r) and the density, cpsd.c:177-194
        if (nbl > 0) {
            c->fft->inv_z(c->g, c1 + (long)lo * c->ldc, c->ldc, c->Tb, nbl, s);
            c->nlaunch += 1;
        }
        mark(c, 1);
        PlaneArgs pa{};
        pa.chunk_b0 = c->bp ? c->chunk_bp : c->chunk_dens;
        pa.rho_part = c->rho_part;
        const int ch0 = c->bp ? c->nchunk_bp[0] : c->nchunk0, ch1 = c->bp ? c->nchunk_bp[1] : c->nchunk1;
        if (ch0 + ch1 > 0) {
            c->fft->plane(PM_DENSITY, c->g, c->Tb, pa, ch0 + ch1, s);
            c->nlaunch += 1;
        }
        mark(c, 2);
        XcArgs xa{c->n3, c->ispin, ch0, ch1, c->rho_part, c->scal1, c->scal2, c->dn, c->xcp, c->xce, c->rfwd};
        if (c->bp) {  // this rank's spin densities; the caller sums them into dn
            density_sum_kernel<<<(unsigned)cdiv(c->n3, 256), 256, 0, s>>>(xa, c->dn_part);
            c->nlaunch += 1;
            CK(cudaGetLastError());
            return CPSD_OK;
        }
        density_xc_kernel<<<(unsigned)cdiv(c->n3, 256), 256, 0, s>>>(xa); c->nlaunch += 1;
        if (c->rec_dn) {
            // while capturing, an external record: a plain one would only be a
            // dependency inside the graph, invisible to a wait outside it (the
            // flag is refused outside a capture)
            cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
            CK(cudaStreamIsCapturing(s, &cap));
            CK(cap == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(c->ev_dn, s, cudaEventRecordExternal)
                                                    : cudaEventRecord(c->ev_dn, s));
        }
        mark(c, 3);
        return CPSD_OK;
    }
    if (phase == 1) {
        if (c->bp) {  // dn holds the densities of all bands now
            XcArgs xa{c->n3, c->ispin, 0, 0, nullptr, c->scal1, c->scal2, c->dn, c->xcp, c->xce, c->rfwd};
            xc_from_density_kernel<<<(unsigned)cdiv(c->n3, 256), 256, 0, s>>>(xa);
            c->nlaunch += 1;
            mark(c, 3);
        }
        // rho(G), cpsd.c:198-205
        PlaneArgs pf{};
        pf.rin = c->rfwd;
        c->fft->plane(PM_FWDREAL, c->g, c->Taux, pf, 1, s); c->nlaunch += 1;
        c->fft->fwd_z_store(c->g, c->Taux, c->dng, c->ldc, 1.0, 1, s); c->nlaunch += 1;
        mark(c, 4);
        if (fork)
            CK(cudaStreamWaitEvent(s, c->ev_sf, 0));
        else
            issue_sf(c, side);
        // V(G), cpsd.c:373-379
        vg_kernel<<<(unsigned)cdiv(c->npw, 128), 128, 0, s>>>(c->npw, c->vall, c->dng, c->vc, c->scal2, c->Vg);
        c->nlaunch += 1;
        if (c->move && c->nion > 0) {  // local, k-space and real-space Ewald forces
            ForceArgs fa{};
            fa.npw = c->npw;
            fa.n = c->n;
            fa.nh = c->nh;
            fa.nion = c->nion;
            fa.pt_i = c->pt_i;
            fa.pt_j = c->pt_j;
            fa.pt_k = c->pt_k;
            fa.katm = c->katm;
            fa.ex1 = c->ex1;
            fa.ex2 = c->ex2;
            fa.ex3 = c->ex3;
            fa.w = c->w;
            fa.G = c->Gv;
            fa.vl = c->vl;
            fa.vg = c->vg;
            fa.zv = c->zv;
            fa.dng = c->dng;
            fa.s = c->sfac;
            fa.scal2 = c->scal2;
            fa.fpart = c->fpart;
            force_local_ewald_kernel<<<dim3(kForceChunks, c->nion), 256, 0, s>>>(fa); c->nlaunch += 1;
            if (c->nion > 1) {
                force_ewald_pairs_kernel<<<c->nion, 256, 0, s>>>(c->nion, c->nsh, c->r1, c->rcell, c->zv, c->katm,
                                                                 c->prm.rcut, c->ewp);
                c->nlaunch += 1;
            }
        }
        mark(c, 5);
        // V_loc + V_H to real space, plus xc per spin (cpsd.c:380-388)
        c->fft->inv_z(c->g, c->Vg, c->ldc, c->Taux, 1, s); c->nlaunch += 1;
        PlaneArgs pv{};
        pv.rout = c->Vr;
        pv.xadd = c->xcp;
        pv.nout = c->ispin;
        c->fft->plane(PM_INVREAL, c->g, c->Taux, pv, 1, s); c->nlaunch += 1;
        mark(c, 6);
        if (!fork) {
            int rc = issue_knl(c, side, c1, c2, lo, nbl);
            if (rc) return rc;
        }
        mark(c, 7);
        // (V + xc) psi back to G, -H psi and the SD step, cpsd.c:384-400
        if (nbl > 0) {
            PlaneArgs pp{};
            pp.chunk_b0 = c->chunk_band;
            pp.V = c->Vr;
            pp.ne0 = (c->ispin == 2) ? std::max(0, c->ne0 - lo) : nbl;
            c->fft->plane(PM_APPLYV, c->g, c->Tb, pp, nbl, s); c->nlaunch += 1;
        }
        mark(c, 8);
        if (fork) CK(cudaStreamWaitEvent(s, c->ev_side, 0));  // kinetic + nonlocal c2 is in place
        if (c->move && c->nion > 0) {  // total force and the ion step r2 = r1 + dti fion
            force_total_kernel<<<(unsigned)cdiv(c->nion, 128), 128, 0, s>>>(
                c->nion, 2.0 * (c->ispin == 1 ? 2.0 : 1.0), c->proj_off, c->lmmax, c->katm, c->fpart, c->fnl, c->ewp,
                c->dti, c->r1, c->fion, c->r2);
            c->nlaunch += 1;
        }
        if (nbl > 0) {
            ZEpilogue e{};
            e.c2 = c2 + (long)lo * c->ldc;
            e.c1 = c1 + (long)lo * c->ldc;
            e.cpsi = c->cpsi + (long)lo * c->ldc;
            e.ldc = c->ldc;
            e.scal1 = c->scal1;
            e.dte = c->dte;
            e.tg = c->tg;
            e.has_nl = c->nproj > 0;
            c->fft->fwd_z_sd(c->g, c->Tb, e, nbl, s); c->nlaunch += 1;
        }
        if (c->mlp) {  // learned step scales per band and |G| shell
            // The residual R = cpsi - C1 (C1' W cpsi) per spin: only R is
            // preconditioned, so the update is plain SD wherever R = 0 and the
            // fixed point H psi = psi Lambda is that of plain SD.
            for (int ms = 0; ms < c->ispin; ++ms) {
                const int m = ms ? c->ne1 : c->ne0;
                const long off = (long)(ms ? c->ne0 : 0) * ldr;
                double *Mt = c->pM + (long)ms * c->ne0 * c->ne0;  // Mt[b][a] = <cpsi_b|c1_a>
                int rc = gemm_tn(c, m, m, K, (const double *)c->cpsi + off, ldr, (const double *)c1 + off, ldr, c->w,
                                 1.0, 0.0, Mt, m, TN_PROJECTOR);
                if (rc) return rc;
                // pR = -C1 Mt; the update adds cpsi (R = cpsi + pR)
                gemm_nn(c, m, K, m, -1.0, Mt, m, (const double *)c1 + off, ldr, 0.0, (double *)c->pR + off, ldr,
                        TN_PROJECTOR);
            }
            band_stats_kernel<<<c->nb, 256, 0, s>>>(c->npw, c->ldc, c->w, c->tg, c1, c->cpsi, c->pstats);
            prec_mlp_kernel<<<mlp_forward_blocks((long)c->nb * kShells), kMlpTileThreads, 0, s>>>(
                c->nb, c->tmax, c->pstats, c->dstep, c->mlp->wq, c->mlp->p, c->py);
            prec_update_kernel<<<(unsigned)cdiv((long)c->nb * c->npw, 256), 256, 0, s>>>(
                c->nb, c->npw, c->ldc, c->shell, c->py, c->pcap, c->dte, c->cpsi, c->pR, c2, c->dstep);
            c->nlaunch += 3;
        }
        mark(c, 9);
        CK(cudaGetLastError());
        return CPSD_OK;
    }
    // phase 2: overlaps and Lagrange multipliers, cpsd.c:415-479
    LagArgs la{};
    la.ispin = c->ispin;
    la.ne0 = c->ne0;
    la.ne1 = c->ne1;
    la.dte = c->dte;
    const long ne02 = (long)c->ne0 * c->ne0;
    for (int ms = 0; ms < c->ispin; ++ms) {
        const int m = ms ? c->ne1 : c->ne0;
        const long off = (long)(ms ? c->ne0 : 0) * ldr;
        const double *C1 = (const double *)c1 + off, *C2 = (const double *)c2 + off;
        // the three overlaps of this spin: C2'WC2, C2'WC1, C1'WC1
        double *Cs[3] = {(double *)Mblk(c, ms, 0), (double *)Mblk(c, ms, 1), (double *)Mblk(c, ms, 2)};
        int rc = overlaps3(c, m, K, ldr, C2, C1, Cs);
        if (rc) return rc;
        la.M22[ms] = Mblk(c, ms, 0);
        la.M21[ms] = Mblk(c, ms, 1);
        la.M11[ms] = Mblk(c, ms, 2);
    }
    mark(c, 10);
    la.s11 = c->lag;
    la.s12 = c->lag + ne02;
    la.s21 = c->lag + 2 * ne02;
    la.s22 = c->lag + 3 * ne02;
    la.st1 = c->lag + 4 * ne02;
    la.X0 = c->lag + 5 * ne02;
    la.X1 = c->lag + 6 * ne02;
    la.lmd = c->lmd;
    la.red = c->red;
    la.fail = c->flags;
    la.lb = c->lag_lb;
    if (c->ne0 <= kLagSmallMax)
        lagrange_small_kernel<<<1, kLagThreads, lag_small_smem_bytes(c->ne0), s>>>(la);
    else if (c->lag_tile) {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kLagTileGrid * kLagTileGrid;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(kLagTileGrid * kLagTileGrid);
        cfg.blockDim = dim3(kLagThreads);
        cfg.dynamicSmemBytes = lagrange_tile_smem(c->ne0);
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, lagrange_tile_kernel, la));
    } else {
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = c->lag_cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(c->lag_cluster);
        cfg.blockDim = dim3(kLagThreads);
        cfg.dynamicSmemBytes = lagrange_cluster_smem(c->ne0, c->lag_cluster, c->lag_lb);
        cfg.stream = s;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, lagrange_kernel, la));
    }
    c->nlaunch += 1;
    mark(c, 11);
    // constraint correction c2 += dte C1 lmd, cpsd.c:482-488
    for (int ms = 0; ms < c->ispin; ++ms) {
        const int m = ms ? c->ne1 : c->ne0;
        const long off = (long)(ms ? c->ne0 : 0) * ldr;
        gemm_nn(c, m, K, m, c->dte, c->lmd + ms * ne02, m, (const double *)c1 + off, ldr, 1.0,
                (double *)c2 + off, ldr, TN_OVERLAPS);
    }
    mark(c, 12);
    CK(cudaGetLastError());
    c->cur ^= 1;
    return CPSD_OK;
}

int one_step(cpsd_gpu_ctx *c)
{
    for (int phase = 0; phase < 3; ++phase) {
        int rc = step_phase(c, phase);
        if (rc) return rc;
    }
    return CPSD_OK;
}

void drop_graphs(cpsd_gpu_ctx *c)
{
    for (auto &g : c->gexec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto &m : c->mgraphs) cudaGraphExecDestroy(m.exec);
    c->mgraphs.clear();
}

// One SD step, replayed from a CUDA graph captured on first use (one graph
// per ping-pong parity of the orbital buffers).
int run_step(cpsd_gpu_ctx *c)
{
    if (!c->use_graph) return one_step(c);
    const int par = c->cur;
    if (!c->gexec[par]) {
        cudaGraph_t g = nullptr;
        const long long before = c->nlaunch;
        CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
        int rc = one_step(c);
        cudaError_t e = cudaStreamEndCapture(c->st, &g);
        c->cur = par;  // capture launched nothing: undo the buffer flip
        c->graph_launches = (int)(c->nlaunch - before);
        c->nlaunch = before;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        CK(e);
        e = cudaGraphInstantiate(&c->gexec[par], g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }
    CK(cudaGraphLaunch(c->gexec[par], c->st));
    c->nlaunch += c->graph_launches;
    c->cur ^= 1;
    return CPSD_OK;
}

// `inner` SD steps as few graph launches: up to kStepsPerGraph steps are
// captured into one graph (per step count and ping-pong parity, the last
// kMultiGraphs kept), so a cpsd() call of 10 steps is one launch.
constexpr int kStepsPerGraph = 32;
constexpr size_t kMultiGraphs = 4;

int run_steps(cpsd_gpu_ctx *c, int inner)
{
    if (!c->use_graph || c->phase_timing) {
        c->rec_dn = true;
        for (int it = 0; it < inner; ++it) {
            int rc = run_step(c);
            if (rc) {
                c->rec_dn = false;
                return rc;
            }
        }
        c->rec_dn = false;
        return CPSD_OK;
    }
    while (inner > 0) {
        const int k = std::min(inner, kStepsPerGraph);
        const int par = c->cur;
        cpsd_gpu_ctx::MultiGraph *m = nullptr;
        for (auto &x : c->mgraphs)
            if (x.steps == k && x.par == par) m = &x;
        if (!m) {
            cudaGraph_t g = nullptr;
            const long long before = c->nlaunch;
            CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
            int rc = CPSD_OK;
            for (int it = 0; it < k && !rc; ++it) {
                c->rec_dn = it == k - 1;  // one record of ev_dn per graph, in its last step
                rc = one_step(c);
            }
            c->rec_dn = false;
            cudaError_t e = cudaStreamEndCapture(c->st, &g);
            c->cur = par;  // capture launched nothing: undo the buffer flips
            const int launches = (int)(c->nlaunch - before);
            c->nlaunch = before;
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            CK(e);
            cudaGraphExec_t ex = nullptr;
            e = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            CK(e);
            if (c->mgraphs.size() >= kMultiGraphs) {
                cudaGraphExecDestroy(c->mgraphs.front().exec);
                c->mgraphs.erase(c->mgraphs.begin());
            }
            c->mgraphs.push_back({k, par, launches, ex});
            m = &c->mgraphs.back();
        }
        CK(cudaGraphLaunch(m->exec, c->st));
        c->nlaunch += m->launches;
        if (k & 1) c->cur ^= 1;
        inner -= k;
    }
    return CPSD_OK;
}

int energies(cpsd_gpu_ctx *c, int inner)
{
    cudaStream_t s = c->st;
    const cx<double> *c2 = c->cbuf[c->cur], *c1 = c->cbuf[c->cur ^ 1];
    const int K = 2 * c->npw_pad;
    const long ldr = 2L * c->npw_pad;
    FinalArgs fa{};
    for (int ms = 0; ms < c->ispin; ++ms) {
        const int m = ms ? c->ne1 : c->ne0;
        const long off = (long)(ms ? c->ne0 : 0) * ldr;
        int rc = gemm_tn(c, m, m, K, (const double *)c1 + off, ldr, (const double *)c->cpsi + off, ldr, c->w,
                         1.0, 0.0, (double *)Mblk(c, ms, 3), m);
        if (rc) return rc;
        fa.Mh[ms] = Mblk(c, ms, 3);
    }
    packed_terms_kernel<<<c->pblocks, 256, 0, s>>>(c->npw, c->w, c->sfac, c->vg, c->dng, c->vc, c->vall,
                                                   c->ppart); c->nlaunch += 1;
    band_terms_kernel<<<dim3(c->bblocks, c->nb), 256, 0, s>>>(c->npw, c->ldc, c->w, c->tg, c1, c2, c->bpart); c->nlaunch += 1;
    grid_terms_kernel<<<c->gblocks, 256, 0, s>>>(c->n3, c->ispin, c->dn, c->xce, c->xcp, c->gpart); c->nlaunch += 1;
    fa.ispin = c->ispin;
    fa.ne0 = c->ne0;
    fa.ne1 = c->ne1;
    fa.nion = c->nion;
    fa.nsh = c->nsh;
    fa.nproj = c->nproj;
    fa.nb = c->nb;
    fa.inner = inner;
    fa.pblocks = c->pblocks;
    fa.bblocks = c->bblocks;
    fa.gblocks = c->gblocks;
    fa.ppart = c->ppart;
    fa.bpart = c->bpart;
    fa.gpart = c->gpart;
    fa.hml = c->hml;
    fa.beta = c->beta;
    fa.vnlnrm_p = c->vnlnrm_p;
    if (c->nion > 1) {
        ewald_real_kernel<<<c->nion - 1, 256, 0, s>>>(c->nion, c->nsh, c->r1, c->rcell, c->zv, c->katm,
                                                      c->prm.rcut, c->epart);
        c->nlaunch += 1;
    }
    fa.ewald_part = c->epart;
    fa.scal2 = c->scal2;
    fa.omega = c->prm.omega;
    fa.dv = c->dv;
    fa.cewald = c->prm.cewald;
    fa.rcut = c->prm.rcut;
    fa.dt = c->prm.dt;
    fa.dte = c->dte;
    fa.E = c->Edev;
    final_energy_kernel<<<1, kFinalThreads, 0, s>>>(fa); c->nlaunch += 1;
    CK(cudaGetLastError());
    return CPSD_OK;
}

}  // namespace

// Full-box (unpruned) single-field transform used by the cr_fft3b_ /
// rc_fft3f_ drop-ins (capi.cu): dir > 0 packed -> real grid, dir < 0 real
// grid -> packed.  Engines are cached per (grid, device); callers serialise.
int cpsd_fft_run_full(int n, int dir, const Geom &g, double *grid, cx<double> *packed, void *Taux,
                      cudaStream_t st, int kx, int *ok)
{
    struct Cached {
        int n, dev;
        DevArena ar;
        std::unique_ptr<FftOps> ops;
        bool inv_ok, fwd_ok;
    };
    static std::vector<std::unique_ptr<Cached>> cache;
    *ok = 0;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    Cached *e = nullptr;
    for (auto &c : cache)
        if (c->n == n && c->dev == dev) e = c.get();
    if (!e) {
        std::unique_ptr<Cached> c(new Cached());
        c->n = n;
        c->dev = dev;
        c->ops = make_fft(n);
        if (!c->ops) return CPSD_ERR_GRID;
        int optin = 0;
        CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        c->inv_ok = (int)plane_need(n, PM_INVREAL, kx, 0) <= optin;
        c->fwd_ok = (int)plane_need(n, PM_FWDREAL, kx, 0) <= optin;
        int rc = c->ops->init(c->ar, kx, 0);
        if (rc) return rc;
        e = c.get();
        cache.push_back(std::move(c));
    }
    if (dir > 0) {
        if (!e->inv_ok) return CPSD_ERR_GRID;
        e->ops->inv_z(g, packed, g.npw, Taux, 1, st);
        PlaneArgs pv{};
        pv.rout = grid;
        pv.nout = 1;
        e->ops->plane(PM_INVREAL, g, Taux, pv, 1, st);
    } else {
        if (!e->fwd_ok) return CPSD_ERR_GRID;
        PlaneArgs pf{};
        pf.rin = grid;
        e->ops->plane(PM_FWDREAL, g, Taux, pf, 1, st);
        e->ops->fwd_z_store(g, Taux, packed, g.npw, 1.0, 1, st);
    }
    CK(cudaGetLastError());
    *ok = 1;
    return CPSD_OK;
}

// ------------------------------------------------------------ batches of cells
// Many independent cells stepped together: one CUDA graph per SD step holds
// one branch per cell (forked from and joined to the batch's stream), so the
// small kernels of uneven cells run concurrently and the whole batch costs
// one graph launch per step.
struct cpsd_gpu_batch {
    std::vector<cpsd_gpu_ctx *> cells;
    cudaStream_t st = nullptr;
    std::vector<cudaEvent_t> ev;  // fork + one join per cell
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_launches = 0;
    long long nlaunch = 0;
};

namespace {

void batch_drop_graphs(cpsd_gpu_batch *b)
{
    for (auto &g : b->gexec)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

int batch_step(cpsd_gpu_batch *b)
{
    const int par = b->cells[0]->cur;
    if (!b->gexec[par]) {
        cudaGraph_t g = nullptr;
        std::vector<long long> before;
        for (auto *c : b->cells) before.push_back(c->nlaunch);
        CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int rc = CPSD_OK;
        cudaError_t e = cudaEventRecord(b->ev[0], b->st);
        for (size_t i = 0; i < b->cells.size() && e == cudaSuccess && rc == CPSD_OK; ++i) {
            cpsd_gpu_ctx *c = b->cells[i];
            e = cudaStreamWaitEvent(c->st, b->ev[0], 0);
            if (e == cudaSuccess) rc = one_step(c);
            c->cur = par;  // capture launched nothing: undo the buffer flip
            if (e == cudaSuccess) e = cudaEventRecord(b->ev[1 + i], c->st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->st, b->ev[1 + i], 0);
        }
        cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
        long long captured = 0;
        for (size_t i = 0; i < b->cells.size(); ++i) {  // capture launched nothing
            captured += b->cells[i]->nlaunch - before[i];
            b->cells[i]->nlaunch = before[i];
        }
        b->graph_launches = (int)captured;
        if (rc || e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
            return rc ? rc : CPSD_ERR_CUDA;
        }
        e = cudaGraphInstantiate(&b->gexec[par], g, 0);
        cudaGraphDestroy(g);
        CK(e);
    }
    CK(cudaGraphLaunch(b->gexec[par], b->st));
    b->nlaunch += b->graph_launches;
    for (auto *c : b->cells) c->cur ^= 1;
    return CPSD_OK;
}

// ------------------------------------------------- host-layout orbitals
// The reference keeps every band on the full half-box grid (nfft3d complex
// values), zero outside the plane-wave sphere (ccpsdv3/cpsd.c:171-205 reads
// and writes c1, c2, cpsi there).  Only the sphere crosses PCIe: host threads
// gather it into pinned staging (checking that the rest is zero) and write
// the grids back as zeros plus the scattered sphere.

// Pinned staging of the packed tables: slices handed out in order (16-byte
// aligned), each copied to its device array by one cudaMemcpyAsync.
struct Stager {
    char *base;
    size_t cap;
    cudaStream_t s;
    size_t off = 0;
    bool full = false;
    cudaError_t err = cudaSuccess;
    long long bytes = 0;
    template <typename T>
    T *slice(size_t n)
    {
        const size_t b = (n * sizeof(T) + 15) / 16 * 16;
        if (off + b > cap) {
            full = true;
            return reinterpret_cast<T *>(base);
        }
        T *p = reinterpret_cast<T *>(base + off);
        off += b;
        return p;
    }
    bool ok() const { return !full; }
    template <typename T>
    void put(T *dst, const T *src, size_t n)
    {
        if (n == 0 || err != cudaSuccess) return;
        err = cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
        bytes += (long long)(n * sizeof(T));
    }
};

// Slices of one band's grid for the host threads (about 512 KB each).
long grid_slices(const cpsd_gpu_ctx *c)
{
    return std::max<long>(1, cdiv(c->nfft3d * (long)sizeof(cx<double>), 512L << 10));
}

// The packed form of the tables (TableArgs, dropin.h): the sphere's values
// in one staging buffer, slices 16-byte aligned in a fixed order.
struct TablePack {
    double *tg, *vc, *vg, *vl, *vnl, *zv, *ug, *rc, *n, *g;
    int *sh, *lm, *k, *o;
    size_t bytes;  // of the buffer used
    int np;        // projectors
    bool motion;   // G vectors and masses given
    double tmax;
};

// Checks the arguments and packs the tables into base (cap bytes): the
// gathers in the grids' memory order (pt_ord), on the host threads when
// threads is set (each table an item), else on the calling thread.
int pack_tables(const cpsd_gpu_ctx *c, const TableArgs &t, char *base, size_t cap, bool threads, TablePack *pk)
{
    if (!t.zv || !t.tg || !t.vc || !t.vg || !t.lmmax || !t.vnlnrm || !t.vl || !t.vnl) return CPSD_ERR_ARG;
    if (c->nion > 0 && (!t.katm || !t.rcell)) return CPSD_ERR_ARG;
    const HostGeom &h = c->hg;
    const int nkatm = c->nkatm;
    for (int ia = 0; ia < nkatm; ++ia)
        if (t.lmmax[ia] < 0 || t.lmmax[ia] > 9) return CPSD_ERR_ARG;
    std::vector<int> off(std::max(c->nion, 1), 0), hk(std::max(c->nion, 1), 0);
    int np = 0;
    for (int ii = 0; ii < c->nion; ++ii) {
        const int ia = t.katm[ii];
        if (ia < 0 || ia >= nkatm) return CPSD_ERR_ARG;
        hk[ii] = ia;
        off[ii] = np;
        np += t.lmmax[ia];
    }
    const bool motion = t.G && t.amass && c->nion > 0;
    if (motion)
        for (int ia = 0; ia < nkatm; ++ia)
            if (!(t.amass[ia] > 0)) return CPSD_ERR_ARG;
    Stager sg{base, cap, nullptr};
    const int npw = c->npw, npw_pad = c->npw_pad;
    const int *pt = h.pt_idx.data();
    TablePack &p = *pk;
    p.tg = sg.slice<double>(npw_pad);
    p.vc = sg.slice<double>(npw_pad);
    p.vg = sg.slice<double>(npw_pad);
    p.sh = sg.slice<int>(npw_pad);
    p.vl = sg.slice<double>((size_t)nkatm * npw);
    p.vnl = sg.slice<double>((size_t)nkatm * 9 * npw);
    p.zv = sg.slice<double>(nkatm);
    p.ug = sg.slice<double>(9);
    p.rc = sg.slice<double>(3 * c->nsh);
    p.lm = sg.slice<int>(nkatm);
    p.k = sg.slice<int>(c->nion);
    p.o = sg.slice<int>(c->nion);
    p.n = sg.slice<double>(np);
    p.g = sg.slice<double>(motion ? (size_t)3 * npw : 0);
    if (!sg.ok()) return CPSD_ERR_ARG;  // more kinds / ions than the context was created for
    p.bytes = sg.off;
    p.np = np;
    p.motion = motion;
    const int *ord = h.pt_ord.data();
    for (int q = npw; q < npw_pad; ++q) p.tg[q] = p.vc[q] = p.vg[q] = 0.0;
    const int ntab = 3 + nkatm * 10 + (motion ? 3 : 0);
    auto gather = [&](int i) {
        const double *src;
        double *d;
        if (i < 3) {
            src = i == 0 ? t.tg : (i == 1 ? t.vc : t.vg);
            d = i == 0 ? p.tg : (i == 1 ? p.vc : p.vg);
        } else if (i < 3 + nkatm * 10) {
            const int ia = (i - 3) / 10, l = (i - 3) % 10;  // l = 0: vl, else vnl channel l - 1
            if (l == 0) {
                src = t.vl + (size_t)ia * c->nfft3d;
                d = p.vl + (size_t)ia * npw;
            } else {
                d = p.vnl + ((size_t)ia * 9 + l - 1) * npw;
                if (l - 1 >= t.lmmax[ia]) {
                    memset(d, 0, sizeof(double) * npw);
                    return;
                }
                src = t.vnl + ((size_t)ia * 9 + l - 1) * c->nfft3d;
            }
        } else {
            const int dd = i - 3 - nkatm * 10;
            src = t.G + (size_t)dd * c->nfft3d;
            d = p.g + (size_t)dd * npw;
        }
        for (int q = 0; q < npw; ++q) {
            const int pp = ord[q];
            d[pp] = src[pt[pp]];
        }
    };
    if (threads)
        cpsd_host::Pool::get().run(ntab, gather);
    else
        for (int i = 0; i < ntab; ++i) gather(i);
    double tmax = 0.0;
    for (int q = 0; q < npw; ++q) tmax = std::max(tmax, p.tg[q]);
    p.tmax = tmax > 0 ? tmax : 1.0;
    for (int q = 0; q < npw_pad; ++q) p.sh[q] = q < npw ? std::min(kShells - 1, (int)(p.tg[q] / p.tmax * kShells)) : 0;
    memcpy(p.zv, t.zv, sizeof(double) * nkatm);
    memcpy(p.ug, c->prm.unitg, sizeof(double) * 9);
    if (c->nsh > 0) memcpy(p.rc, t.rcell, sizeof(double) * 3 * c->nsh);
    memcpy(p.lm, t.lmmax, sizeof(int) * nkatm);
    if (c->nion > 0) {
        memcpy(p.k, hk.data(), sizeof(int) * c->nion);
        memcpy(p.o, off.data(), sizeof(int) * c->nion);
    }
    for (int ii = 0, q = 0; ii < c->nion; ++ii)
        for (int l = 0; l < t.lmmax[hk[ii]]; ++l) p.n[q++] = t.vnlnrm[hk[ii] * 9 + l];
    return CPSD_OK;
}

// Whether tables passed now equal the ones the device holds (the packed
// bytes of the last upload, the masses kept on the host): packed into
// scratch on the calling thread.
bool tables_current(const cpsd_gpu_ctx *c, const TableArgs &t, std::vector<char> &scratch)
{
    if (!c->tables_ok || c->tables_last.empty()) return false;
    scratch.resize(c->tstage_bytes);
    TablePack pk{};
    if (pack_tables(c, t, scratch.data(), scratch.size(), false, &pk)) return false;
    if (pk.np != c->nproj || pk.motion != c->motion_ok) return false;
    if (pk.motion && (c->amass_h.size() != (size_t)c->nkatm ||
                      memcmp(c->amass_h.data(), t.amass, sizeof(double) * c->nkatm)))
        return false;
    return pk.bytes == c->tables_last.size() && !memcmp(scratch.data(), c->tables_last.data(), pk.bytes);
}

// c->hstage[b][p] = full[b][pt_idx[p]], zero past npw; returns the number of
// nonzero points outside the sphere.
long host_gather(cpsd_gpu_ctx *c, const double *full)
{
    const cx<double> *src = reinterpret_cast<const cx<double> *>(full);
    const int *inv = c->hg.inv_idx.data();
    const long S = grid_slices(c), per = cdiv(c->nfft3d, S);
    std::atomic<long> outside{0};
    cpsd_host::Pool::get().run((int)(c->nb * S), [&](int t) {
        const int b = (int)(t / S);
        const long g0 = (t % S) * per, g1 = std::min(c->nfft3d, g0 + per);
        const cx<double> *sb = src + (long)b * c->nfft3d;
        cx<double> *d = c->hstage.p + (long)b * c->ldc;
        long bad = 0;
        for (long g = g0; g < g1; ++g) {
            const int p = inv[g];
            if (p >= 0)
                d[p] = sb[g];
            else
                bad += (sb[g].x != 0.0 || sb[g].y != 0.0);
        }
        if (t % S == 0)
            for (long p = c->npw; p < c->ldc; ++p) d[p] = cx<double>{0.0, 0.0};
        if (bad) outside += bad;
    });
    return outside.load();
}

// c->hstage[b][p] = full[b][pt_idx[p]], zero past npw: the sphere only (the
// rest of the grid is checked separately, see count_outside).
void host_gather_sphere(cpsd_gpu_ctx *c, const double *full)
{
    const cx<double> *src = reinterpret_cast<const cx<double> *>(full);
    const int *pt = c->hg.pt_idx.data(), *ord = c->hg.pt_ord.data();
    cpsd_host::Pool::get().run(c->nb, [&](int b) {
        const cx<double> *sb = src + (long)b * c->nfft3d;
        cx<double> *d = c->hstage.p + (long)b * c->ldc;
        for (int q = 0; q < c->npw; ++q) {
            const int p = ord[q];
            d[p] = sb[pt[p]];
        }
        for (long p = c->npw; p < c->ldc; ++p) d[p] = cx<double>{0.0, 0.0};
    });
}

// Nonzero values outside the sphere in slice t of the band grids (the
// slicing of grid_slices).
long count_outside(const cpsd_gpu_ctx *c, const double *full, int t)
{
    const cx<double> *src = reinterpret_cast<const cx<double> *>(full);
    const int *inv = c->hg.inv_idx.data();
    const long S = grid_slices(c), per = cdiv(c->nfft3d, S);
    const long b = t / S, g0 = (t % S) * per, g1 = std::min(c->nfft3d, g0 + per);
    const cx<double> *sb = src + b * c->nfft3d;
    long bad = 0;
    for (long g = g0; g < g1; ++g) bad += (inv[g] < 0) & (sb[g].x != 0.0 || sb[g].y != 0.0);
    return bad;
}

// Zero n doubles.  On x86-64 with non-temporal stores: the lines are only
// written, so they need not be read for ownership first; scalar stores at
// the unaligned ends, and a store fence so that later stores from other
// threads (the scatter of the sphere) land after these.
void zero_stream(double *p, size_t n)
{
#if defined(__x86_64__)
    size_t i = 0;
    for (; i < n && (reinterpret_cast<uintptr_t>(p + i) & 15) != 0; ++i) p[i] = 0.0;
    const __m128d z = _mm_setzero_pd();
    for (; i + 2 <= n; i += 2) _mm_stream_pd(p + i, z);
    for (; i < n; ++i) p[i] = 0.0;
    _mm_sfence();
#else
    memset(p, 0, sizeof(double) * n);
#endif
}

// Zero every band grid of the listed host arrays (nb x nfft3d complex each).
std::function<void(int)> zero_grids_task(const cpsd_gpu_ctx *c, std::vector<double *> grids, int *items)
{
    const long S = grid_slices(c), per = cdiv(c->nfft3d, S), nb = c->nb, nfft3d = c->nfft3d;
    *items = (int)(grids.size() * nb * S);
    return [grids, S, per, nb, nfft3d](int t) {
        const long gi = t / (nb * S), r = t % (nb * S), b = r / S;
        const long g0 = (r % S) * per, g1 = std::min(nfft3d, g0 + per);
        if (g1 > g0) zero_stream(grids[gi] + 2 * (b * nfft3d + g0), (size_t)2 * (g1 - g0));
    };
}

// Bits of get_state_host's `zeroed`: host grids known to be zero outside the sphere.
enum { ZERO_C1 = 1, ZERO_C2 = 2, ZERO_CPSI = 4 };

int get_state_host(cpsd_gpu_ctx *c, double *c1, double *c2, double *cpsi, double *dn, double *hml, double *lmd,
                   double *r1, double *r2, double *fion, unsigned zeroed)
{
    if (!c) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    cudaStream_t s = c->st;
    const long P = (long)c->nb * c->ldc;
    const size_t pb = sizeof(cx<double>) * P;
    const cx<double> *cc2 = c->cbuf[c->cur], *cc1 = c->ran ? c->cbuf[c->cur ^ 1] : cc2;
    cx<double> *h2 = c->hstage.p, *h1 = c->hstage.p + P;
    double *dst = reinterpret_cast<double *>(c->dstage.p);
    if (c->fetched) {  // c1, c2 and the density are in the staging already
        CK(cudaEventSynchronize(c->ev_fetch));
        c->fetched = false;
    } else {
        if (c2 || cpsi) {
            CK(cudaMemcpyAsync(h2, cc2, pb, cudaMemcpyDeviceToHost, s));
            c->d2h += (long long)pb;
        }
        if (c1 || cpsi) {
            CK(cudaMemcpyAsync(h1, cc1, pb, cudaMemcpyDeviceToHost, s));
            c->d2h += (long long)pb;
        }
        if (dn) {  // unpadded into pinned staging; the host adds the two pad reals per x line
            CK(cudaMemcpyAsync(dst, c->dn, sizeof(double) * c->ispin * c->n3, cudaMemcpyDeviceToHost, s));
            c->d2h += (long long)sizeof(double) * c->ispin * c->n3;
        }
    }
    const long ne02 = (long)c->ne0 * c->ne0, ne12 = (long)c->ne1 * c->ne1;
    c->d2h += (long long)sizeof(double) * ((hml ? ne02 + ne12 : 0) + (lmd ? ne02 + ne12 : 0) +
                                          (c->nion > 0 ? ((r1 ? 3 : 0) + (r2 ? 3 : 0)) * c->nion : 0));
    if (hml) CK(cudaMemcpyAsync(hml, c->hml, sizeof(double) * (ne02 + ne12), cudaMemcpyDeviceToHost, s));
    if (lmd) CK(cudaMemcpyAsync(lmd, c->lmd, sizeof(double) * (ne02 + ne12), cudaMemcpyDeviceToHost, s));
    if (c->nion > 0) {
        if (r1) CK(cudaMemcpyAsync(r1, c->r1, sizeof(double) * 3 * c->nion, cudaMemcpyDeviceToHost, s));
        if (r2) CK(cudaMemcpyAsync(r2, c->r2, sizeof(double) * 3 * c->nion, cudaMemcpyDeviceToHost, s));
        // the forces exist only after a move = 1 run (cpsd.c:246-364); as in
        // the reference, fion is left untouched otherwise
        if (fion && c->move) {
            CK(cudaMemcpyAsync(fion, c->fion, sizeof(double) * 3 * c->nion, cudaMemcpyDeviceToHost, s));
            c->d2h += (long long)sizeof(double) * 3 * c->nion;
        }
    }
    // zero the grids that need it while the copies run, then scatter the sphere
    std::vector<double *> zero;
    if (c1 && !(zeroed & ZERO_C1)) zero.push_back(c1);
    if (c2 && !(zeroed & ZERO_C2)) zero.push_back(c2);
    if (cpsi && !(zeroed & ZERO_CPSI)) zero.push_back(cpsi);
    auto &pool = cpsd_host::Pool::get();
    if (!zero.empty()) {
        int items = 0;
        auto task = zero_grids_task(c, zero, &items);
        pool.run(items, task);
    }
    CK(cudaStreamSynchronize(s));
    if (dn) {  // [ms][z][y][x] -> the reference's [ms][z][y][x(n+2)], pads zero (cpsd.c:185-194)
        const int n = c->n;
        const long lines = (long)c->ispin * n * n, per = 128;  // enough items for every host thread
        pool.run((int)cdiv(lines, per), [&](int t) {
            for (long l = t * per; l < std::min(lines, (t + 1) * per); ++l) {
                memcpy(dn + l * (n + 2), dst + l * n, sizeof(double) * n);
                dn[l * (n + 2) + n] = 0.0;
                dn[l * (n + 2) + n + 1] = 0.0;
            }
        });
    }
    struct Out {
        double *host;
        const cx<double> *a, *sub;
    } outs[3] = {{c1, h1, nullptr}, {c2, h2, nullptr}, {cpsi, h2, h1}};  // cpsi = c2 - c1
    std::vector<Out> todo;
    for (const Out &o : outs)
        if (o.host) todo.push_back(o);
    const int *pt = c->hg.pt_idx.data(), *ord = c->hg.pt_ord.data();
    pool.run((int)(todo.size() * c->nb), [&](int t) {
        const Out &o = todo[t / c->nb];
        const long b = t % c->nb;
        cx<double> *d = reinterpret_cast<cx<double> *>(o.host) + b * c->nfft3d;
        const cx<double> *a = o.a + b * c->ldc;
        if (o.sub) {
            const cx<double> *u = o.sub + b * c->ldc;
            for (int q = 0; q < c->npw; ++q) {
                const int p = ord[q];
                d[pt[p]] = cx<double>{a[p].x - u[p].x, a[p].y - u[p].y};
            }
        } else {
            for (int q = 0; q < c->npw; ++q) {
                const int p = ord[q];
                d[pt[p]] = a[p];
            }
        }
    });
    return CPSD_OK;
}

}  // namespace

// The drop-in's run-and-fetch: c2 has just been read by cpsd_gpu_set_state,
// which checked it is zero outside the sphere, so only its sphere is written
// back; c1 and cpsi are zeroed by host threads while the GPU runs the steps.
int cpsd_dropin_run_fetch(cpsd_gpu_ctx *c, int inner, int move, double *E, double *deltae, double *deltac,
                          double *deltar, double *c1, double *c2, double *cpsi, double *dn, double *hml,
                          double *lmd, double *r1, double *r2, double *fion)
{
    if (!c) return CPSD_ERR_ARG;
    const size_t gb = sizeof(double) * c->nb * c->n2ft3d;
    auto apart = [gb](const double *x, const double *y) {
        return !x || !y || (const char *)x + gb <= (const char *)y || (const char *)y + gb <= (const char *)x;
    };
    const bool separate = c2 && apart(c1, c2) && apart(cpsi, c2) && apart(c1, cpsi);
    std::vector<double *> zero;
    if (separate) {
        if (c1) zero.push_back(c1);
        if (cpsi) zero.push_back(cpsi);
    }
    auto &pool = cpsd_host::Pool::get();
    if (!zero.empty()) {
        int items = 0;
        auto task = zero_grids_task(c, zero, &items);
        pool.start(items, task);  // the pool is held until the wait below
    }
    const int run = cpsd_gpu_run(c, inner, move, E, deltae, deltac, deltar);
    if (!zero.empty()) pool.wait();
    if (run != CPSD_OK && run != CPSD_WARN_LAGRANGE) return run;
    const unsigned zeroed = separate ? (ZERO_C1 | ZERO_C2 | ZERO_CPSI) : 0u;
    const int rc = get_state_host(c, c1, c2, cpsi, dn, hml, lmd, r1, r2, fion, zeroed);
    return rc ? rc : run;
}

// The drop-in's whole call after the tables: c2's sphere is gathered and
// uploaded and the steps start at once; host threads meanwhile check that c2
// is zero outside the sphere (the reference keeps it masked, and the pruned
// transforms rely on it) and only then zero c1 and cpsi for the outputs.  A
// c2 with values outside the sphere returns CPSD_ERR_UNMASKED_PSI with every
// output untouched; the context's device state is then that of a discarded
// run and the next call uploads its own.  Outputs that share memory take the
// serial path (check, run, then zero and scatter).
int cpsd_dropin_state_run_fetch(cpsd_gpu_ctx *c, const double *r2in, int inner, int move, double *E,
                                double *deltae, double *deltac, double *deltar, double *c1, double *c2,
                                double *cpsi, double *dn, double *hml, double *lmd, double *r1, double *r2,
                                double *fion, const DropinCheck *check)
{
    if (!c || !c2 || (c->nion > 0 && !r2in)) return CPSD_ERR_ARG;
    const size_t gb = sizeof(double) * c->nb * c->n2ft3d;
    auto apart = [gb](const double *x, const double *y) {
        return !x || !y || (const char *)x + gb <= (const char *)y || (const char *)y + gb <= (const char *)x;
    };
    if (!(apart(c1, c2) && apart(cpsi, c2) && apart(c1, cpsi))) {
        if (check) return kDropinRedo;  // the serial path checks first: no speculation
        const int rc = cpsd_gpu_set_state(c, c2, r2in);
        if (rc) return rc;
        return cpsd_dropin_run_fetch(c, inner, move, E, deltae, deltac, deltar, c1, c2, cpsi, dn, hml, lmd, r1,
                                     r2, fion);
    }
    CK(cudaSetDevice(c->prm.device));
    cudaStream_t s = c->st;
    CK(cudaStreamSynchronize(s));  // the staging buffer may still feed an earlier copy
    host_gather_sphere(c, c2);
    const size_t pb = sizeof(cx<double>) * c->nb * c->ldc;
    CK(cudaMemcpyAsync(c->cbuf[c->cur], c->hstage.p, pb, cudaMemcpyHostToDevice, s));
    if (c->nion > 0) CK(cudaMemcpyAsync(c->r2, r2in, sizeof(double) * 3 * c->nion, cudaMemcpyHostToDevice, s));
    c->h2d += (long long)pb + (long long)sizeof(double) * 3 * c->nion;
    c->state_ok = true;
    // items [0, ns): the DropinCheck (mask and tables, one item); [ns, ns +
    // nv): the check of c2; then the zeroing of c1 and cpsi, each of which
    // first waits for every check (the items are claimed in order, so every
    // check item is running or done by then) and is skipped after a failed
    // one, so that a refused or redone call leaves the outputs untouched
    const long S = grid_slices(c);
    const int ns = check ? 1 : 0, nv = (int)(c->nb * S);
    std::vector<double *> zero;
    if (c1) zero.push_back(c1);
    if (cpsi) zero.push_back(cpsi);
    int nz = 0;
    auto ztask = zero.empty() ? std::function<void(int)>() : zero_grids_task(c, zero, &nz);
    std::atomic<long> bad{0};
    std::atomic<int> checked{0}, stale{0};
    std::vector<char> scratch;
    auto &pool = cpsd_host::Pool::get();
    pool.start(ns + nv + nz, [&](int t) {
        if (t < ns) {
            const bool same = check->masker_n == (size_t)2 * c->nfft3d &&
                              !memcmp(check->masker, check->masker_ref, sizeof(int) * check->masker_n) &&
                              tables_current(c, check->tables, scratch);
            if (!same) stale = 1;
            checked.fetch_add(1, std::memory_order_release);
            return;
        }
        t -= ns;
        if (t < nv) {
            const long n = count_outside(c, c2, t);
            if (n) bad += n;
            checked.fetch_add(1, std::memory_order_release);
            return;
        }
        while (checked.load(std::memory_order_acquire) < ns + nv) std::this_thread::yield();
        if (bad.load() == 0 && stale.load() == 0) ztask(t - nv);
    });
    // the energies go to the caller only once the check has passed (E[0]
    // comes in as the previous call's energy, for deltae)
    double Et[10], dt3[3] = {0.0, 0.0, 0.0};
    memcpy(Et, E, sizeof(Et));
    c->early_fetch = true;
    const int run = cpsd_gpu_run(c, inner, move, Et, &dt3[0], &dt3[1], &dt3[2]);
    c->early_fetch = false;
    pool.wait();
    if (stale.load() || bad.load() || (run != CPSD_OK && run != CPSD_WARN_LAGRANGE)) {
        if (c->fetched) {  // the staging is free again only once those copies are done
            CK(cudaEventSynchronize(c->ev_fetch));
            c->fetched = false;
        }
    }
    if (stale.load()) {  // the steps ran on another mask or other tables: discarded
        c->state_ok = false;
        return kDropinRedo;
    }
    if (bad.load()) {
        c->state_ok = false;
        return CPSD_ERR_UNMASKED_PSI;
    }
    memcpy(E, Et, sizeof(Et));
    if (deltae) *deltae = dt3[0];
    if (deltac) *deltac = dt3[1];
    if (deltar) *deltar = dt3[2];
    if (run != CPSD_OK && run != CPSD_WARN_LAGRANGE) return run;
    const int rc = get_state_host(c, c1, c2, cpsi, dn, hml, lmd, r1, r2, fion, ZERO_C1 | ZERO_C2 | ZERO_CPSI);
    return rc ? rc : run;
}

// ====================================================================== C ABI
extern "C" {

int cpsd_gpu_batch_create(cpsd_gpu_ctx **cells, int ncells, cpsd_gpu_batch **out)
{
    if (!cells || ncells < 1 || !out) return CPSD_ERR_ARG;
    *out = nullptr;
    const int dev = cells[0]->prm.device;
    for (int i = 0; i < ncells; ++i)
        if (!cells[i] || cells[i]->prm.device != dev || !cells[i]->tables_ok || !cells[i]->state_ok)
            return CPSD_ERR_ARG;
    std::unique_ptr<cpsd_gpu_batch> b(new cpsd_gpu_batch());
    b->cells.assign(cells, cells + ncells);
    CK(cudaSetDevice(dev));
    CK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
    b->ev.resize(ncells + 1);
    for (auto &e : b->ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // every cell must start from the same buffer parity
    for (auto *c : b->cells)
        if (c->cur != b->cells[0]->cur) return CPSD_ERR_ARG;
    *out = b.release();
    return CPSD_OK;
}

int cpsd_gpu_batch_run(cpsd_gpu_batch *b, int inner, double *E, double *deltae, double *deltac)
{
    if (!b || !E || inner < 1) return CPSD_ERR_ARG;
    CK(cudaSetDevice(b->cells[0]->prm.device));
    const int n = (int)b->cells.size();
    for (int i = 0; i < n; ++i) {
        cpsd_gpu_ctx *c = b->cells[i];
        if (c->move) {  // batched cells take fixed-ion steps
            drop_graphs(c);
            batch_drop_graphs(b);
            c->move = 0;
        }
        CK(cudaMemsetAsync(c->flags, 0, 3 * sizeof(int), b->st));
        CK(cudaMemcpyAsync(c->Edev, E + 10 * i, sizeof(double), cudaMemcpyHostToDevice, b->st));
    }
    for (int it = 0; it < inner; ++it) {
        int rc = batch_step(b);
        if (rc) return rc;
    }
    // energies per cell on its own stream after the batch's steps
    CK(cudaEventRecord(b->ev[0], b->st));
    int warn = 0;
    std::vector<double> Eh(16 * n);
    std::vector<int> fails(3 * n, 0);
    for (int i = 0; i < n; ++i) {
        cpsd_gpu_ctx *c = b->cells[i];
        CK(cudaStreamWaitEvent(c->st, b->ev[0], 0));
        int rc = energies(c, inner);
        if (rc) return rc;
        CK(cudaMemcpyAsync(&Eh[16 * i], c->Edev, sizeof(double) * 12, cudaMemcpyDeviceToHost, c->st));
        CK(cudaMemcpyAsync(&fails[3 * i], c->flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    }
    int timeout = 0;
    for (int i = 0; i < n; ++i) {
        cpsd_gpu_ctx *c = b->cells[i];
        CK(cudaStreamSynchronize(c->st));
        for (int k = 0; k < 10; ++k) E[10 * i + k] = Eh[16 * i + k];
        if (deltae) deltae[i] = Eh[16 * i + 10];
        if (deltac) deltac[i] = Eh[16 * i + 11];
        c->lag_fail_total += fails[3 * i];
        c->steps_run += inner;
        c->ran = true;
        warn |= fails[3 * i];
        timeout |= fails[3 * i + 2];
    }
    if (timeout) return CPSD_ERR_TIMEOUT;
    return warn ? CPSD_WARN_LAGRANGE : CPSD_OK;
}

void cpsd_gpu_batch_counters(const cpsd_gpu_batch *b, long long *out)
{
    if (!out) return;
    long long l = b ? b->nlaunch : 0;
    if (b)
        for (auto *c : b->cells) l += c->nlaunch;
    out[0] = l;
}

void *cpsd_gpu_batch_stream(cpsd_gpu_batch *b) { return b ? (void *)b->st : nullptr; }

void cpsd_gpu_batch_destroy(cpsd_gpu_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->cells[0]->prm.device);
    if (b->st) cudaStreamSynchronize(b->st);
    batch_drop_graphs(b);
    for (auto e : b->ev)
        if (e) cudaEventDestroy(e);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}


const char *cpsd_gpu_strerror(int status)
{
    switch (status) {
    case CPSD_OK: return "ok";
    case CPSD_ERR_CUDA: return cudaGetErrorString(last_cuda_error());
    case CPSD_ERR_ARG: return "invalid argument";
    case CPSD_ERR_TIMEOUT: return "a bounded wait on the device ran out (tensor-core pipeline)";
    case CPSD_ERR_SCRATCH: return "M*N exceeds the static scratch of the no-alloc entry point (CPSD_NOALLOC_MAX_DOUBLES)";
    case CPSD_ERR_GRID: return "unsupported FFT grid (nfft must be 16, 24, 32, 48, 64 or 128, and the sphere must fit the plane kernel)";
    case CPSD_ERR_BANDS: return "more than 256 bands in a spin channel";
    case CPSD_ERR_EMPTY_MASK: return "the cutoff mask selects no G vector";
    case CPSD_ERR_UNMASKED_PSI: return "orbital coefficients outside the cutoff mask";
    case CPSD_ERR_MOVE: return "move=1 requested but no G vectors / masses were given";
    case CPSD_ERR_EIG: return "the Jacobi eigen solve of hml did not converge in 60 sweeps";
    case CPSD_ERR_IO: return "an output file could not be written";
    case CPSD_WARN_LAGRANGE: return "ierr=10: Lagrange-multiplier iteration did not converge in 30 steps";
    default: return "unknown status";
    }
}

int cpsd_gpu_create(const cpsd_gpu_params *p, const int *masker1, cpsd_gpu_ctx **out)
{
    if (!p || !masker1 || !out) return CPSD_ERR_ARG;
    *out = nullptr;
    if (!grid_supported(p->nfft)) return CPSD_ERR_GRID;
    if (p->ispin != 1 && p->ispin != 2) return CPSD_ERR_ARG;
    if (p->ne[0] < 1 || p->ne[1] < 0 || (p->ispin == 2 && p->ne[1] > p->ne[0])) return CPSD_ERR_ARG;
    if (p->ispin == 1 && p->ne[1] != 0) return CPSD_ERR_ARG;
    if (p->ne[0] > 256 || p->ne[1] > 256) return CPSD_ERR_BANDS;
    if (p->nion < 0 || p->nkatm < 1 || p->nsh < 0 || p->omega <= 0 || p->fmass <= 0) return CPSD_ERR_ARG;
    std::unique_ptr<cpsd_gpu_ctx> c(new cpsd_gpu_ctx());
    c->prm = *p;
    c->n = p->nfft;
    c->nh = c->n / 2 + 1;
    c->ispin = p->ispin;
    c->ne0 = p->ne[0];
    c->ne1 = p->ne[1];
    c->nb = c->ne0 + c->ne1;
    c->nion = p->nion;
    c->nkatm = p->nkatm;
    c->nsh = p->nsh;
    c->nfft3d = (long)c->nh * c->n * c->n;
    c->n2ft3d = 2 * c->nfft3d;
    c->n3 = (long)c->n * c->n * c->n;
    c->scal1 = 1.0 / ((double)c->n * c->n * c->n);
    c->scal2 = 1.0 / p->omega;
    c->dv = p->omega * c->scal1;
    c->dte = p->dt / sqrt(p->fmass);
    c->use_graph = !getenv("CPSD_B200_NO_GRAPHS");
    c->hg = build_geom(c->n, masker1, false);
    HostGeom &h = c->hg;
    if (h.npw == 0) return CPSD_ERR_EMPTY_MASK;
    c->npw = h.npw;
    c->npw_pad = h.npw_pad;
    c->ldc = h.npw_pad;
    CK(cudaSetDevice(p->device));
    c->sms = device_sms();
    CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_sf, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_side, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c->ev_dn, cudaEventDisableTiming));
    c->cs = c->st;
    // the fused density plane must fit in shared memory
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, p->device));
    if (p->precision != CPSD_PREC_FP64 && p->precision != CPSD_PREC_MIXED) return CPSD_ERR_ARG;
    for (int m = 0; m < 4; ++m)
        if ((int)plane_need(c->n, m, h.KX, h.ncol, p->precision) > optin) return CPSD_ERR_GRID;
    DevArena &ar = c->ar;
    c->fft64 = make_fft(c->n, CPSD_PREC_FP64);
    if (!c->fft64) return CPSD_ERR_GRID;
    int rc = c->fft64->init(ar, h.KX, h.ncol);
    if (rc) return rc;
    if (p->precision == CPSD_PREC_MIXED) {
        c->fft32 = make_fft(c->n, CPSD_PREC_MIXED);
        rc = c->fft32->init(ar, h.KX, h.ncol);
        if (rc) return rc;
        CK(cudaFuncSetAttribute(tc_gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
        CK(cudaFuncSetAttribute(tc_overlaps3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kOvSmem));
        CK(cudaFuncSetAttribute(tc_gemm_nn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    }
    c->precision = p->precision;
    c->fft = (p->precision == CPSD_PREC_MIXED) ? c->fft32.get() : c->fft64.get();
    CK(upload(ar, &c->pt_i, h.pt_i));
    CK(upload(ar, &c->pt_j, h.pt_j));
    CK(upload(ar, &c->pt_k, h.pt_k));
    CK(upload(ar, &c->pt_idx, h.pt_idx));
    CK(upload(ar, &c->inv_idx, h.inv_idx));
    CK(upload(ar, &c->col_i, h.col_i));
    CK(upload(ar, &c->col_j, h.col_j));
    CK(upload(ar, &c->col_ptr, h.col_ptr));
    CK(upload(ar, &c->colidx, h.colidx));
    if (!h.yrun.empty()) CK(upload(ar, &c->yrun, h.yrun));
    CK(upload(ar, &c->w, h.w));
    c->g.n = c->n;
    c->g.nh = c->nh;
    c->g.KX = h.KX;
    c->g.ncol = h.ncol;
    c->g.npw = h.npw;
    c->g.npw_pad = h.npw_pad;
    c->g.col_i = c->col_i;
    c->g.col_j = c->col_j;
    c->g.col_ptr = c->col_ptr;
    c->g.pt_k = c->pt_k;
    c->g.colidx = c->colidx;
    c->g.yrun = c->yrun;

    const long P = c->npw_pad;
    const int nb = c->nb, nkatm = c->nkatm, nion = c->nion;
    CK(ar.alloc(&c->tg, P));
    CK(ar.alloc(&c->vc, P));
    CK(ar.alloc(&c->vg, P));
    CK(ar.alloc(&c->vl, (size_t)nkatm * c->npw));
    CK(ar.alloc(&c->vnl, (size_t)nkatm * 9 * c->npw));
    CK(ar.alloc(&c->zv, nkatm));
    CK(ar.alloc(&c->rcell, 3 * std::max(c->nsh, 1)));
    CK(ar.alloc(&c->unitg, 9));
    CK(ar.alloc(&c->katm, std::max(nion, 1)));
    CK(ar.alloc(&c->lmmax, nkatm));
    CK(ar.alloc(&c->proj_off, std::max(nion, 1)));
    CK(ar.alloc(&c->cbuf[0], (size_t)nb * P));
    CK(ar.alloc(&c->cbuf[1], (size_t)nb * P));
    CK(ar.alloc(&c->cpsi, (size_t)nb * P));
    CK(ar.alloc(&c->r1, 3 * std::max(nion, 1)));
    CK(ar.alloc(&c->r2, 3 * std::max(nion, 1)));
    CK(ar.alloc(&c->fion, 3 * std::max(nion, 1)));
    const size_t tbytes = c->fft64->elem() * (size_t)c->n * h.ncol;  // widest element
    {
        unsigned char *t = nullptr;
        CK(ar.alloc(&t, tbytes * nb));
        c->Tb = t;
        CK(ar.alloc(&t, tbytes));
        c->Taux = t;
    }
    // density chunks (bands summed by one CTA per z plane): the count that
    // minimises waves x bands per CTA over the SMs' resident slots, the
    // smallest such count (fewer partial densities to add); never across spins
    {
        const long slots = (long)c->sms * c->fft->plane_ctas_per_sm(PM_DENSITY) /
                           c->fft->plane_ctas_per_plane(PM_DENSITY);
        auto best_chunks = [&](int bands, int planes_per_chunk_group) {
            int best = 1;
            long best_cost = -1;
            for (int ch = 1; ch <= std::min(bands, 64); ++ch) {
                const long cost = cdiv((long)planes_per_chunk_group * ch, slots) * cdiv(bands, ch);
                if (best_cost < 0 || cost < best_cost) {
                    best_cost = cost;
                    best = ch;
                }
            }
            return best;
        };
        if (c->ispin == 1) {
            c->nchunk0 = best_chunks(c->ne0, c->n);
            c->nchunk1 = 0;
        } else {  // both spins share the launch: plan each with half of the slots
            c->nchunk0 = best_chunks(c->ne0, 2 * c->n);
            c->nchunk1 = c->ne1 > 0 ? best_chunks(c->ne1, 2 * c->n) : 0;
        }
        c->dens_model[0] = c->nchunk0;
        c->dens_model[1] = c->nchunk1;
        // room for up to max(4, 2 x the model's count) chunks per spin (tuning)
        c->dens_cap = std::min(std::max(4, 2 * std::max(c->nchunk0, c->nchunk1)), std::max(c->ne0, c->ne1));
        std::vector<int> b0 = density_chunk_table(c->ne0, c->nchunk0, c->ne1, c->nchunk1);
        b0.resize((size_t)2 * c->dens_cap + 1, 0);
        CK(upload(ar, &c->chunk_dens, b0));
        std::vector<int> bb(nb + 1);
        for (int b = 0; b <= nb; ++b) bb[b] = b;
        CK(upload(ar, &c->chunk_band, bb));
    }
    CK(ar.alloc(&c->rho_part, (size_t)(std::min(c->dens_cap, c->ne0) + std::min(c->dens_cap, c->ne1)) * c->n3));
    CK(ar.alloc(&c->dn, (size_t)c->ispin * c->n3));
    CK(ar.alloc(&c->xcp, (size_t)c->ispin * c->n3));
    CK(ar.alloc(&c->xce, (size_t)c->n3));
    CK(ar.alloc(&c->rfwd, (size_t)c->n3));
    CK(ar.alloc(&c->Vr, (size_t)c->ispin * c->n3));
    CK(ar.alloc(&c->dng, P));
    CK(ar.alloc(&c->vall, P));
    CK(ar.alloc(&c->sfac, P));
    CK(ar.alloc(&c->Vg, P));
    CK(ar.alloc(&c->ex1, (size_t)std::max(nion, 1) * c->nh));
    CK(ar.alloc(&c->ex2, (size_t)std::max(nion, 1) * c->n));
    CK(ar.alloc(&c->ex3, (size_t)std::max(nion, 1) * c->n));
    const long ne02 = (long)c->ne0 * c->ne0;
    CK(ar.alloc(&c->Mov, (size_t)8 * ne02));
    CK(ar.alloc(&c->lag, (size_t)7 * ne02 + 1));
    CK(ar.alloc(&c->lmd, (size_t)2 * ne02));
    CK(ar.alloc(&c->hml, (size_t)2 * ne02));
    CK(ar.alloc(&c->red, 2 * kLagClusterMax));
    CK(ar.alloc(&c->Edev, 16));
    CK(ar.alloc(&c->flags, 4));
    c->gemm_splits_cap = 512;
    // split-K partials: at least 32 MB, and room for one split per SM of the
    // three overlaps of the largest spin
    c->gemm_ws_elems = std::max<size_t>((size_t)4 << 20, (size_t)3 * c->ne0 * c->ne0 * c->sms);
    CK(ar.alloc(&c->gws, c->gemm_ws_elems));
    c->pblocks = c->sms;
    c->bblocks = (int)std::max<long>(1, std::min<long>(64, cdiv(c->npw, 256 * 8)));
    c->gblocks = 296;
    CK(ar.alloc(&c->ppart, 3 * c->pblocks));
    CK(ar.alloc(&c->bpart, (size_t)2 * nb * c->bblocks));
    CK(ar.alloc(&c->gpart, 2 * c->gblocks));
    CK(cudaMallocHost((void **)&c->hstage.p, sizeof(cx<double>) * 2 * nb * c->ldc));
    {
        // every slice cpsd_gpu_set_tables packs, each rounded up to 16 bytes
        const size_t P = (size_t)c->npw_pad, K = (size_t)c->nkatm, I = (size_t)std::max(nion, 1);
        c->tstage_bytes = 8 * (3 * P + P + K * P + 9 * K * P + K + 9 + 3 * (size_t)c->nsh + K + 2 * I + 9 * I +
                               3 * P) + 16 * 16;
        CK(cudaMallocHost((void **)&c->tstage.p, c->tstage_bytes));
        CK(cudaMallocHost((void **)&c->dstage.p, sizeof(double) * c->ispin * c->n3));
    }
    CK(ar.alloc(&c->shell, (size_t)c->npw_pad));
    CK(ar.alloc(&c->dstep, 1));
    CK(ar.alloc(&c->pcap, 2));
    CK(ar.alloc(&c->epart, std::max(nion, 1)));  // zero: the last ion has no pair of its own
    CK(ar.alloc(&c->Gv, (size_t)3 * c->npw));
    CK(ar.alloc(&c->dti, std::max(nion, 1)));
    CK(ar.alloc(&c->fpart, (size_t)kForceChunks * std::max(nion, 1) * 3));
    CK(ar.alloc(&c->fnl, (size_t)27 * std::max(nion, 1)));  // at most 9 projectors per ion
    CK(ar.alloc(&c->ewp, (size_t)3 * std::max<long>(1, (long)nion * (nion - 1) / 2)));
    CK(ar.alloc(&c->pR, (size_t)nb * P));
    CK(ar.alloc(&c->pM, (size_t)c->ispin * c->ne0 * c->ne0));
    CK(ar.alloc(&c->pstats, (size_t)3 * nb));
    CK(ar.alloc(&c->py, (size_t)nb * kShells));
    if (c->ne0 <= kLagSmallMax)
        CK(cudaFuncSetAttribute(lagrange_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)lag_small_smem_bytes(kLagSmallMax)));
    else {
        // 16-CTA clusters where the device can schedule them, else the portable 8
        CK(cudaFuncSetAttribute(lagrange_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        CK(allow_max_smem(lagrange_kernel, optin));
        const size_t limit = (size_t)optin - 1024;
        c->lag_cluster = kLagCluster;
        c->lag_lb = lagrange_lb(c->ne0, kLagCluster, limit);
        const int lb16 = lagrange_lb(c->ne0, kLagClusterMax, limit);
        if (lb16) {
            cudaLaunchConfig_t cfg{};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = kLagClusterMax;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(kLagClusterMax);
            cfg.blockDim = dim3(kLagThreads);
            cfg.dynamicSmemBytes = lagrange_cluster_smem(c->ne0, kLagClusterMax, lb16);
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, lagrange_kernel, &cfg) == cudaSuccess &&
                nclusters >= 1) {
                c->lag_cluster = kLagClusterMax;
                c->lag_lb = lb16;
            }
            (void)cudaGetLastError();
        }
        if (!c->lag_lb) return CPSD_ERR_BANDS;
        // the tiled solver where its 16-CTA clusters fit (CPSD_B200_LAGRANGE=cluster
        // keeps the column solver, for comparisons)
        const char *lag_env = getenv("CPSD_B200_LAGRANGE");
        const size_t tsm = lagrange_tile_smem(c->ne0);
        if (c->ne0 <= kLagTileMax && tsm <= limit) {
            CK(cudaFuncSetAttribute(lagrange_tile_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            CK(allow_max_smem(lagrange_tile_kernel, optin));
            cudaLaunchConfig_t cfg{};
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = kLagTileGrid * kLagTileGrid;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3(kLagTileGrid * kLagTileGrid);
            cfg.blockDim = dim3(kLagThreads);
            cfg.dynamicSmemBytes = tsm;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, lagrange_tile_kernel, &cfg) == cudaSuccess &&
                nclusters >= 1)
                c->lag_tile_ok = true;
            (void)cudaGetLastError();
        }
        c->lag_tile = c->lag_tile_ok && !(lag_env && !strcmp(lag_env, "cluster"));
    }
    CK(cudaDeviceSynchronize());  // allocation memsets run on the legacy stream
    *out = c.release();
    return CPSD_OK;
}

int cpsd_gpu_set_scalars(cpsd_gpu_ctx *c, const double *unitg, double omega, double dt, double fmass,
                         double cewald, double rcut)
{
    if (!c || !unitg || omega <= 0 || fmass <= 0) return CPSD_ERR_ARG;
    // the drop-in passes the same scalars on every call: keep the captured
    // step graphs unless a value changes
    const bool same = !memcmp(c->prm.unitg, unitg, sizeof(c->prm.unitg)) && c->prm.omega == omega &&
                      c->prm.dt == dt && c->prm.fmass == fmass && c->prm.cewald == cewald && c->prm.rcut == rcut;
    if (same) return CPSD_OK;
    memcpy(c->prm.unitg, unitg, sizeof(c->prm.unitg));
    c->prm.omega = omega;
    c->prm.dt = dt;
    c->prm.fmass = fmass;
    c->prm.cewald = cewald;
    c->prm.rcut = rcut;
    c->scal2 = 1.0 / omega;
    c->dv = omega * c->scal1;
    c->dte = dt / sqrt(fmass);
    drop_graphs(c);  // kernel arguments captured by value change
    return CPSD_OK;
}

int cpsd_gpu_set_tables(cpsd_gpu_ctx *c, const int *katm, const double *amass, const double *zv,
                        const double *rcell, const double *G, const double *tg, const double *vc,
                        const double *vg, const int *lmmax, const double *vnlnrm, const double *vl,
                        const double *vnl)
{
    if (!c) return CPSD_ERR_ARG;
    const TableArgs t{katm, amass, zv, rcell, G, tg, vc, vg, lmmax, vnlnrm, vl, vnl};
    CK(cudaSetDevice(c->prm.device));
    // pack into pinned staging (the previous upload from it has finished
    // once the stream is idle), then one asynchronous copy per table
    CK(cudaStreamSynchronize(c->st));
    TablePack pk{};
    int rc = pack_tables(c, t, reinterpret_cast<char *>(c->tstage.p), c->tstage_bytes, true, &pk);
    if (rc) return rc;
    const int np = pk.np, nkatm = c->nkatm, npw = c->npw, npw_pad = c->npw_pad;
    if (np != c->nproj || !c->proj) {
        drop_graphs(c);
        c->tables_last.clear();
        if (np > 0) {
            CK(c->ar.alloc(&c->proj, (size_t)np * c->npw_pad));
            CK(c->ar.alloc(&c->beta, (size_t)np * c->nb));
            CK(c->ar.alloc(&c->coefT, (size_t)np * c->nb));
            CK(c->ar.alloc(&c->vnlnrm_p, (size_t)np));
        }
        c->nproj = np;
    }
    c->tmax = pk.tmax;
    // a driver passes the same tables every call (ccpsdv3/main.c:422-426):
    // the device copies are current when the staged bytes are unchanged
    if (pk.motion) c->amass_h.assign(amass, amass + nkatm);
    if (c->tables_ok && c->tables_last.size() == pk.bytes && !memcmp(c->tables_last.data(), c->tstage.p, pk.bytes)) {
        c->motion_ok = pk.motion;
        return CPSD_OK;
    }
    Stager sg{reinterpret_cast<char *>(c->tstage.p), c->tstage_bytes, c->st};
    sg.put(c->tg, pk.tg, npw_pad);
    sg.put(c->shell, pk.sh, npw_pad);
    sg.put(c->vc, pk.vc, npw_pad);
    sg.put(c->vg, pk.vg, npw_pad);
    sg.put(c->vl, pk.vl, (size_t)nkatm * npw);
    sg.put(c->vnl, pk.vnl, (size_t)nkatm * 9 * npw);
    sg.put(c->zv, pk.zv, nkatm);
    sg.put(c->lmmax, pk.lm, nkatm);
    sg.put(c->unitg, pk.ug, 9);
    if (c->nion > 0) {
        sg.put(c->katm, pk.k, c->nion);
        sg.put(c->proj_off, pk.o, c->nion);
    }
    if (c->nsh > 0) sg.put(c->rcell, pk.rc, 3 * c->nsh);
    if (np > 0) sg.put(c->vnlnrm_p, pk.n, np);
    // ion motion needs the G vectors (packed like tg) and the masses
    c->motion_ok = false;
    if (pk.motion) {
        sg.put(c->Gv, pk.g, (size_t)3 * npw);
        c->motion_ok = true;
    }
    c->tables_last.clear();
    CK(sg.err);
    CK(cudaStreamSynchronize(c->st));
    c->h2d += sg.bytes;
    c->tables_last.assign(reinterpret_cast<const char *>(c->tstage.p),
                          reinterpret_cast<const char *>(c->tstage.p) + pk.bytes);
    c->tables_ok = true;
    return CPSD_OK;
}

int cpsd_gpu_set_state(cpsd_gpu_ctx *c, const double *c2, const double *r2)
{
    if (!c || !c2 || (c->nion > 0 && !r2)) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    cudaStream_t s = c->st;
    CK(cudaStreamSynchronize(s));  // the staging buffer may still feed an earlier copy
    if (host_gather(c, c2)) return CPSD_ERR_UNMASKED_PSI;  // device state untouched
    const size_t pb = sizeof(cx<double>) * c->nb * c->ldc;
    CK(cudaMemcpyAsync(c->cbuf[c->cur], c->hstage.p, pb, cudaMemcpyHostToDevice, s));
    if (c->nion > 0) CK(cudaMemcpyAsync(c->r2, r2, sizeof(double) * 3 * c->nion, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));
    c->h2d += (long long)pb + (long long)sizeof(double) * 3 * c->nion;
    c->state_ok = true;
    return CPSD_OK;
}

static int finish_call(cpsd_gpu_ctx *c, int inner, double *E, double *deltae, double *deltac, double *deltar);

int cpsd_gpu_run(cpsd_gpu_ctx *c, int inner, int move, double *E, double *deltae, double *deltac,
                 double *deltar)
{
    if (!c || !E || inner < 1) return CPSD_ERR_ARG;
    if (!c->tables_ok || !c->state_ok) return CPSD_ERR_ARG;
    if (move && !c->motion_ok) return CPSD_ERR_MOVE;  // no G vectors or masses were given
    CK(cudaSetDevice(c->prm.device));
    if ((move != 0) != (c->move != 0)) {
        drop_graphs(c);
        c->move = move ? 1 : 0;
    }
    if (c->move) {
        if (c->nproj > 0 && !c->Ynl) {
            CK(c->ar.alloc(&c->Ynl, (size_t)c->nproj * c->npw_pad));
            CK(c->ar.alloc(&c->coefP, (size_t)c->nproj * c->nb));
        }
        std::vector<double> dti(c->nion);  // cpsd.c:116-122
        std::vector<int> katm(c->nion);
        CK(cudaMemcpy(katm.data(), c->katm, sizeof(int) * c->nion, cudaMemcpyDeviceToHost));
        for (int ii = 0; ii < c->nion; ++ii) dti[ii] = c->prm.dt / sqrt(c->amass_h[katm[ii]]);
        CK(cudaMemcpy(c->dti, dti.data(), sizeof(double) * c->nion, cudaMemcpyHostToDevice));
    }
    if (c->bp) return CPSD_ERR_ARG;  // band-parallel contexts step by phases
    cudaStream_t s = c->st;
    CK(cudaMemsetAsync(c->flags, 0, 3 * sizeof(int), s));
    CK(cudaMemcpyAsync(c->Edev, E, sizeof(double), cudaMemcpyHostToDevice, s));
    int rc = run_steps(c, inner);
    if (rc) return rc;
    if (c->early_fetch) {  // the energies below only read c1, c2 and the density
        const size_t pb = sizeof(cx<double>) * c->nb * c->ldc;
        if (!c->ev_steps) {
            CK(cudaEventCreateWithFlags(&c->ev_steps, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->ev_fetch, cudaEventDisableTiming));
        }
        // the density and c1 (the last step's input orbitals) as soon as the
        // last step's density pass is done, c2 once the steps are
        CK(cudaStreamWaitEvent(c->st2, c->ev_dn, 0));
        CK(cudaMemcpyAsync(c->dstage.p, c->dn, sizeof(double) * c->ispin * c->n3, cudaMemcpyDeviceToHost, c->st2));
        CK(cudaMemcpyAsync(c->hstage.p + (long)c->nb * c->ldc, c->cbuf[c->cur ^ 1], pb, cudaMemcpyDeviceToHost,
                           c->st2));
        CK(cudaEventRecord(c->ev_steps, s));
        CK(cudaStreamWaitEvent(c->st2, c->ev_steps, 0));
        CK(cudaMemcpyAsync(c->hstage.p, c->cbuf[c->cur], pb, cudaMemcpyDeviceToHost, c->st2));
        CK(cudaEventRecord(c->ev_fetch, c->st2));
        c->d2h += 2LL * (long long)pb + (long long)sizeof(double) * c->ispin * c->n3;
        c->fetched = true;
    }
    return finish_call(c, inner, E, deltae, deltac, deltar);
}

// The energies of a call and what cpsd() returns besides the orbitals
// (cpsd.c:494-672), after its `inner` steps; E[0] on the device holds the
// previous total energy.
static int finish_call(cpsd_gpu_ctx *c, int inner, double *E, double *deltae, double *deltac, double *deltar)
{
    cudaStream_t s = c->st;
    int rc = energies(c, inner);
    if (rc) return rc;
    double Eh[16];
    int fl[3] = {0, 0, 0};
    CK(cudaMemcpyAsync(Eh, c->Edev, sizeof(double) * 12, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(fl, c->flags, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    c->h2d += sizeof(double);
    c->d2h += 12 * sizeof(double) + sizeof(int);
    for (int i = 0; i < 10; ++i) E[i] = Eh[i];
    if (deltae) *deltae = Eh[10];
    if (deltac) *deltac = Eh[11];
    double dr = 0.0;  // the largest force of the last step, cpsd.c:662-672
    if (c->move && c->nion > 0) {
        std::vector<double> f((size_t)3 * c->nion);
        CK(cudaMemcpy(f.data(), c->fion, sizeof(double) * f.size(), cudaMemcpyDeviceToHost));
        c->d2h += (long long)sizeof(double) * f.size();
        for (int ii = 0; ii < c->nion; ++ii) {
            const double a = sqrt(f[3 * ii] * f[3 * ii] + f[3 * ii + 1] * f[3 * ii + 1] + f[3 * ii + 2] * f[3 * ii + 2]);
            if (a > dr) dr = a;
        }
    }
    if (deltar) *deltar = dr;
    const int fails = fl[0];
    c->lag_fail_total += fails;
    c->steps_run += inner;
    c->ran = true;
    if (fl[2]) return CPSD_ERR_TIMEOUT;
    return fails ? CPSD_WARN_LAGRANGE : CPSD_OK;
}

int cpsd_gpu_get_state(cpsd_gpu_ctx *c, double *c1, double *c2, double *cpsi, double *dn, double *hml,
                       double *lmd, double *r1, double *r2, double *fion)
{
    return get_state_host(c, c1, c2, cpsi, dn, hml, lmd, r1, r2, fion, 0u);
}

int cpsd_gpu_epilogue(cpsd_gpu_ctx *c, double *ortho, double *eig, double *vec)
{
    if (!c) return CPSD_ERR_ARG;
    if (!c->ran) return CPSD_ERR_ARG;  // hml and c1 exist only after a run
    CK(cudaSetDevice(c->prm.device));
    cudaStream_t s = c->st;
    const long ne02 = (long)c->ne0 * c->ne0;
    if (!c->eigA) {
        CK(c->ar.alloc(&c->eigA, (size_t)2 * ne02));
        CK(c->ar.alloc(&c->eigV, (size_t)2 * ne02));
        CK(c->ar.alloc(&c->eigD, (size_t)2 * c->ne0));
        CK(c->ar.alloc(&c->eigVec, (size_t)2 * ne02));
        CK(c->ar.alloc(&c->ortho, (size_t)2 * ne02));
        CK(c->ar.alloc(&c->eig_sweeps, 2));
    }
    const cudaStream_t cs_saved = c->cs;
    c->cs = s;
    const int K = 2 * c->npw_pad;
    const long ldr = 2L * c->npw_pad;
    const double *c1 = (const double *)c->cbuf[c->cur ^ 1];
    const double *c2 = (const double *)c->cbuf[c->cur];
    // orthonormality of c1 (main.c:455-467): <c1_i|c1_j>, Gamma-point dots
    if (ortho) {
        for (int ms = 0; ms < c->ispin; ++ms) {
            const int m = ms ? c->ne1 : c->ne0;
            const long off = (long)(ms ? c->ne0 : 0) * ldr;
            // row-major M x M from the TN product equals its column-major transpose (symmetric)
            const int rc = gemm_tn(c, m, m, K, c1 + off, ldr, c1 + off, ldr, c->w, 1.0, 0.0, c->ortho + ms * ne02, m);
            if (rc) {
                c->cs = cs_saved;
                return rc;
            }
        }
    }
    // eigenpairs of hml per spin (main.c:470-479)
    EigArgs ea{};
    ea.hml = c->hml;
    ea.ne[0] = c->ne0;
    ea.ne[1] = c->ispin == 2 ? c->ne1 : 0;
    ea.ne0 = c->ne0;
    ea.A = c->eigA;
    ea.V = c->eigV;
    ea.eig = c->eigD;
    ea.vec = c->eigVec;
    ea.sweeps = c->eig_sweeps;
    jacobi_eig_kernel<<<c->ispin, kEigThreads, 0, s>>>(ea);
    c->nlaunch += 1;
    // c1 <- c2 V per spin (main.c:481-487): band j of c1 = sum_l V[l][j] band l of c2
    double *c1w = (double *)c->cbuf[c->cur ^ 1];
    for (int ms = 0; ms < c->ispin; ++ms) {
        const int m = ms ? c->ne1 : c->ne0;
        const long off = (long)(ms ? c->ne0 : 0) * ldr;
        gemm_nn(c, m, K, m, 1.0, c->eigVec + ms * ne02, m, c2 + off, ldr, 0.0, c1w + off, ldr);
    }
    c->cs = cs_saved;
    CK(cudaGetLastError());
    int sweeps[2] = {0, 0};
    CK(cudaMemcpyAsync(sweeps, c->eig_sweeps, sizeof(int) * c->ispin, cudaMemcpyDeviceToHost, s));
    const long ne12 = (long)c->ne1 * c->ne1;
    if (ortho) {
        CK(cudaMemcpyAsync(ortho, c->ortho, sizeof(double) * ne02, cudaMemcpyDeviceToHost, s));
        if (c->ispin == 2)
            CK(cudaMemcpyAsync(ortho + ne02, c->ortho + ne02, sizeof(double) * ne12, cudaMemcpyDeviceToHost, s));
    }
    if (eig) {
        CK(cudaMemcpyAsync(eig, c->eigD, sizeof(double) * c->ne0, cudaMemcpyDeviceToHost, s));
        if (c->ispin == 2)
            CK(cudaMemcpyAsync(eig + c->ne0, c->eigD + c->ne0, sizeof(double) * c->ne1, cudaMemcpyDeviceToHost, s));
    }
    if (vec) {
        CK(cudaMemcpyAsync(vec, c->eigVec, sizeof(double) * ne02, cudaMemcpyDeviceToHost, s));
        if (c->ispin == 2)
            CK(cudaMemcpyAsync(vec + ne02, c->eigVec + ne02, sizeof(double) * ne12, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    for (int ms = 0; ms < c->ispin; ++ms)
        if (sweeps[ms] > kEigMaxSweeps) return CPSD_ERR_EIG;
    return CPSD_OK;
}

int cpsd_gpu_npw(const cpsd_gpu_ctx *c) { return c ? c->npw : 0; }

int cpsd_gpu_geometry(const cpsd_gpu_ctx *c, int *out)
{
    if (!c || !out) return CPSD_ERR_ARG;
    out[0] = c->npw;
    out[1] = c->npw_pad;
    out[2] = c->hg.ncol;
    out[3] = c->hg.KX;
    out[4] = c->nproj;
    out[5] = c->nchunk0 + c->nchunk1;
    return CPSD_OK;
}

int cpsd_gpu_launches_per_step(const cpsd_gpu_ctx *c)
{
    if (!c) return 0;
    if (c->graph_launches) return c->graph_launches;
    // inv_z, density plane, xc, fwd plane, fwd_z, phase, vloc, inv_z, inv plane,
    // kinetic, [beta gemm + reduce, coef, nn gemm], applyV plane, fwd_z(SD),
    // 3 overlap gemms (+reduce) per spin, lagrange, constraint gemm per spin
    int n = 13 + 2 * 3 * c->ispin + 1 + c->ispin;
    if (c->nproj > 0) n += 4;
    return n;
}

int cpsd_gpu_lagrange_failures(cpsd_gpu_ctx *c) { return c ? c->lag_fail_total : 0; }

int cpsd_gpu_phase_timing(cpsd_gpu_ctx *c, int on)
{
    if (!c) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    drop_graphs(c);  // recapture with (or without) the event records
    if (on && !c->pev[0])
        for (int i = 0; i <= kNumPhases; ++i) CK(cudaEventCreate(&c->pev[i]));
    c->phase_timing = on != 0;
    return CPSD_OK;
}

int cpsd_gpu_phase_times(cpsd_gpu_ctx *c, float *ms, int max)
{
    if (!c || !c->phase_timing || !ms) return 0;
    if (cudaEventSynchronize(c->pev[kNumPhases]) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    int n = std::min(max, kNumPhases);
    for (int i = 0; i < n; ++i)
        if (cudaEventElapsedTime(&ms[i], c->pev[i], c->pev[i + 1]) != cudaSuccess) {
            (void)cudaGetLastError();
            ms[i] = -1.0f;
        }
    return n;
}

const char *cpsd_gpu_phase_name(int i) { return (i >= 0 && i < kNumPhases) ? kPhaseNames[i] : ""; }

int cpsd_gpu_set_preconditioner(cpsd_gpu_ctx *c, cpsd_mlp *m)
{
    if (c && c->bp && m) return CPSD_ERR_ARG;
    if (!c) return CPSD_ERR_ARG;
    if (m && m->device != c->prm.device) return CPSD_ERR_ARG;
    if (m != c->mlp) drop_graphs(c);
    c->mlp = m;
    if (m) {
        // the step feature counts every SD step of this context, and the
        // trust region starts fully open
        CK(cudaSetDevice(c->prm.device));
        const int step = (int)std::min<long long>(c->steps_run, 1 << 30);
        CK(cudaMemcpyAsync(c->dstep, &step, sizeof(int), cudaMemcpyHostToDevice, c->st));
        const float range[2] = {kLogKMin, kLogKMax};
        CK(cudaMemcpyAsync(c->pcap, range, sizeof(range), cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
    }
    return CPSD_OK;
}

int cpsd_gpu_set_preconditioner_range(cpsd_gpu_ctx *c, double min_log_k, double max_log_k)
{
    if (!c || !(min_log_k == min_log_k) || !(max_log_k == max_log_k) || min_log_k > max_log_k)
        return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    auto clamp = [](double v) { return (float)std::max<double>(kLogKMin, std::min<double>(kLogKMax, v)); };
    const float range[2] = {clamp(min_log_k), clamp(max_log_k)};
    CK(cudaMemcpyAsync(c->pcap, range, sizeof(range), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return CPSD_OK;
}

int cpsd_gpu_run_guarded(cpsd_gpu_ctx *c, int blocks, int inner, double *cap, double *E, double *deltae,
                         double *deltac, int *rejected)
{
    if (!c || !cap || !E || blocks < 1 || inner < 1) return CPSD_ERR_ARG;
    if (!c->mlp) return CPSD_ERR_ARG;  // plain SD: cpsd_gpu_run
    const int min_bands = (c->ispin == 2) ? std::min(c->ne0, c->ne1) : c->ne0;
    int last = CPSD_OK;
    for (int blk = 0; blk < blocks; ++blk) {
        const double prev = E[0];
        int rc = cpsd_gpu_save_orbitals(c);
        if (rc) return rc;
        rc = cpsd_gpu_set_preconditioner_range(c, kLogKMin, *cap);
        if (rc) return rc;
        last = cpsd_gpu_run(c, inner, 0, E, deltae, deltac, nullptr);
        if (last != CPSD_OK && last != CPSD_WARN_LAGRANGE) return last;
        // with one band per spin the reference's convergence test can never
        // pass (cpsd.c:471), so its warning says nothing there
        const bool lag_failed = last == CPSD_WARN_LAGRANGE && min_bands > 1;
        if (!std::isfinite(E[0]) || E[0] > prev || lag_failed) {
            // rejected: the block again from its start with plain SD steps
            // (K = 1 exactly: the reference's update, cpsd.c:399-400)
            if (rejected) ++*rejected;
            *cap = std::max<double>(kLogKMin, *cap - kCapShrink);
            rc = cpsd_gpu_restore_orbitals(c);
            if (rc) return rc;
            rc = cpsd_gpu_set_preconditioner_range(c, 0.0, 0.0);
            if (rc) return rc;
            E[0] = prev;
            last = cpsd_gpu_run(c, inner, 0, E, deltae, deltac, nullptr);
            if (last != CPSD_OK && last != CPSD_WARN_LAGRANGE) return last;
        } else {
            *cap = std::min<double>(kLogKMax, *cap + kCapGrow);
        }
    }
    return last;
}

int cpsd_gpu_save_orbitals(cpsd_gpu_ctx *c)
{
    if (!c || !c->state_ok) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    if (!c->saved) {
        CK(c->ar.alloc(&c->saved, (size_t)c->nb * c->npw_pad));
        CK(c->ar.alloc(&c->saved_step, 1));
    }
    CK(cudaMemcpyAsync(c->saved, c->cbuf[c->cur], sizeof(cx<double>) * c->nb * c->npw_pad,
                       cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->saved_step, c->dstep, sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->saved_steps_run = c->steps_run;
    return CPSD_OK;
}

int cpsd_gpu_restore_orbitals(cpsd_gpu_ctx *c)
{
    if (!c || !c->saved) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    CK(cudaMemcpyAsync(c->cbuf[c->cur], c->saved, sizeof(cx<double>) * c->nb * c->npw_pad,
                       cudaMemcpyDeviceToDevice, c->st));
    CK(cudaMemcpyAsync(c->dstep, c->saved_step, sizeof(int), cudaMemcpyDeviceToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->steps_run = c->saved_steps_run;
    return CPSD_OK;
}

int cpsd_gpu_get_packed(cpsd_gpu_ctx *c, double *c1, double *c2, double *cpsi)
{
    if (!c) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    const cx<double> *cc2 = c->cbuf[c->cur], *cc1 = c->ran ? c->cbuf[c->cur ^ 1] : c->cbuf[c->cur];
    double *outs[3] = {c1, c2, cpsi};
    const cx<double> *srcs[3] = {cc1, cc2, c->cpsi};
    for (int k = 0; k < 3; ++k) {
        if (!outs[k]) continue;
        CK(cudaMemcpy2DAsync(outs[k], sizeof(cx<double>) * c->npw, srcs[k], sizeof(cx<double>) * c->ldc,
                             sizeof(cx<double>) * c->npw, c->nb, cudaMemcpyDeviceToHost, c->st));
        c->d2h += (long long)sizeof(cx<double>) * c->npw * c->nb;
    }
    CK(cudaStreamSynchronize(c->st));
    return CPSD_OK;
}

int cpsd_gpu_set_packed(cpsd_gpu_ctx *c, const double *c2)
{
    if (!c || !c2) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    CK(cudaMemsetAsync(c->cbuf[c->cur], 0, sizeof(cx<double>) * c->nb * c->npw_pad, c->st));
    CK(cudaMemcpy2DAsync(c->cbuf[c->cur], sizeof(cx<double>) * c->ldc, c2, sizeof(cx<double>) * c->npw,
                         sizeof(cx<double>) * c->npw, c->nb, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->h2d += (long long)sizeof(cx<double>) * c->npw * c->nb;
    c->state_ok = true;
    return CPSD_OK;
}

int cpsd_gpu_get_sphere(const cpsd_gpu_ctx *c, int *pt_idx, double *weights, int *shell)
{
    if (!c) return CPSD_ERR_ARG;
    for (int p = 0; p < c->npw; ++p) {
        if (pt_idx) pt_idx[p] = c->hg.pt_idx[p];
        if (weights) weights[p] = c->hg.w[p];
    }
    if (shell) CK(cudaMemcpy(shell, c->shell, sizeof(int) * c->npw, cudaMemcpyDeviceToHost));
    return CPSD_OK;
}

// ---------------------------------------------------------------- network
int cpsd_mlp_nparams(void) { return kMlpParams; }

int cpsd_mlp_create(unsigned long long seed, cpsd_mlp **out)
{
    if (!out) return CPSD_ERR_ARG;
    *out = nullptr;
    std::unique_ptr<cpsd_mlp> m(new cpsd_mlp());
    CK(cudaGetDevice(&m->device));
    CK(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    CK(m->ar.alloc(&m->p, kMlpParams));
    CK(m->ar.alloc(&m->m1, kMlpParams));
    CK(m->ar.alloc(&m->m2, kMlpParams));
    CK(m->ar.alloc(&m->g, kMlpParams));
    CK(m->ar.alloc(&m->wq, kMlpParams));
    // Xavier-uniform weights from a splitmix64 stream, zero biases
    std::vector<float> h(kMlpParams, 0.0f);
    uint64_t st = seed;
    auto next = [&]() {
        uint64_t z = (st += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int ofs, int fan_out, int fan_in) {
        const double a = sqrt(6.0 / (fan_in + fan_out));
        for (int i = 0; i < fan_out * fan_in; ++i) h[ofs + i] = (float)((2.0 * next() - 1.0) * a);
    };
    fill(kW1, kMlpHid, kMlpIn);
    fill(kW2, kMlpHid, kMlpHid);
    fill(kW3, kMlpHid, kMlpHid);
    fill(kW4, 1, kMlpHid);
    CK(cudaMemcpy(m->p, h.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    mlp_quantize_kernel<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(kMlpParams, m->p, m->wq);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    *out = m.release();
    return CPSD_OK;
}

namespace {
int mlp_reserve(cpsd_mlp *m, int n)
{
    if (n <= m->cap) return CPSD_OK;
    const int cap = std::max(n, 1024);
    CK(m->ar.alloc(&m->X, (size_t)kMlpIn * cap));
    CK(m->ar.alloc(&m->T, (size_t)cap));
    CK(m->ar.alloc(&m->y, (size_t)cap));
    CK(m->ar.alloc(&m->H, (size_t)3 * kMlpHid * cap));
    CK(m->ar.alloc(&m->D, (size_t)3 * kMlpHid * cap));
    CK(m->ar.alloc(&m->dy, (size_t)cap));
    CK(m->ar.alloc(&m->lp, (size_t)cdiv(cap, 128)));
    CK(cudaDeviceSynchronize());
    m->cap = cap;
    return CPSD_OK;
}

// forward + backward of one batch already in X/T (device); gradient into m->g
int mlp_grad_batch(cpsd_mlp *m, const float *X, const float *T, int n)
{
    const unsigned b128 = (unsigned)cdiv(n, 128);
    mlp_forward_kernel<<<mlp_forward_blocks(n), kMlpTileThreads, 0, m->st>>>(n, X, m->wq, m->p, m->y, m->H);
    mlp_backward_delta_kernel<<<b128, 128, 0, m->st>>>(n, m->y, T, m->wq, m->H, m->D, m->dy, m->lp);
    mlp_wgrad_kernel<<<3 * kMlpHid + 1, kMlpGradThreads, 0, m->st>>>(n, X, m->H, m->D, m->dy, m->g);
    CK(cudaGetLastError());
    return CPSD_OK;
}
}  // namespace

int cpsd_mlp_forward(cpsd_mlp *m, const float *X, int n, float *y)
{
    if (!m || !X || !y || n < 1) return CPSD_ERR_ARG;
    CK(cudaSetDevice(m->device));
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(m->X, X, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->st));
    mlp_forward_kernel<<<mlp_forward_blocks(n), kMlpTileThreads, 0, m->st>>>(n, m->X, m->wq, m->p, m->y, nullptr);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(y, m->y, sizeof(float) * n, cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    return CPSD_OK;
}

int cpsd_mlp_gradient(cpsd_mlp *m, const float *X, const float *T, int n, float *grad, float *loss)
{
    if (!m || !X || !T || n < 1) return CPSD_ERR_ARG;
    CK(cudaSetDevice(m->device));
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(m->X, X, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->T, T, sizeof(float) * n, cudaMemcpyHostToDevice, m->st));
    rc = mlp_grad_batch(m, m->X, m->T, n);
    if (rc) return rc;
    if (grad) CK(cudaMemcpyAsync(grad, m->g, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost, m->st));
    std::vector<float> lp(cdiv(n, 128));
    CK(cudaMemcpyAsync(lp.data(), m->lp, sizeof(float) * lp.size(), cudaMemcpyDeviceToHost, m->st));
    CK(cudaStreamSynchronize(m->st));
    if (loss) {
        double t = 0;
        for (float v : lp) t += v;
        *loss = (float)(t / n);
    }
    return CPSD_OK;
}

int cpsd_mlp_train(cpsd_mlp *m, const float *X, const float *T, int n, int steps, int batch, float lr,
                   float *losses)
{
    if (!m || !X || !T || n < 1 || steps < 1 || batch < 1) return CPSD_ERR_ARG;
    CK(cudaSetDevice(m->device));
    batch = std::min(batch, n);
    int rc = mlp_reserve(m, n);
    if (rc) return rc;
    CK(cudaMemcpyAsync(m->X, X, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice, m->st));
    CK(cudaMemcpyAsync(m->T, T, sizeof(float) * n, cudaMemcpyHostToDevice, m->st));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<float> lp(cdiv(batch, 128));
    for (int it = 0; it < steps; ++it) {
        const int start = (int)(((long)it * batch) % n);
        const int len = std::min(batch, n - start);  // contiguous window of the (pre-shuffled) data
        rc = mlp_grad_batch(m, m->X + (long)kMlpIn * start, m->T + start, len);
        if (rc) return rc;
        ++m->adam_t;
        const float bc1 = 1.0f - powf(b1, (float)m->adam_t), bc2 = 1.0f - powf(b2, (float)m->adam_t);
        mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(kMlpParams, m->p, m->g, m->m1, m->m2, m->wq,
                                                                      lr, b1, b2, eps, bc1, bc2);
        CK(cudaGetLastError());
        if (losses) {
            const int nb = (int)cdiv(len, 128);
            CK(cudaMemcpyAsync(lp.data(), m->lp, sizeof(float) * nb, cudaMemcpyDeviceToHost, m->st));
            CK(cudaStreamSynchronize(m->st));
            double t = 0;
            for (int k = 0; k < nb; ++k) t += lp[k];
            losses[it] = (float)(t / len);
        }
    }
    CK(cudaStreamSynchronize(m->st));
    return CPSD_OK;
}

int cpsd_mlp_get_params(const cpsd_mlp *m, float *p)
{
    if (!m || !p) return CPSD_ERR_ARG;
    CK(cudaMemcpy(p, m->p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    return CPSD_OK;
}

int cpsd_mlp_set_params(cpsd_mlp *m, const float *p)
{
    if (!m || !p) return CPSD_ERR_ARG;
    CK(cudaSetDevice(m->device));
    CK(cudaMemcpy(m->p, p, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    mlp_quantize_kernel<<<(kMlpParams + 255) / 256, 256, 0, m->st>>>(kMlpParams, m->p, m->wq);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(m->st));
    return CPSD_OK;
}

void cpsd_mlp_destroy(cpsd_mlp *m)
{
    if (!m) return;
    cudaSetDevice(m->device);
    if (m->st) cudaStreamSynchronize(m->st);
    m->ar.release();
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
}

void cpsd_gpu_counters(const cpsd_gpu_ctx *c, long long *out)
{
    if (!out) return;
    out[0] = c ? c->nlaunch : 0;
    out[1] = c ? c->h2d : 0;
    out[2] = c ? c->d2h : 0;
}

int cpsd_gpu_set_precision(cpsd_gpu_ctx *c, int precision)
{
    if (!c) return CPSD_ERR_ARG;
    if (precision == CPSD_PREC_FP64) {
        c->fft = c->fft64.get();
    } else if (precision == CPSD_PREC_MIXED) {
        if (!c->fft32) return CPSD_ERR_ARG;  // the context was created FP64-only
        c->fft = c->fft32.get();
    } else {
        return CPSD_ERR_ARG;
    }
    if (precision != c->precision) drop_graphs(c);
    c->precision = precision;
    return CPSD_OK;
}

int cpsd_gpu_set_gemm(cpsd_gpu_ctx *c, int mode)
{
    if (!c) return CPSD_ERR_ARG;
    if (mode != CPSD_GEMM_FP64 && mode != CPSD_GEMM_TF32X3 && mode != CPSD_GEMM_TF32X3_OVERLAPS)
        return CPSD_ERR_ARG;
    if (mode != CPSD_GEMM_FP64 && !c->fft32) return CPSD_ERR_ARG;  // FP64-only context
    if (mode != c->gemm_mode) drop_graphs(c);
    c->gemm_mode = mode;
    return CPSD_OK;
}

int cpsd_gpu_use_graphs(cpsd_gpu_ctx *c, int on)
{
    if (!c) return CPSD_ERR_ARG;
    if (!on) drop_graphs(c);
    c->use_graph = on != 0;
    return CPSD_OK;
}

// ------------------------------------------------------------ band-parallel SD
int cpsd_gpu_set_band_range(cpsd_gpu_ctx *c, int lo, int hi)
{
    if (!c) return CPSD_ERR_ARG;
    if (hi < 0) {  // back to stepping every band
        c->bp = false;
        drop_graphs(c);
        return CPSD_OK;
    }
    if (lo < 0 || lo > hi || hi > c->nb || c->mlp || c->move) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    if (!c->dn_part) {
        CK(c->ar.alloc(&c->dn_part, (size_t)c->ispin * c->n3));
        CK(c->ar.alloc(&c->chunk_bp, (size_t)c->nb + 2));
    }
    // density chunks of this rank's bands: spin 0's [lo, min(hi, ne0)) then
    // spin 1's, at most as many per spin as the whole-cell plan
    const int n0 = std::max(0, std::min(hi, c->ne0) - lo), n1 = (hi - lo) - n0;
    const int ch0 = n0 > 0 ? std::min(std::max(c->nchunk0, 1), n0) : 0;
    const int ch1 = n1 > 0 ? std::min(std::max(c->nchunk1, 1), n1) : 0;
    std::vector<int> tab;
    tab.push_back(0);
    for (int q = 1; q <= ch0; ++q) tab.push_back((int)((long)n0 * q / ch0));
    for (int q = 1; q <= ch1; ++q) tab.push_back(n0 + (int)((long)n1 * q / ch1));
    CK(cudaMemcpyAsync(c->chunk_bp, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    c->nchunk_bp[0] = ch0;
    c->nchunk_bp[1] = ch1;
    c->bp_lo = lo;
    c->bp_hi = hi;
    c->bp = true;
    drop_graphs(c);
    return CPSD_OK;
}

int cpsd_gpu_step_phase(cpsd_gpu_ctx *c, int phase)
{
    if (!c || phase < 0 || phase > 2) return CPSD_ERR_ARG;
    if (!c->tables_ok || !c->state_ok) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    if (phase == 0 && c->move) {  // a band-parallel cell keeps its ions
        drop_graphs(c);
        c->move = 0;
    }
    return step_phase(c, phase);
}

int cpsd_gpu_bp_buffers(cpsd_gpu_ctx *c, double **dn_part, double **dn, double **c2, double **cpsi, long *ld)
{
    if (!c || !c->bp) return CPSD_ERR_ARG;
    if (dn_part) *dn_part = c->dn_part;
    if (dn) *dn = c->dn;
    if (c2) *c2 = (double *)c->cbuf[c->cur ^ 1];
    if (cpsi) *cpsi = (double *)c->cpsi;
    if (ld) *ld = 2L * c->ldc;
    return CPSD_OK;
}

int cpsd_gpu_bp_finish(cpsd_gpu_ctx *c, int inner, double *E, double *deltae, double *deltac)
{
    if (!c || !c->bp || !E || inner < 1) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    cudaStream_t s = c->st;
    CK(cudaMemcpyAsync(c->Edev, E, sizeof(double), cudaMemcpyHostToDevice, s));
    // the projector coefficients of every band (the steps formed only this
    // rank's columns); c1 is the last step's orbitals of all bands
    if (c->nproj > 0) {
        const long ldr = 2L * c->npw_pad;
        int rc = gemm_tn(c, c->nproj, c->nb, 2 * c->npw_pad, (const double *)c->proj, ldr,
                         (const double *)c->cbuf[c->cur ^ 1], ldr, c->w, 1.0, 0.0, c->beta, c->nb, TN_PROJECTOR);
        if (rc) return rc;
    }
    int rc = finish_call(c, inner, E, deltae, deltac, nullptr);
    CK(cudaMemsetAsync(c->flags, 0, 3 * sizeof(int), s));
    return rc;
}

// ------------------------------------------------------------ tuning
int cpsd_gpu_get_tuning(const cpsd_gpu_ctx *c, cpsd_gpu_tuning *t)
{
    if (!c || !t) return CPSD_ERR_ARG;
    for (int m = 0; m < 4; ++m) t->plane_occupancy[m] = c->fft->plane_variant(m);
    t->tn_ctas_per_sm = c->tn_ctas;
    t->density_chunks = c->nchunk0;
    t->lagrange_solver = (c->ne0 <= kLagSmallMax) ? 0 : (c->lag_tile ? 1 : 2);
    return CPSD_OK;
}

int cpsd_gpu_tuning_limits(const cpsd_gpu_ctx *c, cpsd_gpu_tuning *t)
{
    if (!c || !t) return CPSD_ERR_ARG;
    for (int m = 0; m < 4; ++m) t->plane_occupancy[m] = c->fft->plane_variants(m) - 1;
    t->tn_ctas_per_sm = kTuneMaxCtas;
    t->density_chunks = std::min(c->dens_cap, c->ne0);
    t->lagrange_solver = (c->ne0 <= kLagSmallMax) ? 0 : 2;
    return CPSD_OK;
}

int cpsd_gpu_set_tuning(cpsd_gpu_ctx *c, const cpsd_gpu_tuning *t)
{
    if (!c || !t) return CPSD_ERR_ARG;
    for (int m = 0; m < 4; ++m)
        if (t->plane_occupancy[m] < 0 || t->plane_occupancy[m] >= c->fft->plane_variants(m)) return CPSD_ERR_ARG;
    if (t->tn_ctas_per_sm < 1 || t->tn_ctas_per_sm > kTuneMaxCtas) return CPSD_ERR_ARG;
    if (t->density_chunks < 1 || t->density_chunks > std::min(c->dens_cap, c->ne0)) return CPSD_ERR_ARG;
    const bool small = c->ne0 <= kLagSmallMax;
    if (small ? t->lagrange_solver != 0
              : (t->lagrange_solver < 1 || t->lagrange_solver > 2 || (t->lagrange_solver == 1 && !c->lag_tile_ok)))
        return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    const int n0 = t->density_chunks;
    const int n1 = c->ispin == 2 && c->ne1 > 0 ? std::min(t->density_chunks, c->ne1) : 0;
    if (n0 != c->nchunk0 || n1 != c->nchunk1) {
        const std::vector<int> tab = density_chunk_table(c->ne0, n0, c->ne1, n1);
        CK(cudaMemcpyAsync(c->chunk_dens, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice, c->st));
        CK(cudaStreamSynchronize(c->st));
        c->nchunk0 = n0;
        c->nchunk1 = n1;
    }
    for (int m = 0; m < 4; ++m) c->fft->set_plane_variant(m, t->plane_occupancy[m]);
    c->tn_ctas = t->tn_ctas_per_sm;
    if (!small) c->lag_tile = t->lagrange_solver == 1;
    drop_graphs(c);  // the step graphs hold the old choices
    return CPSD_OK;
}

namespace {

struct TuneKey {
    int dev, n, ne0, ne1, npw, nproj, precision, gemm, mlp, move;
    bool operator<(const TuneKey &o) const
    {
        return memcmp(this, &o, sizeof(TuneKey)) < 0;
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, cpsd_gpu_tuning> g_tune_cache;

TuneKey tune_key(const cpsd_gpu_ctx *c)
{
    TuneKey k;
    memset(&k, 0, sizeof(k));
    k.dev = c->prm.device;
    k.n = c->n;
    k.ne0 = c->ne0;
    k.ne1 = c->ne1;
    k.npw = c->npw;
    k.nproj = c->nproj;
    k.precision = c->precision;
    k.gemm = c->gemm_mode;
    k.mlp = c->mlp != nullptr;
    k.move = c->move;
    return k;
}

}  // namespace

int cpsd_gpu_autotune(cpsd_gpu_ctx *c, int steps, int force, float *ms_before, float *ms_after)
{
    if (!c || steps < 1) return CPSD_ERR_ARG;
    if (!c->tables_ok || !c->state_ok) return CPSD_ERR_ARG;
    CK(cudaSetDevice(c->prm.device));
    if (ms_before) *ms_before = -1.0f;
    if (ms_after) *ms_after = -1.0f;
    const TuneKey key = tune_key(c);
    if (!force) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return cpsd_gpu_set_tuning(c, &it->second);
    }
    // the orbitals and step counters are put back after every trial
    const size_t bytes = sizeof(cx<double>) * c->nb * c->npw_pad;
    struct Keep {
        cx<double> *p = nullptr;
        int *step = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Keep()
        {
            if (p) cudaFree(p);
            if (step) cudaFree(step);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } keep;
    CK(cudaMalloc(&keep.p, bytes));
    CK(cudaMalloc(&keep.step, sizeof(int)));
    CK(cudaEventCreate(&keep.e0));
    CK(cudaEventCreate(&keep.e1));
    const int cur0 = c->cur;
    const long long steps0 = c->steps_run, nl0 = c->nlaunch;
    cudaStream_t s = c->st;
    CK(cudaMemcpyAsync(keep.p, c->cbuf[cur0], bytes, cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(keep.step, c->dstep, sizeof(int), cudaMemcpyDeviceToDevice, s));
    auto restore = [&]() -> int {
        c->cur = cur0;
        CK(cudaMemcpyAsync(c->cbuf[cur0], keep.p, bytes, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(c->dstep, keep.step, sizeof(int), cudaMemcpyDeviceToDevice, s));
        return CPSD_OK;
    };
    // time `steps` SD steps of the current choice: best of three after a
    // warm-up step that captures its graphs
    auto trial = [&](float *ms) -> int {
        drop_graphs(c);
        int rc = restore();
        if (!rc) rc = run_steps(c, steps);
        float best = 0.0f;
        for (int rep = 0; rep < 3 && !rc; ++rep) {
            rc = restore();
            if (rc) break;
            CK(cudaEventRecord(keep.e0, s));
            rc = run_steps(c, steps);
            CK(cudaEventRecord(keep.e1, s));
            CK(cudaEventSynchronize(keep.e1));
            float t = 0.0f;
            CK(cudaEventElapsedTime(&t, keep.e0, keep.e1));
            if (rep == 0 || t < best) best = t;
        }
        *ms = best / steps;
        return rc;
    };
    cpsd_gpu_tuning cur{}, lim{};
    cpsd_gpu_get_tuning(c, &cur);
    cpsd_gpu_tuning_limits(c, &lim);
    float t0 = 0.0f;
    int rc = trial(&t0);
    float best = t0;
    // one knob at a time, a choice kept only when it is at least 2% faster
    auto try_value = [&](int *field, int v) -> int {
        const int old = *field;
        if (v == old) return CPSD_OK;
        *field = v;
        if (cpsd_gpu_set_tuning(c, &cur) != CPSD_OK) {
            *field = old;
            return cpsd_gpu_set_tuning(c, &cur);
        }
        float t = 0.0f;
        int r = trial(&t);
        if (r) return r;
        if (t < 0.98f * best) {
            best = t;
            return CPSD_OK;
        }
        *field = old;
        return cpsd_gpu_set_tuning(c, &cur);
    };
    for (int m = 0; m < 4 && !rc; ++m)
        for (int v = 0; v <= lim.plane_occupancy[m] && !rc; ++v) rc = try_value(&cur.plane_occupancy[m], v);
    {
        const int model = c->dens_model[0];
        const int cand[4] = {1, std::max(1, model / 2), model + 1, 2 * model};
        for (int q = 0; q < 4 && !rc; ++q)
            if (cand[q] <= lim.density_chunks) rc = try_value(&cur.density_chunks, cand[q]);
    }
    for (int v : {1, 2, 4}) {
        if (rc) break;
        rc = try_value(&cur.tn_ctas_per_sm, v);
    }
    if (!rc && lim.lagrange_solver == 2)
        for (int v = 1; v <= 2 && !rc; ++v) rc = try_value(&cur.lagrange_solver, v);
    float t1 = best;
    if (!rc) rc = trial(&t1);
    const int rc2 = restore();
    drop_graphs(c);
    CK(cudaStreamSynchronize(s));
    c->steps_run = steps0;
    c->nlaunch = nl0;
    if (rc) return rc;
    if (rc2) return rc2;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = cur;
    }
    if (ms_before) *ms_before = t0;
    if (ms_after) *ms_after = t1;
    return CPSD_OK;
}

void *cpsd_gpu_stream(cpsd_gpu_ctx *c) { return c ? (void *)c->st : nullptr; }

void cpsd_gpu_destroy(cpsd_gpu_ctx *c)
{
    if (!c) return;
    cudaSetDevice(c->prm.device);
    if (c->st) cudaStreamSynchronize(c->st);
    drop_graphs(c);
    for (auto &e : c->pev)
        if (e) cudaEventDestroy(e);
    c->ar.release();
    if (c->st2) cudaStreamSynchronize(c->st2);
    for (cudaEvent_t e : {c->ev_fork, c->ev_sf, c->ev_side, c->ev_steps, c->ev_fetch, c->ev_dn})
        if (e) cudaEventDestroy(e);
    if (c->st2) cudaStreamDestroy(c->st2);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

}  // extern "C"

// ------------------------------------------------------- no-alloc overlaps
// Split-K workspace of cpsd_overlap_tn_noalloc: a file-scope device array,
// so that entry point never allocates.  Its first 256 bytes hold the
// timeout word, the rest (CPSD_NOALLOC_MAX_DOUBLES doubles) the partials.
// Every GPU that loads this library holds the array until the process exits.
constexpr size_t kNoAllocHeadDoubles = 32;
constexpr size_t kNoAllocScratchDoubles = kNoAllocHeadDoubles + CPSD_NOALLOC_MAX_DOUBLES;  // 8 MiB
static __device__ __align__(256) double g_overlap_scratch[kNoAllocScratchDoubles];

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
double *g_noalloc_base[kNoAllocMaxDevices] = {};

// Device address of g_overlap_scratch on the current device: looked up once
// per device, with that device current, then cached (with the tensor-core
// kernel's shared-memory limit set at the same time).
int noalloc_scratch(double **out)
{
    int dev = 0;
    CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return CPSD_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        double *p = nullptr;
        CK(cudaGetSymbolAddress((void **)&p, g_overlap_scratch));
        CK(cudaFuncSetAttribute(tc_gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
        g_noalloc_base[dev] = p;
    }
    *out = g_noalloc_base[dev];
    return CPSD_OK;
}

}  // namespace

extern "C" {

int cpsd_overlap_tn(int method, int M, int N, int K, const double *A, long lda, const double *B, long ldb,
                    const double *w, double *C, long ldc, void *stream)
{
    if (method != CPSD_GEMM_FP64 && method != CPSD_GEMM_TF32X3) return CPSD_ERR_ARG;
    if (M < 0 || N < 0 || K < 0 || lda < K || ldb < K || ldc < N) return CPSD_ERR_ARG;
    if (M == 0 || N == 0) return CPSD_OK;
    if (!A || !B || !C) return CPSD_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    const bool tc = method != CPSD_GEMM_FP64;
    if (tc)
        CK(cudaFuncSetAttribute(tc_gemm_tn_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    const size_t cap = std::max<size_t>((size_t)M * N, (size_t)4 << 20);
    const TnPlan pl = tn_plan(M, N, K, 1, tc, cap, device_sms());
    struct Scratch {
        double *ws = nullptr;
        int *err = nullptr;
        ~Scratch()
        {
            if (ws) cudaFree(ws);
            if (err) cudaFree(err);
        }
    } sc;
    CK(cudaMalloc(&sc.ws, sizeof(double) * (size_t)pl.splits * M * N));
    CK(cudaMalloc(&sc.err, sizeof(int)));
    CK(cudaMemsetAsync(sc.err, 0, sizeof(int), s));
    (void)launch_tn(M, N, K, 1, &A, lda, &B, ldb, w, 1.0, 0.0, &C, ldc, tc, sc.ws, cap, sc.err, s);
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, sc.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return herr ? CPSD_ERR_TIMEOUT : CPSD_OK;
}

int cpsd_overlap_tn_noalloc(int method, int M, int N, int K, const double *A, long lda, const double *B, long ldb,
                            const double *w, double *C, long ldc, void *stream)
{
    if (method != CPSD_GEMM_FP64 && method != CPSD_GEMM_TF32X3) return CPSD_ERR_ARG;
    if (M < 0 || N < 0 || K < 0 || lda < K || ldb < K || ldc < N) return CPSD_ERR_ARG;
    if (M == 0 || N == 0) return CPSD_OK;
    if (!A || !B || !C) return CPSD_ERR_ARG;
    if ((size_t)M * (size_t)N > (size_t)CPSD_NOALLOC_MAX_DOUBLES) return CPSD_ERR_SCRATCH;
    double *base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int *err = reinterpret_cast<int *>(base);  // the timeout word: must start at zero
    double *ws = base + kNoAllocHeadDoubles;   // partials: every one is written before it is read
    CK(cudaMemsetAsync(err, 0, sizeof(int), s));
    (void)launch_tn(M, N, K, 1, &A, lda, &B, ldb, w, 1.0, 0.0, &C, ldc, method != CPSD_GEMM_FP64, ws,
                    (size_t)CPSD_NOALLOC_MAX_DOUBLES, err, s);
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return herr ? CPSD_ERR_TIMEOUT : CPSD_OK;
}

}  // extern "C"
