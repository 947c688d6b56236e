// fft.cuh -- sphere-pruned batched 3-D transforms of the half box.
//
// Layouts (n = nfft, h = n/2, nh = h+1):
//   packed   psi[b][p]      complex, p over the cutoff sphere ordered by
//                           column (kx, ky) then kz (Geom)
//   columns  T[b][z][c]     complex, after the kz transform: c over the
//                           (kx, ky) columns that hold sphere points
//   real     R[z][y][x]     double, x fastest (no padding)
//
// A transform G -> r is   inv_z (packed -> T)   then   plane (T -> real),
// r -> G is               plane (real -> T)     then   fwd_z (T -> packed).
// The plane kernel owns one z plane per CTA: it transforms the kx <= KX-1
// lines along y in shared memory, then every x row (c2r / r2c by the
// half-length complex trick), so the real-space plane never goes to HBM
// unless asked.  Because the reference keeps psi, the density and every
// potential masked to the same sphere (ccpsdv3/cpsd.c:205, 233), columns
// outside the sphere are exact zeros and are skipped.
//
// Semantics match fftpack3d/fftpack3d.f: cr_fft3b drops Im(kx=0) and
// Im(kx=n/2) before the x c2r (:86-89), rc_fft3f sets them to zero after the
// x r2c (:157-161); both are unnormalised.
#pragma once

#include "common.cuh"

struct Geom {
    int n, nh, KX, ncol, npw, npw_pad;
    const int *col_i, *col_j, *col_ptr;  // ncol, ncol, ncol+1
    const int *pt_k;                     // npw
    const int *colidx;                   // KX*n: column of (kx, y) or -1
    // 3 per line kx: first column, a, b -- the line's columns are y in
    // [0, a) then [b, n), column first + y or first + a + (y - b); null:
    // use colidx
    const int *yrun;
};

// The twiddle tables of the y/z length NF, one allocation in this order:
// the line-transform tables of Line<NF> (line_fft order) for the signs +1
// and -1, those of Line<H> (H = NF/2) for both signs, the Line<H> table of
// the transposed transform (line_fft_dif order, sign -1), and the
// real-transform factors e^{+-2 pi i k/NF} (k <= H).
template <int NF>
struct TwLayout {
    static constexpr int H = NF / 2;
    static constexpr int n_inv = 0, n_fwd = NF, h_inv = 2 * NF, h_fwd = 2 * NF + H, h_fwd_dif = 2 * NF + 2 * H,
                         r_inv = 2 * NF + 3 * H, r_fwd = 2 * NF + 4 * H + 1, total = 2 * NF + 5 * H + 2;
};

template <typename T>
struct Twiddles {
    const cx<T> *n_inv, *n_fwd, *h_inv, *h_fwd, *h_fwd_dif, *r_inv, *r_fwd;
    // the tables of one TwLayout<NF> allocation starting at base
    template <int NF>
    CPSD_HD static Twiddles at(const cx<T> *base)
    {
        using L = TwLayout<NF>;
        return Twiddles{base + L::n_inv, base + L::n_fwd,     base + L::h_inv, base + L::h_fwd,
                        base + L::h_fwd_dif, base + L::r_inv, base + L::r_fwd};
    }
};

constexpr int kThreads = 256;

// one complex value global -> shared without a register round trip
// (cp.async: 16 bytes bypassing L1 for FP64, 8 bytes for FP32)
template <typename T>
CPSD_D void cp_async_cx(cx<T> *dst, const cx<T> *src)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(cx<T>) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
CPSD_D void cp_async_commit_all() { asm volatile("cp.async.commit_group;" ::: "memory"); }
CPSD_D void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Shared memory of the z passes: one region (complex values) that holds the
// CTA's column tile ([CPB][NF + 1] or [NF][CPB + 1]) and, once the lines are
// in registers, the line groups' exchange buffers; the twiddle table after it.
template <typename T, int NF>
constexpr int z_tile_elems()
{
    constexpr int CPB = kThreads / Line<NF>::P;
    constexpr int TILE = (CPB * (NF + 1) > NF * (CPB + 1)) ? CPB * (NF + 1) : NF * (CPB + 1);
    constexpr int XB = CPB * group_stride<T, NF>();
    return TILE > XB ? TILE : XB;
}
template <typename T, int NF>
constexpr size_t z_smem_bytes()
{
    return sizeof(cx<T>) * ((size_t)z_tile_elems<T, NF>() + NF);
}

// ------------------------------------------------------------------ inv_z
// packed psi (double) -> T (type T), one CTA = CPB columns of one band
template <typename T, int NF>
__global__ void __launch_bounds__(kThreads)
inv_z_kernel(Geom g, const cx<double> *__restrict__ psi, long ldp, cx<T> *__restrict__ Tb,
             Twiddles<T> tw)
{
    using L = Line<NF>;
    constexpr int P = L::P, Q = L::Q, U = L::U, CPB = kThreads / P;
    constexpr int XS = group_stride<T, NF>();
    constexpr int RS = NF + 1, CS = CPB + 1;  // row / column strides of the tile
    extern __shared__ unsigned char smem_raw[];
    // the exchange buffers reuse the tile once every line is in registers
    cx<T> *tile = reinterpret_cast<cx<T> *>(smem_raw);
    cx<T> *xb = tile;
    cx<T> *twz = tile + z_tile_elems<T, NF>();  // W_NF^m staged once per CTA (read by every line)
    for (int i = threadIdx.x; i < NF; i += kThreads) twz[i] = tw.n_inv[i];

    const int b = blockIdx.y;
    const int c0 = blockIdx.x * CPB;
    const int grp = threadIdx.x / P, t = threadIdx.x % P;
    const int c = c0 + grp;
    cx<T> *row = tile + grp * RS;
    for (int k = t; k < NF; k += P) row[k] = cx<T>{0, 0};
    __syncwarp();
    if (c < g.ncol) {
        // four points per lane in flight: their loads before their stores
        const cx<double> *src = psi + (long)b * ldp;
        const int pe = g.col_ptr[c + 1];
        for (int p0 = g.col_ptr[c] + t; p0 < pe; p0 += 4 * P) {
            cx<double> vv[4];
            int kk[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int p = p0 + u * P;
                kk[u] = (p < pe) ? g.pt_k[p] : -1;
                if (p < pe) vv[u] = src[p];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (kk[u] >= 0) row[kk[u]] = cx<T>{(T)vv[u].x, (T)vv[u].y};
        }
    }
    __syncthreads();  // the rows and the staged table
    cx<T> v[Q];
#pragma unroll
    for (int m = 0; m < Q; ++m) v[m] = row[L::in_index(t, m)];
    __syncthreads();  // every row read: the exchange buffers overwrite the tile
    line_fft<NF, +1, T>(v, t, xb + grp * XS, twz);
    __syncthreads();
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int s = 0; s < P; ++s) tile[L::out_index(t, u, s) * CS + grp] = v[u * P + s];
    __syncthreads();
    cx<T> *dst = Tb + (long)b * NF * g.ncol;
    for (int idx = threadIdx.x; idx < NF * CPB; idx += kThreads) {
        int z = idx / CPB, cl = idx % CPB;
        if (c0 + cl < g.ncol) dst[(long)z * g.ncol + c0 + cl] = tile[z * CS + cl];
    }
}

// ------------------------------------------------------------------ fwd_z
enum { ZEPI_STORE = 0, ZEPI_SD = 1 };

struct ZEpilogue {
    // STORE: out[b*ldo + p] = scale * F
    cx<double> *out;
    long ldo;
    double scale;
    // SD (ccpsdv3/cpsd.c:212-221, 394-400): cpsi = -scal1*F + (-tg c1 + nl);
    // c2 = c1 + dte*cpsi, the kinetic term -tg c1 formed here from the c1
    // the epilogue reads anyway
    cx<double> *c2;        // in: the nonlocal part nl (when has_nl); out: steepest-descent iterate
    const cx<double> *c1;
    cx<double> *cpsi;
    const double *tg;      // G^2/2 per sphere point
    long ldc;
    double scal1, dte;
    int has_nl;            // 0: no projectors, nl = 0 and c2 is not read
};

template <typename T, int NF, int EPI>
__global__ void __launch_bounds__(kThreads)
fwd_z_kernel(Geom g, const cx<T> *__restrict__ Tb, ZEpilogue e, Twiddles<T> tw)
{
    using L = Line<NF>;
    constexpr int P = L::P, Q = L::Q, U = L::U, CPB = kThreads / P;
    constexpr int RS = NF + 1, CS = CPB + 1;
    constexpr int XS = group_stride<T, NF>();
    extern __shared__ unsigned char smem_raw[];
    cx<T> *tile = reinterpret_cast<cx<T> *>(smem_raw);
    cx<T> *xb = tile;  // reuses the tile once every line is in registers

    const int b = blockIdx.y;
    const int c0 = blockIdx.x * CPB;
    const int grp = threadIdx.x / P, t = threadIdx.x % P;
    const int c = c0 + grp;
    cx<T> *twz = tile + z_tile_elems<T, NF>();  // W_NF^-m staged once per CTA
    for (int i = threadIdx.x; i < NF; i += kThreads) twz[i] = tw.n_fwd[i];
    // the column tile by cp.async: every element of a thread in flight at once
    const cx<T> *src = Tb + (long)b * NF * g.ncol;
    for (int idx = threadIdx.x; idx < NF * CPB; idx += kThreads) {
        int z = idx / CPB, cl = idx % CPB;
        if (c0 + cl < g.ncol)
            cp_async_cx(tile + z * CS + cl, src + (long)z * g.ncol + c0 + cl);
        else
            tile[z * CS + cl] = cx<T>{0, 0};
    }
    cp_async_commit_all();
    cp_async_wait_all();
    __syncthreads();
    cx<T> v[Q];
#pragma unroll
    for (int m = 0; m < Q; ++m) v[m] = tile[L::in_index(t, m) * CS + grp];
    __syncthreads();  // every column read: the exchange buffers overwrite the tile
    line_fft<NF, -1, T>(v, t, xb + grp * XS, twz);
    __syncthreads();
    cx<T> *row = tile + grp * RS;
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
        for (int s = 0; s < P; ++s) row[L::out_index(t, u, s)] = v[u * P + s];
    __syncwarp();
    if (c < g.ncol) {
        // four points per lane in flight: every load of the four before any
        // store (the stores to c2 would otherwise keep the next loads back)
        const int pe = g.col_ptr[c + 1];
        for (int p0 = g.col_ptr[c] + t; p0 < pe; p0 += 4 * P) {
            int kk[4];
            cx<double> c2k[4], c1v[4];
            double t[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int p = p0 + u * P;
                kk[u] = (p < pe) ? g.pt_k[p] : -1;
                if constexpr (EPI == ZEPI_SD)
                    if (p < pe) {
                        const long o = (long)b * e.ldc + p;
                        c1v[u] = e.c1[o];
                        t[u] = e.tg[p];
                        c2k[u] = e.has_nl ? e.c2[o] : cx<double>{0.0, 0.0};
                    }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (kk[u] < 0) continue;
                const int p = p0 + u * P;
                const cx<T> F = row[kk[u]];
                if constexpr (EPI == ZEPI_STORE) {
                    e.out[(long)b * e.ldo + p] = cx<double>{e.scale * (double)F.x, e.scale * (double)F.y};
                } else {
                    const long o = (long)b * e.ldc + p;
                    // kinetic + nonlocal: -t c1 + nl (nl absent: the kinetic term alone)
                    const cx<double> kin{-t[u] * c1v[u].x, -t[u] * c1v[u].y};
                    const cx<double> h = e.has_nl ? cx<double>{c2k[u].x + kin.x, c2k[u].y + kin.y} : kin;
                    const cx<double> cp{-e.scal1 * (double)F.x + h.x, -e.scal1 * (double)F.y + h.y};
                    e.cpsi[o] = cp;
                    e.c2[o] = cx<double>{c1v[u].x + e.dte * cp.x, c1v[u].y + e.dte * cp.y};
                }
            }
        }
    }
}

// ------------------------------------------------------------------ plane
enum { PM_DENSITY = 0, PM_APPLYV = 1, PM_INVREAL = 2, PM_FWDREAL = 3 };

struct PlaneArgs {
    const int *chunk_b0;  // band range of blockIdx.y: [chunk_b0[y], chunk_b0[y+1])
    double *rho_part;     // DENSITY: [chunk][z][y][x] sums of psi^2
    const double *V;      // APPLYV: [ispin][z][y][x] total local potential
    int ne0;              // bands b >= ne0 use V of spin 1
    double *rout;         // INVREAL: rout[ms] = psi + xadd[ms], ms < nout
    const double *xadd;
    int nout;
    const double *rin;    // FWDREAL: real input grid
    int nchunks;          // APPLYV with two bands a CTA: chunk_b0 has nchunks + 1 entries
};

template <typename T, int NF>
struct PlaneShape {
    static constexpr int H = NF / 2;
    using LY = Line<NF>;
    using LX = Line<H>;
    // exchange-buffer strides of the y-line groups and the x-row groups
    static constexpr int SY = group_stride<T, NF>();
    static constexpr int SX = group_stride<T, H>();
    // FP64 lines of 8 lanes holding 2 outputs each (NF = 128): a lane stores
    // its outputs 2 apart, so the 8 lanes of a 128-byte phase would meet in
    // 4 of the 8 16-byte slots; one pad slot after every 8 y positions
    // (ymap) spreads them over all 8
    static constexpr bool YSWZ = sizeof(cx<T>) == 16 && LY::P >= 8 && LY::U >= 2;
    static constexpr int YW = NF + (YSWZ ? NF / 8 : 0);
    CPSD_HD static int ymap(int p) { return YSWZ ? p + (p >> 3) : p; }
    // y-line stride: lanes t of an x group read rows k = t + P m of one column
    // and the 8/P groups of a phase read neighbouring columns
    static constexpr int YS = (LX::P >= kSlots<T>) ? pad_to(YW + 1, kSlots<T>, 1)
                                                   : pad_to(YW + 1, kSlots<T>, kSlots<T> / LX::P);
    // y-line groups that hold a line: all of them when there are at least as
    // many lines as groups, else the lines rounded up to whole warps (the
    // warps past them skip the y transforms and need no exchange buffer)
    CPSD_HD static int y_groups(int KX, int ngy)
    {
        const int gpw = 32 / LY::P;
        return KX >= ngy ? ngy : ((KX + gpw - 1) / gpw) * gpw;
    }
    // density rows: one extra complex per row moves the next row's group
    static constexpr int RS = NF + 2;
};

template <typename T, int NF>
__host__ __device__ constexpr int plane_threads(int mode)
{
    return kThreads;
}

// The density pass stages the next band's columns of its plane in shared
// memory (ncol values, rounded to 16 bytes); the other passes take one band
// per CTA and read the columns directly, and so does the density build that
// splits a plane's rows between two CTAs (its two CTAs must fit one SM).
template <typename T>
constexpr size_t stage_elems(int mode, int ncol)
{
    return mode == PM_DENSITY ? ((size_t)ncol * sizeof(cx<T>) + 15) / 16 * 16 / sizeof(cx<T>) : 0;
}

// Bands one CTA of a plane pass takes together.  The V psi pass on grids up
// to 64 takes two: a small plane has few y lines (11 at 64^3 for 32 line
// groups), so with one band most warps wait at the barriers around its y
// phases; two bands fill twice the groups and share each barrier (and each
// V row).  At 128 the second band's line buffer would leave one CTA per SM.
__host__ __device__ constexpr int plane_bands_per_cta(int NF, int mode)
{
    return (mode == PM_APPLYV && NF <= 64) ? 2 : 1;
}

template <typename T, int NF>
size_t plane_smem_bytes(int mode, int KX, int ncol)
{
    using S = PlaneShape<T, NF>;
    const int nt = plane_threads<T, NF>(mode);
    const int lines = plane_bands_per_cta(NF, mode) * KX;
    const size_t ex_y = (size_t)S::y_groups(lines, nt / S::LY::P) * S::SY, ex_x = (size_t)(nt / S::LX::P) * S::SX;
    size_t b = sizeof(cx<T>) * ((size_t)TwLayout<NF>::total + stage_elems<T>(mode, ncol) + (size_t)lines * S::YS +
                                (ex_y > ex_x ? ex_y : ex_x));
    return (b + 15) / 16 * 16;
}

// Every plane variant is built for one and for two CTAs per SM (MINB); the
// host launches the two-CTA build where two planes' shared memory fits an SM
// (it caps registers at 128 per thread).  The density variant at n >= 128
// keeps 64 per-lane sums in registers; its two-CTA build instead splits each
// plane's x rows between two CTAs (blockIdx.z = the half): every CTA redoes
// the plane's y lines (about a quarter of the work) and keeps half the sums.
template <int NF, int MODE>
constexpr bool plane_has_two_cta_build()
{
    return true;
}
template <int NF, int MODE, int MINB>
constexpr int plane_row_split()
{
    return (MODE == PM_DENSITY && NF >= 128 && MINB == 2) ? 2 : 1;
}

template <typename T, int NF, int MODE, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
plane_kernel(Geom g, cx<T> *__restrict__ Tb, PlaneArgs a, Twiddles<T> twg)
{
    using S = PlaneShape<T, NF>;
    using LY = typename S::LY;
    using LX = typename S::LX;
    constexpr int H = S::H;
    constexpr int NT = plane_threads<T, NF>(MODE);
    constexpr int YS = S::YS;  // Ybuf row stride
    constexpr int PY = LY::P, QY = LY::Q, UY = LY::U, NGY = NT / PY;
    constexpr int PX = LX::P, QX = LX::Q, UX = LX::U, NGX = NT / PX;
    constexpr int EXB = (NGY * S::SY > NGX * S::SX) ? NGY * S::SY : NGX * S::SX;
    extern __shared__ unsigned char smem_raw[];
    const int KX = g.KX;
    // the twiddle tables, staged once per CTA: shared-memory reads instead of
    // L1 hits in every line transform, and 32-bit addresses (fewer registers)
    cx<T> *tws = reinterpret_cast<cx<T> *>(smem_raw);
    constexpr int RSPLIT = plane_row_split<NF, MODE, MINB>();
    constexpr bool STAGE = MODE == PM_DENSITY && RSPLIT == 1;
    cx<T> *stage = tws + TwLayout<NF>::total;                          // STAGE: one band's columns
    constexpr int BPC = plane_bands_per_cta(NF, MODE);
    cx<T> *Y = stage + stage_elems<T>(STAGE ? MODE : -1, g.ncol);  // [BPC][KX][YS]
    cx<T> *xball = Y + BPC * KX * YS;                               // group exchange buffers
    for (int i = threadIdx.x; i < TwLayout<NF>::total; i += NT) tws[i] = twg.n_inv[i];
    const Twiddles<T> tw = Twiddles<T>::template at<NF>(tws);
    __syncthreads();
    // DENSITY: each lane owns the same (row, x) points for every band, so the
    // sum of psi^2 over the band chunk stays in registers
    constexpr int NIT = (NF + NGX - 1) / NGX / RSPLIT;  // x-row iterations per lane (of this CTA's rows)
    static_assert(RSPLIT == 1 || NIT * NGX * RSPLIT == NF, "row split");
    const int it0 = (RSPLIT > 1) ? (int)blockIdx.z * NIT : 0;
    double rho[(MODE == PM_DENSITY) ? NIT : 1][(MODE == PM_DENSITY) ? 2 * QX : 1];

    const int z = blockIdx.x;
    // this CTA's bands: chunk blockIdx.y, or chunks BPC y .. BPC y + BPC - 1
    const int cb = (int)blockIdx.y * BPC, ce = (BPC > 1) ? min(cb + BPC, a.nchunks) : cb + 1;
    const int b0 = (MODE == PM_DENSITY || MODE == PM_APPLYV) ? a.chunk_b0[cb] : 0;
    const int b1 = (MODE == PM_DENSITY || MODE == PM_APPLYV) ? a.chunk_b0[ce] : 1;
    const long plane = (long)NF * NF;

    if constexpr (MODE == PM_DENSITY) {
#pragma unroll
        for (int it = 0; it < NIT; ++it)
#pragma unroll
            for (int q = 0; q < 2 * QX; ++q) rho[it][q] = 0.0;
    }

    const int gy = threadIdx.x / PY, ty = threadIdx.x % PY;
    const int gx = threadIdx.x / PX, tx = threadIdx.x % PX;
    cx<T> *xby = xball + gy * S::SY;
    cx<T> *xbx = xball + gx * S::SX;

    // STAGE: band bb's columns of this plane -> stage, asynchronously; the
    // copy of band b+1 is issued once band b's y lines have read the stage
    // and lands while band b's x rows run
    auto prefetch = [&](int bb) {
        const cx<T> *src = Tb + ((long)bb * NF + z) * g.ncol;
        for (int c = threadIdx.x; c < g.ncol; c += NT) cp_async_cx(stage + c, src + c);
        cp_async_commit_all();
    };
    if (STAGE && b0 < b1) prefetch(b0);
    // bands b .. b + nbg - 1 together (nbg = 1 unless BPC > 1); line li of
    // the group is line li % KX of band b + li / KX
    for (int b = b0; b < b1; b += BPC) {
        const int nbg = (BPC == 1) ? 1 : min(BPC, b1 - b);
        const int nl = nbg * KX;
        const int ngy_act = S::y_groups(nl, NGY);  // warp-uniform: whole warps skip the y lines
        const cx<T> *Tcol = STAGE ? stage : Tb + ((long)b * NF + z) * g.ncol;
        if (STAGE) {
            cp_async_wait_all();
            __syncthreads();
        }
        // ---- inverse along y (columns -> lines kx < KX) ------------------
        if constexpr (MODE != PM_FWDREAL) {
            for (int base = 0; base < nl && gy < ngy_act; base += NGY) {
                const int li = base + gy;
                const bool act = li < nl;
                const int kb = (BPC == 1 || !act) ? 0 : li / KX;
                const int i = act ? li - kb * KX : 0;
                const cx<T> *Tp = (BPC == 1) ? Tcol : Tb + ((long)(b + kb) * NF + z) * g.ncol;
                cx<T> v[QY];
                // the line's columns: arithmetic from its two runs (one small
                // load per line), else the colidx table (one load per value).
                // The density pass keeps the table: measured faster there (its
                // band loop reuses the same columns for every band)
                if (MODE != PM_DENSITY && g.yrun) {
                    const int c0 = act ? g.yrun[3 * i] : 0, ra = act ? g.yrun[3 * i + 1] : 0;
                    const int rb = act ? g.yrun[3 * i + 2] : NF;
#pragma unroll
                    for (int m = 0; m < QY; ++m) {
                        const int y = LY::in_index(ty, m);
                        const int c = y < ra ? c0 + y : (y >= rb ? c0 + ra + (y - rb) : -1);
                        v[m] = (c >= 0) ? Tp[c] : cx<T>{0, 0};
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < QY; ++m) {
                        const int c = act ? g.colidx[i * NF + LY::in_index(ty, m)] : -1;
                        v[m] = (c >= 0) ? Tp[c] : cx<T>{0, 0};
                    }
                }
                line_fft<NF, +1, T>(v, ty, xby, tw.n_inv);
                if (act) {
                    cx<T> *Yl = Y + (kb * KX + i) * YS;
#pragma unroll
                    for (int u = 0; u < UY; ++u)
#pragma unroll
                        for (int s = 0; s < PY; ++s) Yl[S::ymap(LY::out_index(ty, u, s))] = v[u * PY + s];
                }
            }
            __syncthreads();
            if (STAGE && b + 1 < b1) prefetch(b + 1);
        }
        // ---- x rows --------------------------------------------------------
        for (int kb = 0; kb < nbg; ++kb) {
            cx<T> *Yb = Y + kb * KX * YS;
#pragma unroll
            for (int it = 0; it < NIT; ++it) {
                const int j = (it0 + it) * NGX + gx;
                const bool act = j < NF;
                const int jj = act ? j : 0;
                cx<T> v[QX];
                if constexpr (MODE != PM_FWDREAL) {
                    // c2r pre-processing: Z_k = E_k + i O_k (half-length packing)
#pragma unroll
                    for (int m = 0; m < QX; ++m) {
                        const int k = LX::in_index(tx, m);
                        const int kk = H - k;
                        cx<T> xa = (k < KX) ? Yb[k * YS + S::ymap(jj)] : cx<T>{0, 0};
                        cx<T> xc = (kk < KX) ? Yb[kk * YS + S::ymap(jj)] : cx<T>{0, 0};
                        if (k == 0) {
                            xa.y = 0;
                            xc.y = 0;
                        }
                        cx<T> E = xa + conj(xc);
                        cx<T> O = cmul(xa - conj(xc), tw.r_inv[k]);
                        v[m] = cx<T>{E.x - O.y, E.y + O.x};
                    }
                    line_fft<H, +1, T>(v, tx, xbx, tw.h_inv);
                    // v[u*PX+s] = (psi(2m), psi(2m+1)), m = out_index
                    if constexpr (MODE == PM_DENSITY) {
#pragma unroll
                        for (int q = 0; q < QX; ++q) {
                            const cx<T> w = v[q];
                            rho[it][2 * q] += (double)w.x * (double)w.x;
                            rho[it][2 * q + 1] += (double)w.y * (double)w.y;
                        }
                    } else if constexpr (MODE == PM_INVREAL) {
                        if (act) {
#pragma unroll
                            for (int u = 0; u < UX; ++u)
#pragma unroll
                                for (int s = 0; s < PX; ++s) {
                                    const int m = LX::out_index(tx, u, s);
                                    cx<T> w = v[u * PX + s];
                                    const long o = (long)z * plane + (long)j * NF + 2 * m;
                                    for (int ms = 0; ms < a.nout; ++ms) {
                                        double *ro = a.rout + ms * NF * plane;
                                        if (a.xadd) {
                                            const double *xa = a.xadd + ms * NF * plane;
                                            ro[o] = (double)w.x + xa[o];
                                            ro[o + 1] = (double)w.y + xa[o + 1];
                                        } else {
                                            ro[o] = (double)w.x;
                                            ro[o + 1] = (double)w.y;
                                        }
                                    }
                                }
                        }
                    } else {  // APPLYV: multiply in place; the DIF forward takes this distribution
                        const double *V = a.V + ((b + kb >= a.ne0) ? NF * plane : 0);
#pragma unroll
                        for (int u = 0; u < UX; ++u)
#pragma unroll
                            for (int s = 0; s < PX; ++s) {
                                const int m = LX::out_index(tx, u, s);
                                const long o = (long)z * plane + (long)jj * NF + 2 * m;
                                const double2 vv = *reinterpret_cast<const double2 *>(V + o);
                                cx<T> &w = v[u * PX + s];
                                w = cx<T>{(T)((double)w.x * vv.x), (T)((double)w.y * vv.y)};
                            }
                    }
                } else {  // FWDREAL: load the real row directly in DIT order
                    const double *r = a.rin + (long)z * plane + (long)jj * NF;
#pragma unroll
                    for (int m = 0; m < QX; ++m) {
                        const int mm = LX::in_index(tx, m);
                        v[m] = cx<T>{(T)r[2 * mm], (T)r[2 * mm + 1]};
                    }
                }
                if constexpr (MODE == PM_APPLYV) {
                    line_fft_dif<H, -1, T>(v, tx, xbx, tw.h_fwd_dif);
#pragma unroll
                    for (int m = 0; m < QX; ++m) xbx[LX::in_index(tx, m)] = v[m];
                    __syncwarp();
                }
                if constexpr (MODE == PM_FWDREAL) {
                    line_fft<H, -1, T>(v, tx, xbx, tw.h_fwd);
#pragma unroll
                    for (int u = 0; u < UX; ++u)
#pragma unroll
                        for (int s = 0; s < PX; ++s) xbx[LX::out_index(tx, u, s)] = v[u * PX + s];
                    __syncwarp();
                }
                if constexpr (MODE == PM_APPLYV || MODE == PM_FWDREAL) {
                    // r2c post-processing for the kx < KX that are kept
                    for (int k = tx; k < KX; k += PX) {
                        cx<T> zk = xbx[k % H];
                        cx<T> zc = conj(xbx[(H - k) % H]);
                        cx<T> E = (T)0.5 * (zk + zc);
                        cx<T> D = (T)0.5 * (zk - zc);
                        cx<T> O{D.y, -D.x};
                        cx<T> X = E + cmul(tw.r_fwd[k], O);
                        if (k == 0 || k == H) X.y = 0;
                        if (act) Yb[k * YS + S::ymap(j)] = X;
                    }
                    __syncwarp();
                }
            }
        }
        __syncthreads();
        // ---- forward along y, keep the columns -----------------------------
        if constexpr (MODE == PM_APPLYV || MODE == PM_FWDREAL) {
            for (int base = 0; base < nl && gy < ngy_act; base += NGY) {
                const int li = base + gy;
                const bool act = li < nl;
                const int lii = act ? li : 0;  // line kb * KX + i of Y
                cx<T> v[QY];
#pragma unroll
                for (int m = 0; m < QY; ++m) v[m] = Y[lii * YS + S::ymap(LY::in_index(ty, m))];
                line_fft<NF, -1, T>(v, ty, xby, tw.n_fwd);
                // each group reads and rewrites only its own line
                if (act) {
#pragma unroll
                    for (int u = 0; u < UY; ++u)
#pragma unroll
                        for (int s = 0; s < PY; ++s) Y[li * YS + S::ymap(LY::out_index(ty, u, s))] = v[u * PY + s];
                }
            }
            __syncthreads();
            for (int c = threadIdx.x; c < g.ncol; c += NT) {
                const int yo = g.col_i[c] * YS + S::ymap(g.col_j[c]);
                for (int kb = 0; kb < nbg; ++kb) Tb[((long)(b + kb) * NF + z) * g.ncol + c] = Y[kb * KX * YS + yo];
            }
            __syncthreads();
        }
    }

    if constexpr (MODE == PM_DENSITY) {
        double *dst = a.rho_part + ((long)blockIdx.y * NF + z) * plane;
#pragma unroll
        for (int it = 0; it < NIT; ++it) {
            const int j = (it0 + it) * NGX + gx;
            if (j < NF) {
#pragma unroll
                for (int u = 0; u < UX; ++u)
#pragma unroll
                    for (int s = 0; s < PX; ++s) {
                        const int m = LX::out_index(tx, u, s);
                        double2 r2 = make_double2(rho[it][2 * (u * PX + s)], rho[it][2 * (u * PX + s) + 1]);
                        *reinterpret_cast<double2 *>(dst + (long)j * NF + 2 * m) = r2;
                    }
            }
        }
    }
}
