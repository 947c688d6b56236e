// tc_gemm.cuh -- weighted TN products on the 5th-generation tensor cores
// (tcgen05, sm_100a) for the mixed-precision path.
//
//   part[prod][split][i][j] = sum_{k in chunk} (w_k A[i][k]) B[j][k]
//
// the same contract as gemm_tn_dmma_kernel (kernels.cuh): A and B FP64 in HBM,
// rows K-contiguous, weight per complex pair.  Each stage converts a 128 x 32
// slab of each operand to a TF32 pair x = hi + lo and one elected thread
// issues the three products hi*hi + hi*lo + lo*hi (tcgen05.mma kind::tf32,
// FP32 accumulation in tensor memory): close to FP32 accuracy from TF32
// tensor cores.  Split-K partials are summed in FP64 by splitk_reduce_kernel.
//
// Shared-memory operand layout: K-major, no swizzle.  The canonical layout
// is built from core matrices of 8 rows x 16 bytes (4 TF32 values); a
// 128 x 32 slab holds 16 row groups x 8 K-chunks of them, core matrix
// (group g, chunk c) at byte (c * 16 + g) * 128.  One MMA consumes K = 8
// (two chunks): descriptor start at chunk 2s, leading-byte offset 2048
// (chunk to chunk), stride-byte offset 128 (row group to row group).
//
// Two slab sets alternate: while the tensor cores work on one, the threads
// load and split the next.  Every wait on an mbarrier is bounded; a wait
// that runs out sets *err, the block stops issuing work, waits (bounded)
// for what it issued, frees its tensor memory and returns.
#pragma once

#include "common.cuh"
#include "kernels.cuh"

constexpr int kTcM = 128, kTcN = 128, kTcBK = 32, kTcThreads = 256;
constexpr int kTcSlabWords = kTcM * kTcBK;               // 4096 words = 16 KB per operand slab
constexpr int kTcStageWords = 4 * kTcSlabWords;          // Ah, Al, Bh, Bl
constexpr size_t kTcSmem = 2 * kTcStageWords * 4 + 128;  // two stages (+ alignment slack)
constexpr long kTcSpinLimit = 1L << 22;                  // polls per mbarrier wait

CPSD_D uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// SWIZZLE_NONE K-major shared-memory matrix descriptor (sm_100 format,
// version 1 at bits 46-47, layout type 0 at bits 61-63)
CPSD_D uint64_t tc_desc(uint32_t saddr)
{
    const uint64_t lbo = 2048 >> 4, sbo = 128 >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// instruction descriptor: D f32 (bits 4-5 = 1), A and B tf32 (bits 7-9,
// 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTcN >> 3) << 17) |
                              ((uint32_t)(kTcM >> 4) << 24);

CPSD_D void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(kTcIdesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

CPSD_D void tc_commit(uint32_t mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

CPSD_D uint32_t tf32_bits(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// true once the mbarrier has completed the phase with this parity; false if
// the poll limit ran out first
CPSD_D bool mbar_wait(uint32_t addr, uint32_t parity)
{
    for (long it = 0; it < kTcSpinLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kTcThreads)
tc_gemm_tn_kernel(int M, int N, int K, long lda, long ldb, const double *__restrict__ w, int kchunk,
                  const __grid_constant__ TnBatch bt, double *__restrict__ part, int *__restrict__ err)
{
    extern __shared__ unsigned char tc_raw[];
    uint32_t *sm = reinterpret_cast<uint32_t *>(((uintptr_t)tc_raw + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int prod = blockIdx.z / bt.splits, split = blockIdx.z % bt.splits;
    const double *__restrict__ A = bt.A[prod];
    const double *__restrict__ B = bt.B[prod];
    const int i0 = blockIdx.x * kTcM, j0 = blockIdx.y * kTcN;
    const int k0 = split * kchunk, k1 = min(K, k0 + kchunk);
    const int nst = k1 > k0 ? (k1 - k0 + kTcBK - 1) / kTcBK : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"((uint32_t)kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    // staging map: a warp covers 8 rows x 4 consecutive k (one 32-byte
    // sector per row in HBM, 32 consecutive words in shared memory)
    const int kq = tid & 3, rlo = (tid >> 2) & 7, chunk = tid >> 5;  // chunk 0..7 of the 32-wide slab
    // the 32 global loads of a stage (and its weight), issued one stage
    // ahead into the other register set so their latency overlaps the split
    // and the MMAs of the stage before
    double ra[16], rb[16], na[16], nb[16], wk = 1.0, nwk = 1.0;
    auto load = [&](int st, double (&xa)[16], double (&xb)[16], double &xw) {
        const int k = k0 + st * kTcBK + chunk * 4 + kq;
        xw = (w && k < k1) ? w[k >> 1] : 1.0;
#pragma unroll
        for (int rhi = 0; rhi < 16; ++rhi) {
            const int r = rhi * 8 + rlo;
            xa[rhi] = (k < k1 && i0 + r < M) ? A[(long)(i0 + r) * lda + k] : 0.0;
            xb[rhi] = (k < k1 && j0 + r < N) ? B[(long)(j0 + r) * ldb + k] : 0.0;
        }
    };
    if (nst > 0) load(0, ra, rb, wk);
    bool fail = false;
    int issued = 0;  // stages whose MMAs were committed
    for (int it = 0; it < nst; ++it) {
        const int b = it & 1;
        uint32_t *Ah = sm + b * kTcStageWords, *Al = Ah + kTcSlabWords, *Bh = Al + kTcSlabWords,
                 *Bl = Bh + kTcSlabWords;
        // the MMAs of stage it-2 read this slab set: wait for them
        if (it >= 2 && !mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((it >> 1) + 1) & 1))) fail = true;
        if (__syncthreads_or(fail)) {
            fail = true;
            break;
        }
        if (it + 1 < nst) load(it + 1, na, nb, nwk);
#pragma unroll
        for (int rhi = 0; rhi < 16; ++rhi) {
            const float a = (float)(ra[rhi] * wk), bv = (float)rb[rhi];
            const uint32_t ah = tf32_bits(a), bh = tf32_bits(bv);
            const int o = ((chunk * 16 + rhi) << 5) + lane;  // = (chunk*16 + rhi)*32 + rlo*4 + kq
            Ah[o] = ah;
            Al[o] = tf32_bits(a - __uint_as_float(ah));
            Bh[o] = bh;
            Bl[o] = tf32_bits(bv - __uint_as_float(bh));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah = smem_u32(Ah), al = smem_u32(Al), bh = smem_u32(Bh), bl = smem_u32(Bl);
#pragma unroll
            for (int s = 0; s < kTcBK / 8; ++s) {
                const uint32_t o = (uint32_t)s * 4096;  // K-chunk 2s
                tc_mma(tmem, tc_desc(ah + o), tc_desc(bh + o), (it > 0 || s > 0) ? 1u : 0u);
                tc_mma(tmem, tc_desc(ah + o), tc_desc(bl + o), 1u);
                tc_mma(tmem, tc_desc(al + o), tc_desc(bh + o), 1u);
            }
            tc_commit(smem_u32(&mbar[b]));
        }
        issued = it + 1;
        if (it + 1 < nst) {
            wk = nwk;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                ra[q] = na[q];
                rb[q] = nb[q];
            }
        }
    }
    // the last commit tracks every MMA this block issued
    bool done = true;
    if (issued > 0) {
        const int last = issued - 1;
        done = mbar_wait(smem_u32(&mbar[last & 1]), (uint32_t)((last >> 1) & 1));
    }
    if (__syncthreads_or(!done)) fail = true;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!fail) {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows), columns
        // 64 (w / 4) .. +63, and writes rows through shared memory
        double *out = part + ((long)prod * bt.splits + split) * M * N;
        double *E = reinterpret_cast<double *>(sm) + warp * 32 * 33;
        const int rbase = 32 * (warp & 3), cbase = 64 * (warp >> 2);
#pragma unroll 1
        for (int cc = 0; cc < 2; ++cc) {
            uint32_t v[32];
            if (issued > 0) {
                const uint32_t ta = tmem + ((uint32_t)rbase << 16) + (uint32_t)(cbase + 32 * cc);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                    "%30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            } else {
#pragma unroll
                for (int q = 0; q < 32; ++q) v[q] = 0u;
            }
#pragma unroll
            for (int q = 0; q < 32; ++q) E[lane * 33 + q] = (double)__uint_as_float(v[q]);
            __syncwarp();
            const int col = j0 + cbase + 32 * cc + lane;
            for (int rr = 0; rr < 32; ++rr) {
                const int row = i0 + rbase + rr;
                if (row < M && col < N) out[(long)row * N + col] = E[rr * 33 + lane];
            }
            __syncwarp();
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcN));
}

// ------------------------------------------------------ the three overlaps
// tc_overlaps3_kernel: the three overlaps of the Lagrange step in one pass
// over the orbitals (m <= 128 bands of a spin):
//
//   part[0][split] = X' W X,  part[1][split] = X' W Y,  part[2][split] = Y' W Y
//
// with X = C2 and Y = C1 (rows K-contiguous).  Both operands are scaled by
// sqrt(w) so one TF32 hi/lo pair of each serves all three products, and the
// three FP32 accumulators (3 x 128 columns) share one 512-column tensor-
// memory allocation.  Raw FP64 slabs arrive by cp.async, kOvRaw stages ahead,
// so the loads are in flight while earlier stages are split and multiplied;
// every operand byte is read once, against three times for three separate
// products.  Same partial layout as tc_gemm_tn_kernel (prod = 0, 1, 2), summed
// by splitk_reduce_kernel.
constexpr int kOvBK = 16;                               // K per stage
constexpr int kOvRaw = 4;                               // raw FP64 stages in flight
constexpr int kOvRow = 20;                              // raw row stride in doubles (160 B: no bank conflicts)
constexpr int kOvSlabWords = kTcM * kOvBK;              // 2048 words = 8 KB per TF32 slab
constexpr int kOvRawDoubles = 2 * kTcM * kOvRow;        // X and Y, [row][k]: 40 KB per stage
constexpr size_t kOvSmem = (size_t)kOvRaw * kOvRawDoubles * 8 + 2 * 4 * kOvSlabWords * 4 + 128;
constexpr uint32_t kOvTmemCols = 512;

CPSD_D void cp_async16(uint32_t dst, const void *src, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}
CPSD_D void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
CPSD_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__global__ void __launch_bounds__(kTcThreads)
tc_overlaps3_kernel(int m, int K, long ld, const double *__restrict__ X, const double *__restrict__ Y,
                    const double *__restrict__ w, int kchunk, int splits, double *__restrict__ part,
                    int *__restrict__ err)
{
    extern __shared__ unsigned char ov_raw[];
    double *raw = reinterpret_cast<double *>(((uintptr_t)ov_raw + 127) & ~(uintptr_t)127);
    uint32_t *slab = reinterpret_cast<uint32_t *>(raw + (size_t)kOvRaw * kOvRawDoubles);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int split = blockIdx.x;
    const int k0 = split * kchunk, k1 = min(K, k0 + kchunk);
    const int nst = k1 > k0 ? (k1 - k0 + kOvBK - 1) / kOvBK : 0;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(kOvTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    // cp.async map: 2 operands x 128 rows x 8 16-byte chunks = 2048 chunks,
    // 8 per thread; rows past m and K past k1 are zero-filled (src bytes 0,
    // source address kept inside the operand)
    auto issue = [&](int st) {
        double *dst = raw + (size_t)(st % kOvRaw) * kOvRawDoubles;
        const int kb = k0 + st * kOvBK;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = tid + q * kTcThreads;  // 0..2047
            const int op = c >> 10, r = (c >> 3) & 127, kc = (c & 7) * 2;
            const double *src = op ? Y : X;
            const int k = kb + kc;
            const bool ok = (r < m) && (k < k1);
            const double *g = ok ? src + (long)r * ld + k : src;
            cp_async16(smem_u32(dst + (size_t)op * kTcM * kOvRow + r * kOvRow + kc), g, ok ? 16u : 0u);
        }
    };
#pragma unroll
    for (int st = 0; st < kOvRaw - 1; ++st) {
        if (st < nst) issue(st);
        cp_async_commit();
    }

    // conversion map: thread -> (chunk c of 4 K values, row group, lane in core matrix)
    const int kq = tid & 3, rlo = (tid >> 2) & 7, chunk = (tid >> 5) & 3, rhalf = tid >> 7;
    bool fail = false;
    int issued = 0;
    for (int it = 0; it < nst; ++it) {
        const int b = it & 1;
        cp_async_wait<kOvRaw - 2>();  // this thread's copies of stage it have landed
        // the MMAs of stage it-2 read slab set b: wait for them
        if (it >= 2 && !mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((it >> 1) + 1) & 1))) fail = true;
        if (__syncthreads_or(fail)) {  // every thread's stage-it copies are visible too
            fail = true;
            break;
        }
        if (it + kOvRaw - 1 < nst) issue(it + kOvRaw - 1);  // into the slot stage it-1 used
        cp_async_commit();
        const double *rs = raw + (size_t)(it % kOvRaw) * kOvRawDoubles;
        uint32_t *Xh = slab + b * 4 * kOvSlabWords, *Xl = Xh + kOvSlabWords, *Yh = Xl + kOvSlabWords,
                 *Yl = Yh + kOvSlabWords;
        const int k = k0 + it * kOvBK + chunk * 4 + kq;
        const double sw = (w && k < k1) ? sqrt(fmax(w[k >> 1], 0.0)) : 1.0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int rhi = rhalf * 8 + j, r = rhi * 8 + rlo;
            const int kl = chunk * 4 + kq;
            const float xv = (float)(rs[r * kOvRow + kl] * sw);
            const float yv = (float)(rs[kTcM * kOvRow + r * kOvRow + kl] * sw);
            const uint32_t xh = tf32_bits(xv), yh = tf32_bits(yv);
            const int o = ((chunk * 16 + rhi) << 5) + lane;  // (chunk*16 + rhi)*32 + rlo*4 + kq
            Xh[o] = xh;
            Xl[o] = tf32_bits(xv - __uint_as_float(xh));
            Yh[o] = yh;
            Yl[o] = tf32_bits(yv - __uint_as_float(yh));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t xh = smem_u32(Xh), xl = smem_u32(Xl), yh = smem_u32(Yh), yl = smem_u32(Yl);
            const uint32_t d0 = tmem, d1 = tmem + kTcN, d2 = tmem + 2 * kTcN;
#pragma unroll
            for (int s = 0; s < kOvBK / 8; ++s) {
                const uint32_t o = (uint32_t)s * 4096;  // K-chunk 2s
                const uint32_t acc0 = (it > 0 || s > 0) ? 1u : 0u;
                tc_mma(d0, tc_desc(xh + o), tc_desc(xh + o), acc0);  // X'X
                tc_mma(d0, tc_desc(xh + o), tc_desc(xl + o), 1u);
                tc_mma(d0, tc_desc(xl + o), tc_desc(xh + o), 1u);
                tc_mma(d1, tc_desc(xh + o), tc_desc(yh + o), acc0);  // X'Y
                tc_mma(d1, tc_desc(xh + o), tc_desc(yl + o), 1u);
                tc_mma(d1, tc_desc(xl + o), tc_desc(yh + o), 1u);
                tc_mma(d2, tc_desc(yh + o), tc_desc(yh + o), acc0);  // Y'Y
                tc_mma(d2, tc_desc(yh + o), tc_desc(yl + o), 1u);
                tc_mma(d2, tc_desc(yl + o), tc_desc(yh + o), 1u);
            }
            tc_commit(smem_u32(&mbar[b]));
        }
        issued = it + 1;
    }
    cp_async_wait<0>();
    bool done = true;
    if (issued > 0) {
        const int last = issued - 1;
        done = mbar_wait(smem_u32(&mbar[last & 1]), (uint32_t)((last >> 1) & 1));
    }
    if (__syncthreads_or(!done)) fail = true;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!fail) {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (rows) and 6 of
        // the 12 32-column chunks (3 products x 128 columns)
        const long MN = (long)m * m;
        double *E = raw + warp * 32 * 33;
        const int rbase = 32 * (warp & 3);
#pragma unroll 1
        for (int cc = (warp >> 2) * 6; cc < (warp >> 2) * 6 + 6; ++cc) {
            const int prod = cc >> 2, c0 = (cc & 3) * 32;
            uint32_t v[32];
            if (issued > 0) {
                const uint32_t ta = tmem + ((uint32_t)rbase << 16) + (uint32_t)(prod * kTcN + c0);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                    "%30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            } else {
#pragma unroll
                for (int q = 0; q < 32; ++q) v[q] = 0u;
            }
#pragma unroll
            for (int q = 0; q < 32; ++q) E[lane * 33 + q] = (double)__uint_as_float(v[q]);
            __syncwarp();
            double *out = part + ((long)prod * splits + split) * MN;
            const int col = c0 + lane;
            for (int rr = 0; rr < 32; ++rr) {
                const int row = rbase + rr;
                if (row < m && col < m) out[(long)row * m + col] = E[rr * 33 + lane];
            }
            __syncwarp();
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kOvTmemCols));
}

// ------------------------------------------------------------- NN products
// tc_gemm_nn_kernel: Out[j][k] = beta Out[j][k] + alpha sum_l Mat[j][l] B[l][k]
// (the contract of gemm_nn_dmma_kernel: back-projection, residual and constraint
// products with K the long grid dimension) in 3xTF32 on tcgen05.  CTA tile:
// 128 rows j x 128 columns k, the reduction over l in slabs of 32.  Mat
// rows are l-contiguous (K-major as loaded); B rows are k-contiguous, so B is
// read along k (coalesced) and transposed into the K-major slab while it is
// split into TF32 hi/lo.  Same pipeline, waits and error handling as
// tc_gemm_tn_kernel; the epilogue stages rows through shared memory.
__global__ void __launch_bounds__(kTcThreads)
tc_gemm_nn_kernel(int NJ, int K, int L, double alpha, const double *__restrict__ Mat, long ldm,
                  const double *__restrict__ B, long ldb, double beta, double *__restrict__ Out, long ldo,
                  int *__restrict__ err)
{
    extern __shared__ unsigned char nn_raw[];
    uint32_t *sm = reinterpret_cast<uint32_t *>(((uintptr_t)nn_raw + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_base;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k0 = blockIdx.x * kTcN, j0 = blockIdx.y * kTcM;
    const int nst = (L + kTcBK - 1) / kTcBK;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"((uint32_t)kTcN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    // Mat slab map (as the A operand of the TN kernel): 8 rows x 4 l per warp
    const int kq = tid & 3, rlo = (tid >> 2) & 7, chunk = tid >> 5;
    // B slab map: thread -> column kk of the tile and 16 consecutive l
    const int kk = tid & 127, lq = tid >> 7;
    // the global loads of a stage, issued one stage ahead into the other
    // register set so their latency overlaps the split and the MMAs
    double ra[16], rb[16], na[16], nb[16];
    auto load = [&](int st, double (&xa)[16], double (&xb)[16]) {
        const int l0 = st * kTcBK;
        const int l = l0 + chunk * 4 + kq;
#pragma unroll
        for (int rhi = 0; rhi < 16; ++rhi) {
            const int r = rhi * 8 + rlo;
            xa[rhi] = (l < L && j0 + r < NJ) ? Mat[(long)(j0 + r) * ldm + l] : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int lb = l0 + lq * 16 + q;
            xb[q] = (lb < L && k0 + kk < K) ? B[(long)lb * ldb + k0 + kk] : 0.0;
        }
    };
    if (nst > 0) load(0, ra, rb);
    bool fail = false;
    int issued = 0;
    for (int it = 0; it < nst; ++it) {
        const int b = it & 1;
        uint32_t *Ah = sm + b * kTcStageWords, *Al = Ah + kTcSlabWords, *Bh = Al + kTcSlabWords,
                 *Bl = Bh + kTcSlabWords;
        if (it >= 2 && !mbar_wait(smem_u32(&mbar[b]), (uint32_t)(((it >> 1) + 1) & 1))) fail = true;
        if (__syncthreads_or(fail)) {
            fail = true;
            break;
        }
        if (it + 1 < nst) load(it + 1, na, nb);
#pragma unroll
        for (int rhi = 0; rhi < 16; ++rhi) {
            const float a = (float)ra[rhi];
            const uint32_t ah = tf32_bits(a);
            const int o = ((chunk * 16 + rhi) << 5) + lane;  // row rhi*8+rlo, l = chunk*4+kq
            Ah[o] = ah;
            Al[o] = tf32_bits(a - __uint_as_float(ah));
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int ll = lq * 16 + q;  // l within the slab
            const float v = (float)rb[q];
            const uint32_t vh = tf32_bits(v);
            const int o = (((ll >> 2) * 16 + (kk >> 3)) << 5) + ((kk & 7) << 2) + (ll & 3);
            Bh[o] = vh;
            Bl[o] = tf32_bits(v - __uint_as_float(vh));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t ah = smem_u32(Ah), al = smem_u32(Al), bh = smem_u32(Bh), bl = smem_u32(Bl);
#pragma unroll
            for (int s = 0; s < kTcBK / 8; ++s) {
                const uint32_t o = (uint32_t)s * 4096;
                tc_mma(tmem, tc_desc(ah + o), tc_desc(bh + o), (it > 0 || s > 0) ? 1u : 0u);
                tc_mma(tmem, tc_desc(ah + o), tc_desc(bl + o), 1u);
                tc_mma(tmem, tc_desc(al + o), tc_desc(bh + o), 1u);
            }
            tc_commit(smem_u32(&mbar[b]));
        }
        issued = it + 1;
        if (it + 1 < nst) {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                ra[q] = na[q];
                rb[q] = nb[q];
            }
        }
    }
    bool done = true;
    if (issued > 0) {
        const int last = issued - 1;
        done = mbar_wait(smem_u32(&mbar[last & 1]), (uint32_t)((last >> 1) & 1));
    }
    if (__syncthreads_or(!done)) fail = true;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    if (!fail) {
        double *E = reinterpret_cast<double *>(sm) + warp * 32 * 33;
        const int rbase = 32 * (warp & 3), cbase = 64 * (warp >> 2);
#pragma unroll 1
        for (int cc = 0; cc < 2; ++cc) {
            uint32_t v[32];
            if (issued > 0) {
                const uint32_t ta = tmem + ((uint32_t)rbase << 16) + (uint32_t)(cbase + 32 * cc);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                    "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
                    "%30, %31}, [%32];"
                    : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                      "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                      "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]),
                      "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]),
                      "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                    : "r"(ta));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            } else {
#pragma unroll
                for (int q = 0; q < 32; ++q) v[q] = 0u;
            }
#pragma unroll
            for (int q = 0; q < 32; ++q) E[lane * 33 + q] = (double)__uint_as_float(v[q]);
            __syncwarp();
            const int col = k0 + cbase + 32 * cc + lane;
            // the 32 rows' old values first (all loads in flight), then the stores
            double ov[32];
#pragma unroll
            for (int rr = 0; rr < 32; ++rr) {
                const int row = j0 + rbase + rr;
                ov[rr] = (beta != 0.0 && row < NJ && col < K) ? Out[(long)row * ldo + col] : 0.0;
            }
#pragma unroll
            for (int rr = 0; rr < 32; ++rr) {
                const int row = j0 + rbase + rr;
                if (row < NJ && col < K) Out[(long)row * ldo + col] = alpha * E[rr * 33 + lane] + beta * ov[rr];
            }
            __syncwarp();
        }
    } else if (tid == 0) {
        atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTcN));
}
