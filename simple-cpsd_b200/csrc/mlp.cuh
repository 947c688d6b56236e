// mlp.cuh -- the small network of the learned SD preconditioner.
//
// y = W4 h3 + b4,  h_k = tanh(W_k h_{k-1} + b_k),  h_0 = x  (4 -> 64 -> 64 -> 64 -> 1)
//
// Inference reads BF16 copies of the weights (FP32 biases) and accumulates
// in FP32.  Training keeps FP32 master weights and Adam moments; the forward
// pass stores the activations of the batch, the backward pass the deltas, and
// each weight gradient is a fixed-order reduction over the batch (no
// atomics), so a training step is bitwise reproducible.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

constexpr int kMlpIn = 4;
constexpr int kMlpHid = 64;
// flat parameter layout (FP32 master copy)
constexpr int kW1 = 0;                            // [64][4]
constexpr int kB1 = kW1 + kMlpHid * kMlpIn;       // [64]
constexpr int kW2 = kB1 + kMlpHid;                // [64][64]
constexpr int kB2 = kW2 + kMlpHid * kMlpHid;      // [64]
constexpr int kW3 = kB2 + kMlpHid;                // [64][64]
constexpr int kB3 = kW3 + kMlpHid * kMlpHid;      // [64]
constexpr int kW4 = kB3 + kMlpHid;                // [64]
constexpr int kB4 = kW4 + kMlpHid;                // [1]
constexpr int kMlpParams = kB4 + 1;               // 8705
constexpr int kMlpGradThreads = 128;

struct MlpDev {
    const __nv_bfloat16 *wq;  // BF16 weights (same layout; biases unused here)
    const float *p;           // FP32 master parameters (biases read from here)
};

// Forward over a batch: y[s], and the activations when H is given
// ([3][n][64]).  One CTA takes kMlpTile samples: the weights are staged once
// per CTA in shared memory, transposed (Wt[i][o]) and widened to FP32, and
// thread t computes output unit o = t % 64 of a hidden layer for
// kMlpTile / 4 samples, so the 64-long dot products of all units run side by
// side instead of one sample's 8k FMAs in a row.  Every unit's sum is
// bias first, then one fmaf per input in ascending order (the order a
// one-sample evaluation takes, so y does not depend on the tiling).
constexpr int kMlpTile = 16;
constexpr int kMlpTileThreads = 256;
constexpr int kMlpTileSpt = kMlpTile / (kMlpTileThreads / kMlpHid);  // samples a thread: 4

// One CTA's tile of the forward pass; xin(e) is input value e = 4 s + k of
// sample s (s < n).
template <typename XIn>
CPSD_D void mlp_tile(int n, const XIn &xin, const __nv_bfloat16 *__restrict__ wq, const float *__restrict__ p,
                     float *__restrict__ y, float *__restrict__ H)
{
    __shared__ float w1t[kMlpIn][kMlpHid];
    // a padded row (65) keeps the transposing writes and the unit-wise reads
    // on distinct banks
    __shared__ float w2t[kMlpHid][kMlpHid + 1], w3t[kMlpHid][kMlpHid + 1];
    __shared__ float w4[kMlpHid], bias[3][kMlpHid];
    __shared__ __align__(16) float act[3][kMlpTile][kMlpHid];  // h1, h2, h3
    __shared__ float x0[kMlpTile][kMlpIn];
    const int t = threadIdx.x;
    const long s0 = (long)blockIdx.x * kMlpTile;
    // stage: row-major W[o][i] read coalesced, written transposed
    for (int k = t; k < kMlpHid * kMlpHid; k += kMlpTileThreads) {
        const int o = k / kMlpHid, i = k % kMlpHid;
        w2t[i][o] = __bfloat162float(wq[kW2 + k]);
        w3t[i][o] = __bfloat162float(wq[kW3 + k]);
    }
    for (int k = t; k < kMlpHid * kMlpIn; k += kMlpTileThreads) w1t[k % kMlpIn][k / kMlpIn] = __bfloat162float(wq[kW1 + k]);
    if (t < kMlpHid) {
        w4[t] = __bfloat162float(wq[kW4 + t]);
        bias[0][t] = p[kB1 + t];
        bias[1][t] = p[kB2 + t];
        bias[2][t] = p[kB3 + t];
    }
    if (t < kMlpTile * kMlpIn) {
        const long e = s0 * kMlpIn + t;
        x0[t / kMlpIn][t % kMlpIn] = (e < (long)n * kMlpIn) ? xin(e) : 0.0f;
    }
    __syncthreads();
    const int o = t % kMlpHid, sg = t / kMlpHid;
    const long nr = (long)n;
    // layer 1 (4 inputs)
#pragma unroll
    for (int k = 0; k < kMlpTileSpt; ++k) {
        const int sl = sg * kMlpTileSpt + k;
        float acc = bias[0][o];
#pragma unroll
        for (int i = 0; i < kMlpIn; ++i) acc = fmaf(w1t[i][o], x0[sl][i], acc);
        act[0][sl][o] = tanhf(acc);
    }
    __syncthreads();
    // layers 2 and 3 (64 inputs): act[0] -> act[1] -> act[2]
#pragma unroll
    for (int layer = 0; layer < 2; ++layer) {
        const float(*wt)[kMlpHid + 1] = layer ? w3t : w2t;
        const float(*in)[kMlpHid] = act[layer];
        float acc[kMlpTileSpt];
#pragma unroll
        for (int k = 0; k < kMlpTileSpt; ++k) acc[k] = bias[1 + layer][o];
#pragma unroll 4
        for (int i = 0; i < kMlpHid; i += 4) {
            float w[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) w[j] = wt[i + j][o];
#pragma unroll
            for (int k = 0; k < kMlpTileSpt; ++k) {
                const float4 h = *reinterpret_cast<const float4 *>(&in[sg * kMlpTileSpt + k][i]);
                acc[k] = fmaf(w[0], h.x, acc[k]);
                acc[k] = fmaf(w[1], h.y, acc[k]);
                acc[k] = fmaf(w[2], h.z, acc[k]);
                acc[k] = fmaf(w[3], h.w, acc[k]);
            }
        }
#pragma unroll
        for (int k = 0; k < kMlpTileSpt; ++k) act[1 + layer][sg * kMlpTileSpt + k][o] = tanhf(acc[k]);
        __syncthreads();
    }
    if (H) {  // training keeps the activations, one coalesced row per sample and layer
#pragma unroll
        for (int k = 0; k < kMlpTileSpt; ++k) {
            const int sl = sg * kMlpTileSpt + k;
            const long s = s0 + sl;
            if (s >= nr) continue;
#pragma unroll
            for (int l = 0; l < 3; ++l) H[((long)l * nr + s) * kMlpHid + o] = act[l][sl][o];
        }
    }
    // output unit: one thread per sample, 64 inputs in order
    if (t < kMlpTile && s0 + t < nr) {
        float acc = p[kB4];
        for (int i = 0; i < kMlpHid; ++i) acc = fmaf(w4[i], act[2][t][i], acc);
        y[s0 + t] = acc;
    }
}

__global__ void __launch_bounds__(kMlpTileThreads) mlp_forward_kernel(int n, const float *__restrict__ X,
                                                                      const __nv_bfloat16 *__restrict__ wq,
                                                                      const float *__restrict__ p,
                                                                      float *__restrict__ y, float *__restrict__ H)
{
    mlp_tile(n, [X](long e) { return X[e]; }, wq, p, y, H);
}

inline unsigned mlp_forward_blocks(long n) { return (unsigned)((n + kMlpTile - 1) / kMlpTile); }

// MSE loss on y - t: dy = 2 (y - t) / n; deltas dZ3, dZ2, dZ1 ([3][n][64]);
// loss partials per block
__global__ void mlp_backward_delta_kernel(int n, const float *__restrict__ y, const float *__restrict__ t,
                                          const __nv_bfloat16 *__restrict__ wq, const float *__restrict__ H,
                                          float *__restrict__ D, float *__restrict__ dy_out,
                                          float *__restrict__ loss_part)
{
    __shared__ float sh[32];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (s < n) {
        const float r = y[s] - t[s];
        l = r * r;
        const float dy = 2.0f * r / (float)n;
        dy_out[s] = dy;
        const float *h1 = H + (long)s * kMlpHid, *h2 = H + ((long)n + s) * kMlpHid, *h3 = H + (2L * n + s) * kMlpHid;
        float *d3 = D + (2L * n + s) * kMlpHid, *d2 = D + ((long)n + s) * kMlpHid, *d1 = D + (long)s * kMlpHid;
        float z3[kMlpHid], z2[kMlpHid];
        for (int o = 0; o < kMlpHid; ++o) {
            const float hv = h3[o];
            z3[o] = dy * __bfloat162float(wq[kW4 + o]) * (1.0f - hv * hv);
            d3[o] = z3[o];
        }
        for (int i = 0; i < kMlpHid; ++i) {
            float acc = 0.0f;
            for (int o = 0; o < kMlpHid; ++o) acc = fmaf(__bfloat162float(wq[kW3 + o * kMlpHid + i]), z3[o], acc);
            const float hv = h2[i];
            z2[i] = acc * (1.0f - hv * hv);
            d2[i] = z2[i];
        }
        for (int i = 0; i < kMlpHid; ++i) {
            float acc = 0.0f;
            for (int o = 0; o < kMlpHid; ++o) acc = fmaf(__bfloat162float(wq[kW2 + o * kMlpHid + i]), z2[o], acc);
            const float hv = h1[i];
            d1[i] = acc * (1.0f - hv * hv);
        }
    }
    // fixed-order block sum of the squared residuals
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
        loss_part[blockIdx.x] = tot;
    }
}

// gradient of one parameter row: blockIdx.x enumerates (layer, output unit);
// each thread strides over the batch, then a fixed-order tree in shared memory.
// grad[param] for W (row o, inputs i) and b[o].
__global__ void __launch_bounds__(kMlpGradThreads) mlp_wgrad_kernel(int n, const float *__restrict__ X,
                                                                    const float *__restrict__ H,
                                                                    const float *__restrict__ D,
                                                                    const float *__restrict__ dy,
                                                                    float *__restrict__ grad)
{
    __shared__ float red[kMlpGradThreads][kMlpHid + 1];
    const int row = blockIdx.x;  // 0..63: layer1, 64..127: layer2, 128..191: layer3, 192: layer4
    int layer, o;
    if (row < 3 * kMlpHid) {
        layer = row / kMlpHid + 1;
        o = row % kMlpHid;
    } else {
        layer = 4;
        o = 0;
    }
    const int nin = (layer == 1) ? kMlpIn : kMlpHid;
    float acc[kMlpHid + 1];
    for (int i = 0; i <= kMlpHid; ++i) acc[i] = 0.0f;
    for (int s = threadIdx.x; s < n; s += blockDim.x) {
        float delta;
        const float *in;
        if (layer == 4) {
            delta = dy[s];
            in = H + (2L * n + s) * kMlpHid;
        } else {
            delta = D[((long)(layer - 1) * n + s) * kMlpHid + o];
            in = (layer == 1) ? X + (long)s * kMlpIn : H + ((long)(layer - 2) * n + s) * kMlpHid;
        }
        for (int i = 0; i < nin; ++i) acc[i] = fmaf(delta, in[i], acc[i]);
        acc[kMlpHid] += delta;  // bias
    }
    for (int i = 0; i < nin; ++i) red[threadIdx.x][i] = acc[i];
    red[threadIdx.x][kMlpHid] = acc[kMlpHid];
    __syncthreads();
    for (int stride = kMlpGradThreads / 2; stride > 0; stride >>= 1) {
        if ((int)threadIdx.x < stride) {
            for (int i = 0; i < nin; ++i) red[threadIdx.x][i] += red[threadIdx.x + stride][i];
            red[threadIdx.x][kMlpHid] += red[threadIdx.x + stride][kMlpHid];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        int wofs, bofs;
        switch (layer) {
        case 1: wofs = kW1 + o * kMlpIn; bofs = kB1 + o; break;
        case 2: wofs = kW2 + o * kMlpHid; bofs = kB2 + o; break;
        case 3: wofs = kW3 + o * kMlpHid; bofs = kB3 + o; break;
        default: wofs = kW4; bofs = kB4; break;
        }
        for (int i = 0; i < nin; ++i) grad[wofs + i] = red[0][i];
        grad[bofs] = red[0][kMlpHid];
    }
}

// Adam on the FP32 master parameters, then refresh the BF16 copy
__global__ void mlp_adam_kernel(int np, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m1,
                                float *__restrict__ m2, __nv_bfloat16 *__restrict__ wq, float lr, float b1, float b2,
                                float eps, float bc1, float bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    const float pi = p[i] - lr * (a / bc1) / (sqrtf(v / bc2) + eps);
    p[i] = pi;
    wq[i] = __float2bfloat16(pi);
}

__global__ void mlp_quantize_kernel(int np, const float *__restrict__ p, __nv_bfloat16 *__restrict__ wq)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) wq[i] = __float2bfloat16(p[i]);
}

// ------------------------------------------------------------ preconditioned SD
// |G| shells of the sphere (by kinetic energy tg = G^2/2) on which the
// network's step scales are tabulated per band.
constexpr int kShells = 64;
// range of the learned log step scale (K from e^-2 to e^4.5, about 0.14 to 90)
constexpr float kLogKMin = -2.0f, kLogKMax = 4.5f;

// per band: KE_b = <c1|T|c1>, h_b = <c1|cpsi>, q_b = <cpsi|cpsi> (Gamma-point weights)
__global__ void band_stats_kernel(int npw, long ldc, const double *__restrict__ w, const double *__restrict__ tg,
                                  const cx<double> *__restrict__ c1, const cx<double> *__restrict__ cpsi,
                                  double *__restrict__ stats)
{
    __shared__ double sh[3][32];
    const int b = blockIdx.x;
    const cx<double> *a = c1 + (long)b * ldc, *g = cpsi + (long)b * ldc;
    double ke = 0, h = 0, q = 0;
    for (int p = threadIdx.x; p < npw; p += blockDim.x) {
        const double ww = w[p];
        const cx<double> x = a[p], y = g[p];
        ke += ww * tg[p] * (x.x * x.x + x.y * x.y);
        h += ww * (x.x * y.x + x.y * y.y);
        q += ww * (y.x * y.x + y.y * y.y);
    }
    double v[3] = {ke, h, q};
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
        if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = v[k];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 3; ++k) {
            double t = 0;
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += sh[k][i];
            stats[3 * b + k] = t;
        }
    }
}

// network input k of sample id = (band b, shell s): tshell/KE, log KE,
// log |residual|^2, step feature (the step counter advances in
// prec_update_kernel, a later launch)
CPSD_D float prec_feature(double tmax, const double *__restrict__ stats, const int *__restrict__ step, long id,
                          int k)
{
    const int b = (int)(id / kShells), s = (int)(id % kShells);
    const double ke = fmax(stats[3 * b], 1e-12);
    switch (k) {
    case 0: return (float)((s + 0.5) * tmax / kShells / ke);
    case 1: return (float)log(ke);
    case 2: {
        const double hh = stats[3 * b + 1], qq = stats[3 * b + 2];
        return (float)log(fmax(qq - hh * hh, 1e-30));  // |cpsi - <c1|cpsi> c1|^2
    }
    default: return (float)(log1p((double)*step) / 10.0);
    }
}

// The step's network pass: the inputs of each (band, shell) formed from the
// band statistics as the tile is staged, then the tiled forward pass.
__global__ void __launch_bounds__(kMlpTileThreads) prec_mlp_kernel(int nb, double tmax,
                                                                   const double *__restrict__ stats,
                                                                   const int *__restrict__ step,
                                                                   const __nv_bfloat16 *__restrict__ wq,
                                                                   const float *__restrict__ p,
                                                                   float *__restrict__ y)
{
    mlp_tile(nb * kShells, [=](long e) { return prec_feature(tmax, stats, step, e / kMlpIn, (int)(e % kMlpIn)); },
             wq, p, y, nullptr);
}

// c2 (= c1 + dte cpsi, the plain SD update) += dte (K[b][shell(p)] - 1) R,
// with R = cpsi + Pm the residual of cpsi outside the occupied subspace (Pm =
// -C1 (C1' W cpsi), the projection's product): the residual is
// stepped by dte K, the part inside the subspace exactly as plain SD.  log K
// is the network output clamped to [range[0], range[1]] (inside [kLogKMin,
// kLogKMax]): the host narrows the upper end after a rejected block (a trust
// region) and sets [0, 0] for plain SD steps (K = 1, c2 unchanged here).
__global__ void prec_update_kernel(int nb, int npw, long ldc, const int *__restrict__ shell,
                                   const float *__restrict__ y, const float *__restrict__ range, double dte,
                                   const cx<double> *__restrict__ cpsi, const cx<double> *__restrict__ Pm,
                                   cx<double> *__restrict__ c2, int *__restrict__ step)
{
    const long id = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id == 0) atomicAdd(step, 1);
    if (id >= (long)nb * npw) return;
    const int b = (int)(id / npw), p = (int)(id % npw);
    const float lo = fmaxf(kLogKMin, range[0]), hi = fminf(kLogKMax, range[1]);
    const float lk = fminf(fmaxf(y[b * kShells + shell[p]], lo), hi);
    const double f = dte * (exp((double)lk) - 1.0);
    const long o = (long)b * ldc + p;
    const cx<double> q = cpsi[o], m = Pm[o], u = c2[o];
    const cx<double> r{q.x + m.x, q.y + m.y};
    c2[o] = cx<double>{u.x + f * r.x, u.y + f * r.y};
}
