// warm.cu -- learned warm start for 2-D cavities: a coordinate network that
// predicts the 13-moment fields of a steady cavity, trained and evaluated by
// hand-written BF16 tensor-core kernels (tcgen05, accumulators in tensor
// memory), and the Grad 13-moment seeding of the distribution from them.
//
// The reference has no learned part: it always starts from the Maxwellian at
// rest (Initialization/InitialConditions.cpp:18-80).  The seeding writes the
// reference's 2-D Chu representation (Core/Types.hpp:248-256: g1 then g2 per
// particle, g2 = (1/2) integral of c_z^2 f over c_z, so that a Maxwellian has
// g2 = R T g1 / 2 as in MLSTransport/MLSBasis.hpp:87-104), and the 13 moments
// are taken with the reference's discrete sums (MomentCalculations/
// Moments.cpp:66-97).
//
// Network (all layers one fused kernel per 128-point tile):
//   Y0 = features(x, y, a, b)                        64 wide
//   Y1..Y4 = tanh(Y_l W_l^T + b_l)                   128 wide
//   O = Y4 W4^T + b4                                 16 wide, 9 used
// Weights are BF16, accumulation FP32 in tensor memory, activations rounded
// to BF16 between layers.  Training keeps FP32 master weights and Adam state.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "alebgk.h"
#include "ctx.h"
#include "umma.cuh"

namespace alebgk {

namespace {

constexpr int kTile = 128;     // points per tile = MMA M = threads per block
constexpr int kIn = 64;        // features
constexpr int kHid = 128;      // hidden width
constexpr int kOut = 16;       // output rows of W4 (9 used)
constexpr int kOutUsed = 9;
constexpr int kFourier = 12;   // sin/cos(k pi x), sin/cos(k pi y), k = 1..12

__host__ __device__ constexpr int layerIn(int l) { return l == 0 ? kIn : kHid; }
__host__ __device__ constexpr int layerOut(int l) { return l == 4 ? kOut : kHid; }

// Flat FP32 parameter vector: W0..W4 row-major [out][in], then b0..b4.
__host__ __device__ constexpr int wOff(int l)
{
    return l == 0 ? 0 : kHid * kIn + (l - 1) * kHid * kHid;
}
constexpr int kWEnd = kHid * kIn + 3 * kHid * kHid + kOut * kHid;   // 59392
__host__ __device__ constexpr int bOff(int l) { return kWEnd + l * kHid; }
constexpr int kNParams = kWEnd + 4 * kHid + kOut;                    // 59920
constexpr int kLossSlot = kNParams;
constexpr int kPartStride = 59936;   // per-tile partial row: gradients + loss, padded

// Forward weight images (rows = out, K = in) and backward images of W^T
// (rows = in, K = out), BF16, swizzled.
__host__ __device__ constexpr uint32_t wImgOff(int l)
{
    return l == 0 ? 0u : (l < 4 ? 16384u + (uint32_t)(l - 1) * 32768u : 114688u);
}
constexpr uint32_t kWImgBytes = 118784;
__host__ __device__ constexpr uint32_t wtImgOff(int l) { return (uint32_t)(l - 1) * 32768u; }
__host__ __device__ constexpr uint32_t wtImgBytesOf(int l) { return l == 4 ? 16384u : 32768u; }
constexpr uint32_t kWTImgBytes = 114688;

// Per-tile activation images Y_l^T (rows = features, K = the tile's points).
__host__ __device__ constexpr uint32_t yImgOff(int l)
{
    return l == 0 ? 0u : 16384u + (uint32_t)(l - 1) * 32768u;
}
__host__ __device__ constexpr uint32_t yImgBytesOf(int l) { return l == 0 ? 16384u : 32768u; }
constexpr uint32_t kYTileBytes = 147456;

struct LossWeights
{
    float w[kOutUsed];
};

// ---------------------------------------------------------------------------
// Features of one point: (x, y) in [0, 1]^2, a = scaled log density,
// b = scaled lid Mach number.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void features(float4 q, float *f)
{
    f[0] = 2.f * q.x - 1.f;
    f[1] = 2.f * q.y - 1.f;
    f[2] = q.z;
    f[3] = q.w;
#pragma unroll
    for (int k = 1; k <= kFourier; ++k)
    {
        float sx, cx, sy, cy;
        sincospif((float)k * q.x, &sx, &cx);
        sincospif((float)k * q.y, &sy, &cy);
        f[4 * k + 0] = sx;
        f[4 * k + 1] = cx;
        f[4 * k + 2] = sy;
        f[4 * k + 3] = cy;
    }
#pragma unroll
    for (int j = 4 + 4 * kFourier; j < kIn; ++j) f[j] = 0.f;
}

// Writes 16 consecutive values (k0 .. k0+15, k0 a multiple of 16) of row r of
// a shared image as two 16-byte chunks.
__device__ __forceinline__ void storeRow16(uint8_t *img, int rows, int r, int k0, const float *v)
{
    uint4 a, b;
    a.x = packBf16(v[0], v[1]);   a.y = packBf16(v[2], v[3]);
    a.z = packBf16(v[4], v[5]);   a.w = packBf16(v[6], v[7]);
    b.x = packBf16(v[8], v[9]);   b.y = packBf16(v[10], v[11]);
    b.z = packBf16(v[12], v[13]); b.w = packBf16(v[14], v[15]);
    *reinterpret_cast<uint4 *>(img + swzOffset(r, k0, rows)) = a;
    *reinterpret_cast<uint4 *>(img + swzOffset(r, k0 + 8, rows)) = b;
}

__device__ __forceinline__ void storeBf16(uint8_t *p, float x)
{
    *reinterpret_cast<uint16_t *>(p) = (uint16_t)(packBf16(x, 0.f) & 0xFFFFu);
}

// Bounded wait, then a block-wide vote so that every thread takes the same
// branch when a wait gives up.
__device__ __forceinline__ bool waitAll(uint64_t *bar, uint32_t parity, bool &dead)
{
    mbarWait(bar, parity, dead);
    dead = __syncthreads_or(dead ? 1 : 0) != 0;
    return !dead;
}

__device__ __forceinline__ void setErr(int *err, int bit)
{
    if (err) atomicOr(err, bit);
}

// Issues the MMAs of one layer product D = A * B^T over K, one thread.
__device__ __forceinline__ void mmaChain(uint32_t d, uint32_t a, int aRows, uint32_t b,
                                         int bRows, int K, uint32_t idesc)
{
    for (int kk = 0; kk < K / 16; ++kk)
        ummaBf16(d, ummaDesc(a, aRows, kk), ummaDesc(b, bRows, kk), idesc, kk > 0 ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// Forward.  One CTA of 128 threads per tile (persistent over tiles); thread t
// owns point t of the tile = row t of every activation and TMEM lane t.
// With yImg, also writes each tile's Y_l^T images for the backward pass.
// ---------------------------------------------------------------------------
constexpr uint32_t kFwdAct = kWImgBytes;                 // activation image, 32 KB
constexpr uint32_t kFwdBias = kFwdAct + 32768;           // 528 floats
constexpr uint32_t kFwdBar = kFwdBias + 2176;            // 2 mbarriers + TMEM slot
constexpr uint32_t kFwdSmem = kFwdBar + 64 + 1024;       // + alignment slack

__global__ void __launch_bounds__(kTile, 1)
k_mlp_forward(const uint8_t *__restrict__ wImg, const float *__restrict__ params,
              const float4 *__restrict__ pts, const int *__restrict__ idx, int n,
              float *__restrict__ out, uint8_t *__restrict__ yImg, int *err)
{
    extern __shared__ uint8_t smemRaw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    uint8_t *act = sm + kFwdAct;
    float *bias = reinterpret_cast<float *>(sm + kFwdBias);
    uint64_t *barW = reinterpret_cast<uint64_t *>(sm + kFwdBar);
    uint64_t *barM = barW + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(barW + 2);
    const int t = threadIdx.x, warp = t >> 5;
    bool dead = false;

    if (t == 0)
    {
        mbarInit(barW, 1);
        mbarInit(barM, 1);
        mbarInitFence();
    }
    if (warp == 0) tmemAlloc(tslot, 128);
    for (int j = t; j < 4 * kHid + kOut; j += kTile) bias[j] = params[kWEnd + j];
    tmemFenceBefore();
    __syncthreads();
    if (t == 0)
    {
        mbarExpectTx(barW, kWImgBytes);
        for (uint32_t o = 0; o < kWImgBytes; o += 16384)
            bulkLoad(sm + o, wImg + o, min(16384u, kWImgBytes - o), barW);
    }
    waitAll(barW, 0, dead);
    tmemFenceAfter();
    const uint32_t tmem = *tslot;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t actS = smemAddr(act), wS = smemAddr(sm);
    uint32_t phase = 0;

    const int ntiles = (n + kTile - 1) / kTile;
    for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x)
    {
        const int p = tile * kTile + t;
        const bool valid = p < n;
        uint8_t *yt = yImg ? yImg + (size_t)tile * kYTileBytes : nullptr;
        {
            float f[kIn];
            if (valid)
                features(pts[idx ? idx[p] : p], f);
            else
                for (int j = 0; j < kIn; ++j) f[j] = 0.f;
#pragma unroll
            for (int k0 = 0; k0 < kIn; k0 += 16) storeRow16(act, kTile, t, k0, f + k0);
            if (yt)
            {
#pragma unroll
                for (int j = 0; j < kIn; ++j)
                    storeBf16(yt + yImgOff(0) + swzOffset(j, t, kIn), f[j]);
            }
        }
        fenceProxyAsync();
        tmemFenceBefore();
        __syncthreads();
#pragma unroll 1
        for (int l = 0; l < 5; ++l)
        {
            const int K = layerIn(l), N = layerOut(l);
            if (t == 0)
            {
                tmemFenceAfter();
                mmaChain(tmem, actS, kTile, wS + wImgOff(l), N, K, ummaIdescBf16(kTile, N));
                ummaCommit(barM);
            }
            if (!waitAll(barM, phase, dead)) break;
            phase ^= 1;
            tmemFenceAfter();
            for (int c0 = 0; c0 < N; c0 += 16)
            {
                float v[16];
                tmemLoad16(tlane + c0, v);
                const float *bl = bias + l * kHid + c0;
                if (l < 4)
                {
#pragma unroll
                    for (int i = 0; i < 16; ++i) v[i] = tanhf(v[i] + bl[i]);
                    storeRow16(act, kTile, t, c0, v);
                    if (yt)
                    {
                        uint8_t *yl = yt + yImgOff(l + 1);
#pragma unroll
                        for (int i = 0; i < 16; ++i)
                            storeBf16(yl + swzOffset(c0 + i, t, kHid), v[i]);
                    }
                }
                else if (valid)
                {
                    float4 *o = reinterpret_cast<float4 *>(out + (size_t)p * kOut + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        o[i] = make_float4(v[4 * i] + bl[4 * i], v[4 * i + 1] + bl[4 * i + 1],
                                           v[4 * i + 2] + bl[4 * i + 2],
                                           v[4 * i + 3] + bl[4 * i + 3]);
                }
            }
            fenceProxyAsync();
            tmemFenceBefore();
            __syncthreads();
        }
    }
    if (dead && t == 0) setErr(err, 1);
    tmemFenceBefore();
    __syncthreads();
    if (warp == 0)
    {
        tmemFenceAfter();
        tmemDealloc(tmem, 128);
    }
}

// ---------------------------------------------------------------------------
// Backward of the tiles a forward pass just wrote.  Per tile and layer l
// (4 .. 0), with dZ_l in shared memory both as rows of points (dZ) and as
// rows of features (dZT):
//   dW_l = dZ_l^T Y_l      (for l = 4 as dW4^T = Y4^T dZ4, so that M = 128)
//   db_l = column sums of dZ_l
//   dZ_{l-1} = (dZ_l W_l) * (1 - Y_l^2)
// The Y_l^T images and the W_l^T images arrive by bulk copies into two
// double-buffered slots.  Gradients go to one FP32 partial row per tile.
// ---------------------------------------------------------------------------
constexpr uint32_t kBwdWT = 0;          // 2 x 32 KB
constexpr uint32_t kBwdY = 65536;       // 2 x 32 KB
constexpr uint32_t kBwdDZ = 131072;     // 32 KB: rows = points, K = out
constexpr uint32_t kBwdDZT = 163840;    // 32 KB: rows = out, K = points
constexpr uint32_t kBwdBar = 196608;    // 5 mbarriers + TMEM slot + loss scratch
constexpr uint32_t kBwdSmem = kBwdBar + 128 + 1024;

__global__ void __launch_bounds__(kTile, 1)
k_mlp_backward(const uint8_t *__restrict__ wtImg, const uint8_t *__restrict__ yImg,
               const float *__restrict__ out, const float *__restrict__ tgt,
               const int *__restrict__ idx, int n, LossWeights lw, float *__restrict__ part,
               int *err)
{
    extern __shared__ uint8_t smemRaw[];
    uint8_t *sm = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smemRaw) + 1023) & ~uintptr_t(1023));
    uint8_t *dz = sm + kBwdDZ, *dzt = sm + kBwdDZT;
    uint64_t *barWT = reinterpret_cast<uint64_t *>(sm + kBwdBar);   // [2]
    uint64_t *barY = barWT + 2;                                      // [2]
    uint64_t *barM = barWT + 4;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(barWT + 5);
    float *red = reinterpret_cast<float *>(barWT + 6);               // 4 floats
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    bool dead = false;

    if (t == 0)
    {
        for (int i = 0; i < 5; ++i) mbarInit(barWT + i, 1);
        mbarInitFence();
    }
    if (warp == 0) tmemAlloc(tslot, 256);
    tmemFenceBefore();
    __syncthreads();
    tmemFenceAfter();
    const uint32_t tmem = *tslot;
    const uint32_t tlane = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t dzS = smemAddr(dz), dztS = smemAddr(dzt);
    uint32_t phM = 0, phWT[2] = {0, 0}, phY[2] = {0, 0};
    const float invN = 1.f / (float)n;

    auto loadWT = [&](int l, int b) {
        mbarExpectTx(barWT + b, wtImgBytesOf(l));
        bulkLoad(sm + kBwdWT + b * 32768, wtImg + wtImgOff(l), wtImgBytesOf(l), barWT + b);
    };
    auto loadY = [&](const uint8_t *yt, int l, int b) {
        mbarExpectTx(barY + b, yImgBytesOf(l));
        bulkLoad(sm + kBwdY + b * 32768, yt + yImgOff(l), yImgBytesOf(l), barY + b);
    };

    const int ntiles = (n + kTile - 1) / kTile;
    for (int tile = blockIdx.x; tile < ntiles && !dead; tile += gridDim.x)
    {
        const uint8_t *yt = yImg + (size_t)tile * kYTileBytes;
        float *pr = part + (size_t)tile * kPartStride;
        if (t == 0)
        {
            loadY(yt, 4, 0);
            loadWT(4, 0);
            loadY(yt, 3, 1);
            loadWT(3, 1);
        }
        // dZ4 = dLoss/dO and the tile's loss.
        {
            const int p = tile * kTile + t;
            float d[kOut], loss = 0.f;
#pragma unroll
            for (int c = 0; c < kOut; ++c) d[c] = 0.f;
            if (p < n)
            {
                const float *o = out + (size_t)p * kOut;
                const float *g = tgt + (size_t)(idx ? idx[p] : p) * kOut;
#pragma unroll
                for (int c = 0; c < kOutUsed; ++c)
                {
                    const float e = o[c] - g[c];
                    loss += lw.w[c] * e * e;
                    d[c] = 2.f * lw.w[c] * e * invN;
                }
            }
            storeRow16(dz, kTile, t, 0, d);
#pragma unroll
            for (int c = 0; c < kOut; ++c) storeBf16(dzt + swzOffset(c, t, kOut), d[c]);
            for (int s = 16; s > 0; s >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, s);
            if (lane == 0) red[warp] = loss;
        }
        fenceProxyAsync();
        tmemFenceBefore();
        __syncthreads();
        if (t == 0) pr[kLossSlot] = (red[0] + red[1]) + (red[2] + red[3]);

#pragma unroll 1
        for (int l = 4; l >= 0; --l)
        {
            const int b = (4 - l) & 1;
            const int in = layerIn(l), outW = layerOut(l);
            const uint32_t yS = smemAddr(sm + kBwdY + b * 32768);
            const uint32_t wtS = smemAddr(sm + kBwdWT + b * 32768);
            if (!waitAll(barY + b, phY[b], dead)) break;
            phY[b] ^= 1;
            if (l > 0)
            {
                if (!waitAll(barWT + b, phWT[b], dead)) break;
                phWT[b] ^= 1;
            }
            if (t == 0)
            {
                tmemFenceAfter();
                if (l == 4)   // dW4^T [in x out] = Y4^T dZ4: A = Y4^T, B = dZ4^T
                    mmaChain(tmem + 128, yS, kHid, dztS, kOut, kTile, ummaIdescBf16(kTile, kOut));
                else          // dW_l [out x in] = dZ_l^T Y_l: A = dZ_l^T, B = Y_l^T
                    mmaChain(tmem + 128, dztS, kHid, yS, in, kTile, ummaIdescBf16(kTile, in));
                if (l > 0)    // dY_l [points x in] = dZ_l W_l: A = dZ_l, B = W_l^T
                    mmaChain(tmem, dzS, kTile, wtS, kHid, outW, ummaIdescBf16(kTile, kHid));
                ummaCommit(barM);
            }
            if (!waitAll(barM, phM, dead)) break;
            phM ^= 1;
            tmemFenceAfter();
            if (t == 0 && l - 2 >= 1) loadWT(l - 2, b);
            // db_l from the BF16 dZ_l the MMAs used.
            if (t < outW)
            {
                float s = 0.f;
                for (int k0 = 0; k0 < kTile; k0 += 8)
                {
                    const uint4 w = *reinterpret_cast<const uint4 *>(dzt + swzOffset(t, k0, outW));
                    s += ((bf16Lo(w.x) + bf16Hi(w.x)) + (bf16Lo(w.y) + bf16Hi(w.y))) +
                         ((bf16Lo(w.z) + bf16Hi(w.z)) + (bf16Lo(w.w) + bf16Hi(w.w)));
                }
                pr[bOff(l) + t] = s;
            }
            // dW_l to the partial row.
            if (l == 4)
            {
                float v[16];
                tmemLoad16(tlane + 128, v);
#pragma unroll
                for (int o = 0; o < kOut; ++o) pr[wOff(4) + o * kHid + t] = v[o];
            }
            else
            {
                for (int c0 = 0; c0 < in; c0 += 16)
                {
                    float v[16];
                    tmemLoad16(tlane + 128 + c0, v);
                    float4 *d4 = reinterpret_cast<float4 *>(pr + wOff(l) + t * in + c0);
#pragma unroll
                    for (int i = 0; i < 4; ++i)
                        d4[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                }
            }
            __syncthreads();   // everyone is done reading dZ / dZT of layer l
            if (l > 0)
            {
                const uint8_t *ys = sm + kBwdY + b * 32768;
                float dzRow[16];
                for (int c0 = 0; c0 < kHid; c0 += 16)
                {
                    tmemLoad16(tlane + c0, dzRow);
#pragma unroll
                    for (int i = 0; i < 16; ++i)
                    {
                        const int j = c0 + i;
                        const uint16_t yb =
                            *reinterpret_cast<const uint16_t *>(ys + swzOffset(j, t, kHid));
                        const float y = __uint_as_float((uint32_t)yb << 16);
                        dzRow[i] = dzRow[i] * (1.f - y * y);
                        storeBf16(dzt + swzOffset(j, t, kHid), dzRow[i]);
                    }
                    storeRow16(dz, kTile, t, c0, dzRow);
                }
            }
            fenceProxyAsync();
            tmemFenceBefore();
            __syncthreads();
            if (t == 0 && l - 2 >= 0) loadY(yt, l - 2, b);
        }
        __syncthreads();
    }
    if (dead && t == 0) setErr(err, 2);
    tmemFenceBefore();
    __syncthreads();
    if (warp == 0)
    {
        tmemFenceAfter();
        tmemDealloc(tmem, 256);
    }
}

// ---------------------------------------------------------------------------
// Gradient = sum of the tile partials in tile order; then either a copy out
// (gradient check) or one Adam step on the FP32 master weights, and the BF16
// images of the new weights.  Rows 9..15 of W4 and b4 stay zero.
// ---------------------------------------------------------------------------
struct AdamArgs
{
    float lr, beta1, beta2, eps, c1, c2;   // c1 = 1 - beta1^t, c2 = 1 - beta2^t
    int apply;
};

__device__ __forceinline__ void writeImages(int i, float w, uint8_t *wImg, uint8_t *wtImg)
{
    if (i >= kWEnd) return;
    int l = 0;
    while (l < 4 && i >= wOff(l + 1)) ++l;
    const int in = layerIn(l), outW = layerOut(l);
    const int o = (i - wOff(l)) / in, k = (i - wOff(l)) % in;
    storeBf16(wImg + wImgOff(l) + swzOffset(o, k, outW), w);
    if (l >= 1) storeBf16(wtImg + wtImgOff(l) + swzOffset(k, o, kHid), w);
}

__device__ __forceinline__ bool isPadParam(int i)
{
    if (i >= wOff(4) && i < kWEnd) return (i - wOff(4)) / kHid >= kOutUsed;
    if (i >= bOff(4) && i < kNParams) return i - bOff(4) >= kOutUsed;
    return false;
}

__global__ void k_mlp_update(const float *__restrict__ part, int ntiles, float *grad,
                             float *params, float *m, float *v, uint8_t *wImg, uint8_t *wtImg,
                             float *loss, AdamArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > kNParams) return;
    float g = 0.f;
    for (int tl = 0; tl < ntiles; ++tl) g += part[(size_t)tl * kPartStride + i];
    if (i == kLossSlot)
    {
        if (loss) *loss = g;
        return;
    }
    if (isPadParam(i)) g = 0.f;
    if (grad) grad[i] = g;
    if (!a.apply) return;
    const float mi = a.beta1 * m[i] + (1.f - a.beta1) * g;
    const float vi = a.beta2 * v[i] + (1.f - a.beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float w = params[i];
    if (!isPadParam(i)) w -= a.lr * (mi / a.c1) / (sqrtf(vi / a.c2) + a.eps);
    params[i] = w;
    writeImages(i, w, wImg, wtImg);
}

__global__ void k_mlp_pack(const float *__restrict__ params, uint8_t *wImg, uint8_t *wtImg)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kWEnd) writeImages(i, params[i], wImg, wtImg);
}

// ---------------------------------------------------------------------------
// Grad 13-moment seed of a 2-D Chu cloud (one warp per particle).  With
// theta = R T, p = rho theta, C = v - u, C2 = |C|^2, A = sigma_ij C_i C_j /
// (2 p theta), B = q.C / (p theta) and sigma_zz = -(sigma_xx + sigma_yy):
//   g1 = M [1 + A + sigma_zz/(2p) + B (C2/(5 theta) - 4/5)]
//   g2 = theta/2 M [1 + A + 3 sigma_zz/(2p) + B (C2/(5 theta) - 2/5)]
// with M = rho/(2 pi theta) exp(-C2/(2 theta)), negative values set to zero.
// These are the c_z integrals of Grad's 13-moment distribution (Grad 1949)
// taken with the Chu weights 1 and c_z^2/2.  The macros of the step are the
// discrete sums of the seeded rows (Moments.cpp:66-97).
// ---------------------------------------------------------------------------
struct Affine
{
    double scale[kOutUsed], shift[kOutUsed];
};

template <typename T>
__global__ void k_seed_grad13(T *f, StepParams p, const float *__restrict__ net, int ldnet,
                              Affine af, double *macro, int *mood)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= p.N) return;
    double m[kOutUsed];
#pragma unroll
    for (int c = 0; c < kOutUsed; ++c)
        m[c] = af.shift[c] + af.scale[c] * (double)net[(size_t)warp * ldnet + c];
    const double rho = fmax(m[0], 1e-30), ux = m[1], uy = m[2];
    const double th = p.R * fmax(m[3], 1e-6), pr = rho * th;
    const double sxx = m[4], sxy = m[5], syy = m[6], qx = m[7], qy = m[8];
    const double szz = -(sxx + syy);
    const double norm = rho / (2.0 * M_PI * th);
    T *row = f + (size_t)warp * p.ldf;
    const int Nv = p.Nv, V = p.V;
    double s0 = 0, s1 = 0, s2 = 0, se = 0;
    for (int k = lane; k < V; k += 32)
    {
        const double vx = p.vmin + (k % Nv) * p.dv, vy = p.vmin + (k / Nv) * p.dv;
        const double cx = vx - ux, cy = vy - uy, c2 = cx * cx + cy * cy;
        const double M = norm * exp(-c2 / (2.0 * th));
        const double A = (sxx * cx * cx + 2.0 * sxy * cx * cy + syy * cy * cy) / (2.0 * pr * th);
        const double B = (qx * cx + qy * cy) / (pr * th);
        const double g1 = fmax(M * (1.0 + A + szz / (2.0 * pr) + B * (c2 / (5.0 * th) - 0.8)), 0.0);
        const double g2 =
            fmax(0.5 * th * M * (1.0 + A + 1.5 * szz / pr + B * (c2 / (5.0 * th) - 0.4)), 0.0);
        const T t1 = (T)g1, t2 = (T)g2;
        row[k] = t1;
        row[V + k] = t2;
        const double d1 = (double)t1, d2 = (double)t2;
        s0 += d1;
        s1 += vx * d1;
        s2 += vy * d1;
        se += (vx * vx + vy * vy) * d1 + 2.0 * d2;
    }
    for (int s = 16; s > 0; s >>= 1)
    {
        s0 += __shfl_xor_sync(0xffffffffu, s0, s);
        s1 += __shfl_xor_sync(0xffffffffu, s1, s);
        s2 += __shfl_xor_sync(0xffffffffu, s2, s);
        se += __shfl_xor_sync(0xffffffffu, se, s);
    }
    if (lane == 0)
    {
        const double dv2 = p.dvN;
        const double r = s0 * dv2;
        double *mc = macro + 6 * (size_t)warp;
        if (r > 1e-30)
        {
            const double u = s1 * dv2 / r, v = s2 * dv2 / r;
            const double T_ = fmax((se * dv2 / r - (u * u + v * v)) / (3.0 * p.R), 1e-6);
            mc[0] = r; mc[1] = u; mc[2] = v; mc[3] = 0.0; mc[4] = T_; mc[5] = r * p.R * T_;
        }
        else
        {
            mc[0] = r; mc[1] = 0; mc[2] = 0; mc[3] = 0; mc[4] = 1e-6; mc[5] = 0;
        }
        mood[warp] = 0;
    }
}

// 13 moments of the current 2-D state (h times the deferred scale), one warp
// per particle: rho, ux, uy, T, sigma_xx, sigma_xy, sigma_yy, q_x, q_y with
// sigma_ij = sum C_i C_j g1 dv^2 - p delta_ij and
// q_i = (1/2) sum C_i (C2 g1 + 2 g2) dv^2.
template <typename T>
__global__ void k_moments13(const T *f, StepParams p, const StepScalars *__restrict__ sc,
                            double *out)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= p.N) return;
    const T *row = f + (size_t)warp * p.ldf;
    const int Nv = p.Nv, V = p.V;
    const double scale = sc->scale, dv2 = p.dvN;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int k = lane; k < V; k += 32)
    {
        const double vx = p.vmin + (k % Nv) * p.dv, vy = p.vmin + (k / Nv) * p.dv;
        const double g1 = (double)row[k];
        s0 += g1;
        s1 += vx * g1;
        s2 += vy * g1;
    }
    for (int s = 16; s > 0; s >>= 1)
    {
        s0 += __shfl_xor_sync(0xffffffffu, s0, s);
        s1 += __shfl_xor_sync(0xffffffffu, s1, s);
        s2 += __shfl_xor_sync(0xffffffffu, s2, s);
    }
    const double rho = s0 * scale * dv2;
    const double ux = s1 / s0, uy = s2 / s0;
    double a[6] = {0, 0, 0, 0, 0, 0};   // Cx^2, CxCy, Cy^2 on g1; energy; qx; qy
    for (int k = lane; k < V; k += 32)
    {
        const double cx = p.vmin + (k % Nv) * p.dv - ux, cy = p.vmin + (k / Nv) * p.dv - uy;
        const double g1 = (double)row[k], g2 = (double)row[V + k];
        const double e = (cx * cx + cy * cy) * g1 + 2.0 * g2;
        a[0] += cx * cx * g1;
        a[1] += cx * cy * g1;
        a[2] += cy * cy * g1;
        a[3] += e;
        a[4] += cx * e;
        a[5] += cy * e;
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
        for (int s = 16; s > 0; s >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], s);
    if (lane == 0)
    {
        const double w = scale * dv2;
        const double th = a[3] * w / (3.0 * rho), pr = rho * th;
        double *o = out + 9 * (size_t)warp;
        o[0] = rho;
        o[1] = ux;
        o[2] = uy;
        o[3] = th / p.R;
        o[4] = a[0] * w - pr;
        o[5] = a[1] * w;
        o[6] = a[2] * w - pr;
        o[7] = 0.5 * a[4] * w;
        o[8] = 0.5 * a[5] * w;
    }
}

}  // namespace

cudaError_t launchSeedGrad13(alebgk_ctx *c, const float *net, int ldnet, const double *scale,
                             const double *shift)
{
    const StepParams &p = c->sp;
    Affine af;
    for (int q = 0; q < kOutUsed; ++q)
    {
        af.scale[q] = scale[q];
        af.shift[q] = shift[q];
    }
    const int blocks = (p.N * 32 + 255) / 256;
    if (c->cfg.precision == 64)
        k_seed_grad13<double><<<blocks, 256, 0, c->stream>>>(
            static_cast<double *>(c->d.f[c->cur]), p, net, ldnet, af, c->d.macro[c->cur],
            c->d.mood);
    else
        k_seed_grad13<float><<<blocks, 256, 0, c->stream>>>(
            static_cast<float *>(c->d.f[c->cur]), p, net, ldnet, af, c->d.macro[c->cur],
            c->d.mood);
    return cudaGetLastError();
}

cudaError_t launchMoments13(alebgk_ctx *c, double *out)
{
    const StepParams &p = c->sp;
    const int blocks = (p.N * 32 + 255) / 256;
    if (c->cfg.precision == 64)
        k_moments13<double><<<blocks, 256, 0, c->stream>>>(
            static_cast<const double *>(c->d.f[c->cur]), p, c->d.sc, out);
    else
        k_moments13<float><<<blocks, 256, 0, c->stream>>>(
            static_cast<const float *>(c->d.f[c->cur]), p, c->d.sc, out);
    return cudaGetLastError();
}

}  // namespace alebgk

// ---------------------------------------------------------------------------
// Network object and its C-ABI.
// ---------------------------------------------------------------------------
using namespace alebgk;

struct alebgk_net
{
    int device = 0;
    cudaStream_t stream = nullptr;
    float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    uint8_t *wImg = nullptr, *wtImg = nullptr;
    uint8_t *yImg = nullptr;
    float *part = nullptr, *out = nullptr;
    int *err = nullptr;
    size_t tilesCap = 0;
    long long adamSteps = 0;
    std::string msg;
};

namespace {

int netFail(alebgk_net *n, int code, const std::string &m)
{
    if (n) n->msg = m;
    return code;
}

#define NCK(call)                                                                     \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return netFail(n, ALEBGK_ECUDA, std::string(#call) + ": " +               \
                                                cudaGetErrorString(e_));              \
    } while (0)

int ensureTiles(alebgk_net *n, size_t tiles)
{
    if (tiles <= n->tilesCap) return ALEBGK_OK;
    cudaFree(n->yImg);
    cudaFree(n->part);
    cudaFree(n->out);
    n->yImg = nullptr; n->part = nullptr; n->out = nullptr;
    n->tilesCap = 0;
    NCK(cudaMalloc(&n->yImg, tiles * kYTileBytes));
    NCK(cudaMalloc(&n->part, tiles * kPartStride * sizeof(float)));
    NCK(cudaMalloc(&n->out, tiles * kTile * kOut * sizeof(float)));
    n->tilesCap = tiles;
    return ALEBGK_OK;
}

int checkErr(alebgk_net *n)
{
    int h = 0;
    NCK(cudaMemcpyAsync(&h, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    if (h) return netFail(n, ALEBGK_ECUDA, "a tensor-core pipeline wait timed out");
    return ALEBGK_OK;
}

int gridFor(const alebgk_net *n, int tiles)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device);
    return tiles < sms ? tiles : sms;
}

// Forward (+ backward) of one batch; leaves the partial rows in n->part.
int runBatch(alebgk_net *n, const float *pts, const float *tgt, const int *idx, int count,
             const float *chanW, bool train, float *outDev)
{
    const int tiles = (count + kTile - 1) / kTile;
    if (train)
    {
        int rc = ensureTiles(n, tiles);
        if (rc) return rc;
    }
    const int grid = gridFor(n, tiles);
    k_mlp_forward<<<grid, kTile, kFwdSmem, n->stream>>>(
        n->wImg, n->params, reinterpret_cast<const float4 *>(pts), idx, count,
        train ? n->out : outDev, train ? n->yImg : nullptr, n->err);
    NCK(cudaGetLastError());
    if (!train) return ALEBGK_OK;
    LossWeights lw;
    for (int c = 0; c < kOutUsed; ++c) lw.w[c] = chanW ? chanW[c] : 1.f;
    k_mlp_backward<<<grid, kTile, kBwdSmem, n->stream>>>(n->wtImg, n->yImg, n->out, tgt, idx,
                                                        count, lw, n->part, n->err);
    NCK(cudaGetLastError());
    return ALEBGK_OK;
}

}  // namespace

extern "C" {

int alebgk_net_nparams(void) { return kNParams; }

int alebgk_net_create(int device, alebgk_net **out)
{
    if (!out) return ALEBGK_EINVAL;
    *out = nullptr;
    alebgk_net *n = new alebgk_net();
    n->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&n->params, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->m, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->v, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->grad, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&n->wImg, kWImgBytes);
    if (e == cudaSuccess) e = cudaMalloc(&n->wtImg, kWTImgBytes);
    if (e == cudaSuccess) e = cudaMalloc(&n->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(n->params, 0, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(n->m, 0, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(n->v, 0, kPartStride * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(n->wImg, 0, kWImgBytes);
    if (e == cudaSuccess) e = cudaMemset(n->wtImg, 0, kWTImgBytes);
    if (e == cudaSuccess) e = cudaMemset(n->err, 0, sizeof(int));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kFwdSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_mlp_backward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kBwdSmem);
    if (e != cudaSuccess)
    {
        alebgk_net_destroy(n);
        return ALEBGK_ECUDA;
    }
    *out = n;
    return ALEBGK_OK;
}

void alebgk_net_destroy(alebgk_net *n)
{
    if (!n) return;
    cudaSetDevice(n->device);
    if (n->stream) cudaStreamSynchronize(n->stream);
    for (void *p : {(void *)n->params, (void *)n->m, (void *)n->v, (void *)n->grad,
                    (void *)n->loss, (void *)n->wImg, (void *)n->wtImg, (void *)n->yImg,
                    (void *)n->part, (void *)n->out, (void *)n->err})
        if (p) cudaFree(p);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
}

const char *alebgk_net_last_error(const alebgk_net *n) { return n ? n->msg.c_str() : ""; }

int alebgk_net_set_params(alebgk_net *n, const float *host)
{
    if (!n || !host) return ALEBGK_EINVAL;
    NCK(cudaSetDevice(n->device));
    std::vector<float> w(host, host + kNParams);
    for (int i = 0; i < kNParams; ++i)
    {
        const bool pad = (i >= wOff(4) && i < kWEnd && (i - wOff(4)) / kHid >= kOutUsed) ||
                         (i >= bOff(4) && i - bOff(4) >= kOutUsed);
        if (pad) w[i] = 0.f;
    }
    NCK(cudaMemcpyAsync(n->params, w.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice,
                        n->stream));
    NCK(cudaMemsetAsync(n->m, 0, kPartStride * sizeof(float), n->stream));
    NCK(cudaMemsetAsync(n->v, 0, kPartStride * sizeof(float), n->stream));
    k_mlp_pack<<<(kWEnd + 255) / 256, 256, 0, n->stream>>>(n->params, n->wImg, n->wtImg);
    NCK(cudaGetLastError());
    NCK(cudaStreamSynchronize(n->stream));
    n->adamSteps = 0;
    return ALEBGK_OK;
}

int alebgk_net_get_params(alebgk_net *n, float *host)
{
    if (!n || !host) return ALEBGK_EINVAL;
    NCK(cudaSetDevice(n->device));
    NCK(cudaMemcpyAsync(host, n->params, kNParams * sizeof(float), cudaMemcpyDeviceToHost,
                        n->stream));
    NCK(cudaStreamSynchronize(n->stream));
    return ALEBGK_OK;
}

int alebgk_net_forward(alebgk_net *n, const float *pts, const int *idx, int count, float *out)
{
    if (!n || !pts || !out || count < 0) return ALEBGK_EINVAL;
    if (count == 0) return ALEBGK_OK;
    NCK(cudaSetDevice(n->device));
    int rc = runBatch(n, pts, nullptr, idx, count, nullptr, false, out);
    if (rc) return rc;
    return checkErr(n);
}

int alebgk_net_grad(alebgk_net *n, const float *pts, const float *tgt, const int *idx,
                    int count, const float *chanW, float *gradHost, float *lossHost)
{
    if (!n || !pts || !tgt || count <= 0) return ALEBGK_EINVAL;
    NCK(cudaSetDevice(n->device));
    int rc = runBatch(n, pts, tgt, idx, count, chanW, true, nullptr);
    if (rc) return rc;
    const int tiles = (count + kTile - 1) / kTile;
    AdamArgs a{};
    a.apply = 0;
    k_mlp_update<<<(kNParams + 1 + 255) / 256, 256, 0, n->stream>>>(
        n->part, tiles, n->grad, n->params, n->m, n->v, n->wImg, n->wtImg, n->loss, a);
    NCK(cudaGetLastError());
    rc = checkErr(n);
    if (rc) return rc;
    if (gradHost)
        NCK(cudaMemcpy(gradHost, n->grad, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
    if (lossHost) NCK(cudaMemcpy(lossHost, n->loss, sizeof(float), cudaMemcpyDeviceToHost));
    return ALEBGK_OK;
}

int alebgk_net_train_step(alebgk_net *n, const float *pts, const float *tgt, const int *idx,
                          int count, const float *chanW, float lr, float beta1, float beta2,
                          float eps, float *lossHost)
{
    if (!n || !pts || !tgt || count <= 0 || !(lr >= 0.f)) return ALEBGK_EINVAL;
    NCK(cudaSetDevice(n->device));
    int rc = runBatch(n, pts, tgt, idx, count, chanW, true, nullptr);
    if (rc) return rc;
    const int tiles = (count + kTile - 1) / kTile;
    n->adamSteps += 1;
    AdamArgs a;
    a.lr = lr;
    a.beta1 = beta1;
    a.beta2 = beta2;
    a.eps = eps;
    a.c1 = 1.f - (float)std::pow((double)beta1, (double)n->adamSteps);
    a.c2 = 1.f - (float)std::pow((double)beta2, (double)n->adamSteps);
    a.apply = 1;
    k_mlp_update<<<(kNParams + 1 + 255) / 256, 256, 0, n->stream>>>(
        n->part, tiles, nullptr, n->params, n->m, n->v, n->wImg, n->wtImg, n->loss, a);
    NCK(cudaGetLastError());
    if (lossHost)
    {
        rc = checkErr(n);
        if (rc) return rc;
        NCK(cudaMemcpy(lossHost, n->loss, sizeof(float), cudaMemcpyDeviceToHost));
    }
    return ALEBGK_OK;
}

int alebgk_net_sync(alebgk_net *n)
{
    if (!n) return ALEBGK_EINVAL;
    NCK(cudaSetDevice(n->device));
    return checkErr(n);
}

}  // extern "C"
