// march.cu -- lattice-marching MLS transport for sm_100a (FP32).
//
// gt(x,y,z;k) = scale * sum_o C[class][o][k] * h(x+o;k) over the 81 lattice
// offsets |o|^2 <= 6, for a cloud that is a complete lattice (march.h).
//
// CTA = one work unit (an 8x4 tile of lattice columns, output planes
// [za, zb)) x one chunk of 32 VPL velocities; lane l holds the VPL adjacent
// velocities k0 + VPL l .. k0 + VPL l + VPL - 1 (VPL = 2: a float2 per lane,
// and every stencil FMA is one packed fma.rn.f32x2 on two velocities, which
// halves the FMA and shared-memory load instructions per update).  The
// chunks of a unit are consecutive CTAs.  The CTA marches through z: every
// input plane of the tile plus a two-column halo (12x8 particles x 32 VPL
// velocities) is brought into a six-slot shared-memory ring by one TMA
// tensor load (cp.async.bulk.tensor.4d, completion on an mbarrier; zero fill
// outside the lattice).  Each warp owns one class-uniform 2x2 block of
// columns; its 81 coefficients for its lane's velocities stay in registers
// for the whole march, and every staged value feeds the FMAs of up to four
// columns and five output planes, held in a 4 x 5 register queue.  An output
// plane is complete two input planes after its own and is stored straight
// from the queue; planes outside the lattice are zero and are skipped.  Long
// segments run every queue slot without tests; short ones (the single-plane
// wall layers) only the slots of their own output planes.  The last warp to
// release a ring slot refills it at once (a shared-memory count per slot),
// so no warp ever waits for the others to free a slot and the loads run as
// far ahead as the ring allows.  Every wait is bounded; a timeout sets the
// step's error word instead of hanging.  Packed and scalar FMAs round alike (each half of
// fma.rn.f32x2 is one fmaf), so both widths give the same bits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <utility>

#include "ctx.h"
#include "march.h"
#include "mbar.cuh"

namespace alebgk {

namespace {

constexpr int kPW = kMarchTileX + 4;      // staged plane: 12 x 8 particles
constexpr int kPH = kMarchTileY + 4;
constexpr int kRing = 6;                  // staged planes
// Bytes of one staged plane at VPL velocities per lane.
template <int VPL>
__host__ __device__ constexpr uint32_t planeBytes() { return kPW * kPH * kMarchChunk * VPL * 4; }


__host__ __device__ constexpr int tidx(int dx, int dy, int dz)
{
    int n = 0;
    for (int z = -2; z <= 2; ++z)
        for (int y = -2; y <= 2; ++y)
            for (int x = -2; x <= 2; ++x)
            {
                if (x * x + y * y + z * z > 6) continue;
                if (x == dx && y == dy && z == dz) return n;
                ++n;
            }
    return -1;
}
static_assert(tidx(2, 1, 1) >= 0 && tidx(2, 2, 0) < 0, "template");

template <int... I, typename F>
__device__ __forceinline__ void unrollImpl(std::integer_sequence<int, I...>, F &&f)
{
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void unroll(F &&f)
{
    unrollImpl(std::make_integer_sequence<int, N>{}, f);
}

// VPL velocities of one lane: a float, or a float2 updated by packed
// fma.rn.f32x2 / mul.rn.f32x2 (sm_100a).
template <int VPL> struct Lanes;
template <> struct Lanes<1>
{
    typedef float T;
    static __device__ __forceinline__ T zero() { return 0.0f; }
    static __device__ __forceinline__ T fma(T a, T b, T c) { return fmaf(a, b, c); }
    static __device__ __forceinline__ T mul(T a, float s) { return a * s; }
};
template <> struct Lanes<2>
{
    typedef float2 T;
    static __device__ __forceinline__ T zero() { return make_float2(0.0f, 0.0f); }
    static __device__ __forceinline__ T fma(T a, T b, T c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ T mul(T a, float s)
    {
        return __fmul2_rn(a, make_float2(s, s));
    }
};

__device__ __forceinline__ void tmaLoadPlane(void *dst, const CUtensorMap *map, uint64_t *bar,
                                             int c0, int c1, int c2, int c3)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smemAddr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
        "r"(smemAddr(bar))
        : "memory");
}

}  // namespace

template <int VPL>
__global__ void __launch_bounds__(kMarchWarps * 32, 3 - VPL)
k_march(const __grid_constant__ CUtensorMap tmapZ, const __grid_constant__ CUtensorMap tmapY,
        const MarchUnit *__restrict__ units, const float *__restrict__ coefTz,
        const float *__restrict__ coefTy, float *__restrict__ out, int ldf, int Nx, int Ny,
        int Nz, int V, int Vpad, StepScalars *sc)
{
    typedef Lanes<VPL> LN;
    typedef typename LN::T VT;
    constexpr int CW = kMarchChunk * VPL;        // velocities per CTA
    constexpr uint32_t kPlaneBytes = planeBytes<VPL>();
    extern __shared__ __align__(128) unsigned char marchSmem[];
    typedef VT Plane[kPH][kPW][kMarchChunk];
    Plane *ring = reinterpret_cast<Plane *>(marchSmem);
    __shared__ __align__(8) uint64_t full[kRing];
    __shared__ int relCnt[kRing];
    __shared__ int giveUp;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // blockIdx.x = velocity chunk, blockIdx.y = unit: the chunks of one unit
    // run back to back and read the same rows of f while they are in L2.
    const MarchUnit &u = units[blockIdx.y];
    const int ux0 = u.x0, uy0 = u.y0, za = u.za, zb = u.zb;
    // Orientation: z-march tiles are (x, y) at one z; y-march tiles (x, z)
    // at one y, with the coefficients in that frame.
    const bool yMarch = u.yMarch != 0;
    const CUtensorMap *tmap = yMarch ? &tmapY : &tmapZ;
    const float *coefT = yMarch ? coefTy : coefTz;
    const int colStride = ldf;
    const int rowStride = yMarch ? ldf * Nx * Ny : ldf * Nx;
    const int planeStride = yMarch ? ldf * Nx : ldf * Nx * Ny;
    const int marchLen = yMarch ? Ny : Nz;
    const int k0 = blockIdx.x * CW;
    const int k = k0 + VPL * lane;               // the lane's first velocity
    const int nin = zb - za + 4;                 // input planes za-2 .. zb+1
    // Planes outside the lattice hold zeros: they are not staged; the queue
    // only moves past them.  Staged plane m is lattice plane zlo + m.
    const int zlo = max(za - 2, 0), zhi = min(zb + 1, marchLen - 1);
    const int nv = zhi - zlo + 1;
    const int moff = zlo - (za - 2);            // staged index m = n - moff
    const bool active = warp < u.nsub;
    const int sub = active ? __ldg(&u.sub[warp]) : 0;
    const int bx = sub & 15, by = (sub >> 4) & 15, mask = (sub >> 8) & 15;
    const int shape = (sub >> 12) & 3, cls = sub >> 14;
    if (threadIdx.x == 0)
    {
        // An earlier CTA that timed out set the error word: skip the work.
        // Read once and shared, so that every thread of the CTA agrees.
        giveUp = *(volatile int *)&sc->err;
        for (int s = 0; s < kRing; ++s)
        {
            mbarInit(&full[s], 1);
            relCnt[s] = 0;
        }
        mbarInitFence();
    }
    __syncthreads();
    if (giveUp) return;
    // Plane z of the march: (x, y) tile rows at lattice z, or in the y-march
    // frame (x, lattice z) rows at lattice y (a box one y deep, eight z).
    auto loadPlane = [&](void *dst, uint64_t *bar, int z) {
        if (yMarch)
            tmaLoadPlane(dst, tmap, bar, k0, ux0 - 2, z, uy0 - 2);
        else
            tmaLoadPlane(dst, tmap, bar, k0, ux0 - 2, uy0 - 2, z);
    };
    if (threadIdx.x == 0)
        for (int m = 0; m < kRing && m < nv; ++m)
        {
            mbarExpectTx(&full[m], kPlaneBytes);
            loadPlane(&ring[m][0][0][0], &full[m], zlo + m);
        }

    // The table is [class][81][Vpad] with Vpad a multiple of CW, so the
    // lane's VPL coefficients of one offset are adjacent and aligned.
    VT coef[kTmplOffsets];
    if (active)
    {
        const VT *cb = reinterpret_cast<const VT *>(coefT + (size_t)cls * kTmplOffsets * Vpad + k);
#pragma unroll
        for (int o = 0; o < kTmplOffsets; ++o) coef[o] = __ldg(cb + (size_t)o * (Vpad / VPL));
    }
    VT acc[4][5];
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 5; ++r) acc[c][r] = LN::zero();
    const float scale = (float)sc->scale;
    // Output column c of the warp's block at plane z:
    // outBase + z planeStride + (c & 1) colStride + (c >> 1) rowStride.
    // With VPL = 2 and an odd V the last pair of a row may end one past V:
    // that float lies in the row padding (ldf rounds V up to a multiple of
    // four), which nothing reads.
    float *outBase = out + (long long)(ux0 + bx) * colStride + (long long)(uy0 + by) * rowStride + k;
    const int smask = (k < V) ? mask : 0;
    bool dead = false;

    // The FMAs of one staged plane into the queue for a warp block of shape
    // SHAPE (column c at (CX(c), CY(c)) from the block origin); with
    // `gated`, only the slots holding the unit's own output planes.
    auto fmaPlane = [&](auto SHAPE, const VT *P, auto GATED, auto inSeg) {
        constexpr int shp = decltype(SHAPE)::value;
        constexpr bool gated = decltype(GATED)::value;
        constexpr auto CX = [](int c) { return shp == kShapeBlock ? (c & 1)
                                               : shp == kShapeColumn ? 0 : c; };
        constexpr auto CY = [](int c) { return shp == kShapeBlock ? (c >> 1)
                                               : shp == kShapeColumn ? c : 0; };
        constexpr int EX = (shp == kShapeRow) ? 8 : (shp == kShapeBlock ? 6 : 5);
        constexpr int EY = (shp == kShapeColumn) ? 8 : (shp == kShapeBlock ? 6 : 5);
        // Outer loop along the block's long side, so that one short line of
        // the neighbourhood (at most six values) is live at a time.
        constexpr bool xMajor = (shp == kShapeRow);
        constexpr int EA = xMajor ? EX : EY, EB = xMajor ? EY : EX;
        unroll<EA>([&](auto A) {
            VT v[EB];
            unroll<EB>([&](auto B) {
                constexpr int dx = (xMajor ? decltype(A)::value : decltype(B)::value) - 2;
                constexpr int dy = (xMajor ? decltype(B)::value : decltype(A)::value) - 2;
                constexpr bool need = tidx(dx - CX(0), dy - CY(0), 0) >= 0 ||
                                      tidx(dx - CX(1), dy - CY(1), 0) >= 0 ||
                                      tidx(dx - CX(2), dy - CY(2), 0) >= 0 ||
                                      tidx(dx - CX(3), dy - CY(3), 0) >= 0;
                if constexpr (need)
                    v[decltype(B)::value] =
                        P[((by + dy + 2) * kPW + (bx + dx + 2)) * kMarchChunk + lane];
            });
            // Value-major: each staged value feeds the queue slots and
            // columns it reaches (up to 20 independent accumulators) before
            // the next value, so FMAs into one accumulator are far apart.
            unroll<EB>([&](auto B) {
                constexpr int dx = (xMajor ? decltype(A)::value : decltype(B)::value) - 2;
                constexpr int dy = (xMajor ? decltype(B)::value : decltype(A)::value) - 2;
                unroll<5>([&](auto R) {
                    constexpr int r = decltype(R)::value;
                    constexpr int dz = 2 - r;
                    if (!gated || inSeg(r))
                    {
                        unroll<4>([&](auto C) {
                            constexpr int c = decltype(C)::value;
                            constexpr int o = tidx(dx - CX(c), dy - CY(c), dz);
                            if constexpr (o >= 0)
                                acc[c][r] = LN::fma(coef[o], v[decltype(B)::value], acc[c][r]);
                        });
                    }
                });
            });
        });
    };
    // Queue slot 0 (output plane zi - 2) is complete: store it, shift.
    auto storeShift = [&](auto SHAPE, float *o, bool store) {
        constexpr int shp = decltype(SHAPE)::value;
        if (store)
        {
            const int s1 = (shp == kShapeColumn) ? rowStride : colStride;
            const int s2 = (shp == kShapeBlock) ? rowStride : 2 * s1;
            const int s3 = (shp == kShapeBlock) ? rowStride + colStride : 3 * s1;
            if (smask & 1) *reinterpret_cast<VT *>(o) = LN::mul(acc[0][0], scale);
            if (smask & 2) *reinterpret_cast<VT *>(o + s1) = LN::mul(acc[1][0], scale);
            if (smask & 4) *reinterpret_cast<VT *>(o + s2) = LN::mul(acc[2][0], scale);
            if (smask & 8) *reinterpret_cast<VT *>(o + s3) = LN::mul(acc[3][0], scale);
        }
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[c][r] = acc[c][r + 1];
            acc[c][4] = LN::zero();
        }
    };
    // Consumer release of staged plane m in ring slot s: the last warp to
    // release the slot refills it at once with plane m + kRing.
    auto release = [&](int m, int s, uint32_t par) {
        __syncwarp();
        if (lane == 0)
        {
            __threadfence_block();
            const int prev = atomicAdd(&relCnt[s], 1);
            if (prev == kMarchWarps - 1)
            {
                __threadfence_block();
                relCnt[s] = 0;
                if (m + kRing < nv)
                {
                    fenceProxyAsync();
                    mbarExpectTx(&full[s], kPlaneBytes);
                    loadPlane(&ring[s][0][0][0], &full[s], zlo + m + kRing);
                }
            }
        }
        (void)par;
    };

    // Long segment: every input plane is staged (the TMA zero-fills any
    // outside the lattice) and every queue slot takes FMAs; a slot outside
    // the segment is never stored and leaves as zero shifts in.
    auto marchLong = [&](auto SHAPE) {
        int s = 0;
        uint32_t par = 0;
        float *o = outBase + (long long)(za - 4) * planeStride;   // plane zi - 2 at n = 0
        for (int n = 0; n < nin; ++n)
        {
            mbarWait(&full[s], par, dead);
            if (active)
            {
                fmaPlane(SHAPE, &ring[s][0][0][0], std::false_type{}, [](int) { return true; });
                storeShift(SHAPE, o, n >= 4);
            }
            release(n, s, par);
            o += planeStride;
            if (++s == kRing) { s = 0; par ^= 1u; }
        }
    };
    // Short segment: planes outside the lattice are not staged, and only the
    // slots of the unit's own planes take FMAs.
    auto marchShort = [&](auto SHAPE) {
        const unsigned L = (unsigned)(zb - za);
        int s = 0;
        uint32_t par = 0;
        float *o = outBase + (long long)(za - 4) * planeStride;
        for (int n = 0; n < nin; ++n)
        {
            const int m = n - moff;
            auto inSeg = [&](int r) { return (unsigned)(n - 4 + r) < L; };
            if (m >= 0 && m < nv)
            {
                mbarWait(&full[s], par, dead);
                if (active) fmaPlane(SHAPE, &ring[s][0][0][0], std::true_type{}, inSeg);
                release(m, s, par);
                if (++s == kRing) { s = 0; par ^= 1u; }
            }
            if (active) storeShift(SHAPE, o, inSeg(0));
            o += planeStride;
        }
    };
    using ShapeBlock = std::integral_constant<int, kShapeBlock>;
    using ShapeColumn = std::integral_constant<int, kShapeColumn>;
    using ShapeRow = std::integral_constant<int, kShapeRow>;
    if (zb - za > 4)
    {
        if (shape == kShapeColumn) marchLong(ShapeColumn{});
        else if (shape == kShapeRow) marchLong(ShapeRow{});
        else marchLong(ShapeBlock{});
    }
    else
    {
        if (shape == kShapeColumn) marchShort(ShapeColumn{});
        else if (shape == kShapeRow) marchShort(ShapeRow{});
        else marchShort(ShapeBlock{});
    }
    if (dead) atomicOr(&sc->err, 2);
}

// ---------------------------------------------------------------------------
// Host side: tensor map over the distribution (dims: velocity, x, y, z).
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

bool encodeMarchMap(void *tmapOut, void *f, int V, int Nx, int Ny, int Nz, int ldf,
                    bool yMarch, int vpl, std::string *err)
{
    static EncodeTiledFn fn = nullptr;
    if (!fn)
    {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !p)
        {
            if (err) *err = "cuTensorMapEncodeTiled is not available";
            return false;
        }
        fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    const cuuint64_t dims[4] = {(cuuint64_t)V, (cuuint64_t)Nx, (cuuint64_t)Ny, (cuuint64_t)Nz};
    const cuuint64_t strides[3] = {(cuuint64_t)ldf * 4, (cuuint64_t)ldf * 4 * Nx,
                                   (cuuint64_t)ldf * 4 * Nx * Ny};
    // z-march: a 12 x 8 (x, y) tile at one z; y-march: a 12 x 8 (x, z) tile
    // at one y.  Both land in shared memory as [8][12][32 vpl velocities].
    const cuuint32_t cw = (cuuint32_t)(kMarchChunk * vpl);
    const cuuint32_t boxZ[4] = {cw, kPW, kPH, 1};
    const cuuint32_t boxY[4] = {cw, kPW, 1, kPH};
    const cuuint32_t *box = yMarch ? boxY : boxZ;
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(reinterpret_cast<CUtensorMap *>(tmapOut), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                    f, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
    {
        if (err) *err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
        return false;
    }
    return true;
}

cudaError_t prepareMarch()
{
    cudaError_t e = cudaFuncSetAttribute(k_march<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kRing * planeBytes<1>()));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_march<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(kRing * planeBytes<2>()));
    return e;
}

cudaError_t launchMarch(alebgk_ctx *c, int from, float *outBuf, cudaStream_t st)
{
    const StepParams &p = c->sp;
    const MarchState &ms = c->march;
    const CUtensorMap *tz = reinterpret_cast<const CUtensorMap *>(ms.tmap[from]);
    const CUtensorMap *ty = reinterpret_cast<const CUtensorMap *>(ms.nunitsY ? ms.tmapY[from]
                                                                              : ms.tmap[from]);
    const float *cy = ms.coefTy ? ms.coefTy : ms.coefT;
    if (ms.vpl == 2)
        k_march<2><<<dim3(ms.Vpad / (2 * kMarchChunk), ms.nunits), kMarchWarps * 32,
                     kRing * planeBytes<2>(), st>>>(*tz, *ty, ms.units, ms.coefT, cy, outBuf,
                                                    p.ldf, ms.Nx, ms.Ny, ms.Nz, p.V, ms.Vpad,
                                                    c->d.sc);
    else
        k_march<1><<<dim3(ms.Vpad / kMarchChunk, ms.nunits), kMarchWarps * 32,
                     kRing * planeBytes<1>(), st>>>(*tz, *ty, ms.units, ms.coefT, cy, outBuf,
                                                    p.ldf, ms.Nx, ms.Ny, ms.Nz, p.V, ms.Vpad,
                                                    c->d.sc);
    return cudaGetLastError();
}

}  // namespace alebgk
