// body_noalloc.cu -- rigid-body surface loads without any device allocation.
//
// Same quantity as alebgk_body_loads (computeBodyLoads,
// RigidBody/BodyDynamics.cpp:17-97): per body the force and torque of the
// surface stress -(P . n) dA summed over the body's wall particles.  The
// allocating entry point stages the body geometry in a cudaMalloc'd buffer and
// frees it after every call; cudaFree synchronises the whole device, so a
// caller that advances several cavities on separate streams of one device
// would stall all of them on every load query, and a caller that has reserved
// the device memory for its own pools may see the allocation fail mid-run.
// This variant allocates nothing: the body geometry travels as a by-value
// kernel argument, and the per-block partial sums and the result live in one
// file-scope device array of fixed size.
//
// The scratch is one per device and shared by every context on that device:
// calls that overlap in time on the same device race on it and must be
// serialised by the caller.  Every call overwrites all of the scratch it reads
// (each block writes all of its partial sums, zeros included), so nothing has
// to start at zero.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "ctx.h"

namespace alebgk {

namespace {

constexpr int kNoAllocBlocks = 148;       // one partial-sum block per SM
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxDevices = 64;
constexpr int kPartialDoubles = kNoAllocBlocks * kNoAllocMaxBodies * 6;
constexpr int kScratchDoubles = kPartialDoubles + kNoAllocMaxBodies * 6;

// [block][body][6] partial sums, then [body][6] totals: 114,432 bytes.
static __device__ __align__(256) double g_bodyScratch[kScratchDoubles];

struct BodyGeom
{
    double centre[kNoAllocMaxBodies][3];
    double area[kNoAllocMaxBodies];
};

std::mutex g_setupMutex;
double *g_scratchPtr[kNoAllocMaxDevices] = {};
unsigned long long g_scratchCtx[kNoAllocMaxDevices] = {};   // context id of that address

// Unique id of the device's current context (cuCtxGetId), or 0 where the
// driver does not offer it.  A device reset destroys the context that an
// address was looked up in; the next context has a new id.
unsigned long long currentContextId()
{
    typedef CUresult (*GetCurrentFn)(CUcontext *);
    typedef CUresult (*GetIdFn)(CUcontext, unsigned long long *);
    static GetCurrentFn getCurrent = nullptr;
    static GetIdFn getId = nullptr;
    static bool looked = false;
    if (!looked)
    {
        looked = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            getCurrent = reinterpret_cast<GetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            getId = reinterpret_cast<GetIdFn>(p);
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (getCurrent && getId && getCurrent(&ctx) == CUDA_SUCCESS && ctx &&
        getId(ctx, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}

__device__ __forceinline__ double warpSum6(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-order block sum of six values; thread 0 receives the totals.
__device__ __forceinline__ void blockSum6(double (&v)[6], double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 6; ++q) v[q] = warpSum6(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q) sh[q * 32 + wid] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 6; ++q)
        {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[q * 32 + w];
            v[q] = s;
        }
    __syncthreads();
}

// Block b takes particles b, b + gridDim.x, ... in order and sums their
// contributions per body; it then writes its sums for every body.
template <typename T>
__global__ void __launch_bounds__(kNoAllocThreads)
k_body_partial(const T *__restrict__ g, StepParams p, const int *__restrict__ bodyId,
               const int *__restrict__ boundary, const double *__restrict__ pos,
               const double *__restrict__ wall, BodyGeom geom, int nbodies,
               const StepScalars *__restrict__ sc, double *__restrict__ partial)
{
    __shared__ double acc[kNoAllocMaxBodies * 6];
    __shared__ double sh[6 * 32];
    for (int t = threadIdx.x; t < kNoAllocMaxBodies * 6; t += blockDim.x) acc[t] = 0.0;
    __syncthreads();
    const double scale = sc->scale;
    for (int i = blockIdx.x; i < p.N; i += gridDim.x)
    {
        const int b = bodyId[i];
        if (!boundary[i] || b < 0) continue;          // uniform over the block
        const T *gr = g + (size_t)i * p.ldf;
        const double *w = wall + 7 * (size_t)i;
        double v[6] = {0, 0, 0, 0, 0, 0};
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            const int iv = k % p.Nv, jv = (k / p.Nv) % p.Nv;
            const int kv = (p.dim == 3) ? k / (p.Nv * p.Nv) : 0;
            const double vx = fma((double)iv, p.dv, p.vmin);
            const double vy = fma((double)jv, p.dv, p.vmin);
            const double vz = (p.dim == 3) ? fma((double)kv, p.dv, p.vmin) : 0.0;
            const double cx = vx - w[3], cy = vy - w[4], cz = vz - w[5];
            const double f = (double)gr[k] * scale * p.dvN;
            v[0] += f * cx * cx; v[1] += f * cy * cy; v[2] += f * cz * cz;
            v[3] += f * cx * cy; v[4] += f * cx * cz; v[5] += f * cy * cz;
        }
        blockSum6(v, sh);
        if (threadIdx.x == 0)
        {
            const double a = geom.area[b];
            const double cdx = pos[3 * i] - geom.centre[b][0];
            const double cdy = pos[3 * i + 1] - geom.centre[b][1];
            const double cdz = pos[3 * i + 2] - geom.centre[b][2];
            double o[6];
            if (p.dim == 3)
            {
                const double tx = -(w[0] * v[0] + w[1] * v[3] + w[2] * v[4]);
                const double ty = -(w[0] * v[3] + w[1] * v[1] + w[2] * v[5]);
                const double tz = -(w[0] * v[4] + w[1] * v[5] + w[2] * v[2]);
                o[0] = a * tx; o[1] = a * ty; o[2] = a * tz;
                o[3] = a * (cdy * tz - cdz * ty);
                o[4] = a * (cdz * tx - cdx * tz);
                o[5] = a * (cdx * ty - cdy * tx);
            }
            else
            {
                const double valX = -w[0] * v[0] - w[1] * v[3];
                const double valY = -w[0] * v[3] - w[1] * v[1];
                o[0] = a * valX; o[1] = a * valY; o[2] = 0.0;
                o[3] = 0.0; o[4] = 0.0; o[5] = a * (cdx * valY - cdy * valX);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[6 * b + q] += o[q];
        }
    }
    __syncthreads();
    double *dst = partial + (size_t)blockIdx.x * kNoAllocMaxBodies * 6;
    for (int t = threadIdx.x; t < nbodies * 6; t += blockDim.x) dst[t] = acc[t];
}

// One thread per (body, component): the block partials summed in block order.
__global__ void k_body_total(const double *__restrict__ partial, int nbodies,
                             double *__restrict__ out)
{
    const int t = threadIdx.x;
    if (t >= nbodies * 6) return;
    double s = 0.0;
    for (int b = 0; b < kNoAllocBlocks; ++b) s += partial[(size_t)b * kNoAllocMaxBodies * 6 + t];
    out[t] = s;
}

// Device address of this device's scratch, looked up with that device
// current the first time a context of the device calls (and again after a
// device reset has replaced the context).  Not to be first called inside a
// stream capture.
cudaError_t scratchFor(int device, double **ptr)
{
    if (device < 0 || device >= kNoAllocMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setupMutex);
    const unsigned long long ctxId = currentContextId();
    if (!g_scratchPtr[device] || g_scratchCtx[device] != ctxId)
    {
        double *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void **)&p, g_bodyScratch);
        if (e != cudaSuccess) return e;
        g_scratchPtr[device] = p;
        g_scratchCtx[device] = ctxId;
    }
    *ptr = g_scratchPtr[device];
    return cudaSuccess;
}

template <typename T>
cudaError_t launchT(alebgk_ctx *c, int nbodies, const BodyGeom &geom, double *scratch)
{
    const StepParams &p = c->sp;
    k_body_partial<T><<<kNoAllocBlocks, kNoAllocThreads, 0, c->stream>>>(
        static_cast<const T *>(c->d.f[c->cur]), p, c->d.bodyId, c->d.boundary, c->d.pos,
        c->d.wall, geom, nbodies, c->d.sc, scratch);
    k_body_total<<<1, kNoAllocMaxBodies * 6, 0, c->stream>>>(scratch, nbodies,
                                                            scratch + kPartialDoubles);
    return cudaGetLastError();
}

}  // namespace

cudaError_t bodyLoadsNoAlloc(alebgk_ctx *c, int nbodies, const double *centre,
                             const double *area, double *out, std::string *err)
{
    if (nbodies < 1 || nbodies > kNoAllocMaxBodies)
    {
        if (err)
            *err = "body loads without allocation take 1.." +
                   std::to_string(kNoAllocMaxBodies) + " bodies, got " +
                   std::to_string(nbodies);
        return cudaErrorInvalidValue;
    }
    double *scratch = nullptr;
    cudaError_t e = scratchFor(c->cfg.device, &scratch);
    if (e != cudaSuccess)
    {
        if (err) *err = std::string("scratch lookup: ") + cudaGetErrorString(e);
        return e;
    }
    BodyGeom geom{};
    for (int b = 0; b < nbodies; ++b)
    {
        for (int d = 0; d < 3; ++d) geom.centre[b][d] = centre[3 * b + d];
        geom.area[b] = area[b];
    }
    e = (c->cfg.precision == 64) ? launchT<double>(c, nbodies, geom, scratch)
                                 : launchT<float>(c, nbodies, geom, scratch);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, scratch + kPartialDoubles, 48 * (size_t)nbodies,
                            cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess && err) *err = std::string("body loads: ") + cudaGetErrorString(e);
    return e;
}

}  // namespace alebgk
