// api.cpp -- the C-ABI of include/alebgk.h: contexts, upload/download,
// coefficient build, CUDA-graph step, body loads, host case set-up.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cases.h"
#include "coeffs.h"
#include "ctx.h"
#include "march.h"

using namespace alebgk;

namespace {

std::string gCreateError;
int gCoeffBuilder = 0;   // 0: classes and tables on the device where possible, 1: host,
                         // 2: host classes with device tables (the hash-collision path)

int fail(alebgk_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg; else gCreateError = msg;
    return code;
}

#define CK(call)                                                              \
    do {                                                                      \
        cudaError_t e_ = (call);                                              \
        if (e_ != cudaSuccess)                                                \
            return fail(c, ALEBGK_ECUDA, std::string(#call) + ": " +          \
                                              cudaGetErrorString(e_));        \
    } while (0)

template <typename P>
cudaError_t dalloc(P **p, size_t n)
{
    return cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(P));
}

// The row kernel visits the interior particles first, then the wall
// particles (each in index order), so that the warps of an SM run the same
// code at the same time: the wall rows' diffuse-wall code and the interior
// rows' collision code then do not evict each other from the instruction
// cache.  Rows are independent; the order changes no result.
cudaError_t putRowOrder(alebgk_ctx *c, const int *boundary, int N)
{
    std::vector<int> order;
    order.reserve(N);
    for (int pass = 0; pass < 2; ++pass)
        for (int i = 0; i < N; ++i)
            if ((boundary[i] != 0) == (pass == 1)) order.push_back(i);
    return cudaMemcpy(c->d.rowOrder, order.data(), 4 * (size_t)N, cudaMemcpyHostToDevice);
}

// The neighbour lists of a cloud: counts within 0..ALEBGK_MAX_NEIGH, indices
// of other particles.  Checked on the host's OpenMP threads; the error names
// the first particle that fails, as a serial check would.
int checkNeighbours(alebgk_ctx *c, const alebgk_cloud *cl, int N)
{
    auto bad = [&](int i) -> int {
        if (cl->nnb[i] < 0 || cl->nnb[i] > ALEBGK_MAX_NEIGH) return 1;
        for (int s = 0; s < cl->nnb[i]; ++s)
        {
            const int j = cl->nbr[(size_t)i * ALEBGK_MAX_NEIGH + s];
            if (j < 0 || j >= N || j == i) return 2;
        }
        return 0;
    };
    int first = N;
#pragma omp parallel for schedule(static) reduction(min : first)
    for (int i = 0; i < N; ++i)
        if (i < first && bad(i)) first = i;
    if (first == N) return ALEBGK_OK;
    return fail(c, ALEBGK_EINVAL,
                std::string(bad(first) == 1 ? "neighbour count" : "neighbour index") +
                    " out of range at particle " + std::to_string(first));
}

// Pinned host staging of at least `bytes` bytes, kept for the context's
// life (grown when a larger cloud needs more), and the ring's events.
cudaError_t pinnedStaging(alebgk_ctx *c, size_t bytes)
{
    for (auto &ev : c->pinEv)
        if (!ev)
        {
            const cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    if (c->pinBytes >= bytes) return cudaSuccess;
    if (c->pin)
    {
        const cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) return e;
        cudaFreeHost(c->pin);
        c->pin = nullptr;
        c->pinBytes = 0;
    }
    const cudaError_t e = cudaHostAlloc(&c->pin, bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) c->pinBytes = bytes;
    else c->pin = nullptr;
    return e;
}

void freeBuffers(alebgk_ctx *c)
{
    DeviceBuffers &d = c->d;
    void *ptrs[] = {d.f[0], d.f[1], d.coef, d.coefLin, d.pos, d.meshv, d.wall,
                    d.boundary, d.bodyId, d.cls, d.nslot, d.slots, d.macro[0],
                    d.macro[1], d.mood, d.flag, d.flagList, d.degList, d.massPos, d.massEnd, d.minG, d.nad, d.redPartial,
                    d.dpx, d.bodyTmp, d.bodyOut, d.stage, d.surfList, d.bodyIO, d.rankAll, d.sc,
                    d.rowOrder};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    d = DeviceBuffers();
    if (c->macSnap) { cudaFree(c->macSnap); c->macSnap = nullptr; }
    c->snapSteps = -1;
    c->hostSteps = 0;
    if (c->march.units) cudaFree(c->march.units);
    if (c->march.coefT) cudaFree(c->march.coefT);
    if (c->march.coefTy) cudaFree(c->march.coefTy);
    c->march = MarchState();
    for (auto &g : c->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    c->uploaded = false;
}

}  // namespace

extern "C" {

int alebgk_create(const alebgk_config *cfg, alebgk_ctx **out)
{
    alebgk_ctx *c = nullptr;
    if (!cfg || !out) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    *out = nullptr;
    if (cfg->dim != 2 && cfg->dim != 3)
        return fail(nullptr, ALEBGK_EINVAL, "dim must be 2 or 3");
    if (cfg->N <= 0 || cfg->Nv < 2)
        return fail(nullptr, ALEBGK_EINVAL, "N must be > 0 and Nv >= 2");
    if (cfg->precision != 32 && cfg->precision != 64)
        return fail(nullptr, ALEBGK_EINVAL, "precision must be 32 or 64");
    if (cfg->mls_order != 1 && cfg->mls_order != 2)
        return fail(nullptr, ALEBGK_EINVAL, "mls_order must be 1 or 2");
    if (cfg->limiter != 0 && cfg->limiter != 2)
        return fail(nullptr, ALEBGK_EINVAL, "limiter must be 0 (none) or 2 (MOOD)");
    if (cfg->transport < 0 || cfg->transport > 2)
        return fail(nullptr, ALEBGK_EINVAL, "the transport selector is 0, 1 or 2");
    if (cfg->particle < 0 || cfg->particle > 3)
        return fail(nullptr, ALEBGK_EINVAL, "the particle selector is 0, 1, 2 or 3");
    if (!(cfg->tau > 0) || !(cfg->R > 0) || !(cfg->dv > 0) || !(cfg->radius > 0))
        return fail(nullptr, ALEBGK_EINVAL, "tau, R, dv and radius must be > 0");
    const int gs = (cfg->dim == 3) ? cfg->Nv * cfg->Nv * cfg->Nv : 2 * cfg->Nv * cfg->Nv;
    if ((size_t)gs * (cfg->precision == 64 ? 8 : 4) > 160 * 1024)
        return fail(nullptr, ALEBGK_EINVAL,
                    "a particle's distribution exceeds the 160 KB shared-memory row "
                    "of the particle kernel");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(nullptr, ALEBGK_ECUDA, "no CUDA device available");
    if (cfg->device < 0 || cfg->device >= ndev)
        return fail(nullptr, ALEBGK_EINVAL, "device ordinal out of range");
    c = new (std::nothrow) alebgk_ctx();
    if (!c) return fail(nullptr, ALEBGK_ENOMEM, "host allocation failed");
    c->cfg = *cfg;
    cudaError_t e = cudaSetDevice(cfg->device);
    // The step's stream at the highest priority, the side stream (the NAD
    // ranges beside the transport) at the lowest: the transport's CTAs are
    // placed first, the side work fills the SMs the transport's last wave
    // leaves idle.
    int prLeast = 0, prGreatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prGreatest);
    if (e == cudaSuccess)
        e = cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, prLeast);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evFork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->evJoin, cudaEventDisableTiming);
    if (e != cudaSuccess)
    {
        gCreateError = std::string("stream creation: ") + cudaGetErrorString(e);
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->stream2) cudaStreamDestroy(c->stream2);
        if (c->evFork) cudaEventDestroy(c->evFork);
        delete c;
        return ALEBGK_ECUDA;
    }
    StepParams &p = c->sp;
    p.N = cfg->N; p.dim = cfg->dim; p.Nv = cfg->Nv;
    p.V = (cfg->dim == 3) ? cfg->Nv * cfg->Nv * cfg->Nv : cfg->Nv * cfg->Nv;
    p.L = (cfg->dim == 3) ? 1 : 2;
    p.gs = p.V * p.L;
    const int align = (cfg->precision == 64) ? 2 : 4;   // 16-byte rows
    p.ldf = (p.gs + align - 1) / align * align;
    p.limiter = cfg->limiter; p.tauVar = cfg->tau_variable;
    p.mlsOrder = cfg->mls_order;
    for (int a = 0; a < 3; ++a) { p.periodic[a] = cfg->periodic[a]; p.Lp[a] = cfg->L[a]; }
    p.R = cfg->R; p.tau = cfg->tau; p.dHS = cfg->dHS;
    p.vmin = cfg->vmin; p.dv = cfg->dv;
    p.dvN = (cfg->dim == 3) ? cfg->dv * cfg->dv * cfg->dv : cfg->dv * cfg->dv;
    p.h = cfg->radius;
    p.nadNoise = (cfg->precision == 32) ? 64.0 * 0x1p-24 : 0.0;
    *out = c;
    return ALEBGK_OK;
}

int alebgk_destroy(alebgk_ctx *c)
{
    if (!c) return ALEBGK_OK;
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    freeBuffers(c);
    freeClassScratch(c->clsScratch);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->stream2) cudaStreamDestroy(c->stream2);
    if (c->evFork) cudaEventDestroy(c->evFork);
    if (c->evJoin) cudaEventDestroy(c->evJoin);
    for (auto ev : c->pinEv)
        if (ev) cudaEventDestroy(ev);
    if (c->pin) cudaFreeHost(c->pin);
    delete c;
    return ALEBGK_OK;
}

int alebgk_last_error(const alebgk_ctx *c, char *buf, size_t len)
{
    if (!buf || len == 0) return ALEBGK_EINVAL;
    const std::string &s = c ? c->err : gCreateError;
    size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
    return ALEBGK_OK;
}

// The geometry part of alebgk_upload (tables, march plan, buffers); with
// withState also the state (g and macros) from the cloud.
static int uploadCloud(alebgk_ctx *c, const alebgk_cloud *cl, double dt, bool withState)
{
    if (!c || !cl) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!cl->xyz || !cl->meshv || !cl->wall || !cl->boundary || !cl->body_id ||
        !cl->nnb || !cl->nbr || (withState && (!cl->g || !cl->macro)))
        return fail(c, ALEBGK_EINVAL, "alebgk_upload needs every cloud member");
    if (!(dt > 0)) return fail(c, ALEBGK_EINVAL, "dt must be > 0");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    freeBuffers(c);
    StepParams &p = c->sp;
    p.dt = dt;
    p.lam = dt / p.tau;
    p.c1 = 1.0 / (1.0 + p.lam);
    p.inv3R = 1.0 / (3.0 * p.R);
    const int N = p.N;
    if (const int r = checkNeighbours(c, cl, N)) return r;
    CoeffInput in;
    in.dim = p.dim; in.N = N; in.Nv = p.Nv; in.mlsOrder = p.mlsOrder;
    in.dt = dt; in.h = p.h; in.vmin = p.vmin; in.dv = p.dv;
    for (int a = 0; a < 3; ++a) { in.periodic[a] = p.periodic[a] != 0; in.L[a] = p.Lp[a]; }
    in.xyz = cl->xyz; in.meshv = cl->meshv; in.wall = cl->wall;
    in.boundary = cl->boundary; in.nnb = cl->nnb; in.nbr = cl->nbr;
    in.maxNeigh = ALEBGK_MAX_NEIGH;
    CoeffTables tb, tl;
    std::string err;
    // The tables are solved on the device, except where the lattice march
    // may take the cloud: its plan re-lays the host tables.
    const bool f64cloud = c->cfg.precision == 64;
    bool anyBody = false;
    for (int i = 0; i < N && !anyBody; ++i) anyBody = cl->body_id[i] >= 0;
    const bool devTables =
        (gCoeffBuilder == 0 || gCoeffBuilder == 2) &&
        !(!f64cloud && c->cfg.transport != 1 && !anyBody &&
          marchEligible(cl->xyz, N, p.dim, cl->nnb, cl->nbr, ALEBGK_MAX_NEIGH));
    CoeffInput inLin = in;
    inLin.mlsOrder = 1;
    DeviceBuffers &d = c->d;
    // With tables solved on the device, the geometry goes up first and the
    // stencil classes and slot lists are built there too.
    bool devClasses = false;
    if (devTables)
    {
        int maxnn = 0;
        for (int i = 0; i < N; ++i) maxnn = std::max(maxnn, cl->nnb[i]);
        const size_t slotsN = (size_t)N * (1 + maxnn);
        CK(dalloc(&d.pos, 3 * (size_t)N));
        CK(dalloc(&d.meshv, 3 * (size_t)N));
        CK(dalloc(&d.wall, 7 * (size_t)N));
        CK(dalloc(&d.boundary, N));
        CK(dalloc(&d.bodyId, N));
        CK(dalloc(&d.cls, N));
        CK(dalloc(&d.nslot, N));
        CK(dalloc(&d.slots, slotsN));
        CK(cudaMemcpy(d.pos, cl->xyz, 24 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.meshv, cl->meshv, 24 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.wall, cl->wall, 56 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.boundary, cl->boundary, 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.bodyId, cl->body_id, 4 * (size_t)N, cudaMemcpyHostToDevice));
        bool collision = false;
        if (gCoeffBuilder == 2)
            collision = true;
        else
            CK(buildClassesDevice(in, d.pos, d.meshv, d.wall, d.boundary, d.cls, d.nslot,
                                  d.slots, slotsN, c->clsScratch, tb, collision, c->stream));
        devClasses = !collision;
        // two keys share a hash: the host builder compares every key
        if (collision && !buildClasses(in, tb, &err)) return fail(c, ALEBGK_EINVAL, err);
    }
    else
    {
        if (!buildCoefficients(in, tb, &err)) return fail(c, ALEBGK_EINVAL, err);
        // Linear tables for the MOOD redo (mlsTransportCompute(..., 1, true)),
        // on the same classes and slot order.
        if (p.limiter == 2)
        {
            if (!buildCoefficients(inLin, tl, &err)) return fail(c, ALEBGK_EINVAL, err);
            if (tl.cls != tb.cls || tl.slots != tb.slots || tl.S != tb.S)
                return fail(c, ALEBGK_EINVAL, "linear and quadratic stencil classes differ");
        }
    }
    p.S = tb.S;
    c->ncls = tb.ncls;

    const bool f64 = c->cfg.precision == 64;
    const size_t es = f64 ? 8 : 4;
    const size_t fBytes = (size_t)N * p.ldf * es;
    CK(cudaMalloc(&d.f[0], fBytes));
    CK(cudaMalloc(&d.f[1], fBytes));
    CK(cudaMemsetAsync(d.f[0], 0, fBytes, c->stream));
    CK(cudaMemsetAsync(d.f[1], 0, fBytes, c->stream));
    const size_t ncoef = (size_t)tb.ncls * tb.S * tb.V;
    auto putTable = [&](void **dst, const std::vector<double> &src) -> cudaError_t {
        cudaError_t e = cudaMalloc(dst, std::max<size_t>(ncoef, 1) * es);
        if (e != cudaSuccess || src.empty()) return e;
        if (f64) return cudaMemcpy(*dst, src.data(), ncoef * 8, cudaMemcpyHostToDevice);
        std::vector<float> cf(ncoef);
        const size_t per = (size_t)tb.S * tb.V;
        for (int c = 0; c < tb.ncls; ++c)
            roundCoefFP32(&src[c * per], &cf[c * per], tb.S, tb.V);
        return cudaMemcpy(*dst, cf.data(), ncoef * 4, cudaMemcpyHostToDevice);
    };
    c->coefCap = std::max<size_t>(ncoef, 1);
    c->slotsCap = (size_t)N * tb.S;
    if (devTables)
    {
        CK(cudaMalloc(&d.coef, std::max<size_t>(ncoef, 1) * es));
        CK(cudaMalloc(&d.coefLin, std::max<size_t>(ncoef, 1) * es));
        CK(buildTablesDevice(in, tb, p.mlsOrder, d.coef, f64, tb.degenerate, c->stream));
        std::vector<int> degLin;
        CK(buildTablesDevice(in, tb, p.limiter == 2 ? 1 : p.mlsOrder, d.coefLin, f64, degLin,
                             c->stream));
    }
    else
    {
        CK(putTable(&d.coef, tb.coef));
        CK(putTable(&d.coefLin, p.limiter == 2 ? tl.coef : tb.coef));
    }
    c->degenerateParticles = 0;
    for (int k = 0; k < tb.ncls; ++k)
        if (tb.degenerate[k]) c->degenerateParticles += tb.members[k];
    if (!devTables)
    {
        CK(dalloc(&d.pos, 3 * (size_t)N));
        CK(dalloc(&d.meshv, 3 * (size_t)N));
        CK(dalloc(&d.wall, 7 * (size_t)N));
        CK(dalloc(&d.boundary, N));
        CK(dalloc(&d.bodyId, N));
        CK(dalloc(&d.cls, N));
        CK(dalloc(&d.nslot, N));
        CK(dalloc(&d.slots, (size_t)N * tb.S));
    }
    CK(dalloc(&d.macro[0], 6 * (size_t)N));
    CK(dalloc(&d.macro[1], 6 * (size_t)N));
    CK(dalloc(&d.mood, N));
    CK(dalloc(&d.flag, N));
    CK(dalloc(&d.flagList, N));
    CK(dalloc(&d.degList, N));
    CK(dalloc(&d.massPos, N));
    CK(dalloc(&d.massEnd, N));
    CK(dalloc(&d.minG, N));
    CK(dalloc(&d.nad, 2 * (size_t)N));
    CK(dalloc(&d.redPartial, 256));
    CK(dalloc(&d.dpx, N));
    CK(dalloc(&d.bodyTmp, 6 * (size_t)N));
    CK(dalloc(&d.bodyOut, 64 * 6));
    CK(dalloc(&d.sc, 1));
    CK(dalloc(&d.stage, (size_t)N * p.gs));
    CK(dalloc(&d.rowOrder, N));
    CK(putRowOrder(c, cl->boundary, N));
    c->surfHost.clear();
    for (int i = 0; i < N; ++i)
        if (cl->boundary[i] && cl->body_id[i] >= 0) c->surfHost.push_back(i);
    c->surfCap = std::max<size_t>(c->surfHost.size(), 1);
    CK(dalloc(&d.surfList, c->surfHost.size()));
    CK(dalloc(&d.bodyIO, (size_t)kBodyIOHead + 13 * c->surfHost.size()));
    if (!c->surfHost.empty())
        CK(cudaMemcpy(d.surfList, c->surfHost.data(), 4 * c->surfHost.size(),
                      cudaMemcpyHostToDevice));
    c->geometryDirty = false;
    if (!devTables)
    {
        CK(cudaMemcpy(d.pos, cl->xyz, 24 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.meshv, cl->meshv, 24 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.wall, cl->wall, 56 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.boundary, cl->boundary, 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.bodyId, cl->body_id, 4 * (size_t)N, cudaMemcpyHostToDevice));
    }
    if (!devClasses)
    {
        CK(cudaMemcpy(d.cls, tb.cls.data(), 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.nslot, tb.nslot.data(), 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.slots, tb.slots.data(), 4 * (size_t)N * tb.S, cudaMemcpyHostToDevice));
    }
    CK(cudaMemset(d.dpx, 0, 8 * (size_t)N));
    CK(cudaMemset(d.sc, 0, sizeof(StepScalars)));
    CK(prepareKernels(c));
    if ((c->cfg.particle == 2 || c->cfg.particle == 3) && !c->pStream)
        return fail(c, ALEBGK_EINVAL,
                    "the streamed particle kernel needs a 3-D cloud whose rows fit in "
                    "shared memory");
    // Lattice-marching transport (FP32, complete 3-D lattice; such clouds
    // always take the host tables, which the plan re-lays).
    if (!f64 && c->cfg.transport != 1 && !devTables)
    {
        MarchPlan plan;
        buildMarchPlan(cl->xyz, N, p.dim, cl->nnb, cl->nbr, ALEBGK_MAX_NEIGH, tb,
                       nullptr, plan);
        if (plan.ok)
        {
            MarchState &m = c->march;
            m.vpl = c->tune.marchVpl;
            // one list, the long y-march units first
            std::vector<MarchUnit> all(plan.unitsY);
            all.insert(all.end(), plan.units.begin(), plan.units.end());
            m.nunits = (int)all.size();
            m.nunitsY = (int)plan.unitsY.size();
            m.Vpad = plan.Vpad; m.Nx = plan.Nx; m.Ny = plan.Ny; m.Nz = plan.Nz;
            CK(cudaMalloc(&m.units, sizeof(MarchUnit) * m.nunits));
            CK(cudaMemcpy(m.units, all.data(), sizeof(MarchUnit) * m.nunits,
                          cudaMemcpyHostToDevice));
            CK(cudaMalloc(&m.coefT, plan.coefT.size() * 4));
            CK(cudaMemcpy(m.coefT, plan.coefT.data(), plan.coefT.size() * 4,
                          cudaMemcpyHostToDevice));
            if (m.nunitsY > 0)
            {
                CK(cudaMalloc(&m.coefTy, plan.coefTy.size() * 4));
                CK(cudaMemcpy(m.coefTy, plan.coefTy.data(), plan.coefTy.size() * 4,
                              cudaMemcpyHostToDevice));
            }
            for (int b = 0; b < 2; ++b)
            {
                if (!encodeMarchMap(m.tmap[b], d.f[b], p.V, m.Nx, m.Ny, m.Nz, p.ldf, false,
                                    m.vpl, &err))
                    return fail(c, ALEBGK_ECUDA, err);
                if (m.nunitsY > 0 &&
                    !encodeMarchMap(m.tmapY[b], d.f[b], p.V, m.Nx, m.Ny, m.Nz, p.ldf, true,
                                    m.vpl, &err))
                    return fail(c, ALEBGK_ECUDA, err);
            }
            CK(prepareMarch());
            m.enabled = true;
        }
    }
    if (c->cfg.transport == 2 && !c->march.enabled)
        return fail(c, ALEBGK_EINVAL,
                    "the lattice march needs FP32 and a complete 3-D lattice cloud");
    c->bodyIdHost.assign(cl->body_id, cl->body_id + N);
    c->maxBodyId = -1;
    for (int b : c->bodyIdHost) c->maxBodyId = std::max(c->maxBodyId, b);
    c->boundaryHost.assign(cl->boundary, cl->boundary + N);
    c->cur = 0;
    c->uploaded = true;
    ++c->epoch;
    return withState ? alebgk_upload_state(c, cl->g, cl->macro) : ALEBGK_OK;
}

int alebgk_upload(alebgk_ctx *c, const alebgk_cloud *cl, double dt)
{
    // without g and macros: the geometry only (the state follows separately)
    return uploadCloud(c, cl, dt, !(cl && !cl->g && !cl->macro));
}

int alebgk_set_coeff_builder(int which)
{
    if (which < 0 || which > 2) return ALEBGK_EINVAL;
    gCoeffBuilder = which;
    return ALEBGK_OK;
}

}  // extern "C"

namespace {

// Geometry refresh in place: the distribution, macros, moodCheck flags,
// step scalars and every per-particle buffer stay where they are; the
// geometry arrays, stencil classes and slot lists (built on the device from
// the uploaded geometry) and MLS tables (solved on the device) are written
// over the old ones, and only buffers that must grow are reallocated.  Returns 1 (nothing done) where it does not apply: tables the
// host builds, or a cloud the lattice march takes.
int refreshGeometryInPlace(alebgk_ctx *c, const alebgk_cloud *cl, double dt)
{
    StepParams &p = c->sp;
    const int N = p.N;
    if (gCoeffBuilder == 1 || c->march.enabled) return 1;
    bool anyBody = false;
    for (int i = 0; i < N && !anyBody; ++i) anyBody = cl->body_id[i] >= 0;
    const bool f64 = c->cfg.precision == 64;
    if (!f64 && c->cfg.transport != 1 && !anyBody &&
        marchEligible(cl->xyz, N, p.dim, cl->nnb, cl->nbr, ALEBGK_MAX_NEIGH))
        return 1;
    if (const int r = checkNeighbours(c, cl, N)) return r;
    p.dt = dt;
    p.lam = dt / p.tau;
    p.c1 = 1.0 / (1.0 + p.lam);
    CoeffInput in;
    in.dim = p.dim; in.N = N; in.Nv = p.Nv; in.mlsOrder = p.mlsOrder;
    in.dt = dt; in.h = p.h; in.vmin = p.vmin; in.dv = p.dv;
    for (int a = 0; a < 3; ++a) { in.periodic[a] = p.periodic[a] != 0; in.L[a] = p.Lp[a]; }
    in.xyz = cl->xyz; in.meshv = cl->meshv; in.wall = cl->wall;
    in.boundary = cl->boundary; in.nnb = cl->nnb; in.nbr = cl->nbr;
    in.maxNeigh = ALEBGK_MAX_NEIGH;
    CoeffTables tb;
    std::string err;
    DeviceBuffers &d = c->d;
    const size_t es = f64 ? 8 : 4;
    // What the captured step graphs hold: the step parameters (by value) and
    // the buffers the refresh may reallocate.  When none of them changes,
    // the graphs stay valid and are kept.
    unsigned char spBefore[sizeof(StepParams)];
    std::memcpy(spBefore, &p, sizeof p);
    const void *bufBefore[] = {d.coef, d.coefLin, d.slots, d.surfList, d.bodyIO};
    // Geometry first: the class keys are computed from the device copy.
    CK(cudaMemcpy(d.pos, cl->xyz, 24 * (size_t)N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.meshv, cl->meshv, 24 * (size_t)N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.wall, cl->wall, 56 * (size_t)N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.boundary, cl->boundary, 4 * (size_t)N, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.bodyId, cl->body_id, 4 * (size_t)N, cudaMemcpyHostToDevice));
    int maxnn = 0;
    for (int i = 0; i < N; ++i) maxnn = std::max(maxnn, cl->nnb[i]);
    if ((size_t)N * (1 + maxnn) > c->slotsCap)
    {
        cudaFree(d.slots);
        d.slots = nullptr;
        CK(dalloc(&d.slots, (size_t)N * (1 + maxnn)));
        c->slotsCap = (size_t)N * (1 + maxnn);
    }
    bool collision = gCoeffBuilder == 2;
    if (!collision)
        CK(buildClassesDevice(in, d.pos, d.meshv, d.wall, d.boundary, d.cls, d.nslot, d.slots,
                              c->slotsCap, c->clsScratch, tb, collision, c->stream));
    if (collision)
    {
        // two keys share a hash: the host builder compares every key
        if (!buildClasses(in, tb, &err)) return fail(c, ALEBGK_EINVAL, err);
        CK(cudaMemcpy(d.cls, tb.cls.data(), 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.nslot, tb.nslot.data(), 4 * (size_t)N, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d.slots, tb.slots.data(), 4 * (size_t)N * tb.S, cudaMemcpyHostToDevice));
    }
    const size_t ncoef = std::max<size_t>((size_t)tb.ncls * tb.S * tb.V, 1);
    if (ncoef > c->coefCap)
    {
        cudaFree(d.coef);
        cudaFree(d.coefLin);
        d.coef = d.coefLin = nullptr;
        CK(cudaMalloc(&d.coef, ncoef * es));
        CK(cudaMalloc(&d.coefLin, ncoef * es));
        c->coefCap = ncoef;
    }
    p.S = tb.S;
    c->ncls = tb.ncls;
    CK(buildTablesDevice(in, tb, p.mlsOrder, d.coef, f64, tb.degenerate, c->stream));
    std::vector<int> degLin;
    CK(buildTablesDevice(in, tb, p.limiter == 2 ? 1 : p.mlsOrder, d.coefLin, f64, degLin,
                         c->stream));
    c->degenerateParticles = 0;
    for (int k = 0; k < tb.ncls; ++k)
        if (tb.degenerate[k]) c->degenerateParticles += tb.members[k];
    c->surfHost.clear();
    for (int i = 0; i < N; ++i)
        if (cl->boundary[i] && cl->body_id[i] >= 0) c->surfHost.push_back(i);
    if (c->surfHost.size() > c->surfCap)
    {
        cudaFree(d.surfList);
        cudaFree(d.bodyIO);
        d.surfList = nullptr;
        d.bodyIO = nullptr;
        CK(dalloc(&d.surfList, c->surfHost.size()));
        CK(dalloc(&d.bodyIO, (size_t)kBodyIOHead + 13 * c->surfHost.size()));
        c->surfCap = c->surfHost.size();
    }
    if (!c->surfHost.empty())
        CK(cudaMemcpy(d.surfList, c->surfHost.data(), 4 * c->surfHost.size(),
                      cudaMemcpyHostToDevice));
    CK(putRowOrder(c, cl->boundary, N));
    CK(cudaStreamSynchronize(c->stream));
    // The step graphs hold the slot stride and the table pointers: rebuilt
    // when either changed.
    const void *bufAfter[] = {d.coef, d.coefLin, d.slots, d.surfList, d.bodyIO};
    bool same = std::memcmp(spBefore, &p, sizeof p) == 0;
    for (int k = 0; k < 5 && same; ++k) same = bufBefore[k] == bufAfter[k];
    if (!same)
        for (auto &g : c->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    if (c->macSnap) { cudaFree(c->macSnap); c->macSnap = nullptr; }
    c->snapSteps = -1;
    c->bodyIdHost.assign(cl->body_id, cl->body_id + N);
    c->maxBodyId = -1;
    for (int b : c->bodyIdHost) c->maxBodyId = std::max(c->maxBodyId, b);
    c->boundaryHost.assign(cl->boundary, cl->boundary + N);
    c->geometryDirty = false;
    ++c->epoch;
    return ALEBGK_OK;
}

}  // namespace

extern "C" {

int alebgk_upload_geometry(alebgk_ctx *c, const alebgk_cloud *cl, double dt)
{
    if (!c || !cl) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (!cl->xyz || !cl->meshv || !cl->wall || !cl->boundary || !cl->body_id || !cl->nnb ||
        !cl->nbr)
        return fail(c, ALEBGK_EINVAL, "alebgk_upload_geometry needs the geometry members");
    if (!(dt > 0)) return fail(c, ALEBGK_EINVAL, "dt must be > 0");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    {
        const int r = refreshGeometryInPlace(c, cl, dt);
        if (r != 1) return r;
    }
    const StepParams &p = c->sp;
    const size_t es = (c->cfg.precision == 64) ? 8 : 4;
    const size_t fBytes = (size_t)p.N * p.ldf * es;
    const size_t N = p.N;
    void *tf = nullptr;
    double *tm = nullptr;
    int *tmood = nullptr;
    StepScalars sc{};
    auto freeTemps = [&]() {
        if (tf) cudaFree(tf);
        if (tm) cudaFree(tm);
        if (tmood) cudaFree(tmood);
    };
    cudaError_t e = cudaMalloc(&tf, fBytes);
    if (e == cudaSuccess) e = cudaMalloc(&tm, 48 * N);
    if (e == cudaSuccess) e = cudaMalloc(&tmood, 4 * N);
    if (e == cudaSuccess) e = cudaMemcpy(tf, c->d.f[c->cur], fBytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tm, c->d.macro[c->cur], 48 * N, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(tmood, c->d.mood, 4 * N, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(&sc, c->d.sc, sizeof sc, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
    {
        freeTemps();
        return fail(c, ALEBGK_ECUDA, std::string("geometry upload: ") + cudaGetErrorString(e));
    }
    const long long steps = c->hostSteps;
    int rc = uploadCloud(c, cl, dt, false);
    if (rc)
    {
        freeTemps();
        return rc;
    }
    e = cudaMemcpy(c->d.f[0], tf, fBytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d.macro[0], tm, 48 * N, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d.mood, tmood, 4 * N, cudaMemcpyDeviceToDevice);
    sc.redCount = 0;
    if (e == cudaSuccess) e = cudaMemcpy(c->d.sc, &sc, sizeof sc, cudaMemcpyHostToDevice);
    freeTemps();
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("geometry upload: ") + cudaGetErrorString(e));
    c->hostSteps = steps;
    return ALEBGK_OK;
}

int alebgk_upload_state(alebgk_ctx *c, const double *g, const double *macro)
{
    if (!c || !g || !macro) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    const StepParams &p = c->sp;
    const size_t N = p.N, gs = p.gs, ldf = p.ldf;
    // Staging: the macros (N x 6 doubles), the MOOD flags (N ints), and for
    // FP32 clouds of at least 32 MB of rows a ring of row chunks of about
    // 8 MB.  Smaller clouds copy the FP64 rows and convert on the device, so
    // that a batch of many small contexts pins little host memory.
    const size_t rowBytes = 4 * ldf;
    const bool fp32 = c->cfg.precision != 64 && N * rowBytes >= (size_t(32) << 20);
    const size_t macBytes = 48 * N, moodOff = macBytes, moodBytes = (4 * N + 15) / 16 * 16;
    const size_t chunkRows = std::max<size_t>(1, (size_t(8) << 20) / rowBytes);
    const size_t ringOff = moodOff + moodBytes;
    const size_t need = ringOff + (fp32 ? alebgk_ctx::kPinChunks * chunkRows * rowBytes : 0);
    cudaError_t e = pinnedStaging(c, need);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("state upload staging: ") + cudaGetErrorString(e));
    char *pin = static_cast<char *>(c->pin);
    double *mac = reinterpret_cast<double *>(pin);
    int *mood = reinterpret_cast<int *>(pin + moodOff);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)N; ++i)
    {
        for (int q = 0; q < 6; ++q) mac[6 * i + q] = macro[7 * i + q];
        mood[i] = macro[7 * i + 6] != 0.0;
    }
    e = cudaMemcpyAsync(c->d.macro[c->cur], mac, macBytes, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->d.mood, mood, 4 * N, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && fp32)
    {
        // FP32: the host rounds each value to FP32 (round to nearest, as the
        // device conversion does) into a ring chunk while the copy engine
        // moves the previous chunk, so half the bytes cross the bus and the
        // conversion overlaps the transfer.
        float *ring = reinterpret_cast<float *>(pin + ringOff);
        float *f = static_cast<float *>(c->d.f[c->cur]);
        int slot = 0;
        for (size_t r0 = 0; r0 < N && e == cudaSuccess; r0 += chunkRows)
        {
            const size_t r1 = std::min(N, r0 + chunkRows);
            if (r0 >= alebgk_ctx::kPinChunks * chunkRows) e = cudaEventSynchronize(c->pinEv[slot]);
            if (e != cudaSuccess) break;
            float *dst = ring + (size_t)slot * chunkRows * ldf;
#pragma omp parallel for schedule(static)
            for (long long i = (long long)r0; i < (long long)r1; ++i)
            {
                const double *src = g + (size_t)i * gs;
                float *row = dst + (size_t)(i - r0) * ldf;
                for (size_t k = 0; k < gs; ++k) row[k] = (float)src[k];
                for (size_t k = gs; k < ldf; ++k) row[k] = 0.0f;
            }
            e = cudaMemcpyAsync(f + r0 * ldf, dst, (r1 - r0) * rowBytes, cudaMemcpyHostToDevice,
                                c->stream);
            if (e == cudaSuccess) e = cudaEventRecord(c->pinEv[slot], c->stream);
            slot = (slot + 1) % alebgk_ctx::kPinChunks;
        }
    }
    else if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(c->d.stage, g, N * gs * 8, cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess) e = launchConvertIn(c, c->d.stage, c->cur);
    }
    if (e == cudaSuccess) e = launchMassInit(c);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess)
    {
        cudaStreamSynchronize(c->stream);
        return fail(c, ALEBGK_ECUDA, std::string("state upload: ") + cudaGetErrorString(e));
    }
    return ALEBGK_OK;
}

struct alebgk_rows
{
    int device = 0, n = 0, gs = 0;
    double *rows = nullptr;
};

int alebgk_rows_build(alebgk_ctx *c, int n, const int *a, const int *b, int nfresh,
                      const double *fresh, alebgk_rows **out)
{
    if (!c || !a || !b || !out || n < 1 || nfresh < 0 || (nfresh > 0 && !fresh))
        return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    *out = nullptr;
    const int N = c->sp.N, gs = c->sp.gs;
    for (int j = 0; j < n; ++j)
        if (a[j] >= N || (a[j] < 0 && -1 - a[j] >= nfresh) || b[j] < -1 || b[j] >= N ||
            (a[j] < 0 && b[j] >= 0))
            return fail(c, ALEBGK_EINVAL, "row plan entry out of range");
    CK(cudaSetDevice(c->cfg.device));
    auto *r = new (std::nothrow) alebgk_rows();
    if (!r) return fail(c, ALEBGK_ENOMEM, "host allocation failed");
    r->device = c->cfg.device; r->n = n; r->gs = gs;
    int *da = nullptr, *db = nullptr;
    double *df = nullptr;
    cudaError_t e = cudaMalloc(&r->rows, 8 * (size_t)n * gs);
    if (e == cudaSuccess) e = cudaMalloc(&da, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&db, 4 * (size_t)n);
    if (e == cudaSuccess) e = cudaMalloc(&df, 8 * (size_t)std::max(nfresh, 1) * gs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(da, a, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, b, 4 * (size_t)n, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess && nfresh)
        e = cudaMemcpyAsync(df, fresh, 8 * (size_t)nfresh * gs, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launchRowsBuild(c, n, da, db, df, r->rows);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    for (void *q : {(void *)da, (void *)db, (void *)df})
        if (q) cudaFree(q);
    if (e != cudaSuccess)
    {
        alebgk_rows_free(r);
        return fail(c, ALEBGK_ECUDA, std::string("rows build: ") + cudaGetErrorString(e));
    }
    *out = r;
    return ALEBGK_OK;
}

int alebgk_upload_rows(alebgk_ctx *c, alebgk_rows *r, const double *macro)
{
    if (!c || !r || !macro) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (r->n != c->sp.N || r->gs != c->sp.gs || r->device != c->cfg.device)
        return fail(c, ALEBGK_EINVAL, "the rows do not fit this context (N, gstride or device)");
    CK(cudaSetDevice(c->cfg.device));
    const int N = c->sp.N;
    std::vector<double> mac(6 * (size_t)N);
    std::vector<int> mood(N);
    for (int i = 0; i < N; ++i)
    {
        for (int q = 0; q < 6; ++q) mac[6 * (size_t)i + q] = macro[7 * (size_t)i + q];
        mood[i] = macro[7 * (size_t)i + 6] != 0.0;
    }
    CK(cudaMemcpy(c->d.macro[c->cur], mac.data(), mac.size() * 8, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d.mood, mood.data(), 4 * (size_t)N, cudaMemcpyHostToDevice));
    cudaError_t e = launchConvertIn(c, r->rows, c->cur);
    if (e == cudaSuccess) e = launchMassInit(c);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    alebgk_rows_free(r);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("rows upload: ") + cudaGetErrorString(e));
    return ALEBGK_OK;
}

void alebgk_rows_free(alebgk_rows *r)
{
    if (!r) return;
    if (r->rows)
    {
        cudaSetDevice(r->device);
        cudaFree(r->rows);
    }
    delete r;
}

int alebgk_moments13(alebgk_ctx *c, double *out)
{
    if (!c || !out) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (c->sp.dim != 2) return fail(c, ALEBGK_EINVAL, "13 moments are defined for 2-D clouds");
    CK(cudaSetDevice(c->cfg.device));
    CK(launchMoments13(c, out));
    CK(cudaStreamSynchronize(c->stream));
    return ALEBGK_OK;
}

int alebgk_seed_grad13(alebgk_ctx *c, const float *net, int ldnet, const double *scale,
                       const double *shift)
{
    if (!c || !net || !scale || !shift) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (c->sp.dim != 2) return fail(c, ALEBGK_EINVAL, "the Grad-13 seed is for 2-D clouds");
    if (ldnet < 9) return fail(c, ALEBGK_EINVAL, "ldnet must be >= 9");
    CK(cudaSetDevice(c->cfg.device));
    cudaError_t e = launchSeedGrad13(c, net, ldnet, scale, shift);
    if (e == cudaSuccess) e = launchMassInit(c);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("grad13 seed: ") + cudaGetErrorString(e));
    c->snapSteps = -1;
    return ALEBGK_OK;
}

int alebgk_step(alebgk_ctx *c, int nsteps)
{
    if (!c) return ALEBGK_EINVAL;
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (nsteps < 0) return fail(c, ALEBGK_EINVAL, "nsteps must be >= 0");
    if (c->geometryDirty)
        return fail(c, ALEBGK_ESTATE,
                    "a body step moved the surface particles: upload the cloud again");
    CK(cudaSetDevice(c->cfg.device));
    for (int n = 0; n < nsteps; ++n)
    {
        const int from = c->cur;
        if (!c->graph[from])
        {
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
            cudaError_t le = launchStep(c, from);
            cudaError_t ee = cudaStreamEndCapture(c->stream, &g);
            if (le != cudaSuccess || ee != cudaSuccess)
            {
                if (g) cudaGraphDestroy(g);
                return fail(c, ALEBGK_ECUDA,
                            std::string("step capture: ") +
                                cudaGetErrorString(le != cudaSuccess ? le : ee));
            }
            cudaError_t ie =
                cudaGraphInstantiate(&c->graph[from], g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess)
                return fail(c, ALEBGK_ECUDA, std::string("graph instantiate: ") +
                                                 cudaGetErrorString(ie));
        }
        CK(cudaGraphLaunch(c->graph[from], c->stream));
        c->cur = 1 - from;
        ++c->hostSteps;
    }
    return ALEBGK_OK;
}

int alebgk_sync(alebgk_ctx *c)
{
    if (!c) return ALEBGK_EINVAL;
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    if (c->uploaded)
    {
        StepScalars s;
        CK(cudaMemcpy(&s, c->d.sc, sizeof s, cudaMemcpyDeviceToHost));
        if (s.err) return fail(c, ALEBGK_EDEVICE, "device error word " + std::to_string(s.err));
    }
    return ALEBGK_OK;
}

int alebgk_step_timed(alebgk_ctx *c, int nsteps, float *ms)
{
    if (!c || !ms) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    // Capture the graphs first so that instantiation stays outside the
    // timed region.
    for (int from = 0; from < 2 && nsteps > 0; ++from)
        if (!c->graph[from])
        {
            int r = alebgk_step(c, 1);
            if (r) return r;
        }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, c->stream));
    int r = alebgk_step(c, nsteps);
    CK(cudaEventRecord(e1, c->stream));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return r;
}

int alebgk_profile_steps(alebgk_ctx *c, int nsteps, float *ms)
{
    if (!c || !ms) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    // launch order -> stage index of include/alebgk.h
    static const int stageOf[ALEBGK_NSTAGES] = {9, 0, 1, 2, 3, 4, 5, 6, 7, 8};
    cudaEvent_t ev[ALEBGK_NSTAGES + 1];
    for (auto &e : ev) CK(cudaEventCreate(&e));
    for (int q = 0; q < ALEBGK_NSTAGES; ++q) ms[q] = 0.0f;
    int rc = ALEBGK_OK;
    for (int n = 0; n < nsteps && rc == ALEBGK_OK; ++n)
    {
        cudaError_t e = launchStep(c, c->cur, ev);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[ALEBGK_NSTAGES]);
        if (e != cudaSuccess)
        {
            rc = fail(c, ALEBGK_ECUDA, std::string("profiled step: ") + cudaGetErrorString(e));
            break;
        }
        for (int q = 0; q < ALEBGK_NSTAGES; ++q)
        {
            float t = 0.0f;
            cudaEventElapsedTime(&t, ev[q], ev[q + 1]);
            ms[stageOf[q]] += t;
        }
        c->cur = 1 - c->cur;
    }
    for (auto &e : ev) cudaEventDestroy(e);
    return rc;
}

int alebgk_download_moments(alebgk_ctx *c, double *macro)
{
    if (!c || !macro) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    const size_t N = c->sp.N;
    const size_t macBytes = 48 * N;
    CK(pinnedStaging(c, macBytes + 4 * N));
    double *mac = static_cast<double *>(c->pin);
    int *mood = reinterpret_cast<int *>(static_cast<char *>(c->pin) + macBytes);
    CK(cudaMemcpyAsync(mac, c->d.macro[c->cur], macBytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(mood, c->d.mood, 4 * N, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)N; ++i)
    {
        for (int q = 0; q < 6; ++q) macro[7 * i + q] = mac[6 * i + q];
        macro[7 * i + 6] = mood[i];
    }
    return ALEBGK_OK;
}

int alebgk_download_full(alebgk_ctx *c, double *g, double *macro)
{
    if (!c || !g) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    const StepParams &p = c->sp;
    cudaError_t e = launchConvertOut(c, c->d.stage, c->cur);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(g, c->d.stage, (size_t)p.N * p.gs * 8, cudaMemcpyDeviceToHost,
                            c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("download: ") + cudaGetErrorString(e));
    return macro ? alebgk_download_moments(c, macro) : ALEBGK_OK;
}

int alebgk_get_counters(alebgk_ctx *c, alebgk_counters *out)
{
    if (!c || !out) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    StepScalars s;
    CK(cudaMemcpy(&s, c->d.sc, sizeof s, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->steps = s.steps;
    out->transport_flags = s.nflag;
    out->positivity_fixes = s.nfix;
    out->mood_fail = s.moodfail;
    out->mls_degenerate = c->degenerateParticles;
    out->mass_after_transport = s.massNew;
    out->mass_scale = s.sigma;
    out->mass_end = s.massEnd;
    out->mass_before = s.sigma * s.massNew;
    out->error_word = s.err;
    out->transport_kernel = c->march.enabled ? 2 : 1;
    out->particle_kernel = c->pStream ? (c->pRows ? 3 : 2) : 1;
    return ALEBGK_OK;
}

int alebgk_total_mass(alebgk_ctx *c, double *mass)
{
    if (!c || !mass) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    StepScalars s;
    CK(cudaMemcpy(&s, c->d.sc, sizeof s, cudaMemcpyDeviceToHost));
    *mass = s.massOld;
    return ALEBGK_OK;
}

int alebgk_wall_momentum(alebgk_ctx *c, double *dpx)
{
    if (!c || !dpx) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaMemcpyAsync(dpx, c->d.dpx, 8 * (size_t)c->sp.N, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return ALEBGK_OK;
}

int alebgk_device_state(alebgk_ctx *c, void **f, int *ldf, int *elem_bytes)
{
    if (!c) return ALEBGK_EINVAL;
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (f) *f = c->d.f[c->cur];
    if (ldf) *ldf = c->sp.ldf;
    if (elem_bytes) *elem_bytes = c->cfg.precision == 64 ? 8 : 4;
    return ALEBGK_OK;
}

int alebgk_body_loads(alebgk_ctx *c, int nbodies, const double *centre,
                      const double *area, double *out)
{
    if (!c || !centre || !area || !out) return fail(c, ALEBGK_EINVAL, "null argument");
    if (nbodies <= 0 || nbodies > 64) return fail(c, ALEBGK_EINVAL, "1..64 bodies");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (c->maxBodyId >= nbodies)
        return fail(c, ALEBGK_EINVAL, "a particle's body id exceeds nbodies");
    CK(cudaSetDevice(c->cfg.device));
    double *dc = nullptr;
    CK(cudaMalloc(&dc, 4 * 64 * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(dc, centre, 24 * (size_t)nbodies, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dc + 3 * 64, area, 8 * (size_t)nbodies, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launchBodyLoads(c, nbodies, dc, dc + 3 * 64);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, c->d.bodyOut, 48 * (size_t)nbodies, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dc);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("body loads: ") + cudaGetErrorString(e));
    return ALEBGK_OK;
}

int alebgk_body_loads_noalloc(alebgk_ctx *c, int nbodies, const double *centre,
                              const double *area, double *out)
{
    if (!c || !centre || !area || !out) return fail(c, ALEBGK_EINVAL, "null argument");
    if (nbodies <= 0 || nbodies > ALEBGK_NOALLOC_MAX_BODIES)
        return fail(c, ALEBGK_EINVAL,
                    "body loads without allocation take 1.." +
                        std::to_string(ALEBGK_NOALLOC_MAX_BODIES) + " bodies, got " +
                        std::to_string(nbodies));
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (c->maxBodyId >= nbodies)
        return fail(c, ALEBGK_EINVAL, "a particle's body id exceeds nbodies");
    CK(cudaSetDevice(c->cfg.device));
    std::string err;
    if (alebgk::bodyLoadsNoAlloc(c, nbodies, centre, area, out, &err) != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, err);
    return ALEBGK_OK;
}

int alebgk_body_set_surface_velocity(alebgk_ctx *c, int nbodies,
                                     const double *centre, const double *state)
{
    if (!c || !centre || !state) return fail(c, ALEBGK_EINVAL, "null argument");
    if (nbodies <= 0 || nbodies > 64) return fail(c, ALEBGK_EINVAL, "1..64 bodies");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (c->maxBodyId >= nbodies)
        return fail(c, ALEBGK_EINVAL, "a particle's body id exceeds nbodies");
    CK(cudaSetDevice(c->cfg.device));
    double *dc = nullptr;
    CK(cudaMalloc(&dc, 9 * 64 * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(dc, centre, 24 * (size_t)nbodies, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dc + 3 * 64, state, 48 * (size_t)nbodies, cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) e = launchSetSurfaceVelocity(c, nbodies, dc, dc + 3 * 64);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(dc);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("surface velocity: ") + cudaGetErrorString(e));
    return ALEBGK_OK;
}

int alebgk_body_step(alebgk_ctx *c, int nbodies, alebgk_body *bodies, const double *box,
                     double dx, double dt)
{
    if (!c || !bodies || !box) return fail(c, ALEBGK_EINVAL, "null argument");
    if (nbodies <= 0 || nbodies > kMaxBodyIO) return fail(c, ALEBGK_EINVAL, "1..64 bodies");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    if (!(dt > 0)) return fail(c, ALEBGK_EINVAL, "dt must be > 0");
    for (int b = 0; b < nbodies; ++b)
    {
        const alebgk_body &B = bodies[b];
        if (B.kind < 0 || B.kind > 3 || (B.kind >= 2) != (c->sp.dim == 3))
            return fail(c, ALEBGK_EINVAL, "body kind does not match the cloud's dimension");
        if (!(B.state[19] > 0) || !(B.state[20] > 0))
            return fail(c, ALEBGK_EINVAL, "body mass and moment of inertia must be > 0");
    }
    if (c->maxBodyId >= nbodies)
        return fail(c, ALEBGK_EINVAL, "a particle's body id exceeds nbodies");
    CK(cudaSetDevice(c->cfg.device));
    std::string err;
    const cudaError_t e = bodyStep(c, nbodies, bodies, box, dx, dt, &err);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, "body step: " + err + ": " + cudaGetErrorString(e));
    c->geometryDirty = !c->surfHost.empty();
    return ALEBGK_OK;
}

int alebgk_download_geometry(alebgk_ctx *c, double *xyz, double *meshv, double *wall)
{
    if (!c) return ALEBGK_EINVAL;
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    CK(cudaStreamSynchronize(c->stream));
    const size_t N = c->sp.N;
    if (xyz) CK(cudaMemcpy(xyz, c->d.pos, 24 * N, cudaMemcpyDeviceToHost));
    if (meshv) CK(cudaMemcpy(meshv, c->d.meshv, 24 * N, cudaMemcpyDeviceToHost));
    if (wall) CK(cudaMemcpy(wall, c->d.wall, 56 * N, cudaMemcpyDeviceToHost));
    return ALEBGK_OK;
}

int alebgk_checkpoint_header(const char *path, alebgk_ckpt_header *out)
{
    if (!path || !out) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    std::string err;
    const int rc = checkpointHeader(path, out, &err);
    return rc ? fail(nullptr, rc, err) : ALEBGK_OK;
}

int alebgk_checkpoint_read(const char *path, const alebgk_ckpt_header *expect,
                           alebgk_cloud *cloud, int *voxel, alebgk_body *bodies)
{
    if (!path || !expect || !cloud) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    std::string err;
    const int rc = checkpointRead(path, expect, cloud, voxel, bodies, &err);
    return rc ? fail(nullptr, rc, err) : ALEBGK_OK;
}

int alebgk_checkpoint_save(alebgk_ctx *c, const char *path, int64_t step, double t,
                           const double *vgrid, const int *voxel, int nbodies,
                           const alebgk_body *bodies)
{
    if (!c || !path) return fail(c, ALEBGK_EINVAL, "null argument");
    if (nbodies < 0 || (nbodies > 0 && !bodies))
        return fail(c, ALEBGK_EINVAL, "bodies missing");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    CK(cudaSetDevice(c->cfg.device));
    std::string err;
    const int rc = checkpointSave(c, path, step, t, vgrid, voxel, nbodies, bodies, &err);
    return rc ? fail(c, rc, "checkpoint: " + err) : ALEBGK_OK;
}

// ---------------------------------------------------------------------------
// Host-side coefficient tables
// ---------------------------------------------------------------------------
struct alebgk_coeffs
{
    CoeffTables t;
    int N = 0;
    int degenerateParticles = 0;
};

int alebgk_coeff_build(const alebgk_config *cfg, const alebgk_cloud *cl, double dt,
                       alebgk_coeffs **out)
{
    if (!cfg || !cl || !out || !cl->xyz || !cl->meshv || !cl->wall || !cl->boundary ||
        !cl->nnb || !cl->nbr)
        return fail(nullptr, ALEBGK_EINVAL, "null argument");
    *out = nullptr;
    CoeffInput in;
    in.dim = cfg->dim; in.N = cfg->N; in.Nv = cfg->Nv; in.mlsOrder = cfg->mls_order;
    in.dt = dt; in.h = cfg->radius; in.vmin = cfg->vmin; in.dv = cfg->dv;
    for (int a = 0; a < 3; ++a) { in.periodic[a] = cfg->periodic[a] != 0; in.L[a] = cfg->L[a]; }
    in.xyz = cl->xyz; in.meshv = cl->meshv; in.wall = cl->wall;
    in.boundary = cl->boundary; in.nnb = cl->nnb; in.nbr = cl->nbr;
    in.maxNeigh = ALEBGK_MAX_NEIGH;
    auto *t = new (std::nothrow) alebgk_coeffs();
    if (!t) return fail(nullptr, ALEBGK_ENOMEM, "host allocation failed");
    std::string err;
    if (!buildCoefficients(in, t->t, &err))
    {
        delete t;
        return fail(nullptr, ALEBGK_EINVAL, err);
    }
    t->N = cfg->N;
    for (int k = 0; k < t->t.ncls; ++k)
        if (t->t.degenerate[k]) t->degenerateParticles += t->t.members[k];
    *out = t;
    return ALEBGK_OK;
}

int alebgk_coeff_info(const alebgk_coeffs *t, int *info)
{
    if (!t || !info) return ALEBGK_EINVAL;
    info[0] = t->t.ncls; info[1] = t->t.S; info[2] = t->t.V;
    info[3] = t->degenerateParticles; info[4] = t->N;
    return ALEBGK_OK;
}

int alebgk_coeff_get(const alebgk_coeffs *t, int *cls, int *nslot, int *slots,
                     double *coef)
{
    if (!t) return ALEBGK_EINVAL;
    if (cls) std::memcpy(cls, t->t.cls.data(), t->t.cls.size() * sizeof(int));
    if (nslot) std::memcpy(nslot, t->t.nslot.data(), t->t.nslot.size() * sizeof(int));
    if (slots) std::memcpy(slots, t->t.slots.data(), t->t.slots.size() * sizeof(int));
    if (coef) std::memcpy(coef, t->t.coef.data(), t->t.coef.size() * sizeof(double));
    return ALEBGK_OK;
}

void alebgk_coeff_free(alebgk_coeffs *t) { delete t; }

// ---------------------------------------------------------------------------
// Host case set-up
// ---------------------------------------------------------------------------
struct alebgk_case
{
    Cloud cloud;
};

int alebgk_case_build(const char *name, int Nx, int Nv, double dt, int mls_order,
                      int fixed_body, double body_scale, alebgk_case **out)
{
    if (!name || !out) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    *out = nullptr;
    int id = 0;
    if (!caseByName(name, &id)) return fail(nullptr, ALEBGK_EINVAL, std::string("unknown case ") + name);
    CaseParams prm;
    if (!configureCase(id, Nx, Nv, dt, mls_order, fixed_body != 0, prm))
        return fail(nullptr, ALEBGK_EINVAL, "configureCase failed");
    auto *c = new (std::nothrow) alebgk_case();
    if (!c) return fail(nullptr, ALEBGK_ENOMEM, "host allocation failed");
    std::string err;
    if (!buildCloud(prm, body_scale, c->cloud, &err))
    {
        delete c;
        return fail(nullptr, ALEBGK_EINVAL, err);
    }
    *out = c;
    return ALEBGK_OK;
}

int alebgk_case_build_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                         int fixed_body, double body_scale, double lid_speed, double rho0,
                         double tau, alebgk_case **out)
{
    if (!name || !out) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    *out = nullptr;
    int id = 0;
    if (!caseByName(name, &id)) return fail(nullptr, ALEBGK_EINVAL, std::string("unknown case ") + name);
    CaseParams prm;
    if (!configureCase(id, Nx, Nv, dt, mls_order, fixed_body != 0, prm))
        return fail(nullptr, ALEBGK_EINVAL, "configureCase failed");
    if (lid_speed > 0) prm.lidSpeed = lid_speed;
    if (rho0 > 0) prm.rho0 = rho0;
    if (tau > 0) prm.tau = tau;
    auto *c = new (std::nothrow) alebgk_case();
    if (!c) return fail(nullptr, ALEBGK_ENOMEM, "host allocation failed");
    std::string err;
    if (!buildCloud(prm, body_scale, c->cloud, &err))
    {
        delete c;
        return fail(nullptr, ALEBGK_EINVAL, err);
    }
    *out = c;
    return ALEBGK_OK;
}

void alebgk_case_free(alebgk_case *c) { delete c; }

static void caseInfo(const CaseParams &p, int N, int gStride, int nbodies, int *info,
                     double *prm)
{
    if (info)
    {
        info[0] = N; info[1] = p.dim; info[2] = p.Nv; info[3] = gStride;
        info[4] = nbodies; info[5] = p.mlsOrder; info[6] = p.Nx;
        info[7] = p.movingBodies ? 1 : 0;
    }
    if (prm)
    {
        double v[24] = {p.dt, p.tau, p.R, p.dx, p.dy, p.dz, p.radius, p.minDist,
                        p.dv, p.VMin, p.VMax, p.rho0, p.Tw, p.xleft, p.xright,
                        p.ybottom, p.ytop, p.zfront, p.zback, p.dtRequested,
                        p.tfinal, p.dHS, p.lidSpeed, (double)p.saveEvery};
        std::memcpy(prm, v, sizeof v);
    }
}

int alebgk_case_info(const alebgk_case *cs, int *info, double *prm)
{
    if (!cs) return ALEBGK_EINVAL;
    const Cloud &c = cs->cloud;
    caseInfo(c.prm, c.N, c.gStride, (int)c.bodies.size(), info, prm);
    return ALEBGK_OK;
}

// ---- lattice set-up on the device -------------------------------------------
// The case parameters of a box cavity without bodies, as buildCloud sets
// them, without building the cloud.
static int latticeCase(const char *name, int Nx, int Nv, double dt, int mls_order,
                       int fixed_body, double lid_speed, double rho0, double tau,
                       CaseParams &prm)
{
    if (!name) return fail(nullptr, ALEBGK_EINVAL, "null argument");
    int id = 0;
    if (!caseByName(name, &id))
        return fail(nullptr, ALEBGK_EINVAL, std::string("unknown case ") + name);
    if (!configureCase(id, Nx, Nv, dt, mls_order, fixed_body != 0, prm))
        return fail(nullptr, ALEBGK_EINVAL, "configureCase failed");
    if (prm.Nx < 3 || prm.Nv < 2)
        return fail(nullptr, ALEBGK_EINVAL, "Nx must be >= 3 and Nv >= 2");
    if (lid_speed > 0) prm.lidSpeed = lid_speed;
    if (rho0 > 0) prm.rho0 = rho0;
    if (tau > 0) prm.tau = tau;
    latticeParams(prm);
    clampDt(prm);
    return ALEBGK_OK;
}

static size_t latticeN(const CaseParams &p)
{
    return (size_t)p.Nx * p.Ny * (p.dim == 3 ? p.Nz : 1);
}

namespace {

struct LatticeBuffers
{
    LatticeDev d;
    ~LatticeBuffers()
    {
        for (void *q : {(void *)d.xyz, (void *)d.wall, (void *)d.meshv, (void *)d.boundary,
                        (void *)d.bodyId, (void *)d.voxel, (void *)d.voxCount, (void *)d.voxStart,
                        (void *)d.voxCursor, (void *)d.voxList, (void *)d.nnb, (void *)d.nbr})
            if (q) cudaFree(q);
    }
    cudaError_t alloc(const CaseParams &p, size_t N)
    {
        const size_t nvox = (size_t)p.nbhBox * p.nbvBox * p.nbwBox;
        cudaError_t e = dalloc(&d.xyz, 3 * N);
        if (e == cudaSuccess) e = dalloc(&d.wall, 7 * N);
        if (e == cudaSuccess) e = dalloc(&d.meshv, 3 * N);
        if (e == cudaSuccess) e = dalloc(&d.boundary, N);
        if (e == cudaSuccess) e = dalloc(&d.bodyId, N);
        if (e == cudaSuccess) e = dalloc(&d.voxel, N);
        if (e == cudaSuccess) e = dalloc(&d.voxCount, nvox);
        if (e == cudaSuccess) e = dalloc(&d.voxStart, nvox + 1);
        if (e == cudaSuccess) e = dalloc(&d.voxCursor, nvox);
        if (e == cudaSuccess) e = dalloc(&d.voxList, N);
        if (e == cudaSuccess) e = dalloc(&d.nnb, N);
        if (e == cudaSuccess) e = dalloc(&d.nbr, N * ALEBGK_MAX_NEIGH);
        return e;
    }
};

// Host copies of the device-built geometry, laid out as an alebgk_cloud.
struct LatticeHost
{
    std::vector<double> xyz, wall, meshv;
    std::vector<int> boundary, bodyId, nnb, nbr;
    cudaError_t fetch(const LatticeDev &d, size_t N)
    {
        xyz.resize(3 * N); wall.resize(7 * N); meshv.resize(3 * N);
        boundary.resize(N); bodyId.resize(N); nnb.resize(N);
        nbr.resize(N * ALEBGK_MAX_NEIGH);
        cudaError_t e = cudaMemcpy(xyz.data(), d.xyz, 24 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(wall.data(), d.wall, 56 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(meshv.data(), d.meshv, 24 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(boundary.data(), d.boundary, 4 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(bodyId.data(), d.bodyId, 4 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(nnb.data(), d.nnb, 4 * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess)
            e = cudaMemcpy(nbr.data(), d.nbr, 4 * N * ALEBGK_MAX_NEIGH, cudaMemcpyDeviceToHost);
        return e;
    }
};

// The whole device set-up of a lattice case into b: the lattice, then (for
// a case with bodies) the bodies embedded on the device, and the neighbour
// lists.  *N = the particle count.
cudaError_t deviceSetup(const CaseParams &p, double bodyScale, LatticeBuffers &b, size_t *N,
                        cudaStream_t st)
{
    const size_t NL = latticeN(p);
    if (!p.hasBody)
    {
        *N = NL;
        cudaError_t e = b.alloc(p, NL);
        return e == cudaSuccess ? buildLatticeDevice(p, b.d, st) : e;
    }
    std::vector<Body> bodies;
    caseBodies(p, bodyScale, bodies);
    std::vector<double> sx, sw;
    std::vector<int> s0;
    bodySurface(p, bodies, sx, sw, s0);
    LatticeBuffers raw;
    cudaError_t e = raw.alloc(p, NL);
    if (e == cudaSuccess) e = buildLatticeDevice(p, raw.d, st, false);
    if (e == cudaSuccess) e = b.alloc(p, NL + sx.size() / 3);
    int n = 0;
    if (e == cudaSuccess) e = embedLatticeDevice(p, bodies, sx, sw, s0, raw.d, (int)NL, b.d, &n, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    *N = (size_t)n;
    return e;
}

// The body descriptor the host API uses (32 doubles, alebgk_case_bodies).
void bodyState(const Body &r, double *o)
{
    double v[22] = {r.cx, r.cy, r.cz, r.velx, r.vely, r.velz, r.angularVel,
                    r.omx, r.omy, r.omz, r.forcex, r.forcey, r.forcez,
                    r.torque, r.tqx, r.tqy, r.tqz, r.ox, r.oy, r.mass,
                    r.inertia(), r.T};
    std::memcpy(o, v, sizeof v);
    for (int k = 0; k < 9; ++k) o[22 + k] = r.Rm[k];
    o[31] = r.surfaceArea();
}

}  // namespace

int alebgk_lattice_info_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                           int fixed_body, double body_scale, double lid_speed, double rho0,
                           double tau, int device, int *info, double *prm)
{
    alebgk_ctx *c = nullptr;
    CaseParams p;
    int rc = latticeCase(name, Nx, Nv, dt, mls_order, fixed_body, lid_speed, rho0, tau, p);
    if (rc) return rc;
    const int gs = (p.dim == 3) ? p.Nv * p.Nv * p.Nv : 2 * p.Nv * p.Nv;
    size_t N = latticeN(p);
    int nb = 0;
    if (p.hasBody)
    {
        // the count after the embedding is known once the device has run it
        std::vector<Body> bodies;
        caseBodies(p, body_scale, bodies);
        nb = (int)bodies.size();
        CK(cudaSetDevice(device));
        LatticeBuffers b;
        CK(deviceSetup(p, body_scale, b, &N, nullptr));
    }
    caseInfo(p, (int)N, gs, nb, info, prm);
    return ALEBGK_OK;
}

int alebgk_lattice_info(const char *name, int Nx, int Nv, double dt, int mls_order,
                        double lid_speed, double rho0, double tau, int *info, double *prm)
{
    return alebgk_lattice_info_ex(name, Nx, Nv, dt, mls_order, 0, 1.0, lid_speed, rho0, tau, 0,
                                  info, prm);
}

int alebgk_lattice_bodies(const char *name, int Nx, int Nv, double dt, int mls_order,
                          int fixed_body, double body_scale, int *nbodies, double *state,
                          int *kind, int *rotates, double *size)
{
    CaseParams p;
    int rc = latticeCase(name, Nx, Nv, dt, mls_order, fixed_body, -1.0, -1.0, -1.0, p);
    if (rc) return rc;
    std::vector<Body> bodies;
    if (p.hasBody) caseBodies(p, body_scale, bodies);
    if (nbodies) *nbodies = (int)bodies.size();
    for (size_t b = 0; b < bodies.size(); ++b)
    {
        if (state) bodyState(bodies[b], state + 32 * b);
        if (kind) kind[b] = bodies[b].kind;
        if (rotates) rotates[b] = bodies[b].rotates ? 1 : 0;
        if (size) size[b] = bodies[b].size;
    }
    return ALEBGK_OK;
}

int alebgk_lattice_build_device_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                                   int fixed_body, double body_scale, double lid_speed,
                                   double rho0, double tau, int device, double *xyz,
                                   double *wall, int *boundary, int *body_id, int *nnb, int *nbr)
{
    alebgk_ctx *c = nullptr;
    CaseParams p;
    int rc = latticeCase(name, Nx, Nv, dt, mls_order, fixed_body, lid_speed, rho0, tau, p);
    if (rc) return rc;
    CK(cudaSetDevice(device));
    LatticeBuffers b;
    size_t N = 0;
    CK(deviceSetup(p, body_scale, b, &N, nullptr));
    CK(cudaDeviceSynchronize());
    LatticeHost h;
    CK(h.fetch(b.d, N));
    if (xyz) std::memcpy(xyz, h.xyz.data(), 24 * N);
    if (wall) std::memcpy(wall, h.wall.data(), 56 * N);
    if (boundary) std::memcpy(boundary, h.boundary.data(), 4 * N);
    if (body_id) std::memcpy(body_id, h.bodyId.data(), 4 * N);
    if (nnb) std::memcpy(nnb, h.nnb.data(), 4 * N);
    if (nbr) std::memcpy(nbr, h.nbr.data(), 4 * N * ALEBGK_MAX_NEIGH);
    return ALEBGK_OK;
}

int alebgk_lattice_build_device(const char *name, int Nx, int Nv, double dt, int mls_order,
                                double lid_speed, double rho0, double tau, int device,
                                double *xyz, double *wall, int *boundary, int *nnb, int *nbr)
{
    return alebgk_lattice_build_device_ex(name, Nx, Nv, dt, mls_order, 0, 1.0, lid_speed, rho0,
                                          tau, device, xyz, wall, boundary, nullptr, nnb, nbr);
}

int alebgk_neighbours_device(alebgk_ctx *c, const double *grid, const int *boxes, int *nnb,
                             int *nbr)
{
    if (!c || !grid || !boxes || !nnb || !nbr) return fail(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return fail(c, ALEBGK_ESTATE, "upload the cloud first");
    NeighbourGrid g;
    g.dim = c->sp.dim;
    g.x0 = grid[0]; g.y0 = grid[1]; g.z0 = grid[2];
    g.hx = grid[3]; g.hy = grid[4]; g.hz = grid[5]; g.radius = grid[6];
    g.nx = boxes[0]; g.ny = boxes[1]; g.nz = boxes[2];
    // box sizes carry the sign of the axis (the z lattice of the 3-D body
    // cases runs from zfront = L down to zback = 0)
    if (g.nx < 1 || g.ny < 1 || g.nz < 1 || (g.dim == 2 && g.nz != 1) || !(g.hx != 0) ||
        !(g.hy != 0) || !(g.hz != 0) || !(g.radius > 0))
        return fail(c, ALEBGK_EINVAL, "bad voxel grid");
    CK(cudaSetDevice(c->cfg.device));
    const size_t N = c->sp.N;
    const size_t nvox = (size_t)g.nx * g.ny * g.nz;
    LatticeBuffers b;
    CK(dalloc(&b.d.voxel, N));
    CK(dalloc(&b.d.voxCount, nvox));
    CK(dalloc(&b.d.voxStart, nvox + 1));
    CK(dalloc(&b.d.voxCursor, nvox));
    CK(dalloc(&b.d.voxList, N));
    CK(dalloc(&b.d.nnb, N));
    CK(dalloc(&b.d.nbr, N * ALEBGK_MAX_NEIGH));
    CK(buildNeighboursDevice(g, c->d.pos, (int)N, b.d, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    CK(cudaMemcpy(nnb, b.d.nnb, 4 * N, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nbr, b.d.nbr, 4 * N * ALEBGK_MAX_NEIGH, cudaMemcpyDeviceToHost));
    return ALEBGK_OK;
}

int alebgk_upload_lattice_ex(alebgk_ctx *c, const char *name, int Nx, int Nv, double dt,
                             int mls_order, int fixed_body, double body_scale, double lid_speed,
                             double rho0, double tau)
{
    if (!c) return ALEBGK_EINVAL;
    CaseParams p;
    int rc = latticeCase(name, Nx, Nv, dt, mls_order, fixed_body, lid_speed, rho0, tau, p);
    if (rc) return fail(c, rc, gCreateError);
    const StepParams &sp = c->sp;
    CK(cudaSetDevice(c->cfg.device));
    LatticeBuffers b;
    size_t N = 0;
    CK(deviceSetup(p, body_scale, b, &N, c->stream));
    if ((size_t)sp.N != N || sp.dim != p.dim || sp.Nv != p.Nv || sp.mlsOrder != p.mlsOrder ||
        sp.vmin != p.VMin || sp.dv != p.dv || sp.h != p.radius || sp.tau != p.tau ||
        sp.R != p.R)
        return fail(c, ALEBGK_EINVAL,
                    "the context's configuration does not match this lattice case "
                    "(N, dim, Nv, MLS order, velocity grid, radius, tau or R)");
    CK(cudaStreamSynchronize(c->stream));
    LatticeHost h;
    CK(h.fetch(b.d, N));
    alebgk_cloud view{};
    view.xyz = h.xyz.data(); view.meshv = h.meshv.data(); view.wall = h.wall.data();
    view.boundary = h.boundary.data(); view.body_id = h.bodyId.data();
    view.nnb = h.nnb.data(); view.nbr = h.nbr.data();
    rc = uploadCloud(c, &view, p.dt, false);
    if (rc) return rc;
    std::vector<double> row;
    restRow(p, row);
    double *rowDev = nullptr;
    CK(cudaMalloc(&rowDev, row.size() * 8));
    cudaError_t e = cudaMemcpy(rowDev, row.data(), row.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launchRestState(c, rowDev, p.rho0, 270.0);
    if (e == cudaSuccess) e = launchMassInit(c);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(rowDev);
    if (e != cudaSuccess)
        return fail(c, ALEBGK_ECUDA, std::string("lattice state: ") + cudaGetErrorString(e));
    return ALEBGK_OK;
}

int alebgk_upload_lattice(alebgk_ctx *c, const char *name, int Nx, int Nv, double dt,
                          int mls_order, double lid_speed, double rho0, double tau)
{
    return alebgk_upload_lattice_ex(c, name, Nx, Nv, dt, mls_order, 0, 1.0, lid_speed, rho0,
                                    tau);
}

int alebgk_case_view(alebgk_case *cs, alebgk_cloud *v)
{
    if (!cs || !v) return ALEBGK_EINVAL;
    Cloud &c = cs->cloud;
    c.xyz.resize(3 * (size_t)c.N);
    for (int i = 0; i < c.N; ++i)
    {
        c.xyz[3 * (size_t)i] = c.x[i];
        c.xyz[3 * (size_t)i + 1] = c.y[i];
        c.xyz[3 * (size_t)i + 2] = c.z[i];
    }
    v->xyz = c.xyz.data();
    v->meshv = c.meshv.data();
    v->wall = c.wall.data();
    v->boundary = c.boundary.data();
    v->body_id = c.bodyId.data();
    v->nnb = c.nnb.data();
    v->nbr = c.nbr.data();
    v->g = c.g.data();
    v->macro = c.macro.data();
    return ALEBGK_OK;
}

int alebgk_case_bodies(const alebgk_case *cs, double *out)
{
    if (!cs || !out) return ALEBGK_EINVAL;
    const Cloud &c = cs->cloud;
    for (size_t b = 0; b < c.bodies.size(); ++b)
    {
        bodyState(c.bodies[b], out + 32 * b);
    }
    return ALEBGK_OK;
}

int alebgk_case_body_shapes(const alebgk_case *cs, int *kind, int *rotates, double *size)
{
    if (!cs || !kind || !rotates || !size) return ALEBGK_EINVAL;
    const Cloud &c = cs->cloud;
    for (size_t b = 0; b < c.bodies.size(); ++b)
    {
        kind[b] = c.bodies[b].kind;
        rotates[b] = c.bodies[b].rotates ? 1 : 0;
        size[b] = c.bodies[b].size;
    }
    return ALEBGK_OK;
}

int alebgk_case_config(const alebgk_case *cs, int precision, int device,
                       alebgk_config *cfg)
{
    if (!cs || !cfg) return ALEBGK_EINVAL;
    const Cloud &c = cs->cloud;
    const CaseParams &p = c.prm;
    std::memset(cfg, 0, sizeof *cfg);
    cfg->dim = p.dim; cfg->N = c.N; cfg->Nv = p.Nv; cfg->mls_order = p.mlsOrder;
    cfg->precision = precision; cfg->limiter = 2; cfg->tau_variable = 0;
    cfg->device = device; cfg->R = p.R; cfg->tau = p.tau; cfg->dHS = p.dHS;
    cfg->vmin = p.VMin; cfg->dv = p.dv; cfg->radius = p.radius;
    return ALEBGK_OK;
}

}  // extern "C"
