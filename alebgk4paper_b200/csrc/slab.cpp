// slab.cpp -- one large cavity split into slabs, one context per slab: the
// B200 form of the reference's decomposed mode (Solver/MpiExchange.cpp:
// 114-466), with the contexts driven from one process.
//
// Each slab holds its owned lattice rows plus ghost rows (copies of the
// neighbouring slabs' rows) on each side.  Per step, every slab runs the
// step in four segments; between segments one combine kernel adds the slabs'
// owned-range partial sums in slab order (the rank-ordered Allgather of
// MomentCalculations/Conservation.cpp:76-84) and ORs the moodCheck flags
// (Conservation.cpp:33-36), writing the global values into every slab's
// scalars.  After the step the ghost rows' distributions and macros are
// refreshed from their owners (alebgk_haloExchange, MpiExchange.cpp:
// 405-466) by one copy per ghost block.  Contexts on different devices read
// each other's scalars and rows over peer access (NVLink); the combine runs
// on the first slab's device.
//
// Multi-process runs (alebgk_rank_slab_*): each process holds one slab.  The
// host runs a segment, reads the slab's four combine words (owned-range
// partial sums and the moodCheck flag), exchanges them with the other ranks
// (an all-gather in rank order, MPI_Allgather in the reference), and hands
// every rank's words back; the combine kernel then applies, for this slab,
// exactly what the single-process combine writes.  Ghost rows travel
// through host buffers between the last segment and the end of the step.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "ctx.h"

using namespace alebgk;

struct alebgk_slab
{
    int device = 0;
    std::vector<alebgk_ctx *> ctx;
    StepScalars **scs = nullptr;          // device array of the slabs' scalars
    cudaStream_t master = nullptr;
    cudaEvent_t combined = nullptr;
    std::vector<cudaEvent_t> done;
    struct Copy
    {
        int dst, dstStart, src, srcStart, count;
    };
    std::vector<Copy> copies;
};

namespace {

int failS(alebgk_ctx *c, int code, const std::string &m)
{
    if (c) c->err = m;
    return code;
}

#define CKS(call)                                                                        \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return failS(c, ALEBGK_ECUDA, std::string(#call) + ": " +                   \
                                              cudaGetErrorString(e_));                   \
    } while (0)

// Ghost rows of the new state (f and macros of buffer `buf`) from their owners.
cudaError_t haloCopies(alebgk_slab *g, int buf)
{
    for (const alebgk_slab::Copy &cp : g->copies)
    {
        alebgk_ctx *d = g->ctx[cp.dst], *s = g->ctx[cp.src];
        const size_t es = (d->cfg.precision == 64) ? 8 : 4;
        const size_t row = (size_t)d->sp.ldf * es;
        cudaError_t e = cudaMemcpyPeerAsync(
            static_cast<char *>(d->d.f[buf]) + row * cp.dstStart, d->cfg.device,
            static_cast<const char *>(s->d.f[buf]) + row * cp.srcStart, s->cfg.device,
            row * cp.count, g->master);
        if (e == cudaSuccess)
            e = cudaMemcpyPeerAsync(d->d.macro[buf] + 6 * (size_t)cp.dstStart, d->cfg.device,
                                    s->d.macro[buf] + 6 * (size_t)cp.srcStart, s->cfg.device,
                                    48 * (size_t)cp.count, g->master);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Every slab's stream waits for the master; the master then waits for them.
cudaError_t joinAll(alebgk_slab *g)
{
    for (size_t i = 0; i < g->ctx.size(); ++i)
    {
        cudaError_t e = cudaEventRecord(g->done[i], g->ctx[i]->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(g->master, g->done[i], 0);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t forkAll(alebgk_slab *g)
{
    cudaError_t e = cudaEventRecord(g->combined, g->master);
    for (size_t i = 0; i < g->ctx.size() && e == cudaSuccess; ++i)
        e = cudaStreamWaitEvent(g->ctx[i]->stream, g->combined, 0);
    return e;
}

}  // namespace

extern "C" {

int alebgk_slab_create(int n, alebgk_ctx **ctxs, const int *own_lo, const int *own_hi,
                       int ncopies, const int *copies, alebgk_slab **out)
{
    if (n < 1 || !ctxs || !own_lo || !own_hi || !out || (ncopies > 0 && !copies))
        return ALEBGK_EINVAL;
    *out = nullptr;
    alebgk_ctx *c = ctxs[0];
    for (int i = 0; i < n; ++i)
    {
        alebgk_ctx *x = ctxs[i];
        if (!x || !x->uploaded) return failS(c, ALEBGK_ESTATE, "every slab must be uploaded");
        if (own_lo[i] < 0 || own_hi[i] <= own_lo[i] || own_hi[i] > x->sp.N)
            return failS(c, ALEBGK_EINVAL, "owned range out of bounds for slab " +
                                                std::to_string(i));
        if (x->cfg.precision != c->cfg.precision || x->sp.ldf != c->sp.ldf ||
            x->sp.gs != c->sp.gs || x->cur != c->cur)
            return failS(c, ALEBGK_EINVAL, "slabs differ in precision, row size or parity");
        if (!x->bodyIdHost.empty())
            for (int b : x->bodyIdHost)
                if (b >= 0) return failS(c, ALEBGK_EINVAL, "slab groups take clouds without bodies");
    }
    auto *g = new alebgk_slab();
    g->device = c->cfg.device;
    g->ctx.assign(ctxs, ctxs + n);
    for (int q = 0; q < ncopies; ++q)
    {
        alebgk_slab::Copy cp{copies[5 * q], copies[5 * q + 1], copies[5 * q + 2],
                             copies[5 * q + 3], copies[5 * q + 4]};
        const bool ok = cp.dst >= 0 && cp.dst < n && cp.src >= 0 && cp.src < n &&
                        cp.count > 0 && cp.dstStart >= 0 && cp.srcStart >= 0 &&
                        cp.dstStart + cp.count <= ctxs[cp.dst]->sp.N &&
                        cp.srcStart + cp.count <= ctxs[cp.src]->sp.N;
        if (!ok)
        {
            delete g;
            return failS(c, ALEBGK_EINVAL, "ghost copy " + std::to_string(q) + " out of bounds");
        }
        g->copies.push_back(cp);
    }
    auto bail = [&](cudaError_t e) {
        alebgk_slab_destroy(g);
        return failS(c, ALEBGK_ECUDA, std::string("slab set-up: ") + cudaGetErrorString(e));
    };
    cudaError_t e = cudaSetDevice(g->device);
    for (int i = 0; i < n && e == cudaSuccess; ++i)
    {
        const int d = ctxs[i]->cfg.device;
        if (d == g->device) continue;
        int can = 0;
        e = cudaDeviceCanAccessPeer(&can, g->device, d);
        if (e == cudaSuccess && !can) e = cudaErrorPeerAccessUnsupported;
        if (e == cudaSuccess)
        {
            e = cudaDeviceEnablePeerAccess(d, 0);
            if (e == cudaErrorPeerAccessAlreadyEnabled) { cudaGetLastError(); e = cudaSuccess; }
        }
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g->master, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->combined, cudaEventDisableTiming);
    g->done.assign(n, nullptr);
    for (int i = 0; i < n && e == cudaSuccess; ++i)
    {
        e = cudaSetDevice(ctxs[i]->cfg.device);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->done[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaSetDevice(g->device);
    std::vector<StepScalars *> host(n);
    for (int i = 0; i < n; ++i) host[i] = ctxs[i]->d.sc;
    if (e == cudaSuccess) e = cudaMalloc(&g->scs, sizeof(StepScalars *) * n);
    if (e == cudaSuccess)
        e = cudaMemcpy(g->scs, host.data(), sizeof(StepScalars *) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return bail(e);
    // owned ranges, then the whole domain's mass as every slab's start
    for (int i = 0; i < n; ++i)
    {
        ctxs[i]->sp.ownLo = own_lo[i];
        ctxs[i]->sp.ownHi = own_hi[i];
    }
    e = forkAll(g);
    for (int i = 0; i < n && e == cudaSuccess; ++i)
    {
        e = cudaSetDevice(ctxs[i]->cfg.device);
        if (e == cudaSuccess) e = launchSlabInitSum(ctxs[i], ctxs[i]->stream);
    }
    if (e == cudaSuccess) e = cudaSetDevice(g->device);
    if (e == cudaSuccess) e = joinAll(g);
    if (e == cudaSuccess) e = launchSlabCombine(g->scs, n, 4, g->master);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->master);
    if (e != cudaSuccess) return bail(e);
    *out = g;
    return ALEBGK_OK;
}

int alebgk_slab_step(alebgk_slab *g, int nsteps)
{
    if (!g || nsteps < 0) return ALEBGK_EINVAL;
    alebgk_ctx *c = g->ctx[0];
    const int n = (int)g->ctx.size();
    for (alebgk_ctx *x : g->ctx)
        if (x->cur != c->cur) return failS(c, ALEBGK_ESTATE, "a slab left the lockstep");
    for (int s = 0; s < nsteps; ++s)
    {
        const int from = c->cur;
        CKS(cudaSetDevice(g->device));
        CKS(forkAll(g));
        for (int seg = 0; seg < 4; ++seg)
        {
            for (int i = 0; i < n; ++i)
            {
                CKS(cudaSetDevice(g->ctx[i]->cfg.device));
                CKS(launchSlabSegment(g->ctx[i], from, seg, g->ctx[i]->stream));
            }
            CKS(cudaSetDevice(g->device));
            CKS(joinAll(g));
            CKS(launchSlabCombine(g->scs, n, seg, g->master));
            if (seg < 3) CKS(forkAll(g));
        }
        CKS(haloCopies(g, 1 - from));
        CKS(forkAll(g));
        for (alebgk_ctx *x : g->ctx)
        {
            x->cur = 1 - from;
            ++x->hostSteps;
        }
    }
    return ALEBGK_OK;
}

int alebgk_rank_slab_init(alebgk_ctx *c, int nranks, int own_lo, int own_hi, double *words)
{
    if (!c || !words || nranks < 1) return ALEBGK_EINVAL;
    if (!c->uploaded) return failS(c, ALEBGK_ESTATE, "upload the slab first");
    if (own_lo < 0 || own_hi <= own_lo || own_hi > c->sp.N)
        return failS(c, ALEBGK_EINVAL, "owned range out of bounds");
    for (int b : c->bodyIdHost)
        if (b >= 0) return failS(c, ALEBGK_EINVAL, "slabs take clouds without bodies");
    CKS(cudaSetDevice(c->cfg.device));
    CKS(cudaStreamSynchronize(c->stream));
    DeviceBuffers &d = c->d;
    if (d.rankAllCap < nranks)
    {
        if (d.rankAll) cudaFree(d.rankAll);
        d.rankAll = nullptr;
        d.rankAllCap = 0;
        CKS(cudaMalloc(&d.rankAll, 32 * (size_t)nranks));
        d.rankAllCap = nranks;
    }
    c->sp.ownLo = own_lo;
    c->sp.ownHi = own_hi;
    for (auto &gr : c->graph)
        if (gr) { cudaGraphExecDestroy(gr); gr = nullptr; }
    CKS(launchSlabInitSum(c, c->stream));
    StepScalars sc{};
    CKS(cudaMemcpyAsync(&sc, d.sc, sizeof sc, cudaMemcpyDeviceToHost, c->stream));
    CKS(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 3; ++q) words[q] = sc.slabPart[q];
    words[3] = sc.moodfail;
    return ALEBGK_OK;
}

int alebgk_rank_slab_segment(alebgk_ctx *c, int seg, double *words)
{
    if (!c || !words || seg < 0 || seg > 3) return ALEBGK_EINVAL;
    if (c->sp.ownHi <= c->sp.ownLo || c->d.rankAllCap < 1)
        return failS(c, ALEBGK_ESTATE, "alebgk_rank_slab_init first");
    CKS(cudaSetDevice(c->cfg.device));
    CKS(launchSlabSegment(c, c->cur, seg, c->stream));
    StepScalars sc{};
    CKS(cudaMemcpyAsync(&sc, c->d.sc, sizeof sc, cudaMemcpyDeviceToHost, c->stream));
    CKS(cudaStreamSynchronize(c->stream));
    for (int q = 0; q < 3; ++q) words[q] = sc.slabPart[q];
    words[3] = sc.moodfail;
    return ALEBGK_OK;
}

int alebgk_rank_slab_combine(alebgk_ctx *c, int phase, int nranks, const double *all)
{
    if (!c || !all || phase < 0 || phase > 4 || nranks < 1) return ALEBGK_EINVAL;
    if (nranks > c->d.rankAllCap)
        return failS(c, ALEBGK_EINVAL, "more ranks than alebgk_rank_slab_init was given");
    CKS(cudaSetDevice(c->cfg.device));
    CKS(cudaMemcpyAsync(c->d.rankAll, all, 32 * (size_t)nranks, cudaMemcpyHostToDevice,
                        c->stream));
    CKS(launchRankCombine(c, c->d.rankAll, nranks, phase, c->stream));
    CKS(cudaStreamSynchronize(c->stream));
    return ALEBGK_OK;
}

int alebgk_rank_slab_rows(alebgk_ctx *c, int start, int count, void *f_rows,
                          double *macro_rows, int put)
{
    if (!c || !f_rows || !macro_rows || count < 1 || start < 0) return ALEBGK_EINVAL;
    if (!c->uploaded || start + count > c->sp.N)
        return failS(c, ALEBGK_EINVAL, "rows out of bounds");
    CKS(cudaSetDevice(c->cfg.device));
    CKS(cudaStreamSynchronize(c->stream));
    const int buf = 1 - c->cur;        // the state the step in progress writes
    const size_t es = (c->cfg.precision == 64) ? 8 : 4;
    const size_t row = (size_t)c->sp.ldf * es;
    char *f = static_cast<char *>(c->d.f[buf]) + row * start;
    double *m = c->d.macro[buf] + 6 * (size_t)start;
    // The copies run on the context's own (non-blocking) stream and are
    // waited for before returning: a pageable host-to-device copy may return
    // before its DMA has landed, and the next step's kernels on this stream
    // must see the ghost rows.
    if (put)
    {
        CKS(cudaMemcpyAsync(f, f_rows, row * count, cudaMemcpyHostToDevice, c->stream));
        CKS(cudaMemcpyAsync(m, macro_rows, 48 * (size_t)count, cudaMemcpyHostToDevice,
                            c->stream));
    }
    else
    {
        CKS(cudaMemcpyAsync(f_rows, f, row * count, cudaMemcpyDeviceToHost, c->stream));
        CKS(cudaMemcpyAsync(macro_rows, m, 48 * (size_t)count, cudaMemcpyDeviceToHost,
                            c->stream));
    }
    CKS(cudaStreamSynchronize(c->stream));
    return ALEBGK_OK;
}

int alebgk_rank_slab_finish(alebgk_ctx *c)
{
    if (!c) return ALEBGK_EINVAL;
    CKS(cudaSetDevice(c->cfg.device));
    CKS(cudaStreamSynchronize(c->stream));
    c->cur = 1 - c->cur;
    ++c->hostSteps;
    return ALEBGK_OK;
}

int alebgk_slab_sync(alebgk_slab *g)
{
    if (!g) return ALEBGK_EINVAL;
    alebgk_ctx *c = g->ctx[0];
    CKS(cudaSetDevice(g->device));
    CKS(cudaStreamSynchronize(g->master));
    for (alebgk_ctx *x : g->ctx)
    {
        CKS(cudaSetDevice(x->cfg.device));
        CKS(cudaStreamSynchronize(x->stream));
    }
    CKS(cudaSetDevice(g->device));
    return ALEBGK_OK;
}

int alebgk_slab_destroy(alebgk_slab *g)
{
    if (!g) return ALEBGK_EINVAL;
    cudaSetDevice(g->device);
    if (g->master) cudaStreamSynchronize(g->master);
    for (alebgk_ctx *x : g->ctx)
        if (x)
        {
            x->sp.ownLo = 0;
            x->sp.ownHi = 0;
        }
    for (cudaEvent_t e : g->done)
        if (e) cudaEventDestroy(e);
    if (g->combined) cudaEventDestroy(g->combined);
    if (g->master) cudaStreamDestroy(g->master);
    if (g->scs) cudaFree(g->scs);
    delete g;
    return ALEBGK_OK;
}

}  // extern "C"
