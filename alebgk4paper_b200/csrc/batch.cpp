// batch.cpp -- launch-shape autotuning, the steady residual, and batches of
// independent cavities advanced by one CUDA graph per step.
//
// A batch holds contexts on one device that advance in lockstep, one graph
// launch per step.  When every context has the same precision and Chu
// layers and runs the plain transport and particle kernels, the contexts
// are split into up to four groups of about equal work, and the graph holds
// per group one launch per stage of the step over the group's contexts
// (step.cu's batch kernels: a block finds its context from per-stage block
// offsets), each group on its own branch: a few dozen nodes whatever the
// batch size, and the short stages of one group overlap the long ones of
// another.  Otherwise one graph per ping-pong parity holds every context's
// whole step (and its residual) as a parallel branch: a master stream forks
// to each context's stream and joins them again.  A third form (mode 2)
// puts the whole step of all contexts into one persistent cooperative
// launch: every stage's blocks spread over the resident grid, a bounded
// grid-wide barrier between stages.  All forms compute each context exactly
// as its own step does.
#include <algorithm>
#include <cuda_runtime.h>

#include <string>
#include <cmath>
#include <vector>

#include "ctx.h"

using namespace alebgk;

struct alebgk_batch
{
    std::vector<alebgk_ctx *> ctx;
    int device = 0;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    double *resid = nullptr;              // device, one per context
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int mode = 0;                         // 0 stage launches when possible, 1 branches,
                                          // 2 one persistent launch when possible
    bool staged = false;                  // the graphs hold stage launches
    bool planned = false;                 // the stage groups were tried
    std::vector<BatchLaunch> groups;      // stage launches per group
    std::vector<int> groupStream;         // context whose stream runs the group
    int ngroups = 4;                      // stage groups wanted
    long long spinCap = 1ll << 24;        // grid-barrier polls before giving up (mode 2)
    std::vector<unsigned long long> epochs;   // the contexts' epochs of the captured graphs
    std::string err;
};

namespace {

int failc(alebgk_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

#define CKC(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return failc(c, ALEBGK_ECUDA, std::string(#call) + ": " +                 \
                                              cudaGetErrorString(e_));                 \
    } while (0)

void dropGraphs(alebgk_ctx *c)
{
    for (auto &g : c->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

void freeGroups(alebgk_batch *b)
{
    for (BatchLaunch &bl : b->groups) freeBatchLaunch(bl);
    b->groups.clear();
    b->groupStream.clear();
    b->staged = false;
    b->planned = false;
}

// Splits the contexts into groups of about equal work (particles x nodes x
// layers; largest first onto the lightest group) and builds each group's
// stage launches.  cudaErrorNotSupported when the contexts cannot share
// stage launches.
cudaError_t planGroups(alebgk_batch *b)
{
    const int n = (int)b->ctx.size();
    // one persistent launch holds the whole batch: a second one beside it
    // could not be resident at the same time
    const int G = b->mode == 2 ? 1 : std::max(1, std::min(b->ngroups, n));
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    auto cost = [&](int i) {
        const StepParams &p = b->ctx[i]->sp;
        return (double)p.N * p.V * p.L;
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
    std::vector<std::vector<int>> member(G);
    std::vector<double> load(G, 0.0);
    for (int i : order)
    {
        const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        member[g].push_back(i);
        load[g] += cost(i);
    }
    b->groups.assign(G, BatchLaunch());
    for (int g = 0; g < G; ++g)
    {
        std::sort(member[g].begin(), member[g].end());
        std::vector<alebgk_ctx *> cs;
        std::vector<double *> rs;
        for (int i : member[g])
        {
            cs.push_back(b->ctx[i]);
            rs.push_back(b->resid + i);
        }
        cudaError_t e = buildBatchLaunch(cs.data(), (int)cs.size(), rs.data(), b->groups[g]);
        b->groups[g].persistent = b->mode == 2;
        b->groups[g].spinCap = b->spinCap;
        if (e == cudaSuccess) e = prepareBatchLaunch(b->groups[g]);
        if (e != cudaSuccess) return e;
        b->groupStream.push_back(member[g][0]);
    }
    return cudaSuccess;
}

}  // namespace

extern "C" {

int alebgk_set_launch(alebgk_ctx *c, int transport_threads, int particle_warps)
{
    if (!c) return ALEBGK_EINVAL;
    if (transport_threads != 0 &&
        (transport_threads < 32 || transport_threads > 256 || transport_threads % 32))
        return failc(c, ALEBGK_EINVAL,
                     "transport threads: 0 (fused into the particle kernel) or a multiple of 32 "
                     "in 32..256");
    if (particle_warps < 0 || particle_warps > 8)
        return failc(c, ALEBGK_EINVAL, "particle warps: 0 (as many as fit) or 1..8");
    if (c->tune.transportThreads != transport_threads || c->tune.particleWarps != particle_warps)
    {
        c->tune.transportThreads = transport_threads;
        c->tune.particleWarps = particle_warps;
        dropGraphs(c);
    }
    return ALEBGK_OK;
}

int alebgk_set_march_width(alebgk_ctx *c, int velocities_per_lane)
{
    if (!c) return ALEBGK_EINVAL;
    if (velocities_per_lane != 1 && velocities_per_lane != 2)
        return failc(c, ALEBGK_EINVAL, "march width: 1 or 2 velocities per lane");
    c->tune.marchVpl = velocities_per_lane;
    MarchState &m = c->march;
    if (!m.enabled || m.vpl == velocities_per_lane) return ALEBGK_OK;
    m.vpl = velocities_per_lane;
    const StepParams &p = c->sp;
    std::string err;
    for (int b = 0; b < 2; ++b)
    {
        if (!encodeMarchMap(m.tmap[b], c->d.f[b], p.V, m.Nx, m.Ny, m.Nz, p.ldf, false, m.vpl,
                            &err) ||
            (m.nunitsY > 0 && !encodeMarchMap(m.tmapY[b], c->d.f[b], p.V, m.Nx, m.Ny, m.Nz,
                                              p.ldf, true, m.vpl, &err)))
            return failc(c, ALEBGK_ECUDA, err);
    }
    dropGraphs(c);
    return ALEBGK_OK;
}

int alebgk_set_nad_floor(alebgk_ctx *c, double rel)
{
    if (!c) return ALEBGK_EINVAL;
    if (!(rel >= 0.0) || rel > 1e-2)
        return failc(c, ALEBGK_EINVAL, "the NAD rounding floor is a relative slack in [0, 1e-2]");
    c->sp.nadNoise = rel;
    dropGraphs(c);
    return ALEBGK_OK;
}

int alebgk_set_residual_speed(alebgk_ctx *c, double speed)
{
    if (!c) return ALEBGK_EINVAL;
    if (!std::isfinite(speed)) return failc(c, ALEBGK_EINVAL, "the residual speed is finite");
    c->sp.resU = speed;
    dropGraphs(c);
    return ALEBGK_OK;
}

int alebgk_get_launch(alebgk_ctx *c, int *transport_threads, int *particle_warps)
{
    if (!c || !transport_threads || !particle_warps) return ALEBGK_EINVAL;
    *transport_threads = c->tune.transportThreads;
    *particle_warps = c->tune.particleWarps;
    return ALEBGK_OK;
}

int alebgk_autotune(alebgk_ctx *c, int steps, float *best_ms)
{
    if (!c) return ALEBGK_EINVAL;
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    if (steps < 1) return failc(c, ALEBGK_EINVAL, "steps must be >= 1");
    CKC(cudaSetDevice(c->cfg.device));
    CKC(cudaStreamSynchronize(c->stream));
    // Snapshot of everything a step reads: the current distribution and
    // macros, the moodCheck flags and the step scalars.
    const StepParams &p = c->sp;
    const size_t es = (c->cfg.precision == 64) ? 8 : 4;
    const size_t fBytes = (size_t)p.N * p.ldf * es, mBytes = 48 * (size_t)p.N;
    const int cur0 = c->cur;
    void *snapF = nullptr, *snapM = nullptr, *snapMood = nullptr, *snapSc = nullptr;
    CKC(cudaMalloc(&snapF, fBytes));
    CKC(cudaMalloc(&snapM, mBytes));
    CKC(cudaMalloc(&snapMood, 4 * (size_t)p.N));
    CKC(cudaMalloc(&snapSc, sizeof(StepScalars)));
    cudaError_t e = cudaMemcpy(snapF, c->d.f[cur0], fBytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(snapM, c->d.macro[cur0], mBytes, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(snapMood, c->d.mood, 4 * (size_t)p.N, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(snapSc, c->d.sc, sizeof(StepScalars), cudaMemcpyDeviceToDevice);
    auto restore = [&]() {
        c->cur = cur0;
        cudaError_t r = cudaMemcpy(c->d.f[cur0], snapF, fBytes, cudaMemcpyDeviceToDevice);
        if (r == cudaSuccess)
            r = cudaMemcpy(c->d.macro[cur0], snapM, mBytes, cudaMemcpyDeviceToDevice);
        if (r == cudaSuccess) r = cudaMemcpy(c->d.mood, snapMood, 4 * (size_t)p.N, cudaMemcpyDeviceToDevice);
        if (r == cudaSuccess) r = cudaMemcpy(c->d.sc, snapSc, sizeof(StepScalars), cudaMemcpyDeviceToDevice);
        return r;
    };
    const int tts[] = {0, 64, 128, 256};
    const int pws[] = {1, 2, 4, 0};
    float best = -1.0f;
    int bestT = c->tune.transportThreads, bestW = c->tune.particleWarps;
    int rc = ALEBGK_OK;
    for (int tt : tts)
    {
        for (int pw : pws)
        {
            if (e != cudaSuccess || rc != ALEBGK_OK) break;
            rc = alebgk_set_launch(c, tt, pw);
            float ms = 0.0f;
            if (rc == ALEBGK_OK) rc = alebgk_step(c, 2);      // captures both graphs
            if (rc == ALEBGK_OK) rc = alebgk_step_timed(c, steps, &ms);
            e = restore();
            if (rc == ALEBGK_OK && e == cudaSuccess && (best < 0 || ms < best))
            {
                best = ms;
                bestT = tt;
                bestW = pw;
            }
        }
    }
    cudaFree(snapF);
    cudaFree(snapM);
    cudaFree(snapMood);
    cudaFree(snapSc);
    if (e != cudaSuccess)
        return failc(c, ALEBGK_ECUDA, std::string("autotune: ") + cudaGetErrorString(e));
    if (rc != ALEBGK_OK) return rc;
    rc = alebgk_set_launch(c, bestT, bestW);
    if (best_ms) *best_ms = best / steps;
    return rc;
}

int alebgk_residual(alebgk_ctx *c, double *res)
{
    if (!c || !res) return ALEBGK_EINVAL;
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    CKC(cudaSetDevice(c->cfg.device));
    CKC(launchResidual(c, c->d.redPartial, c->stream));
    CKC(cudaMemcpyAsync(res, c->d.redPartial, 8, cudaMemcpyDeviceToHost, c->stream));
    CKC(cudaStreamSynchronize(c->stream));
    return ALEBGK_OK;
}

int alebgk_residual_interval(alebgk_ctx *c, double *res)
{
    if (!c || !res) return ALEBGK_EINVAL;
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    CKC(cudaSetDevice(c->cfg.device));
    const size_t mBytes = 48 * (size_t)c->sp.N;
    if (!c->macSnap) CKC(cudaMalloc(&c->macSnap, mBytes));
    *res = -1.0;
    const long long k = c->hostSteps - c->snapSteps;
    if (c->snapSteps >= 0 && k > 0)
    {
        // residual of "one step" from the snapshot to now, per step
        const int keep = c->cur;
        double *old = c->d.macro[1 - keep];
        c->d.macro[1 - keep] = c->macSnap;
        const cudaError_t e = launchResidual(c, c->d.redPartial, c->stream);
        c->d.macro[1 - keep] = old;
        CKC(e);
        CKC(cudaMemcpyAsync(res, c->d.redPartial, 8, cudaMemcpyDeviceToHost, c->stream));
        CKC(cudaStreamSynchronize(c->stream));
        *res /= (double)k;
    }
    CKC(cudaMemcpyAsync(c->macSnap, c->d.macro[c->cur], mBytes, cudaMemcpyDeviceToDevice,
                        c->stream));
    CKC(cudaStreamSynchronize(c->stream));
    c->snapSteps = c->hostSteps;
    return ALEBGK_OK;
}

int alebgk_batch_create(int n, alebgk_ctx **ctxs, alebgk_batch **out)
{
    if (!ctxs || !out || n < 1) return ALEBGK_EINVAL;
    *out = nullptr;
    for (int i = 0; i < n; ++i)
    {
        alebgk_ctx *c = ctxs[i];
        if (!c || !c->uploaded) return ALEBGK_ESTATE;
        if (c->geometryDirty) return failc(c, ALEBGK_ESTATE, "upload the cloud again first");
        if (c->cfg.device != ctxs[0]->cfg.device)
            return failc(c, ALEBGK_EINVAL, "a batch lives on one device");
        if (c->cur != ctxs[0]->cur)
            return failc(c, ALEBGK_EINVAL, "the contexts of a batch must be in step");
        for (int j = 0; j < i; ++j)
            if (ctxs[j] == c) return failc(c, ALEBGK_EINVAL, "a context appears twice");
    }
    auto *b = new (std::nothrow) alebgk_batch();
    if (!b) return ALEBGK_ENOMEM;
    b->ctx.assign(ctxs, ctxs + n);
    b->device = ctxs[0]->cfg.device;
    b->join.assign(n, nullptr);
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int i = 0; i < n && e == cudaSuccess; ++i)
        e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc(&b->resid, 8 * (size_t)n);
    if (e == cudaSuccess) e = cudaMemset(b->resid, 0, 8 * (size_t)n);
    if (e != cudaSuccess)
    {
        alebgk_batch_destroy(b);
        return ALEBGK_ECUDA;
    }
    *out = b;
    return ALEBGK_OK;
}

int alebgk_batch_step(alebgk_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return ALEBGK_EINVAL;
    alebgk_ctx *c = b->ctx[0];
    CKC(cudaSetDevice(b->device));
    for (alebgk_ctx *x : b->ctx)
        if (!x->uploaded || x->geometryDirty || x->cur != c->cur)
            return failc(x, ALEBGK_ESTATE, "a context of the batch left the lockstep");
    // A context uploaded or refreshed since the capture: its buffers and slot
    // stride may have changed, so the graphs and stage launches are rebuilt.
    bool stale = b->epochs.size() != b->ctx.size();
    for (size_t i = 0; i < b->ctx.size() && !stale; ++i) stale = b->epochs[i] != b->ctx[i]->epoch;
    if (stale)
    {
        CKC(cudaStreamSynchronize(b->master));
        for (auto &g : b->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        freeGroups(b);
        b->epochs.clear();
        for (alebgk_ctx *x : b->ctx) b->epochs.push_back(x->epoch);
    }
    for (int n = 0; n < nsteps; ++n)
    {
        const int from = c->cur;
        if (b->mode != 1 && !b->planned)
        {
            const cudaError_t be = planGroups(b);
            if (be != cudaSuccess)
            {
                freeGroups(b);
                if (be != cudaErrorNotSupported) CKC(be);
            }
            else b->staged = true;
            b->planned = true;
        }
        if (!b->graph[from])
        {
            cudaGraph_t g = nullptr;
            CKC(cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal));
            cudaError_t le = cudaEventRecord(b->fork, b->master);
            for (size_t q = 0; q < b->groups.size() && le == cudaSuccess && b->staged; ++q)
            {
                cudaStream_t gs = b->ctx[b->groupStream[q]]->stream;
                le = cudaStreamWaitEvent(gs, b->fork, 0);
                if (le == cudaSuccess) le = launchBatchStep(b->groups[q], from, gs);
                if (le == cudaSuccess) le = cudaEventRecord(b->join[q], gs);
                if (le == cudaSuccess) le = cudaStreamWaitEvent(b->master, b->join[q], 0);
            }
            for (size_t i = 0; i < b->ctx.size() && le == cudaSuccess && !b->staged; ++i)
            {
                alebgk_ctx *x = b->ctx[i];
                le = cudaStreamWaitEvent(x->stream, b->fork, 0);
                if (le == cudaSuccess) le = launchStep(x, from);
                // the residual compares the new macros with the old ones
                const int keep = x->cur;
                x->cur = 1 - from;
                if (le == cudaSuccess) le = launchResidual(x, b->resid + i, x->stream);
                x->cur = keep;
                if (le == cudaSuccess) le = cudaEventRecord(b->join[i], x->stream);
                if (le == cudaSuccess) le = cudaStreamWaitEvent(b->master, b->join[i], 0);
            }
            cudaError_t ee = cudaStreamEndCapture(b->master, &g);
            if (le != cudaSuccess || ee != cudaSuccess)
            {
                if (g) cudaGraphDestroy(g);
                return failc(c, ALEBGK_ECUDA,
                             std::string("batch capture: ") +
                                 cudaGetErrorString(le != cudaSuccess ? le : ee));
            }
            cudaError_t ie = cudaGraphInstantiate(&b->graph[from], g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess)
                return failc(c, ALEBGK_ECUDA, std::string("batch graph: ") + cudaGetErrorString(ie));
        }
        CKC(cudaGraphLaunch(b->graph[from], b->master));
        for (alebgk_ctx *x : b->ctx)
        {
            x->cur = 1 - from;
            ++x->hostSteps;
        }
    }
    // the contexts' own streams see the batch's work before their next call
    CKC(cudaEventRecord(b->fork, b->master));
    for (alebgk_ctx *x : b->ctx) CKC(cudaStreamWaitEvent(x->stream, b->fork, 0));
    return ALEBGK_OK;
}

int alebgk_batch_set_mode(alebgk_batch *b, int mode)
{
    if (!b || mode < 0 || mode > 2) return ALEBGK_EINVAL;
    if (mode != b->mode)
    {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->master);
        for (auto &g : b->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        freeGroups(b);
        b->mode = mode;
    }
    return ALEBGK_OK;
}

int alebgk_batch_get_mode(alebgk_batch *b, int *mode, int *staged)
{
    if (!b || !mode || !staged) return ALEBGK_EINVAL;
    *mode = b->mode;
    *staged = b->staged ? (int)b->groups.size() : 0;
    return ALEBGK_OK;
}

int alebgk_batch_set_groups(alebgk_batch *b, int groups)
{
    if (!b || groups < 1 || groups > 64) return ALEBGK_EINVAL;
    if (groups != b->ngroups)
    {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->master);
        for (auto &g : b->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        freeGroups(b);
        b->ngroups = groups;
    }
    return ALEBGK_OK;
}

int alebgk_batch_set_spin_limit(alebgk_batch *b, long long polls)
{
    if (!b || polls < 0) return ALEBGK_EINVAL;
    if (polls != b->spinCap)
    {
        cudaSetDevice(b->device);
        cudaStreamSynchronize(b->master);
        for (auto &g : b->graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        freeGroups(b);
        b->spinCap = polls;
    }
    return ALEBGK_OK;
}

int alebgk_batch_autotune(alebgk_batch *b, int steps, float *best_ms)
{
    if (!b || steps < 1) return ALEBGK_EINVAL;
    alebgk_ctx *c = b->ctx[0];
    CKC(cudaSetDevice(b->device));
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CKC(cudaEventCreate(&t0));
    CKC(cudaEventCreate(&t1));
    // candidates: stage launches in 1, 2, 4, 8 groups, one persistent
    // launch, then branches
    struct Cand { int mode, groups; };
    std::vector<Cand> cands;
    for (int g : {1, 2, 4, 8})
        if (g <= (int)b->ctx.size()) cands.push_back({0, g});
    cands.push_back({2, 1});
    cands.push_back({1, b->ngroups});
    float best = -1.0f;
    Cand pick = {b->mode, b->ngroups};
    int rc = ALEBGK_OK;
    for (const Cand &cd : cands)
    {
        rc = alebgk_batch_set_mode(b, cd.mode);
        if (rc == ALEBGK_OK) rc = alebgk_batch_set_groups(b, cd.groups);
        if (rc == ALEBGK_OK) rc = alebgk_batch_step(b, 2);     // captures both graphs
        if (rc != ALEBGK_OK) break;
        // (contexts that cannot share stage launches run as branches here)
        float ms = 0.0f;
        cudaError_t e = cudaEventRecord(t0, b->master);
        if (e == cudaSuccess) rc = alebgk_batch_step(b, steps);
        if (rc != ALEBGK_OK) break;
        if (e == cudaSuccess) e = cudaEventRecord(t1, b->master);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        if (e != cudaSuccess)
        {
            rc = failc(c, ALEBGK_ECUDA, std::string("batch autotune: ") + cudaGetErrorString(e));
            break;
        }
        if (best < 0 || ms < best)
        {
            best = ms;
            pick = cd;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rc != ALEBGK_OK) return rc;
    rc = alebgk_batch_set_mode(b, pick.mode);
    if (rc == ALEBGK_OK) rc = alebgk_batch_set_groups(b, pick.groups);
    if (best_ms) *best_ms = best / steps;
    return rc;
}

int alebgk_batch_residuals(alebgk_batch *b, double *out)
{
    if (!b || !out) return ALEBGK_EINVAL;
    alebgk_ctx *c = b->ctx[0];
    CKC(cudaSetDevice(b->device));
    CKC(cudaMemcpyAsync(out, b->resid, 8 * b->ctx.size(), cudaMemcpyDeviceToHost, b->master));
    CKC(cudaStreamSynchronize(b->master));
    return ALEBGK_OK;
}

int alebgk_batch_sync(alebgk_batch *b)
{
    if (!b) return ALEBGK_EINVAL;
    alebgk_ctx *c = b->ctx[0];
    CKC(cudaSetDevice(b->device));
    CKC(cudaStreamSynchronize(b->master));
    return ALEBGK_OK;
}

int alebgk_batch_destroy(alebgk_batch *b)
{
    if (!b) return ALEBGK_OK;
    cudaSetDevice(b->device);
    if (b->master) cudaStreamSynchronize(b->master);
    for (auto &g : b->graph)
        if (g) cudaGraphExecDestroy(g);
    freeGroups(b);
    for (auto &e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->resid) cudaFree(b->resid);
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
    return ALEBGK_OK;
}

}  // extern "C"
