// step.cu -- device kernels of the ALE-BGK time step for sm_100a.
//
// One step (the CPU step order of Solver/Solver.cpp:632-705):
//   k_step_begin      reset the step's counters (and the NAD neighbour ranges
//                     of the streamed particle kernel)
//   k_transport       gt[i][k] = scale * sum_s coef[class][s][k] * h[slot s][k]
//                     (k_march in march.cu for lattice clouds; by default the
//                     gather runs inside k_particle, each warp building its
//                     particle's row in shared memory)
//   k_particle        per particle (one warp; k_particle_stream for 3-D clouds):
//                     positivity repair, MOOD PAD/NAD
//                     screen with linear redo, diffuse wall or moments + BGK
//                     collision + moments, without the global rescale
//   k_sigma           deterministic mass sums -> global rescale sigma
//   k_scale_mood      sigma on the macros, moodCheck
//   k_recollide       second collision when moodCheck failed (else exits)
//   k_mass_end        end-of-step mass after a second collision (else exits)
// k_batch_* run the same stage bodies for a batch of clouds, one launch per
// stage over all of them (a block finds its cloud from block offsets).
// The stored state h is the true distribution divided by StepScalars::scale.
// All reductions are FP64 and in a fixed order, so a step is bitwise
// reproducible.  No kernel waits on another block, so none can hang.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "ctx.h"
#include "mbar.cuh"

namespace alebgk {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kNT = 256;   // threads per particle block

__device__ __forceinline__ double warpSum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warpMin(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ double warpMax(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sums K values over the block in a fixed order; every thread receives the
// totals.  sh must hold K * (NT/32) doubles.
template <int K>
__device__ __forceinline__ void blockSums(double (&v)[K], double *sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) v[q] = warpSum(v[q]);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < K; ++q) sh[q * 32 + wid] = v[q];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < K; ++q)
    {
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += sh[q * 32 + w];
        v[q] = s;
    }
    __syncthreads();
}

// Node index -> velocity (iv fastest, MLSTransport.cpp:142).
__device__ __forceinline__ void nodeVel(int k, int Nv, int dim, double vmin,
                                        double dv, double &vx, double &vy,
                                        double &vz)
{
    int iv = k % Nv, jv = (k / Nv) % Nv, kv = (dim == 3) ? k / (Nv * Nv) : 0;
    vx = fma((double)iv, dv, vmin);
    vy = fma((double)jv, dv, vmin);
    vz = (dim == 3) ? fma((double)kv, dv, vmin) : 0.0;
}

// Wall-normal velocity (v - U_w).n in the FMA-contracted form the reference's
// -O3 -march=native build evaluates in its wall loops
// (BoundaryConditions/DiffuseWall.cpp:58,83,110,133): only the x-term is
// fused.  The form decides the exact ties cn = 0 of edge and corner particles.
__device__ __forceinline__ double bcCn(int dim, double vx, double vy, double vz,
                                       const double *w)
{
    double c = fma(vx - w[3], w[0], (vy - w[4]) * w[1]);
    if (dim == 3) c = __dadd_rn(c, __dmul_rn(vz - w[5], w[2]));
    return c;
}

__device__ __forceinline__ double minImage(double d, double L)
{
    return d - L * round(d / L);
}

}  // namespace

// ---------------------------------------------------------------------------
// Transport: coefficient gather.  Warp = one particle and one chunk of its
// velocity nodes; lane = nodes k = k0 + lane + 32 q for q < qn <= kTransportQ,
// so one slot's row index and coefficient row serve qn nodes per lane and
// qn (or 2 qn in 2-D) independent loads are in flight per slot.  The node's
// coefficients are shared by both Chu layers in 2-D.  Every node sums its
// slots in slot order, whatever the chunking.  The output is scaled by the
// stored-state scale so that gt carries the true magnitude.
// ---------------------------------------------------------------------------
constexpr int kTransportQ = 8;

// Chunks of a row: the 32-node groups of V split as evenly as possible into
// chunks of at most kTransportQ groups.
__host__ __device__ __forceinline__ int transportChunks(int V)
{
    const int groups = (V + 31) / 32;
    return (groups + kTransportQ - 1) / kTransportQ;
}

// Accumulates the slots of one chunk of a row: nodes k0 + 32 q for q < qn
// (k0 = first node of the chunk + lane), both Chu layers when L = 2.
template <typename T, int L>
__device__ __forceinline__ void gatherChunk(const T *__restrict__ f, const T *__restrict__ cc,
                                            const int *__restrict__ sl, int ns, int V, int ldf,
                                            int k0, int qn, T (&a0)[kTransportQ],
                                            T (&a1)[kTransportQ])
{
#pragma unroll
    for (int q = 0; q < kTransportQ; ++q) { a0[q] = T(0); a1[q] = T(0); }
    // the lanes past V in the last group neither load nor store
    const bool tail = k0 + 32 * (qn - 1) >= V;
    for (int s = 0; s < ns; ++s)
    {
        const T *cs = cc + (size_t)s * V;
        const T *fr = f + (size_t)__ldg(sl + s) * ldf + k0;
#pragma unroll
        for (int q = 0; q < kTransportQ; ++q)
        {
            if (q < qn && (!tail || k0 + 32 * q < V))
            {
                const T w = __ldg(cs + 32 * q);
                a0[q] = fma(w, __ldg(fr + 32 * q), a0[q]);
                if (L == 2) a1[q] = fma(w, __ldg(fr + V + 32 * q), a1[q]);
            }
        }
    }
}

// One chunk of particle i's transported row, stored to out = row of g.
template <typename T, int L>
__device__ __forceinline__ void transportRow(const T *__restrict__ f, T *__restrict__ g,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int V, int ldf, T scale, int i, int chunk, int nch, int lane)
{
    const int groups = (V + 31) / 32;
    const int per = (groups + nch - 1) / nch;
    const int g0 = chunk * per;
    const int qn = min(per, groups - g0);        // warp-uniform
    if (qn <= 0) return;
    const int k0 = g0 * 32 + lane;
    const int c = __ldg(cls + i), ns = __ldg(nslot + i);
    T a0[kTransportQ], a1[kTransportQ];
    gatherChunk<T, L>(f, coef + (size_t)c * S * V + k0, slots + (size_t)i * S, ns, V, ldf, k0,
                      qn, a0, a1);
    T *out = g + (size_t)i * ldf + k0;
#pragma unroll
    for (int q = 0; q < kTransportQ; ++q)
    {
        if (q < qn && k0 + 32 * q < V)
        {
            out[32 * q] = a0[q] * scale;
            if (L == 2) out[V + 32 * q] = a1[q] * scale;
        }
    }
}

// Particle i's whole transported row into a warp's shared-memory row copy
// (the fused transport of the particle kernel): the same sums as
// transportRow, chunk by chunk.
template <typename T, int L>
__device__ __forceinline__ void transportRowShared(const T *__restrict__ f, T *__restrict__ buf,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int V, int ldf, T scale, int i, int lane)
{
    const int groups = (V + 31) / 32;
    const int nch = transportChunks(V);
    const int per = (groups + nch - 1) / nch;
    const int c = __ldg(cls + i), ns = __ldg(nslot + i);
    const T *cc = coef + (size_t)c * S * V;
    const int *sl = slots + (size_t)i * S;
    for (int g0 = 0; g0 < groups; g0 += per)
    {
        const int qn = min(per, groups - g0);
        const int k0 = g0 * 32 + lane;
        T a0[kTransportQ], a1[kTransportQ];
        gatherChunk<T, L>(f, cc + k0, sl, ns, V, ldf, k0, qn, a0, a1);
#pragma unroll
        for (int q = 0; q < kTransportQ; ++q)
        {
            if (q < qn && k0 + 32 * q < V)
            {
                buf[k0 + 32 * q] = a0[q] * scale;
                if (L == 2) buf[V + k0 + 32 * q] = a1[q] * scale;
            }
        }
    }
    __syncwarp();
}

// Block = consecutive particles, one per warp, at one velocity chunk: the
// particles share most of their neighbours, so the block's gathers of
// neighbour rows hit L1 after the first.
template <typename T>
__device__ __forceinline__ void k_transport_body(const T *__restrict__ f, T *__restrict__ g,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int N, int V, int L, int ldf, const StepScalars *__restrict__ sc, int chunk,
            int tile)
{
    const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int i = tile * nw + warp;
    if (i >= N) return;
    const T scale = T(sc->scale);
    const int nch = transportChunks(V);
    if (L == 2)
        transportRow<T, 2>(f, g, coef, cls, nslot, slots, S, V, ldf, scale, i, chunk, nch,
                           threadIdx.x & 31);
    else
        transportRow<T, 1>(f, g, coef, cls, nslot, slots, S, V, ldf, scale, i, chunk, nch,
                           threadIdx.x & 31);
}

// Grid (velocity chunks, particle tiles of blockDim.x / 32).
template <typename T>
__global__ void __launch_bounds__(kNT)
k_transport(const T *__restrict__ f, T *__restrict__ g,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int N, int V, int L, int ldf, const StepScalars *__restrict__ sc)
{
    k_transport_body(f, g, coef, cls, nslot, slots, S, N, V, L, ldf, sc, blockIdx.x, blockIdx.y);
}

// Walks the nodes k = lane, lane + 32, ... of a particle row and keeps the
// node's grid indices (iv fastest, MLSTransport.cpp:142) without divisions.
struct NodeWalk
{
    int iv, jv, kv, k;
    int dI, dJ, dK, Nv;
    __device__ NodeWalk(int k0, int Nv_, int dim) : k(k0), Nv(Nv_)
    {
        iv = k0 % Nv; jv = (k0 / Nv) % Nv; kv = (dim == 3) ? k0 / (Nv * Nv) : 0;
        dI = 32 % Nv; dJ = (32 / Nv) % Nv; dK = (dim == 3) ? 32 / (Nv * Nv) : 0;
    }
    __device__ void next()
    {
        k += 32;
        iv += dI;
        int c = iv >= Nv;
        iv -= c * Nv;
        jv += dJ + c;
        c = jv >= Nv;
        jv -= c * Nv;
        kv += dK + c;
    }
};

constexpr int kMaxNv = 48;    // Core/Types.hpp:16 (MAX_NV)

// Positivity repair (MLSTransport.cpp:189-200 in 3-D, 283-309 in 2-D) of a
// transported row, as sums: returns pos, neg and whether any value is not
// finite.  The repair itself is applied lazily through posv().
template <typename T>
__device__ __forceinline__ void rowSigns(const T *row, int V, int lane,
                                         double &pos, double &neg, bool &bad)
{
    double p = 0.0, n = 0.0;
    int b = 0;
    for (int k = lane; k < V; k += 32)
    {
        double v = (double)row[k];
        b |= !isfinite(v);
        if (v >= 0.0) p += v; else n += v;
    }
    pos = warpSum(p);
    neg = warpSum(n);
    bad = __any_sync(0xffffffffu, b) != 0;
}

struct Positivity
{
    bool fix;
    double s;
    __device__ Positivity(double pos, double neg)
    {
        fix = (neg < -1.0e-30 && pos > 1.0e-30 && (pos + neg) > 0.0);
        s = fix ? (pos + neg) / pos : 1.0;
    }
    // g1 layer value, and the g2 value whose fate follows the g1 sign.
    __device__ __forceinline__ double v1(double g1) const
    {
        return fix ? (g1 < 0.0 ? 0.0 : g1 * s) : g1;
    }
    __device__ __forceinline__ double v2(double g1, double g2) const
    {
        return fix ? (g1 < 0.0 ? 0.0 : g2 * s) : g2;
    }
};

// Per-particle arguments of the stages after transport.
template <typename T>
struct ParticleArgs
{
    T *g;                     // in: gt (true scale); out: h (unscaled by sigma)
    const T *fold;            // previous stored h (scale sc->scale)
    const T *coef;            // MLS tables (the fused transport)
    const T *coefLin;         // linear MLS tables (MOOD redo)
    const int *boundary, *cls, *nslot, *slots;
    const double *wall, *macPrev;
    double *macNew, *massPos, *massEnd, *minG, *dpx;
    const double *nad;        // NAD neighbour density range (lo, hi) per particle
    int *flag, *flagList, *degList;
    StepScalars *sc;
    const int *rowOrder;      // visiting order of the row kernel
};

// A particle row staged in shared memory for the passes of one warp: loaded
// once with coalesced loads (many in flight per lane), then every pass reads
// and writes the copy, and flush() stores it back.
template <typename T, int L>
struct RowRegs
{
    T *buf;
    T *row;
    int V, lane;

    __device__ RowRegs(T *row_, T *buf_, const StepParams &p, int lane_)
        : buf(buf_), row(row_), V(p.V), lane(lane_)
    {
        const int n = L * V;
#pragma unroll 8
        for (int k = lane; k < n; k += 32) buf[k] = row[k];
        __syncwarp();
    }
    // Over a copy that is already staged in buf.
    __device__ RowRegs(T *row_, T *buf_, const StepParams &p, int lane_, bool)
        : buf(buf_), row(row_), V(p.V), lane(lane_)
    {
    }
    // Calls f(k, iv, jv, kv, g1&, g2&) for every node of the row.
    template <typename F>
    __device__ __forceinline__ void pass(const StepParams &p, bool, F &&f)
    {
        for (NodeWalk nw(lane, p.Nv, p.dim); nw.k < V; nw.next())
            f(nw.k, nw.iv, nw.jv, nw.kv, buf[nw.k], buf[L == 2 ? V + nw.k : nw.k]);
        __syncwarp();
    }
    __device__ __forceinline__ void flush()
    {
        const int n = L * V;
#pragma unroll 8
        for (int k = lane; k < n; k += 32) row[k] = buf[k];
    }
};

// Positivity repair sums (MLSTransport.cpp:189-200 in 3-D, 283-309 in 2-D)
// over the mass layer of a register row.
template <typename T, int L>
__device__ __forceinline__ void regSigns(RowRegs<T, L> &r, const StepParams &p,
                                         double &pos, double &neg, bool &bad)
{
    double ps = 0.0, ng = 0.0;
    int b = 0;
    r.pass(p, false, [&](int, int, int, int, T &g1, T &) {
        double v = (double)g1;
        b |= !isfinite(v);
        if (v >= 0.0) ps += v; else ng += v;
    });
    pos = warpSum(ps);
    neg = warpSum(ng);
    bad = __any_sync(0xffffffffu, b) != 0;
}

// Finishes one particle on one warp after its positivity decision: diffuse
// wall (BoundaryConditions/DiffuseWall.cpp:19-154) or moments + implicit BGK
// collision + moments (Moments.cpp:17-97, Collision.cpp:70-139).  The global
// rescale sigma of the step is not known yet; every operation here is
// homogeneous of degree one in g, so the row is finished without it and
// sigma is applied afterwards (k_scale_mood).  The exception is an interior
// particle whose repaired row has no positive mass: the reference then keeps
// its previous (absolute) macros, which breaks homogeneity, so the particle
// is left untouched, listed, and finished by k_fixup once sigma is known.
// Maxwellians are evaluated as products of per-axis exponentials.
// With flushDeferred the row of a deferred particle is written back first
// (its staged copy was never in g: the fused transport built it in place).
template <typename T, int L>
__device__ void finishParticle(const ParticleArgs<T> &a, const StepParams &p, int i,
                               RowRegs<T, L> &r, const Positivity &pv, double (*tb)[kMaxNv],
                               bool flushDeferred = false)
{
    const int lane = r.lane;
    const int Nv = p.Nv, dim = p.dim;
    double *mac = a.macNew + 6 * (size_t)i;
    const double *mp = a.macPrev + 6 * (size_t)i;
    auto vel = [&](int q) { return fma((double)q, p.dv, p.vmin); };

    if (a.boundary[i])
    {
        const double *w = a.wall + 7 * (size_t)i;
        const double Ux = w[3], Uy = w[4], Uz = w[5], Tw = w[6];
        const double RT2w = 2.0 * p.R * Tw;
        const double norm = (dim == 3) ? pow(kPi * RT2w, 1.5) : kPi * RT2w;
        for (int q = lane; q < Nv; q += 32)
        {
            double va = vel(q);
            tb[0][q] = exp(-(va - Ux) * (va - Ux) / RT2w) / norm;
            tb[1][q] = exp(-(va - Uy) * (va - Uy) / RT2w);
            tb[2][q] = (dim == 3) ? exp(-(va - Uz) * (va - Uz) / RT2w) : 1.0;
        }
        __syncwarp();
        double iM = 0.0, iP = 0.0;
        r.pass(p, false, [&](int, int iv, int jv, int kv, T &g1, T &) {
            const double cn = bcCn(dim, vel(iv), vel(jv), (dim == 3) ? vel(kv) : 0.0, w);
            if (cn < 0.0) iM += cn * pv.v1((double)g1) * p.dvN;
            else if (cn > 0.0) iP += cn * (tb[0][iv] * tb[1][jv] * tb[2][kv]) * p.dvN;
        });
        iM = warpSum(iM);
        iP = warpSum(iP);
        const double rhow = (iP > 1.0e-30) ? (-iM / iP) : 1.0;
        double dp = 0.0, ms = 0.0;
        r.pass(p, true, [&](int, int iv, int jv, int kv, T &g1, T &g2) {
            const double vx = vel(iv);
            const double cn = bcCn(dim, vx, vel(jv), (dim == 3) ? vel(kv) : 0.0, w);
            const double x1 = (double)g1;
            double h1 = pv.v1(x1);
            double h2 = (L == 2) ? pv.v2(x1, (double)g2) : 0.0;
            if (cn > 0.0)
            {
                const double Mw = rhow * (tb[0][iv] * tb[1][jv] * tb[2][kv]);
                dp += vx * (Mw - h1) * p.dvN;
                h1 = Mw;
                h2 = 0.5 * p.R * Tw * Mw;
            }
            g1 = T(h1);
            ms += (double)g1;
            if (L == 2) g2 = T(h2);
        });
        r.flush();
        dp = warpSum(dp);
        ms = warpSum(ms);
        if (lane == 0)
        {
            mac[0] = rhow; mac[1] = Ux; mac[2] = Uy;
            mac[3] = (dim == 3) ? Uz : mp[3];
            mac[4] = Tw; mac[5] = rhow * p.R * Tw;
            a.dpx[i] = dp;
            a.massEnd[i] = ms * p.dvN;
            a.minG[i] = 0.0;
        }
        return;
    }

    // Interior: moments of the repaired row.
    double M0 = 0, Mx = 0, My = 0, Mz = 0, ME = 0;
    r.pass(p, false, [&](int, int iv, int jv, int kv, T &g1, T &g2) {
        const double vx = vel(iv), vy = vel(jv), vz = (dim == 3) ? vel(kv) : 0.0;
        const double x1 = (double)g1;
        const double f1 = pv.v1(x1) * p.dvN;
        M0 += f1; Mx += vx * f1; My += vy * f1; Mz += vz * f1;
        ME += (vx * vx + vy * vy + vz * vz) * f1;
        if (L == 2) ME += 2.0 * pv.v2(x1, (double)g2) * p.dvN;
    });
    M0 = warpSum(M0); Mx = warpSum(Mx); My = warpSum(My); Mz = warpSum(Mz); ME = warpSum(ME);
    if (!(M0 > 1.0e-30) || p.tauVar)
    {
        // No positive mass (macros kept from the previous step), or a
        // relaxation time tau(rho, T) that is not homogeneous in rho: the
        // particle is finished on true magnitudes once sigma is known.
        if (flushDeferred) r.flush();
        if (lane == 0) a.degList[atomicAdd(&a.sc->ndeg, 1)] = i;
        return;
    }
    const double rho = M0, ux = Mx / M0, uy = My / M0;
    const double uz = (dim == 3) ? Mz / M0 : mp[3];
    const double Tt = fmax((ME / M0 - (ux * ux + uy * uy + uz * uz)) / (3.0 * p.R), 1.0e-6);
    const double lam = p.dt / p.tau;
    const double c1 = 1.0 / (1.0 + lam);
    const double twoRT = 2.0 * p.R * Tt;
    const double A = (dim == 3) ? rho / pow(kPi * twoRT, 1.5) : rho / (kPi * twoRT);
    for (int q = lane; q < Nv; q += 32)
    {
        double va = vel(q);
        tb[0][q] = lam * A * exp(-(va - ux) * (va - ux) / twoRT);
        tb[1][q] = exp(-(va - uy) * (va - uy) / twoRT);
        tb[2][q] = (dim == 3) ? exp(-(va - uz) * (va - uz) / twoRT) : 1.0;
    }
    __syncwarp();
    double N0 = 0, Nx = 0, Ny = 0, Nz = 0, NE = 0, mn = INFINITY;
    const double halfRT = 0.5 * p.R * Tt;
    r.pass(p, true, [&](int, int iv, int jv, int kv, T &g1, T &g2) {
        const double vx = vel(iv), vy = vel(jv), vz = (dim == 3) ? vel(kv) : 0.0;
        const double x1 = (double)g1;
        const double lM = tb[0][iv] * tb[1][jv] * tb[2][kv];
        const T h1s = T(c1 * (pv.v1(x1) + lM));
        const double f1 = (double)h1s * p.dvN;
        N0 += f1; Nx += vx * f1; Ny += vy * f1; Nz += vz * f1;
        NE += (vx * vx + vy * vy + vz * vz) * f1;
        mn = fmin(mn, (double)h1s);
        if (L == 2)
        {
            const T h2s = T(c1 * (pv.v2(x1, (double)g2) + halfRT * lM));
            NE += 2.0 * (double)h2s * p.dvN;
            g2 = h2s;
        }
        g1 = h1s;
    });
    r.flush();
    N0 = warpSum(N0); Nx = warpSum(Nx); Ny = warpSum(Ny); Nz = warpSum(Nz); NE = warpSum(NE);
    mn = warpMin(mn);
    if (lane == 0)
    {
        double r2 = rho, x2 = ux, y2 = uy, z2 = uz, T2 = Tt;
        if (N0 > 1.0e-30)
        {
            r2 = N0; x2 = Nx / N0; y2 = Ny / N0;
            z2 = (dim == 3) ? Nz / N0 : uz;
            T2 = fmax((NE / N0 - (x2 * x2 + y2 * y2 + z2 * z2)) / (3.0 * p.R), 1.0e-6);
        }
        mac[0] = r2; mac[1] = x2; mac[2] = y2; mac[3] = z2; mac[4] = T2;
        mac[5] = r2 * p.R * T2;
        a.dpx[i] = 0.0;
        a.massEnd[i] = N0;
        a.minG[i] = mn;
    }
}

// MOOD PAD/NAD screen of one transported row (MLSTransport.cpp:325-379)
// against the neighbours' pre-transport densities.  Returns 1 if flagged.
template <typename T>
__device__ int screen(const ParticleArgs<T> &a, const StepParams &p, int i, int lane,
                      double m, bool bad)
{
    if (p.limiter != 2 || a.boundary[i]) return 0;
    if (bad || m <= 0.0) return 1;
    const int ns = a.nslot[i];
    const int *sl = a.slots + (size_t)i * p.S;
    double lo = INFINITY, hi = -INFINITY;
    for (int s = 1 + lane; s < ns; s += 32)
    {
        double rr = a.macPrev[6 * (size_t)sl[s]];
        lo = fmin(lo, rr);
        hi = fmax(hi, rr);
    }
    lo = warpMin(lo);
    hi = warpMax(hi);
    if (isfinite(lo) && isfinite(hi))
    {
        double rn = m * p.dvN;
        double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9 +
                       p.nadNoise * fmax(fabs(lo), fabs(hi));
        if (rn < lo - slack || rn > hi + slack) return 1;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Positivity + MOOD screen + finish, one warp per particle.  A particle the
// screen flags is listed for k_redo and left as is.  Fused: the warp first
// builds the particle's transported row in its shared-memory copy
// (transportRowShared, the sums of k_transport) instead of loading it from
// g; a flagged particle's row is then not stored (k_redo rebuilds it), a
// deferred one's is.
// ---------------------------------------------------------------------------
template <typename T, int L, bool Fused = false>
__device__ __forceinline__ void k_particle_body(const ParticleArgs<T> &a, const StepParams &p,
                                                int warpsPerBlock, int bx)
{
    __shared__ double tab[kNT / 32][3][kMaxNv];
    extern __shared__ __align__(16) unsigned char rowSmem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= warpsPerBlock) return;
    const int i = bx * warpsPerBlock + warp;
    if (i >= p.N) return;                        // warp-uniform
    T *buf = reinterpret_cast<T *>(rowSmem) + (size_t)warp * L * p.V;
    if (Fused)
        transportRowShared<T, L>(a.fold, buf, a.coef, a.cls, a.nslot, a.slots, p.S, p.V, p.ldf,
                                 T(a.sc->scale), i, lane);
    RowRegs<T, L> r = Fused ? RowRegs<T, L>(a.g + (size_t)i * p.ldf, buf, p, lane, true)
                            : RowRegs<T, L>(a.g + (size_t)i * p.ldf, buf, p, lane);
    double pos, neg;
    bool bad;
    regSigns(r, p, pos, neg, bad);
    const double m = pos + neg;
    const Positivity pv(pos, neg);
    const int flagged = screen(a, p, i, lane, m, bad);
    if (lane == 0)
    {
        a.flag[i] = flagged;
        if (pv.fix) atomicAdd(&a.sc->nfix, 1);
        if (flagged) a.flagList[atomicAdd(&a.sc->nflag, 1)] = i;
        else a.massPos[i] = m * p.dvN;
    }
    if (flagged) return;
    finishParticle(a, p, i, r, pv, tab[warp], Fused);
}

template <typename T, int L, bool Fused>
__global__ void __launch_bounds__(kNT)
k_particle(ParticleArgs<T> a, StepParams p, int warpsPerBlock)
{
    k_particle_body<T, L, Fused>(a, p, warpsPerBlock, blockIdx.x);
}

// ---------------------------------------------------------------------------
// The same stages for a 3-D single-layer cloud, streamed: persistent warps
// take particles i = w, w + W, ...; each warp double-buffers its particles'
// rows in shared memory with one bulk copy per row (the next row is in
// flight while the current one is processed).  Per node the velocity
// (vx, vy, vz, |v|^2) and the grid indices come from tables built once per
// block, and the NAD neighbour density range comes from k_step_begin.  An
// interior row takes two passes:
//   1. positivity sums and the moments of the row,
//   2. the implicit BGK collision h = (g + lam M) / (1 + lam), written out.
// The post-collision moments are not summed over the row: by linearity they
// are c1 (moments of g + lam * moments of M), and the moments of the
// separable discrete Maxwellian are products of per-axis sums over Nv nodes
// (Collision.cpp:70-139 then Moments.cpp:17-97 give the same numbers up to
// rounding).  Each lane sums its nodes in the storage type T -- at most
// ceil(V/32) terms -- and the lanes' sums are combined in FP64.  Wall
// particles take finishParticle on the staged row.
// ---------------------------------------------------------------------------

// Node velocity table of the streamed kernel, in the storage type.
template <typename T> struct VelNode;
template <> struct __align__(16) VelNode<float>
{
    float vx, vy, vz, v2;
};
template <> struct __align__(16) VelNode<double>
{
    double vx, vy, vz, v2;
};

// Shared-memory layout of k_particle_stream: velocity table, node index
// table, then two rows per warp.
template <typename T>
__host__ __device__ inline size_t streamRowsOffset(int V)
{
    return ((size_t)V * (sizeof(VelNode<T>) + sizeof(int)) + 127) / 128 * 128;
}

template <typename T>
__host__ __device__ inline size_t streamSmemBytes(int V, int ldf, int wpb)
{
    return streamRowsOffset<T>(V) + (size_t)wpb * 2 * ldf * sizeof(T);
}

// Sums K <= 8 values over the warp with 9 shuffle rounds instead of 5K:
// each round halves the set a lane keeps and adds its partner's other half.
// Every lane receives all K totals.
template <int K>
__device__ __forceinline__ void warpSumMany(double (&v)[K], int lane)
{
    static_assert(K >= 1 && K <= 8, "up to eight values");
    double w[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) w[q] = q < K ? v[q] : 0.0;
#pragma unroll
    for (int half = 4, bit = 16; half >= 1; half >>= 1, bit >>= 1)
    {
        const bool up = (lane & bit) != 0;
#pragma unroll
        for (int q = 0; q < half; ++q)
        {
            const double keep = up ? w[q + half] : w[q];
            const double give = up ? w[q] : w[q + half];
            w[q] = keep + __shfl_xor_sync(0xffffffffu, give, bit);
        }
    }
    // w[0] now holds value index (b4 b3 b2 of the lane) summed over the lanes
    // that share those bits; finish over bits 1 and 0.
    w[0] += __shfl_xor_sync(0xffffffffu, w[0], 2);
    w[0] += __shfl_xor_sync(0xffffffffu, w[0], 1);
#pragma unroll
    for (int q = 0; q < K; ++q)
    {
        const int src = ((q >> 2) & 1) << 4 | ((q >> 1) & 1) << 3 | (q & 1) << 2;
        v[q] = __shfl_sync(0xffffffffu, w[0], src);
    }
}

// NAD neighbour density range of every interior particle
// (MLSTransport.cpp:325-379) from the previous step's macros, one warp per
// particle; the streamed particle kernel reads it instead of gathering.
__device__ void nadRanges(const double *__restrict__ macPrev, const int *__restrict__ boundary,
                          const int *__restrict__ nslot, const int *__restrict__ slots,
                          int S, int N, double *__restrict__ nad)
{
    const int lane = threadIdx.x & 31;
    const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = w0; i < N; i += nw)
    {
        if (boundary[i]) continue;
        double lo = INFINITY, hi = -INFINITY;
        const int ns = nslot[i];
        const int *sl = slots + (size_t)i * S;
        for (int s = 1 + lane; s < ns; s += 32)
        {
            const double rr = macPrev[6 * (size_t)sl[s]];
            lo = fmin(lo, rr);
            hi = fmax(hi, rr);
        }
        lo = warpMin(lo);
        hi = warpMax(hi);
        if (lane == 0)
        {
            nad[2 * (size_t)i] = lo;
            nad[2 * (size_t)i + 1] = hi;
        }
    }
}

// Diffuse wall (BoundaryConditions/DiffuseWall.cpp:19-154) of a staged 3-D
// row, as finishParticle's wall branch computes it, with the node velocities
// read from the exact FP64 per-axis table velD and no divergent branches.
// The wall-normal velocity keeps the reference's contracted form (bcCn),
// which decides the cn = 0 ties.
template <typename T>
__device__ __forceinline__ void finishWallStream(const ParticleArgs<T> &a, const StepParams &p,
                                                 int i, const T *row, const int *idxT,
                                                 const double *velD, const Positivity &pv,
                                                 double (*tb)[kMaxNv], int lane)
{
    const double *w = a.wall + 7 * (size_t)i;
    const double Ux = w[3], Uy = w[4], Uz = w[5], Tw = w[6];
    const double RT2w = 2.0 * p.R * Tw;
    const double norm = pow(kPi * RT2w, 1.5);
    const double dvN = p.dvN;
    for (int q = lane; q < p.Nv; q += 32)
    {
        const double va = velD[q];
        tb[0][q] = exp(-(va - Ux) * (va - Ux) / RT2w) / norm;
        tb[1][q] = exp(-(va - Uy) * (va - Uy) / RT2w);
        tb[2][q] = exp(-(va - Uz) * (va - Uz) / RT2w);
    }
    __syncwarp();
    double iM[2] = {0, 0}, iP[2] = {0, 0};
    auto passA = [&](int u, int k) {
        const int id = idxT[k];
        const int iv = id & 255, jv = (id >> 8) & 255, kv = id >> 16;
        const double cn = bcCn(3, velD[iv], velD[jv], velD[kv], w);
        const double x = pv.v1((double)row[k]);
        const double mw = tb[0][iv] * tb[1][jv] * tb[2][kv];
        iM[u] += cn < 0.0 ? cn * x * dvN : 0.0;
        iP[u] += cn > 0.0 ? cn * mw * dvN : 0.0;
    };
    int k1 = lane;
#pragma unroll 2
    for (; k1 + 32 < p.V; k1 += 64)
    {
        passA(0, k1);
        passA(1, k1 + 32);
    }
    if (k1 < p.V) passA(0, k1);
    double r[2] = {iM[0] + iM[1], iP[0] + iP[1]};
    warpSumMany<2>(r, lane);
    const double rhow = (r[1] > 1.0e-30) ? (-r[0] / r[1]) : 1.0;
    T *gout = a.g + (size_t)i * p.ldf;
    double dp[2] = {0, 0}, ms[2] = {0, 0};
    auto passB = [&](int u, int k) {
        const int id = idxT[k];
        const int iv = id & 255, jv = (id >> 8) & 255, kv = id >> 16;
        const double vx = velD[iv];
        const double cn = bcCn(3, vx, velD[jv], velD[kv], w);
        const double h1 = pv.v1((double)row[k]);
        const double Mw = rhow * (tb[0][iv] * tb[1][jv] * tb[2][kv]);
        dp[u] += cn > 0.0 ? vx * (Mw - h1) * dvN : 0.0;
        const T g1 = T(cn > 0.0 ? Mw : h1);
        gout[k] = g1;
        ms[u] += (double)g1;
    };
    k1 = lane;
#pragma unroll 2
    for (; k1 + 32 < p.V; k1 += 64)
    {
        passB(0, k1);
        passB(1, k1 + 32);
    }
    if (k1 < p.V) passB(0, k1);
    double r2[2] = {dp[0] + dp[1], ms[0] + ms[1]};
    warpSumMany<2>(r2, lane);
    if (lane == 0)
    {
        double *mac = a.macNew + 6 * (size_t)i;
        mac[0] = rhow; mac[1] = Ux; mac[2] = Uy; mac[3] = Uz;
        mac[4] = Tw; mac[5] = rhow * p.R * Tw;
        a.dpx[i] = r2[0];
        a.massEnd[i] = r2[1] * dvN;
        a.minG[i] = 0.0;
    }
}

template <typename T>
__global__ void __launch_bounds__(kNT)
k_particle_stream(ParticleArgs<T> a, StepParams p, int wpb)
{
    __shared__ double tab[kNT / 32][3][kMaxNv];
    __shared__ float tabF[kNT / 32][sizeof(T) == 4 ? 3 : 1][kMaxNv];
    __shared__ double velD[kMaxNv];
    __shared__ __align__(8) uint64_t full[kNT / 32][2];
    extern __shared__ __align__(128) unsigned char streamSmem[];
    VelNode<T> *velT = reinterpret_cast<VelNode<T> *>(streamSmem);
    int *idxT = reinterpret_cast<int *>(velT + p.V);
    T *rows = reinterpret_cast<T *>(streamSmem + streamRowsOffset<T>(p.V));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int V = p.V, Nv = p.Nv;

    for (int k = threadIdx.x; k < V; k += blockDim.x)
    {
        const int iv = k % Nv, jv = (k / Nv) % Nv, kv = k / (Nv * Nv);
        const double vx = fma((double)iv, p.dv, p.vmin);
        const double vy = fma((double)jv, p.dv, p.vmin);
        const double vz = fma((double)kv, p.dv, p.vmin);
        velT[k] = VelNode<T>{T(vx), T(vy), T(vz), T(vx * vx + vy * vy + vz * vz)};
        idxT[k] = iv | jv << 8 | kv << 16;
    }
    for (int q = threadIdx.x; q < Nv; q += blockDim.x) velD[q] = fma((double)q, p.dv, p.vmin);
    if (lane == 0 && warp < wpb)
    {
        mbarInit(&full[warp][0], 1);
        mbarInit(&full[warp][1], 1);
        mbarInitFence();
    }
    __syncthreads();
    if (warp >= wpb) return;

    const int W = gridDim.x * wpb;
    int i = blockIdx.x * wpb + warp;
    auto rb = [&](int b) { return rows + (size_t)(2 * warp + b) * p.ldf; };
    const uint32_t rowBytes = (uint32_t)(p.ldf * sizeof(T));
    if (lane == 0 && i < p.N)
    {
        mbarExpectTx(&full[warp][0], rowBytes);
        bulkLoad(rb(0), a.g + (size_t)i * p.ldf, rowBytes, &full[warp][0]);
    }
    double(*tb)[kMaxNv] = tab[warp];
    // Maxwellian factors in T for the node loop: the double table itself,
    // or the warp's single-precision copy.
    T(*tt)[kMaxNv] = sizeof(T) == 4 ? reinterpret_cast<T(*)[kMaxNv]>(&tabF[warp][0][0])
                                    : reinterpret_cast<T(*)[kMaxNv]>(&tb[0][0]);
    const double dvN = p.dvN;
    bool dead = false;

    for (int it = 0; i < p.N; ++it, i += W)
    {
        const int b = it & 1;
        const int inext = i + W;
        if (lane == 0 && inext < p.N)
        {
            fenceProxyAsync();     // the warp's accesses to rb(b ^ 1) are done
            mbarExpectTx(&full[warp][b ^ 1], rowBytes);
            bulkLoad(rb(b ^ 1), a.g + (size_t)inext * p.ldf, rowBytes, &full[warp][b ^ 1]);
        }
        // Independent loads, first used after pass 1.
        const int wallI = a.boundary[i];
        const double2 nadI = p.limiter == 2 ? reinterpret_cast<const double2 *>(a.nad)[i]
                                            : make_double2(INFINITY, -INFINITY);

        mbarWait(&full[warp][b], (uint32_t)(it >> 1) & 1u, dead);
        if (__any_sync(0xffffffffu, dead))
        {
            // The row never arrived: report, let the other copy land, stop.
            if (lane == 0)
            {
                atomicOr(&a.sc->err, 4);
                bool d2 = false;
                if (inext < p.N) mbarWait(&full[warp][b ^ 1], (uint32_t)((it + 1) >> 1) & 1u, d2);
            }
            __syncwarp();
            return;
        }
        const T *row = rb(b);

        // Pass 1: positivity sums and moments of the transported row, two
        // interleaved partial sums per quantity.
        T s0[4] = {0, 0, 0, 0}, sn[4] = {0, 0, 0, 0}, mx[4] = {0, 0, 0, 0},
          my[4] = {0, 0, 0, 0}, mz[4] = {0, 0, 0, 0}, me[4] = {0, 0, 0, 0};
        auto acc = [&](int u, int k) {
            const T x = row[k];
            const VelNode<T> v = velT[k];
            s0[u] += x;
            sn[u] += x < T(0) ? x : T(0);
            mx[u] = fma(v.vx, x, mx[u]);
            my[u] = fma(v.vy, x, my[u]);
            mz[u] = fma(v.vz, x, mz[u]);
            me[u] = fma(v.v2, x, me[u]);
        };
        int k1 = lane;
        for (; k1 + 96 < V; k1 += 128)
        {
            acc(0, k1);
            acc(1, k1 + 32);
            acc(2, k1 + 64);
            acc(3, k1 + 96);
        }
        if (k1 < V) acc(0, k1);
        if (k1 + 32 < V) acc(1, k1 + 32);
        if (k1 + 64 < V) acc(2, k1 + 64);
        auto sum4 = [](const T (&v)[4]) {
            return ((double)v[0] + (double)v[1]) + ((double)v[2] + (double)v[3]);
        };
        double r1[6] = {sum4(s0), sum4(sn), sum4(mx), sum4(my), sum4(mz), sum4(me)};
        warpSumMany<6>(r1, lane);
        const bool wallP = wallI != 0;
        const bool screenP = p.limiter == 2 && !wallP;
        const double lo = nadI.x, hi = nadI.y;
        const bool bad = !isfinite(r1[0]) || !isfinite(r1[1]);
        const double pos = r1[0] - r1[1], neg = r1[1];
        const double m = pos + neg;
        const Positivity pv(pos, neg);
        int flagged = 0;
        if (screenP)
        {
            if (bad || m <= 0.0) flagged = 1;
            else if (isfinite(lo) && isfinite(hi))
            {
                const double rn = m * dvN;
                const double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9 +
                                     p.nadNoise * fmax(fabs(lo), fabs(hi));
                flagged = (rn < lo - slack || rn > hi + slack);
            }
        }
        if (lane == 0)
        {
            a.flag[i] = flagged;
            if (pv.fix) atomicAdd(&a.sc->nfix, 1);
            if (flagged) a.flagList[atomicAdd(&a.sc->nflag, 1)] = i;
            else a.massPos[i] = m * dvN;
        }
        if (flagged)
        {
            __syncwarp();
            continue;
        }
        if (wallP)
        {
            finishWallStream(a, p, i, row, idxT, velD, pv, tb, lane);
            __syncwarp();
            continue;
        }

        // Moments of the repaired row (Moments.cpp:17-97).
        double M0 = r1[0] * dvN, Mx = r1[2] * dvN, My = r1[3] * dvN, Mz = r1[4] * dvN,
               ME = r1[5] * dvN;
        if (pv.fix)
        {
            // Rare: the repair zeroes the negative nodes and scales the rest,
            // so the repaired moments are s times those of the positive part.
            T q[5] = {0, 0, 0, 0, 0};
            for (int k = lane; k < V; k += 32)
            {
                const T x = row[k] < T(0) ? T(0) : row[k];
                const VelNode<T> v = velT[k];
                q[0] += x;
                q[1] = fma(v.vx, x, q[1]);
                q[2] = fma(v.vy, x, q[2]);
                q[3] = fma(v.vz, x, q[3]);
                q[4] = fma(v.v2, x, q[4]);
            }
            double r2[5] = {(double)q[0], (double)q[1], (double)q[2], (double)q[3], (double)q[4]};
            warpSumMany<5>(r2, lane);
            const double f = pv.s * dvN;
            M0 = r2[0] * f; Mx = r2[1] * f; My = r2[2] * f; Mz = r2[3] * f; ME = r2[4] * f;
        }
        if (!(M0 > 1.0e-30) || p.tauVar)
        {
            if (lane == 0) a.degList[atomicAdd(&a.sc->ndeg, 1)] = i;
            __syncwarp();
            continue;
        }
        const double iM0 = 1.0 / M0;
        const double rho = M0, ux = Mx * iM0, uy = My * iM0, uz = Mz * iM0;
        const double Tt = fmax((ME * iM0 - (ux * ux + uy * uy + uz * uz)) * p.inv3R, 1.0e-6);
        const double lam = p.lam, c1 = p.c1;
        const double twoRT = 2.0 * p.R * Tt;
        const double piT = kPi * twoRT;
        const double A = rho / (piT * sqrt(piT));
        const double i2RT = 1.0 / twoRT;

        // Per-axis Maxwellian factors, one (axis, node) per lane, in FP64 and
        // in T for the node loop; then lane 3d + m sums velocity^m times the
        // axis-d factors over the Nv nodes.
        for (int j = lane; j < 3 * Nv; j += 32)
        {
            const int d = j / Nv, q = j - d * Nv;
            const double va = velD[q];
            const double u = d == 0 ? ux : (d == 1 ? uy : uz);
            const double e = (d == 0 ? lam * A : 1.0) * exp(-(va - u) * (va - u) * i2RT);
            tb[d][q] = e;
            tt[d][q] = T(e);
        }
        __syncwarp();
        double Sl = 0.0;
        if (lane < 9)
        {
            const int d = lane / 3, mom = lane - 3 * d;
            for (int q = 0; q < Nv; ++q)
            {
                const double va = velD[q], e = tb[d][q];
                Sl += mom == 0 ? e : (mom == 1 ? va * e : va * va * e);
            }
        }
        double S[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) S[j] = __shfl_sync(0xffffffffu, Sl, j);

        // Pass 2: collision, written straight to the distribution.
        T *gout = a.g + (size_t)i * p.ldf;
        const T c1t = T(c1), st = T(pv.s);
        T mn = T(INFINITY);
#pragma unroll 8
        for (int k = lane; k < V; k += 32)
        {
            const int id = idxT[k];
            const T lM = tt[0][id & 255] * tt[1][(id >> 8) & 255] * tt[2][id >> 16];
            T x = row[k];
            if (pv.fix) x = x < T(0) ? T(0) : x * st;
            const T h = c1t * (x + lM);
            mn = mn < h ? mn : h;
            gout[k] = h;
        }
        const double mnd = warpMin((double)mn);
        if (lane == 0)
        {
            const double N0 = c1 * (M0 + dvN * S[0] * S[3] * S[6]);
            const double Nx = c1 * (Mx + dvN * S[1] * S[3] * S[6]);
            const double Ny = c1 * (My + dvN * S[0] * S[4] * S[6]);
            const double Nz = c1 * (Mz + dvN * S[0] * S[3] * S[7]);
            const double NE = c1 * (ME + dvN * (S[2] * S[3] * S[6] + S[0] * S[5] * S[6] +
                                                S[0] * S[3] * S[8]));
            double r2 = rho, x2 = ux, y2 = uy, z2 = uz, T2 = Tt;
            if (N0 > 1.0e-30)
            {
                const double iN0 = 1.0 / N0;
                r2 = N0; x2 = Nx * iN0; y2 = Ny * iN0; z2 = Nz * iN0;
                T2 = fmax((NE * iN0 - (x2 * x2 + y2 * y2 + z2 * z2)) * p.inv3R, 1.0e-6);
            }
            double *mac = a.macNew + 6 * (size_t)i;
            mac[0] = r2; mac[1] = x2; mac[2] = y2; mac[3] = z2; mac[4] = T2;
            mac[5] = r2 * p.R * T2;
            a.dpx[i] = 0.0;
            a.massEnd[i] = N0;
            a.minG[i] = mnd;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// The same stages for a 3-D single-layer FP32 cloud with Nv = NV <= 10, the
// row held in registers: one warp per row (a persistent grid walks the
// rows).  A row of NV^3 velocities is NV^2 lines of NV contiguous values
// (fixed ky, kz; kx = 0..NV-1); lane l holds lines l, l + 32, ... .  One
// load of the row serves the whole stage:
//   - positivity sums and the moments of the positive part, in FP32 per lane
//     (the kx loop runs over compile-time velocity registers, the line's vy,
//     vz apply once per line), combined over the warp in FP64;
//   - the decisions and the Maxwellian's parameters, on every lane alike;
//   - the per-axis Maxwellian factors, one (axis, node) per lane in FP64,
//     and their per-axis moment sums by one warp reduction;
//   - the collision h = a max(g, lo) + c1 lam A ex ey ez written back, with
//     a = c1 s and lo = 0 when the repair fires, else a = c1 and lo = -inf;
//   - the macros of the collided row by linearity, as in k_particle_stream.
// Wall rows take the diffuse wall (finishWallStream) after their positivity
// sums.  The moments of the repaired row are those of the positive part
// (times the repair scale when the repair fires); without a repair any
// negative values sum to less than 1e-30 in magnitude (Positivity), below the
// rounding of the FP64 moments, and rows of no positive mass are deferred to
// k_fixup as before.
// ---------------------------------------------------------------------------
constexpr int kRowsThreads = 128;   // four warps per block of the register-row stage

// Lane l's lines l, l + 32, ... of a row of NV^3 values (zeros past the
// row's NV^2 lines).
template <int NV>
__device__ __forceinline__ void loadRowLines(const float *row, int lane,
                                             float (&x)[(NV * NV + 31) / 32][NV])
{
    constexpr int LINES = NV * NV, LPL = (LINES + 31) / 32;
#pragma unroll
    for (int j = 0; j < LPL; ++j)
    {
        const int L = lane + 32 * j;
        if (L < LINES)
        {
            const float *ln = row + L * NV;
            if constexpr (NV % 2 == 0)
            {
#pragma unroll
                for (int q = 0; q < NV; q += 2)
                {
                    const float2 v2 = *reinterpret_cast<const float2 *>(ln + q);
                    x[j][q] = v2.x;
                    x[j][q + 1] = v2.y;
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < NV; ++q) x[j][q] = ln[q];
            }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < NV; ++q) x[j][q] = 0.0f;
        }
    }
}

template <int NV>
__global__ void __launch_bounds__(kRowsThreads, 4)
k_particle_rows(ParticleArgs<float> a, StepParams p)
{
    constexpr int LINES = NV * NV;
    constexpr int LPL = (LINES + 31) / 32;       // lines per lane
    constexpr int V = NV * NV * NV;
    static_assert(NV <= 10 && 3 * NV <= 32, "rows of at most 10^3 velocities");
    __shared__ double wtab[kRowsThreads / 32][3][kMaxNv];  // diffuse-wall tables
    __shared__ double velD[kMaxNv];
    __shared__ float velF[kMaxNv];
    __shared__ int idxT[V];
    // Two staged rows per warp: the row being processed (the wall rows' flux
    // balance reads it from here) and the next one, arriving by one bulk copy.
    constexpr int LDF = (V + 3) / 4 * 4;
    __shared__ __align__(16) float rowBuf[kRowsThreads / 32][2][LDF];
    __shared__ __align__(8) uint64_t rowBar[kRowsThreads / 32][2];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
    {
        mbarInit(&rowBar[warp][0], 1);
        mbarInit(&rowBar[warp][1], 1);
        mbarInitFence();
    }
    for (int k = threadIdx.x; k < V; k += blockDim.x)
    {
        const int iv = k % NV, jv = (k / NV) % NV, kv = k / (NV * NV);
        idxT[k] = iv | jv << 8 | kv << 16;
    }
    for (int q = threadIdx.x; q < NV; q += blockDim.x)
    {
        velD[q] = fma((double)q, p.dv, p.vmin);
        velF[q] = (float)velD[q];
    }
    __syncthreads();
    float vx[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) vx[q] = velF[q];
    // this lane's axis node of the per-axis factors
    const int myAxis = lane / NV, myNode = lane - (lane / NV) * NV;
    const double myV = lane < 3 * NV ? velD[myNode] : 0.0;
    const double dvN = p.dvN, c1 = p.c1;
    const int W = gridDim.x * (blockDim.x >> 5);
    constexpr uint32_t kRowBytes = 4u * LDF;
    // The warp's rows: t, t + W, ...; the index, wall flag and screen range
    // of the next row are loaded one row ahead, and the next row itself is
    // staged into the other rowBuf by one bulk copy while the current row is
    // processed.
    int t = blockIdx.x * (blockDim.x >> 5) + warp;
    int inext = t < p.N ? a.rowOrder[t] : 0;
    int wallN = t < p.N ? a.boundary[inext] : 0;
    double2 nadN = (t < p.N && p.limiter == 2) ? reinterpret_cast<const double2 *>(a.nad)[inext]
                                                 : make_double2(INFINITY, -INFINITY);
    int inext2 = t + W < p.N ? a.rowOrder[t + W] : 0;
    if (lane == 0 && t < p.N)
    {
        mbarExpectTx(&rowBar[warp][0], kRowBytes);
        bulkLoad(&rowBuf[warp][0][0], a.g + (size_t)inext * p.ldf, kRowBytes, &rowBar[warp][0]);
    }
    bool dead = false;
    for (uint32_t it = 0; t < p.N; t += W, ++it)
    {
        const int i = inext;
        const int wallI = wallN;
        const double2 nadI = nadN;
        const bool more = t + W < p.N;
        inext = inext2;
        // loads for the next row, first used in the next iteration
        wallN = more ? a.boundary[inext] : 0;
        nadN = (more && p.limiter == 2) ? reinterpret_cast<const double2 *>(a.nad)[inext]
                                        : make_double2(INFINITY, -INFINITY);
        inext2 = t + 2 * W < p.N ? a.rowOrder[t + 2 * W] : 0;
        float *row = a.g + (size_t)i * p.ldf;
        float x[LPL][NV];
        const int b = it & 1;
        const uint32_t par = (it >> 1) & 1u;
        mbarWait(&rowBar[warp][b], par, dead);
        if (__any_sync(0xffffffffu, dead))
        {
            // The row never arrived: report, give the copy a second bounded
            // wait, stop.
            if (lane == 0)
            {
                atomicOr(&a.sc->err, 4);
                bool d2 = false;
                mbarWait(&rowBar[warp][b], par, d2);
            }
            __syncwarp();
            return;
        }
        loadRowLines<NV>(&rowBuf[warp][b][0], lane, x);
        __syncwarp();
        if (lane == 0 && more)
        {
            fenceProxyAsync();     // the warp's reads of the other buffer are done
            mbarExpectTx(&rowBar[warp][b ^ 1], kRowBytes);
            bulkLoad(&rowBuf[warp][b ^ 1][0], a.g + (size_t)inext * p.ldf, kRowBytes,
                     &rowBar[warp][b ^ 1]);
        }
        float s0 = 0.f, sn = 0.f, sx = 0.f, sy = 0.f, sz = 0.f, se = 0.f;
#pragma unroll
        for (int j = 0; j < LPL; ++j)
        {
            const int L = lane + 32 * j;
            float ls = 0.f, lx = 0.f, le = 0.f;
#pragma unroll
            for (int q = 0; q < NV; ++q)
            {
                const float xp = fmaxf(x[j][q], 0.0f);
                ls += xp;
                sn += fminf(x[j][q], 0.0f);
                lx = fmaf(vx[q], xp, lx);
                le = fmaf(vx[q] * vx[q], xp, le);
            }
            if (L < LINES)
            {
                const float vy = velF[L % NV], vz = velF[L / NV];
                s0 += ls;
                sx += lx;
                sy = fmaf(vy, ls, sy);
                sz = fmaf(vz, ls, sz);
                se += le + (vy * vy + vz * vz) * ls;
            }
        }
        double r6[6] = {(double)s0, (double)sn, (double)sx, (double)sy, (double)sz, (double)se};
        warpSumMany<6>(r6, lane);
        const double pos = r6[0], neg = r6[1];
        const bool bad = !isfinite(pos) || !isfinite(neg) || !isfinite(r6[5]);
        const double m = pos + neg;
        const Positivity pv(pos, neg);
        if (wallI)
        {
            if (lane == 0)
            {
                a.flag[i] = 0;
                if (pv.fix) atomicAdd(&a.sc->nfix, 1);
                a.massPos[i] = m * dvN;
            }
            finishWallStream(a, p, i, (const float *)&rowBuf[warp][b][0], idxT, velD, pv,
                             wtab[warp], lane);
            __syncwarp();
            continue;
        }
        int flagged = 0;
        if (p.limiter == 2)
        {
            const double2 nad = nadI;
            if (bad || m <= 0.0) flagged = 1;
            else if (isfinite(nad.x) && isfinite(nad.y))
            {
                const double rn = m * dvN;
                const double slack = 0.1 * fmax(nad.y - nad.x, 1.0e-12) + 1.0e-9 +
                                     p.nadNoise * fmax(fabs(nad.x), fabs(nad.y));
                flagged = (rn < nad.x - slack || rn > nad.y + slack);
            }
        }
        if (lane == 0)
        {
            a.flag[i] = flagged;
            if (pv.fix) atomicAdd(&a.sc->nfix, 1);
            if (flagged) a.flagList[atomicAdd(&a.sc->nflag, 1)] = i;
            else a.massPos[i] = m * dvN;
        }
        if (flagged) continue;
        // Moments of the repaired row (Moments.cpp:17-97): s times the
        // positive part's when the repair fires.
        const double f = (pv.fix ? pv.s : 1.0) * dvN;
        const double M0 = pv.fix ? pos * f : m * dvN;
        if (!(M0 > 1.0e-30) || p.tauVar)
        {
            if (lane == 0) a.degList[atomicAdd(&a.sc->ndeg, 1)] = i;
            continue;
        }
        const double iM0 = 1.0 / M0;
        const double Mx = r6[2] * f, My = r6[3] * f, Mz = r6[4] * f, ME = r6[5] * f;
        const double ux = Mx * iM0, uy = My * iM0, uz = Mz * iM0;
        const double Tt = fmax((ME * iM0 - (ux * ux + uy * uy + uz * uz)) * p.inv3R, 1.0e-6);
        const double twoRT = 2.0 * p.R * Tt;
        const double piT = kPi * twoRT;
        const double lamA = p.lam * M0 / (piT * sqrt(piT));
        // Per-axis factors: lane d NV + q holds axis d, node q; their
        // per-axis sums of velocity^0,1,2 by one reduction (eight values,
        // then the ninth).
        double e = 0.0;
        if (lane < 3 * NV)
        {
            const double u = myAxis == 0 ? ux : (myAxis == 1 ? uy : uz);
            e = (myAxis == 0 ? lamA : 1.0) * exp(-(myV - u) * (myV - u) / twoRT);
        }
        double S8[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            const int d = j / 3, pw = j - 3 * d;
            S8[j] = (lane < 3 * NV && myAxis == d)
                        ? (pw == 0 ? e : (pw == 1 ? myV * e : myV * myV * e)) : 0.0;
        }
        warpSumMany<8>(S8, lane);
        const double S22 = warpSum(lane < 3 * NV && myAxis == 2 ? myV * myV * e : 0.0);
        const float ef = (float)(lane < NV ? c1 * e : e);
        float ex[NV];
#pragma unroll
        for (int q = 0; q < NV; ++q) ex[q] = __shfl_sync(0xffffffffu, ef, q);
        const float am = (float)(c1 * (pv.fix ? pv.s : 1.0));
        const float lo = pv.fix ? 0.0f : -INFINITY;
        float mn = INFINITY;
#pragma unroll
        for (int j = 0; j < LPL; ++j)
        {
            const int L = lane + 32 * j;
            const int Lc = L < LINES ? L : 0;
            const float eyz = __shfl_sync(0xffffffffu, ef, NV + Lc % NV) *
                              __shfl_sync(0xffffffffu, ef, 2 * NV + Lc / NV);
            if (L < LINES)
            {
                float h[NV];
#pragma unroll
                for (int q = 0; q < NV; ++q)
                {
                    h[q] = fmaf(am, fmaxf(x[j][q], lo), ex[q] * eyz);
                    mn = fminf(mn, h[q]);
                }
                float *ln = row + L * NV;
                if constexpr (NV % 2 == 0)
                {
#pragma unroll
                    for (int q = 0; q < NV; q += 2)
                        *reinterpret_cast<float2 *>(ln + q) = make_float2(h[q], h[q + 1]);
                }
                else
                {
#pragma unroll
                    for (int q = 0; q < NV; ++q) ln[q] = h[q];
                }
            }
        }
        const double mnd = warpMin((double)mn);
        if (lane == 0)
        {
            const double *S = S8;
            const double N0 = c1 * (M0 + dvN * S[0] * S[3] * S[6]);
            const double Nx = c1 * (Mx + dvN * S[1] * S[3] * S[6]);
            const double Ny = c1 * (My + dvN * S[0] * S[4] * S[6]);
            const double Nz = c1 * (Mz + dvN * S[0] * S[3] * S[7]);
            const double NE = c1 * (ME + dvN * (S[2] * S[3] * S[6] + S[0] * S[5] * S[6] +
                                                S[0] * S[3] * S22));
            double r2 = M0, x2 = ux, y2 = uy, z2 = uz, T2 = Tt;
            if (N0 > 1.0e-30)
            {
                const double iN0 = 1.0 / N0;
                r2 = N0; x2 = Nx * iN0; y2 = Ny * iN0; z2 = Nz * iN0;
                T2 = fmax((NE * iN0 - (x2 * x2 + y2 * y2 + z2 * z2)) * p.inv3R, 1.0e-6);
            }
            double *mac = a.macNew + 6 * (size_t)i;
            mac[0] = r2; mac[1] = x2; mac[2] = y2; mac[3] = z2; mac[4] = T2;
            mac[5] = r2 * p.R * T2;
            a.dpx[i] = 0.0;
            a.massEnd[i] = N0;
            a.minG[i] = mnd;
        }
    }
}

// Launch of the register-row stage for the cloud's Nv (nullptr when no
// instance covers it).
typedef void (*RowsKernel)(ParticleArgs<float>, StepParams);
static RowsKernel rowsKernel(int Nv)
{
    switch (Nv)
    {
    case 4: return k_particle_rows<4>;
    case 5: return k_particle_rows<5>;
    case 6: return k_particle_rows<6>;
    case 8: return k_particle_rows<8>;
    case 10: return k_particle_rows<10>;
    default: return nullptr;
    }
}

// ---------------------------------------------------------------------------
// Linear MLS redo of the flagged particles (Solver/Solver.cpp:641-646:
// mlsTransportCompute(..., 1, onlyFlagged=true)) from the pre-transport
// state, one block per particle, then positivity and finish on warp 0.
// ---------------------------------------------------------------------------
template <typename T, int L>
__device__ __forceinline__ void k_redo_body(const ParticleArgs<T> &a, const StepParams &p, int bx,
                                            int gx)
{
    __shared__ double tab[3][kMaxNv];
    extern __shared__ __align__(16) unsigned char rowSmem[];
    const int nflag = a.sc->nflag;
    const T scale = T(a.sc->scale);
    for (int li = bx; li < nflag; li += gx)
    {
        const int i = a.flagList[li];
        const int ns = a.nslot[i];
        const int *sl = a.slots + (size_t)i * p.S;
        const T *cl = a.coefLin + (size_t)a.cls[i] * p.S * p.V;
        T *row = a.g + (size_t)i * p.ldf;
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            T a0 = T(0), a1 = T(0);
            for (int s = 0; s < ns; ++s)
            {
                const T cs = cl[(size_t)s * p.V + k];
                const T *fr = a.fold + (size_t)sl[s] * p.ldf + k;
                a0 = fma(cs, fr[0], a0);
                if (p.L == 2) a1 = fma(cs, fr[p.V], a1);
            }
            row[k] = a0 * scale;
            if (p.L == 2) row[p.V + k] = a1 * scale;
        }
        __syncthreads();
        if (threadIdx.x < 32)
        {
            const int lane = threadIdx.x;
            RowRegs<T, L> r(row, reinterpret_cast<T *>(rowSmem), p, lane);
            double pos, neg;
            bool bad;
            regSigns(r, p, pos, neg, bad);
            const Positivity pv(pos, neg);
            if (lane == 0) a.massPos[i] = (pos + neg) * p.dvN;
            finishParticle(a, p, i, r, pv, tab);
        }
        __syncthreads();
    }
}

template <typename T, int L>
__global__ void __launch_bounds__(kNT)
k_redo(ParticleArgs<T> a, StepParams p)
{
    k_redo_body<T, L>(a, p, blockIdx.x, gridDim.x);
}

// Finishes the listed particles once sigma is known, on true magnitudes:
// moments (kept from the previous step when the row has no positive mass,
// Moments.cpp:89), collision, moments; stored as h = g / sigma with the
// macros' density and pressure divided by sigma, as k_scale_mood expects.
template <typename T>
__device__ __forceinline__ void k_fixup_body(const ParticleArgs<T> &a, const StepParams &p, int bx,
                                             int gx)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ndeg = a.sc->ndeg;
    const double sigma = a.sc->sigma;
    const int V = p.V, dim = p.dim;
    for (int li = bx * (kNT / 32) + warp; li < ndeg; li += gx * (kNT / 32))
    {
        const int i = a.degList[li];
        T *row = a.g + (size_t)i * p.ldf;
        double pos, neg;
        bool bad;
        rowSigns((const T *)row, V, lane, pos, neg, bad);
        const Positivity pv(pos, neg);
        const double *mp = a.macPrev + 6 * (size_t)i;
        double mac[6] = {mp[0], mp[1], mp[2], mp[3], mp[4], mp[5]};
        auto moments = [&](bool post) {
            double S0 = 0, Sx = 0, Sy = 0, Sz = 0, SE = 0;
            for (NodeWalk nw(lane, p.Nv, dim); nw.k < V; nw.next())
            {
                double vx = fma((double)nw.iv, p.dv, p.vmin);
                double vy = fma((double)nw.jv, p.dv, p.vmin);
                double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
                const double g1 = (double)row[nw.k];
                const double f1 = (post ? g1 * sigma : sigma * pv.v1(g1)) * p.dvN;
                S0 += f1; Sx += vx * f1; Sy += vy * f1; Sz += vz * f1;
                SE += (vx * vx + vy * vy + vz * vz) * f1;
                if (p.L == 2)
                {
                    const double g2 = (double)row[V + nw.k];
                    SE += 2.0 * (post ? g2 * sigma : sigma * pv.v2(g1, g2)) * p.dvN;
                }
            }
            S0 = warpSum(S0); Sx = warpSum(Sx); Sy = warpSum(Sy); Sz = warpSum(Sz);
            SE = warpSum(SE);
            if (S0 > 1.0e-30)
            {
                mac[0] = S0; mac[1] = Sx / S0; mac[2] = Sy / S0;
                if (dim == 3) mac[3] = Sz / S0;
                mac[4] = fmax((SE / S0 - (mac[1] * mac[1] + mac[2] * mac[2] + mac[3] * mac[3])) /
                                  (3.0 * p.R), 1.0e-6);
                mac[5] = S0 * p.R * mac[4];
            }
            return S0;
        };
        moments(false);
        double lam = p.dt / p.tau;
        if (p.tauVar)
        {
            const double kB = 1.380649e-23;
            double l = kB / (sqrt(2.0) * kPi * mac[0] * p.R * p.dHS * p.dHS);
            double cbar = sqrt(8.0 * p.R * mac[4] / kPi);
            lam = p.dt / (4.0 * l / (kPi * cbar));
        }
        const double c1 = 1.0 / (1.0 + lam);
        const double twoRT = 2.0 * p.R * mac[4];
        const double A = (dim == 3) ? mac[0] / pow(kPi * twoRT, 1.5) : mac[0] / (kPi * twoRT);
        double mn = INFINITY;
        for (NodeWalk nw(lane, p.Nv, dim); nw.k < V; nw.next())
        {
            const int k = nw.k;
            double vx = fma((double)nw.iv, p.dv, p.vmin);
            double vy = fma((double)nw.jv, p.dv, p.vmin);
            double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
            double e = (vx - mac[1]) * (vx - mac[1]) + (vy - mac[2]) * (vy - mac[2]);
            if (dim == 3) e += (vz - mac[3]) * (vz - mac[3]);
            const double M = A * exp(-e / twoRT);
            const double g1 = (double)row[k];
            const T h1 = T(c1 * (sigma * pv.v1(g1) + lam * M) / sigma);
            if (p.L == 2)
            {
                const double g2 = (double)row[V + k];
                row[V + k] = T(c1 * (sigma * pv.v2(g1, g2) + lam * 0.5 * p.R * mac[4] * M) / sigma);
            }
            row[k] = h1;
            mn = fmin(mn, (double)h1);
        }
        __syncwarp();
        const double S0 = moments(true);
        mn = warpMin(mn);
        if (lane == 0)
        {
            double *out = a.macNew + 6 * (size_t)i;
            out[0] = mac[0] / sigma; out[1] = mac[1]; out[2] = mac[2]; out[3] = mac[3];
            out[4] = mac[4]; out[5] = mac[5] / sigma;
            a.massEnd[i] = S0 / sigma;
            a.minG[i] = mn;
            a.dpx[i] = 0.0;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(kNT)
k_fixup(ParticleArgs<T> a, StepParams p)
{
    k_fixup_body(a, p, blockIdx.x, gridDim.x);
}

// Deterministic single-block sums: thread t sums elements t, t + nt, ...
// (coalesced) into four interleaved partial sums, combined in a fixed order.
template <int K>
__device__ void blockReduceArrays(const double *const (&a)[K], int N, double (&out)[K],
                                  double *sh)
{
    const int t = threadIdx.x, nt = blockDim.x;
    double v[K];
#pragma unroll
    for (int q = 0; q < K; ++q)
    {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int i = t;
        for (; i + 3 * nt < N; i += 4 * nt)
        {
            s0 += a[q][i];
            s1 += a[q][i + nt];
            s2 += a[q][i + 2 * nt];
            s3 += a[q][i + 3 * nt];
        }
        for (; i < N; i += nt) s0 += a[q][i];
        v[q] = (s0 + s1) + (s2 + s3);
    }
    blockSums<K>(v, sh);
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = v[q];
}

// Deterministic grid sum of a[0..N) over kRedBlocks blocks: block b sums the
// fixed strided subset b*nt + t + k*stride into partial[b]; the last block to
// finish (ticket on sc->redCount) adds the partials in block order and
// resets the ticket.  Returns true in thread 0 of that block, with *total.
constexpr int kRedBlocks = 64;
constexpr int kRedThreads = 256;

__device__ bool gridSumLast(const double *__restrict__ a, int N, double *partial,
                            StepScalars *sc, double *total, int bx = -1, int gx = -1)
{
    __shared__ double sh[32];
    __shared__ bool last;
    if (bx < 0) { bx = blockIdx.x; gx = gridDim.x; }
    const int t = threadIdx.x, stride = gx * blockDim.x;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int i = bx * blockDim.x + t;
    for (; i + 3 * stride < N; i += 4 * stride)
    {
        s0 += a[i];
        s1 += a[i + stride];
        s2 += a[i + 2 * stride];
        s3 += a[i + 3 * stride];
    }
    for (; i < N; i += stride) s0 += a[i];
    double v[1] = {(s0 + s1) + (s2 + s3)};
    blockSums<1>(v, sh);
    if (t == 0)
    {
        partial[bx] = v[0];
        __threadfence();
        last = atomicAdd(&sc->redCount, 1u) == (unsigned)gx - 1;
    }
    __syncthreads();
    if (!last || t != 0) return false;
    __threadfence();
    double s = 0.0;
    for (int b = 0; b < gx; ++b) s += ((volatile double *)partial)[b];
    sc->redCount = 0;
    *total = s;
    return true;
}

// Global mass rescale (Solver/Solver.cpp:650-655): sigma = massOld/massNew.
__global__ void __launch_bounds__(kRedThreads)
k_sigma(const double *__restrict__ massPos, int N, double *partial, StepScalars *sc)
{
    double m;
    if (gridSumLast(massPos, N, partial, sc, &m))
    {
        sc->massNew = m;
        sc->sigma = (m > 1.0e-30) ? sc->massOld / m : 1.0;
    }
}

// Mass at the end of the step (the next step's massOld); the stored state
// now carries the scale sigma.
__global__ void __launch_bounds__(kRedThreads)
k_mass_sum(const double *__restrict__ massEnd, int N, double *partial, StepScalars *sc)
{
    double m;
    if (gridSumLast(massEnd, N, partial, sc, &m))
    {
        const double sigma = sc->sigma;
        sc->massEnd = sigma * m;
        sc->massOld = sc->massEnd;
        sc->scale = sigma;
        sc->steps += 1;
    }
}

// Applies sigma to the macros and runs moodCheck (Conservation.cpp:16-38,
// MLSBasis.hpp:208-222) on the true values.
__device__ __forceinline__ void k_scale_mood_body(const StepParams &p, const int *__restrict__ boundary,
                             double *__restrict__ macNew, const double *__restrict__ minG,
                             int *__restrict__ mood, StepScalars *sc, int bx)
{
    const int i = bx * blockDim.x + threadIdx.x;
    if (i >= p.N) return;
    const double sigma = sc->sigma;
    double *mac = macNew + 6 * (size_t)i;
    mac[0] *= sigma;
    mac[5] *= sigma;
    if (p.limiter != 2) return;
    if (boundary[i]) { mood[i] = 0; return; }
    // a slab's ghost rows are copies: their moodCheck belongs to their owner
    if (p.ownHi > p.ownLo && (i < p.ownLo || i >= p.ownHi)) { mood[i] = 0; return; }
    const int fail = (mac[0] < 1.0e-10) || (mac[4] < 1.0e-6) || (sigma * minG[i] < -1.0e-14);
    mood[i] = fail;
    if (fail) atomicOr(&sc->moodfail, 1);
}

__global__ void 
k_scale_mood(StepParams p, const int *__restrict__ boundary,
                             double *__restrict__ macNew, const double *__restrict__ minG,
                             int *__restrict__ mood, StepScalars *sc)
{
    k_scale_mood_body(p, boundary, macNew, minG, mood, sc, blockIdx.x);
}

// Second collision + moments of every interior particle when moodCheck
// failed (Solver/Solver.cpp:685-693).  Exits at once otherwise.
template <typename T>
__device__ __forceinline__ void k_recollide_body(T *__restrict__ g, const StepParams &p, const int *__restrict__ boundary,
            double *__restrict__ macNew, double *__restrict__ massEnd, StepScalars *sc, int bx, int gx)
{
    if (sc->moodfail == 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = bx * (kNT / 32) + warp; i < p.N; i += gx * (kNT / 32))
    {
    if (boundary[i]) continue;
    const double sigma = sc->sigma;
    T *row = g + (size_t)i * p.ldf;
    double *mac = macNew + 6 * (size_t)i;
    const int V = p.V, dim = p.dim;
    const double rho = mac[0], ux = mac[1], uy = mac[2], uz = mac[3], Tt = mac[4];
    double lam = p.dt / p.tau;
    if (p.tauVar)
    {
        const double kB = 1.380649e-23;
        double l = kB / (sqrt(2.0) * kPi * rho * p.R * p.dHS * p.dHS);
        double cbar = sqrt(8.0 * p.R * Tt / kPi);
        lam = p.dt / (4.0 * l / (kPi * cbar));
    }
    const double c1 = 1.0 / (1.0 + lam);
    const double twoRT = 2.0 * p.R * Tt;
    const double A = (dim == 3) ? rho / pow(kPi * twoRT, 1.5) : rho / (kPi * twoRT);
    double N0 = 0, Nx = 0, Ny = 0, Nz = 0, NE = 0;
    NodeWalk nw(lane, p.Nv, dim);
    for (; nw.k < V; nw.next())
    {
        const int k = nw.k;
        double vx = fma((double)nw.iv, p.dv, p.vmin);
        double vy = fma((double)nw.jv, p.dv, p.vmin);
        double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
        double e = (vx - ux) * (vx - ux) + (vy - uy) * (vy - uy);
        if (dim == 3) e += (vz - uz) * (vz - uz);
        const double M = A * exp(-e / twoRT);
        const double g1 = c1 * (sigma * (double)row[k] + lam * M);
        const T g1s = T(g1 / sigma);
        row[k] = g1s;
        const double f1 = (double)g1s * sigma * p.dvN;
        N0 += f1; Nx += vx * f1; Ny += vy * f1; Nz += vz * f1;
        NE += (vx * vx + vy * vy + vz * vz) * f1;
        if (p.L == 2)
        {
            const double g2 = c1 * (sigma * (double)row[V + k] + lam * 0.5 * p.R * Tt * M);
            const T g2s = T(g2 / sigma);
            row[V + k] = g2s;
            NE += 2.0 * (double)g2s * sigma * p.dvN;
        }
    }
    N0 = warpSum(N0); Nx = warpSum(Nx); Ny = warpSum(Ny); Nz = warpSum(Nz); NE = warpSum(NE);
    if (lane == 0)
    {
        if (N0 > 1.0e-30)
        {
            mac[0] = N0; mac[1] = Nx / N0; mac[2] = Ny / N0;
            if (dim == 3) mac[3] = Nz / N0;
            double u2 = mac[1] * mac[1] + mac[2] * mac[2] + mac[3] * mac[3];
            mac[4] = fmax((NE / N0 - u2) / (3.0 * p.R), 1.0e-6);
            mac[5] = N0 * p.R * mac[4];
        }
        massEnd[i] = N0 / sigma;
    }
    }
}

template <typename T>
__global__ void __launch_bounds__(kNT)
k_recollide(T *__restrict__ g, StepParams p, const int *__restrict__ boundary,
            double *__restrict__ macNew, double *__restrict__ massEnd, StepScalars *sc)
{
    k_recollide_body(g, p, boundary, macNew, massEnd, sc, blockIdx.x, gridDim.x);
}

// Mass at the end of a step whose moodCheck failed (after k_recollide).
__global__ void __launch_bounds__(kRedThreads)
k_mass_end(const double *__restrict__ massEnd, int N, double *partial, StepScalars *sc)
{
    if (sc->moodfail == 0) return;
    double m;
    if (gridSumLast(massEnd, N, partial, sc, &m))
    {
        sc->massEnd = sc->sigma * m;
        sc->massOld = sc->massEnd;
    }
}

// ---------------------------------------------------------------------------
// Slab groups.  The global sums of the step (Conservation.cpp:48-109, the
// moodCheck flag of Conservation.cpp:16-38) become, per slab, a sum over the
// owned range into slabPart[q], then one combine over all slabs in slab
// order -- the rank-ordered Allgather of the reference's decomposed mode
// (Conservation.cpp:76-84) -- that writes the global values back to every
// slab's scalars.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kRedThreads)
k_sum_range(const double *__restrict__ a, int n, double *partial, StepScalars *sc, int q,
            int gate)
{
    if (gate && sc->moodfail == 0) return;
    double m;
    if (gridSumLast(a, n, partial, sc, &m)) sc->slabPart[q] = m;
}

__global__ void k_slab_combine(StepScalars *const *scs, int n, int phase)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    StepScalars *s0 = scs[0];
    auto total = [&](int q) {
        double m = 0.0;
        for (int i = 0; i < n; ++i) m += scs[i]->slabPart[q];
        return m;
    };
    if (phase == 0)            // k_sigma
    {
        const double m = total(0);
        const double sigma = (m > 1.0e-30) ? s0->massOld / m : 1.0;
        for (int i = 0; i < n; ++i) { scs[i]->massNew = m; scs[i]->sigma = sigma; }
    }
    else if (phase == 1)       // k_mass_sum
    {
        const double sigma = s0->sigma;
        const double me = sigma * total(1);
        for (int i = 0; i < n; ++i)
        {
            scs[i]->massEnd = me;
            scs[i]->massOld = me;
            scs[i]->scale = sigma;
            scs[i]->steps += 1;
        }
    }
    else if (phase == 2)       // moodCheck: any slab failed
    {
        int f = 0;
        for (int i = 0; i < n; ++i) f |= scs[i]->moodfail;
        for (int i = 0; i < n; ++i) scs[i]->moodfail = f;
    }
    else if (phase == 3)       // k_mass_end
    {
        if (s0->moodfail == 0) return;
        const double me = s0->sigma * total(2);
        for (int i = 0; i < n; ++i) { scs[i]->massEnd = me; scs[i]->massOld = me; }
    }
    else                       // set-up: k_mass_init over the whole domain
    {
        const double m = total(1);
        for (int i = 0; i < n; ++i)
        {
            scs[i]->massOld = m;
            scs[i]->massEnd = m;
            scs[i]->scale = 1.0;
            scs[i]->sigma = 1.0;
        }
    }
}

// One slab of a multi-process slab run: k_slab_combine's arithmetic for
// this slab alone.  The totals add every rank's word in rank order, as
// k_slab_combine adds the slabs; massOld, sigma and moodfail are the same in
// every slab when a phase starts, so the slab's own copies stand in for
// slab 0's.
__global__ void k_rank_combine(StepScalars *sc, const double *__restrict__ all, int n, int phase)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    auto total = [&](int q) {
        double m = 0.0;
        for (int i = 0; i < n; ++i) m += all[4 * i + q];
        return m;
    };
    if (phase == 0)
    {
        const double m = total(0);
        sc->sigma = (m > 1.0e-30) ? sc->massOld / m : 1.0;
        sc->massNew = m;
    }
    else if (phase == 1)
    {
        const double sigma = sc->sigma;
        const double me = sigma * total(1);
        sc->massEnd = me;
        sc->massOld = me;
        sc->scale = sigma;
        sc->steps += 1;
    }
    else if (phase == 2)
    {
        int f = 0;
        for (int i = 0; i < n; ++i) f |= all[4 * i + 3] != 0.0;
        sc->moodfail = f;
    }
    else if (phase == 3)
    {
        if (sc->moodfail == 0) return;
        const double me = sc->sigma * total(2);
        sc->massEnd = me;
        sc->massOld = me;
    }
    else
    {
        const double m = total(1);
        sc->massOld = m;
        sc->massEnd = m;
        sc->scale = 1.0;
        sc->sigma = 1.0;
    }
}

// Resets the step's counters; with a NAD range buffer also computes the
// neighbour density ranges of the streamed particle kernel.
__global__ void __launch_bounds__(kNT)
k_step_begin(StepScalars *sc, int reset, const double *__restrict__ macPrev,
             const int *__restrict__ boundary, const int *__restrict__ nslot,
             const int *__restrict__ slots, int S, int N, double *__restrict__ nad)
{
    if (reset && blockIdx.x == 0 && threadIdx.x == 0)
    {
        sc->nflag = 0;
        sc->ndeg = 0;
        sc->nfix = 0;
        sc->moodfail = 0;
    }
    if (nad) nadRanges(macPrev, boundary, nslot, slots, S, N, nad);
}

// Particle masses of an uploaded state (scale 1).
template <typename T>
__global__ void __launch_bounds__(kNT)
k_particle_mass(const T *g, StepParams p, double *massEnd)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kNT / 32) + warp;
    if (i >= p.N) return;
    const T *row = g + (size_t)i * p.ldf;
    double s = 0.0;
    for (int k = lane; k < p.V; k += 32) s += (double)row[k];
    s = warpSum(s);
    if (lane == 0) massEnd[i] = s * p.dvN;
}

__global__ void __launch_bounds__(kRedThreads)
k_mass_init(const double *__restrict__ massEnd, int N, double *partial, StepScalars *sc)
{
    double m;
    if (gridSumLast(massEnd, N, partial, sc, &m))
    {
        sc->massOld = m;
        sc->massEnd = m;
        sc->scale = 1.0;
        sc->sigma = 1.0;
    }
}

// ---------------------------------------------------------------------------
// Rigid-body surface-stress loads (RigidBody/BodyDynamics.cpp:17-97): one
// block per particle writes its contribution; a single block then sums the
// contributions in particle order, as the reference's serial loop does.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_body_contrib(const T *g, StepParams p, const int *__restrict__ bodyId,
               const int *__restrict__ boundary, const double *__restrict__ pos,
               const double *__restrict__ wall, const double *__restrict__ centre,
               const double *__restrict__ area, double *tmp,
               const StepScalars *__restrict__ sc)
{
    __shared__ double sh[6 * 32];
    const int i = blockIdx.x;
    const int b = bodyId[i];
    if (!boundary[i] || b < 0) return;
    const T *gr = g + (size_t)i * p.ldf;
    const double *w = wall + 7 * (size_t)i;
    const double scale = sc->scale;
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < p.V; k += blockDim.x)
    {
        double vx, vy, vz;
        nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
        double cx = vx - w[3], cy = vy - w[4], cz = vz - w[5];
        double f = (double)gr[k] * scale * p.dvN;
        v[0] += f * cx * cx; v[1] += f * cy * cy; v[2] += f * cz * cz;
        v[3] += f * cx * cy; v[4] += f * cx * cz; v[5] += f * cy * cz;
    }
    blockSums<6>(v, sh);
    if (threadIdx.x == 0)
    {
        const double a = area[b];
        const double cdx = pos[3 * i] - centre[3 * b];
        const double cdy = pos[3 * i + 1] - centre[3 * b + 1];
        const double cdz = pos[3 * i + 2] - centre[3 * b + 2];
        double *o = tmp + 6 * (size_t)i;
        if (p.dim == 3)
        {
            double tx = -(w[0] * v[0] + w[1] * v[3] + w[2] * v[4]);
            double ty = -(w[0] * v[3] + w[1] * v[1] + w[2] * v[5]);
            double tz = -(w[0] * v[4] + w[1] * v[5] + w[2] * v[2]);
            o[0] = a * tx; o[1] = a * ty; o[2] = a * tz;
            o[3] = a * (cdy * tz - cdz * ty);
            o[4] = a * (cdz * tx - cdx * tz);
            o[5] = a * (cdx * ty - cdy * tx);
        }
        else
        {
            double valX = -w[0] * v[0] - w[1] * v[3];
            double valY = -w[0] * v[3] - w[1] * v[1];
            o[0] = a * valX; o[1] = a * valY; o[2] = 0.0;
            o[3] = 0.0; o[4] = 0.0; o[5] = a * (cdx * valY - cdy * valX);
        }
    }
}

__global__ void k_body_sum(const double *tmp, const int *bodyId,
                           const int *boundary, int N, int nbodies, double *out)
{
    // One thread per (body, component): serial sum in particle order.
    const int t = threadIdx.x;
    if (t >= nbodies * 6) return;
    const int b = t / 6, q = t % 6;
    double s = 0.0;
    for (int i = 0; i < N; ++i)
        if (boundary[i] && bodyId[i] == b) s += tmp[6 * (size_t)i + q];
    out[t] = s;
}

// Wall velocity V + w x r on body-surface particles
// (RigidBody/BodyDynamics.cpp:103-125).
__global__ void k_set_surface_velocity(int N, int dim, const int *bodyId,
                                       const int *boundary, const double *pos,
                                       double *wall, const double *centre,
                                       const double *state)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int b = bodyId[i];
    if (!boundary[i] || b < 0) return;
    const double *s = state + 6 * b;
    double rx = pos[3 * i] - centre[3 * b];
    double ry = pos[3 * i + 1] - centre[3 * b + 1];
    double rz = pos[3 * i + 2] - centre[3 * b + 2];
    double *w = wall + 7 * (size_t)i;
    w[3] = s[0] + s[4] * rz - s[5] * ry;
    w[4] = s[1] + s[5] * rx - s[3] * rz;
    if (dim == 3) w[5] = s[2] + s[3] * ry - s[4] * rx;
}

template <typename T>
__global__ void k_convert_in(const double *src, T *dst, int N, int gs, int ldf)
{
    size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t tot = (size_t)N * gs;
    for (; idx < tot; idx += (size_t)gridDim.x * blockDim.x)
    {
        size_t i = idx / gs, k = idx % gs;
        dst[i * ldf + k] = T(src[idx]);
    }
}

// The distribution of a managed cloud from the current one (the row plan of
// the cloud management): what k_convert_out, the host management and
// k_convert_in give, without the round trip.  A kept row is the stored row
// at true scale; a merged row the mean of two such rows, rounded as the
// host rounds it (products kept separate from the sum); a refill row comes
// from the host.
template <typename T>
__global__ void k_rows_build(const T *__restrict__ src, int ldf, int gs, int n,
                             const int *__restrict__ a, const int *__restrict__ b,
                             const double *__restrict__ fresh,
                             const StepScalars *__restrict__ sc, double *__restrict__ out)
{
    const double scale = sc->scale;
    const size_t tot = (size_t)n * gs;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < tot;
         idx += (size_t)gridDim.x * blockDim.x)
    {
        const size_t j = idx / gs, k = idx % gs;
        const int ia = a[j];
        double v;
        if (ia >= 0)
        {
            const double va = __dmul_rn((double)src[(size_t)ia * ldf + k], scale);
            const int ib = b[j];
            v = (ib >= 0) ? 0.5 * (va + __dmul_rn((double)src[(size_t)ib * ldf + k], scale)) : va;
        }
        else
            v = fresh[(size_t)(-1 - ia) * gs + k];
        out[idx] = v;
    }
}

template <typename T>
__global__ void k_convert_out(const T *src, double *dst, int N, int gs, int ldf,
                              const StepScalars *__restrict__ sc)
{
    const double scale = sc->scale;
    size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t tot = (size_t)N * gs;
    for (; idx < tot; idx += (size_t)gridDim.x * blockDim.x)
    {
        size_t i = idx / gs, k = idx % gs;
        dst[idx] = (double)src[i * ldf + k] * scale;
    }
}

// ---------------------------------------------------------------------------
// Steady residual of the last step, over the interior particles:
//   max( |d rho| / |rho|, |d(rho ux)| / |rho c|, |d(rho uy)| / |rho c|,
//        |d(rho E)| / |rho E| ),  |.| the 2-norm over particles,
// E = |u|^2 / 2 + 3 R T / 2 (monatomic gas) and c the momentum speed scale:
// uRef when it is positive (the lid speed of a driven cavity), the flow
// speed |u| itself when it is negative (momentum changes against the flow's
// own momentum), else sqrt(R T), the thermal speed, which does not vanish
// for a gas at rest.  The reference defines no
// residual; this is the convergence measure of a run to steady state.  One
// block, fixed order: deterministic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void k_residual_body(const double *__restrict__ macNew, const double *__restrict__ macOld,
           const int *__restrict__ boundary, int N, double R, double *out, double uRef)
{
    __shared__ double sh[8 * 32];
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < N; i += blockDim.x)
    {
        if (boundary[i]) continue;
        const double *a = macNew + 6 * (size_t)i, *b = macOld + 6 * (size_t)i;
        const double ea = 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) + 1.5 * R * a[4];
        const double eb = 0.5 * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]) + 1.5 * R * b[4];
        const double mn[4] = {a[0], a[0] * a[1], a[0] * a[2], a[0] * ea};
        const double mo[4] = {b[0], b[0] * b[1], b[0] * b[2], b[0] * eb};
        const double thermal2 =                                  // (rho c)^2
            uRef > 0.0 ? b[0] * b[0] * uRef * uRef
                       : (uRef < 0.0 ? b[0] * b[0] * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3])
                                     : b[0] * b[0] * R * b[4]);
        const double ref[4] = {b[0] * b[0], thermal2, thermal2, mo[3] * mo[3]};
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const double d = mn[q] - mo[q];
            v[q] += d * d;
            v[4 + q] += ref[q];
        }
    }
    blockSums<8>(v, sh);
    if (threadIdx.x == 0)
    {
        double r = 0.0;
        for (int q = 0; q < 4; ++q)
            if (v[4 + q] > 0.0) r = fmax(r, sqrt(v[q] / v[4 + q]));
        *out = r;
    }
}

__global__ void __launch_bounds__(1024)
k_residual(const double *__restrict__ macNew, const double *__restrict__ macOld,
           const int *__restrict__ boundary, int N, double R, double *out, double uRef)
{
    k_residual_body(macNew, macOld, boundary, N, R, out, uRef);
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
// Warps (particles) per block of k_particle: as many of the eight as fit
// their shared-memory row copies in 160 KB.
static int particleWarpsPerBlock(const StepParams &p, size_t es)
{
    const size_t rowBytes = (size_t)p.L * p.V * es;
    int w = (int)((160u * 1024u) / rowBytes);
    return w < 1 ? 1 : (w > kNT / 32 ? kNT / 32 : w);
}

// The streamed particle stage of a 3-D single-layer cloud: batched (FP32)
// or one warp per particle.
template <typename T>
static void launchParticleStream(alebgk_ctx *c, const ParticleArgs<T> &pa, const StepParams &p,
                                 cudaStream_t st)
{
    if constexpr (sizeof(T) == 4)
    {
        if (c->pRows)
        {
            rowsKernel(p.Nv)<<<c->pRowsBlocks, kRowsThreads, 0, st>>>(pa, p);
            return;
        }
    }
    k_particle_stream<T><<<c->pStreamBlocks, kNT, c->pStreamSmem, st>>>(pa, p, c->pStreamWpb);
}

// Launches one step.  With ev != nullptr an event is recorded before each
// launch and after the last one (ev[0..ALEBGK_NSTAGES]), in launch order:
// step_begin, transport, particle, redo, sigma, fixup, mass_sum, scale_mood,
// recollide, mass_end.
template <typename T>
static cudaError_t stepT(alebgk_ctx *c, int from, cudaEvent_t *ev)
{
    const StepParams &p = c->sp;
    DeviceBuffers &d = c->d;
    cudaStream_t st = c->stream;
    T *fa = static_cast<T *>(d.f[from]);
    T *fb = static_cast<T *>(d.f[1 - from]);
    double *macA = d.macro[from], *macB = d.macro[1 - from];
    ParticleArgs<T> pa;
    pa.g = fb; pa.fold = fa; pa.coefLin = static_cast<const T *>(d.coefLin);
    pa.coef = static_cast<const T *>(d.coef);
    pa.boundary = d.boundary; pa.cls = d.cls; pa.nslot = d.nslot; pa.slots = d.slots;
    pa.rowOrder = d.rowOrder;
    pa.wall = d.wall; pa.macPrev = macA; pa.macNew = macB;
    pa.massPos = d.massPos; pa.massEnd = d.massEnd; pa.minG = d.minG; pa.dpx = d.dpx;
    pa.flag = d.flag; pa.flagList = d.flagList; pa.degList = d.degList; pa.sc = d.sc;
    pa.nad = d.nad;
    int q = 0;
    auto mark = [&]() { if (ev) cudaEventRecord(ev[q++], st); };
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    const int listBlocks = min(p.N, 296);
    mark();
    const bool nadOn = c->pStream && p.limiter == 2;
    const int nadBlocks = min((p.N + kNT / 32 - 1) / (kNT / 32), 1184);
    // The NAD ranges depend only on the previous step's macros: in a step
    // graph they run on a side stream beside the transport; when stages are
    // timed they run in step_begin.
    const bool fork = nadOn && !ev && c->stream2;
    if (fork)
    {
        k_step_begin<<<1, kNT, 0, st>>>(d.sc, 1, macA, d.boundary, d.nslot, d.slots, p.S, p.N,
                                        nullptr);
        cudaEventRecord(c->evFork, st);
        cudaStreamWaitEvent(c->stream2, c->evFork, 0);
        k_step_begin<<<nadBlocks, kNT, 0, c->stream2>>>(d.sc, 0, macA, d.boundary, d.nslot,
                                                        d.slots, p.S, p.N, d.nad);
        cudaEventRecord(c->evJoin, c->stream2);
    }
    else
        k_step_begin<<<nadOn ? nadBlocks : 1, kNT, 0, st>>>(
            d.sc, 1, macA, d.boundary, d.nslot, d.slots, p.S, p.N, nadOn ? d.nad : nullptr);
    mark();
    const bool march = sizeof(T) == 4 && c->march.enabled;
    // Transport fused into the particle kernel (transport threads 0), except
    // when stages are timed: then it runs as its own kernel, with the same
    // sums, so that its time is seen.
    const bool fused = !march && !c->pStream && c->tune.transportThreads == 0 && !ev;
    if (march)
    {
        cudaError_t e = launchMarch(c, from, reinterpret_cast<float *>(fb), st);
        if (e != cudaSuccess) return e;
    }
    else if (!fused)
    {
        const int tt = c->tune.transportThreads > 0 ? c->tune.transportThreads : kNT;
        dim3 gt(transportChunks(p.V), (p.N + tt / 32 - 1) / (tt / 32));
        k_transport<T><<<gt, tt, 0, st>>>(fa, fb, static_cast<const T *>(d.coef),
                                           d.cls, d.nslot, d.slots, p.S, p.N, p.V, p.L,
                                           p.ldf, d.sc);
    }
    mark();
    if (fork) cudaStreamWaitEvent(st, c->evJoin, 0);
    const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
    const int wmax = particleWarpsPerBlock(p, sizeof(T));
    const int wpb = (c->tune.particleWarps > 0 && c->tune.particleWarps < wmax)
                        ? c->tune.particleWarps : wmax;
    const int ppBlocks = (p.N + wpb - 1) / wpb;
    if (c->pStream)
        launchParticleStream<T>(c, pa, p, st);
    else if (fused)
    {
        if (p.L == 2) k_particle<T, 2, true><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
        else k_particle<T, 1, true><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
    }
    else if (p.L == 2) k_particle<T, 2, false><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
    else k_particle<T, 1, false><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
    mark();
    if (p.L == 2) k_redo<T, 2><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
    else k_redo<T, 1><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
    mark();
    k_sigma<<<kRedBlocks, kRedThreads, 0, st>>>(d.massPos, p.N, d.redPartial, d.sc);
    mark();
    k_fixup<T><<<min(pBlocks, 296), kNT, 0, st>>>(pa, p);
    mark();
    k_mass_sum<<<kRedBlocks, kRedThreads, 0, st>>>(d.massEnd, p.N, d.redPartial, d.sc);
    mark();
    k_scale_mood<<<(p.N + 255) / 256, 256, 0, st>>>(p, d.boundary, macB, d.minG, d.mood, d.sc);
    mark();
    if (p.limiter == 2)
        k_recollide<T><<<min(pBlocks, 592), kNT, 0, st>>>(fb, p, d.boundary, macB, d.massEnd,
                                                         d.sc);
    mark();
    if (p.limiter == 2)
        k_mass_end<<<kRedBlocks, kRedThreads, 0, st>>>(d.massEnd, p.N, d.redPartial, d.sc);
    mark();
    return cudaGetLastError();
}

template <typename T>
static cudaError_t prepareT(alebgk_ctx *c)
{
    const StepParams &p = c->sp;
    const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
    const int wpb = particleWarpsPerBlock(p, sizeof(T));
    // The dynamic shared-memory cap is an attribute of the kernel, shared by
    // every context in the process, so it is raised to the device's opt-in
    // maximum rather than set to this context's need: contexts of different
    // row sizes (a batch of uneven cavities) then all stay launchable.
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    auto set = [&](const void *fn, size_t bytes) {
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        const size_t cap = (size_t)optin - fa.sharedSizeBytes;   // minus static shared memory
        if (e == cudaSuccess && bytes > cap) e = cudaErrorInvalidValue;
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    };
    set((const void *)k_particle<T, 1, false>, wpb * rowBytes);
    set((const void *)k_particle<T, 2, false>, wpb * rowBytes);
    set((const void *)k_particle<T, 1, true>, wpb * rowBytes);
    set((const void *)k_particle<T, 2, true>, wpb * rowBytes);
    set((const void *)k_redo<T, 1>, rowBytes);
    set((const void *)k_redo<T, 2>, rowBytes);

    // Streamed particle kernel: 3-D single layer, two rows per warp, at
    // least four warps per block in 200 KB of shared memory.
    c->pStream = false;
    if (e == cudaSuccess && p.dim == 3 && p.L == 1 && p.Nv <= 255 && c->cfg.particle != 1)
    {
        int w = kNT / 32;
        while (w >= 4 && streamSmemBytes<T>(p.V, p.ldf, w) > 200u * 1024u) --w;
        if (w >= 4)
        {
            const size_t smem = streamSmemBytes<T>(p.V, p.ldf, w);
            set((const void *)k_particle_stream<T>, smem);
            int occ = 0, sms = 0;
            if (e == cudaSuccess)
                e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                    &occ, k_particle_stream<T>, kNT, smem);
            if (e == cudaSuccess && occ > 0)
            {
                const int need = (p.N + w - 1) / w;
                c->pStream = true;
                c->pStreamWpb = w;
                c->pStreamSmem = smem;
                c->pStreamBlocks = need < sms * occ ? need : sms * occ;
            }
        }
        // The register-row form of the same stages (FP32, Nv of an
        // instance): the default, unless the shared-memory form is asked for.
        c->pRows = false;
        // (Its staged rows are (V + 3) / 4 * 4 floats, the FP32 row stride.)
        const RowsKernel rk = rowsKernel(p.Nv);
        if (e == cudaSuccess && c->pStream && sizeof(T) == 4 && c->cfg.particle != 3 && rk &&
            p.dim == 3 && p.ldf == (p.V + 3) / 4 * 4)
        {
            int occ = 0, sms = 0;
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, rk, kRowsThreads, 0);
            if (e == cudaSuccess && occ > 0)
            {
                const int need = (p.N + kRowsThreads / 32 - 1) / (kRowsThreads / 32);
                c->pRows = true;
                c->pRowsBlocks = std::min(need, sms * occ);
            }
        }
    }
    return e;
}



cudaError_t prepareKernels(alebgk_ctx *c)
{
    return (c->cfg.precision == 64) ? prepareT<double>(c) : prepareT<float>(c);
}

cudaError_t launchStep(alebgk_ctx *c, int from, cudaEvent_t *ev)
{
    return (c->cfg.precision == 64) ? stepT<double>(c, from, ev)
                                    : stepT<float>(c, from, ev);
}

// ---------------------------------------------------------------------------
// Batches of small clouds: one launch per stage of the step over every cloud
// of the batch.  Block b of a stage belongs to the cloud c with
// off[c] <= b < off[c + 1] and runs that cloud's kernel body with the
// virtual block index b - off[c] and the cloud's own grid size, so every
// cloud computes exactly what its own launches compute (same bodies, same
// block-sum order); only the number of launches changes.
// ---------------------------------------------------------------------------
template <typename T>
struct BatchCtx
{
    ParticleArgs<T> pa;        // parity `from`: pa.g = f[1 - from], pa.fold = f[from]
    StepParams p;
    double *redPartial;
    double *resid;
    int *mood;
    int wpb;                   // particles (warps) per block of the particle stage
};

// Stages: 0 begin, 1 transport (empty: fused into the particle stage, the
// slot keeps the numbering of the cloud's own launch order), 2 particle,
// 3 redo, 4 sigma, 5 fixup, 6 mass sum, 7 scale + moodCheck, 8 recollide,
// 9 end mass, 10 residual.
constexpr int kBatchStages = 11;

__device__ __forceinline__ int batchCtxOf(const int *__restrict__ off, int n, int b)
{
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// The block's cloud descriptor is copied to shared memory: its fields are
// then read from there as needed instead of occupying registers (read from
// global memory through a restricted pointer instead, the particle stage
// kept them in registers and ran 19 % slower on the 96-cavity batch).
template <typename T>
__device__ __forceinline__ const BatchCtx<T> &batchStage(const BatchCtx<T> *__restrict__ ctx,
                                                         const int *__restrict__ off, int n,
                                                         int stage, int &vb, int &vg,
                                                         int gb = -1)
{
    __shared__ __align__(16) unsigned char raw[sizeof(BatchCtx<T>)];
    static_assert(sizeof(BatchCtx<T>) % 8 == 0, "descriptor words");
    if (gb < 0) gb = blockIdx.x;
    const int *o = off + stage * (n + 1);
    const int c = batchCtxOf(o, n, gb);
    vb = gb - o[c];
    vg = o[c + 1] - o[c];
    const unsigned long long *src = reinterpret_cast<const unsigned long long *>(ctx + c);
    unsigned long long *dst = reinterpret_cast<unsigned long long *>(raw);
    for (int w = threadIdx.x; w < (int)(sizeof(BatchCtx<T>) / 8); w += blockDim.x)
        dst[w] = src[w];
    __syncthreads();
    return *reinterpret_cast<const BatchCtx<T> *>(raw);
}

#define BATCH_CTX(stage)                                                          \
    int vb, vg;                                                                    \
    const BatchCtx<T> &B = batchStage<T>(ctx, off, n, (stage), vb, vg);            \
    (void)vg

template <typename T>
__global__ void __launch_bounds__(kNT)
k_batch_begin(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(0);
    if (vb == 0 && threadIdx.x == 0)
    {
        StepScalars *sc = B.pa.sc;
        sc->nflag = 0;
        sc->ndeg = 0;
        sc->nfix = 0;
        sc->moodfail = 0;
    }
}

template <typename T, int L>
__global__ void __launch_bounds__(kNT)
k_batch_particle(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(2);
    k_particle_body<T, L, true>(B.pa, B.p, B.wpb, vb);
}

template <typename T, int L>
__global__ void __launch_bounds__(kNT)
k_batch_redo(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(3);
    k_redo_body<T, L>(B.pa, B.p, vb, vg);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
k_batch_sigma(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(4);
    StepScalars *sc = B.pa.sc;
    double m;
    if (gridSumLast(B.pa.massPos, B.p.N, B.redPartial, sc, &m, vb, vg))
    {
        sc->massNew = m;
        sc->sigma = (m > 1.0e-30) ? sc->massOld / m : 1.0;
    }
}

template <typename T>
__global__ void __launch_bounds__(kNT)
k_batch_fixup(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(5);
    k_fixup_body<T>(B.pa, B.p, vb, vg);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
k_batch_mass_sum(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(6);
    StepScalars *sc = B.pa.sc;
    double m;
    if (gridSumLast(B.pa.massEnd, B.p.N, B.redPartial, sc, &m, vb, vg))
    {
        const double sigma = sc->sigma;
        sc->massEnd = sigma * m;
        sc->massOld = sc->massEnd;
        sc->scale = sigma;
        sc->steps += 1;
    }
}

template <typename T>
__global__ void __launch_bounds__(256)
k_batch_scale_mood(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(7);
    k_scale_mood_body(B.p, B.pa.boundary, B.pa.macNew, B.pa.minG, B.mood, B.pa.sc, vb);
}

template <typename T>
__global__ void __launch_bounds__(kNT)
k_batch_recollide(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(8);
    k_recollide_body<T>(B.pa.g, B.p, B.pa.boundary, B.pa.macNew, B.pa.massEnd, B.pa.sc, vb, vg);
}

template <typename T>
__global__ void __launch_bounds__(kRedThreads)
k_batch_mass_end(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(9);
    StepScalars *sc = B.pa.sc;
    if (sc->moodfail == 0) return;
    double m;
    if (gridSumLast(B.pa.massEnd, B.p.N, B.redPartial, sc, &m, vb, vg))
    {
        sc->massEnd = sc->sigma * m;
        sc->massOld = sc->massEnd;
    }
}

template <typename T>
__global__ void __launch_bounds__(1024)
k_batch_residual(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off, int n)
{
    BATCH_CTX(10);
    k_residual_body(B.pa.macNew, B.pa.macPrev, B.pa.boundary, B.p.N, B.p.R, B.resid, B.p.resU);
}

// The residual's 1024-thread block (k_residual_body) on a 256-thread block:
// each thread runs four virtual threads t + 256 j with their own strided
// sums, a warp reduces virtual warp wid + 8 j, and the 32 virtual warps'
// sums are added in virtual-warp order -- the operations and order of the
// 1024-thread block, so the same bits.
__device__ void residualBody1024(const double *__restrict__ macNew,
                                 const double *__restrict__ macOld,
                                 const int *__restrict__ boundary, int N, double R, double *out,
                                 double uRef)
{
    __shared__ double sh[8 * 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll 1
    for (int j = 0; j < 4; ++j)
    {
        double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = threadIdx.x + 256 * j; i < N; i += 1024)
        {
            if (boundary[i]) continue;
            const double *a = macNew + 6 * (size_t)i, *b = macOld + 6 * (size_t)i;
            const double ea = 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) + 1.5 * R * a[4];
            const double eb = 0.5 * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]) + 1.5 * R * b[4];
            const double mn[4] = {a[0], a[0] * a[1], a[0] * a[2], a[0] * ea};
            const double mo[4] = {b[0], b[0] * b[1], b[0] * b[2], b[0] * eb};
            const double thermal2 =
                uRef > 0.0 ? b[0] * b[0] * uRef * uRef
                           : (uRef < 0.0 ? b[0] * b[0] * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3])
                                         : b[0] * b[0] * R * b[4]);
            const double ref[4] = {b[0] * b[0], thermal2, thermal2, mo[3] * mo[3]};
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
                const double d = mn[q] - mo[q];
                v[q] += d * d;
                v[4 + q] += ref[q];
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = warpSum(v[q]);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < 8; ++q) sh[q * 32 + wid + 8 * j] = v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            double sum = 0.0;
            for (int w = 0; w < 32; ++w) sum += sh[q * 32 + w];
            v[q] = sum;
        }
        double r = 0.0;
        for (int q = 0; q < 4; ++q)
            if (v[4 + q] > 0.0) r = fmax(r, sqrt(v[q] / v[4 + q]));
        *out = r;
    }
    __syncthreads();
}

// Grid-wide barrier of the persistent batch step: bar[0] counts the blocks
// in, bar[kBarLine] is the generation, bar[2 kBarLine] an abort flag, and
// bar[(3 + s) kBarLine] stage s's block counter, each on its own 128-byte
// line so that the polls of the waiting blocks do not contend with the
// arrivals' atomics.  Polls back off with __nanosleep.  Every wait gives up
// after `cap` polls (or when another block has given up), raises the abort
// flag and returns false; the caller then leaves the kernel.  The host
// clears bar before every launch.
constexpr int kBarLine = 32;
constexpr int kBarWords = (3 + kBatchStages) * kBarLine;

__device__ __forceinline__ bool gridBarrier(unsigned *bar, long long cap)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile unsigned *gen = bar + kBarLine, *abort = bar + 2 * kBarLine;
        ok = 1;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1)
        {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + kBarLine, 1u);
        }
        else
        {
            long long it = 0;
            unsigned ns = 32;
            while (*gen == g0)
            {
                if (it >= cap || *abort != 0u)
                {
                    ok = 0;
                    atomicExch(bar + 2 * kBarLine, 1u);
                    break;
                }
                ++it;
                __nanosleep(ns);
                if (ns < 256) ns <<= 1;
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Stage bodies of the persistent batch step, each its own (not inlined)
// function: register allocation is per function, so the particle body gets
// the registers it gets in its own launch instead of sharing them with the
// other stages' state (inlined together they spilled).
template <typename T, int L>
__device__ __noinline__ void persistentParticle(const BatchCtx<T> &B, int vb)
{
    k_particle_body<T, L, true>(B.pa, B.p, B.wpb, vb);
}

template <typename T, int L>
__device__ __noinline__ void persistentRedo(const BatchCtx<T> &B, int vb, int vg)
{
    k_redo_body<T, L>(B.pa, B.p, vb, vg);
}

template <typename T>
__device__ __noinline__ void persistentRecollide(const BatchCtx<T> &B, int vb, int vg)
{
    k_recollide_body<T>(B.pa.g, B.p, B.pa.boundary, B.pa.macNew, B.pa.massEnd, B.pa.sc, vb, vg);
}

template <typename T>
__device__ __noinline__ void persistentResidual(const BatchCtx<T> &B)
{
    residualBody1024(B.pa.macNew, B.pa.macPrev, B.pa.boundary, B.p.N, B.p.R, B.resid, B.p.resU);
}

// The whole batch step in one launch: every stage of every cloud as
// virtual blocks (the bodies, virtual block indices and grid sizes of the
// stage launches, so every cloud computes what its own launches compute),
// handed out to the resident blocks by a per-stage counter (the next index
// is fetched while the current one runs), and a bounded grid-wide barrier
// between stages.  vmap[s] is the start of stage s's virtual-block ->
// cloud table within vmap.  A block keeps its cloud's descriptor in shared
// memory while consecutive virtual blocks stay in that cloud.  A barrier
// that gives up sets bit 8 of the first cloud's error word and ends the
// launch.
template <typename T, int L>
__global__ void __launch_bounds__(kNT, 3)
k_batch_persistent(const BatchCtx<T> *__restrict__ ctx, const int *__restrict__ off,
                   const int *__restrict__ vmap, int n, unsigned *bar, long long cap)
{
    __shared__ __align__(16) unsigned char raw[sizeof(BatchCtx<T>)];
    __shared__ int sNext[2];
    static_assert(sizeof(BatchCtx<T>) % 8 == 0, "descriptor words");
    const BatchCtx<T> &B = *reinterpret_cast<const BatchCtx<T> *>(raw);
    // Only the iteration count and the cached cloud stay live across a
    // body (the particle body needs every register it can get): the stage's
    // tables are re-derived from the parameters, and the next index is
    // fetched into shared memory by the last warp at the start of each
    // virtual block.
    int cached = -1, it = 0;
    bool alive = true;
    auto run = [&](auto stageC, auto &&body) {
        constexpr int stage = decltype(stageC)::value;
        if (!alive) return;
        if (threadIdx.x == 0) sNext[it & 1] = (int)atomicAdd(bar + (3 + stage) * kBarLine, 1u);
        __syncthreads();
        for (;;)
        {
            const int gb = sNext[it & 1];
            const int *o = off + stage * (n + 1);
            if (gb >= o[n]) break;
            if (threadIdx.x == kNT - 32)
                sNext[(it + 1) & 1] = (int)atomicAdd(bar + (3 + stage) * kBarLine, 1u);
            const int c = vmap[vmap[stage] + gb];
            if (c != cached)
            {
                const unsigned long long *src =
                    reinterpret_cast<const unsigned long long *>(ctx + c);
                unsigned long long *dst = reinterpret_cast<unsigned long long *>(raw);
                for (int w = threadIdx.x; w < (int)(sizeof(BatchCtx<T>) / 8); w += blockDim.x)
                    dst[w] = src[w];
                cached = c;
                __syncthreads();
            }
            body(o[c + 1] - o[c], gb - o[c]);
            ++it;
            __syncthreads();
        }
        if (gridBarrier(bar, cap)) return;
        if (threadIdx.x == 0) atomicOr(&ctx[0].pa.sc->err, 8);
        alive = false;
    };
    // 0: counters
    run(std::integral_constant<int, 0>{}, [&](int, int vb) {
        if (vb == 0 && threadIdx.x == 0)
        {
            StepScalars *sc = B.pa.sc;
            sc->nflag = 0; sc->ndeg = 0; sc->nfix = 0; sc->moodfail = 0;
        }
    });
    // 2: transport + particle stage (fused)
    run(std::integral_constant<int, 2>{}, [&](int, int vb) { persistentParticle<T, L>(B, vb); });
    // 3: linear redo of the flagged particles
    run(std::integral_constant<int, 3>{}, [&](int vg, int vb) { persistentRedo<T, L>(B, vb, vg); });
    // 4: sigma
    run(std::integral_constant<int, 4>{}, [&](int vg, int vb) {
        StepScalars *sc = B.pa.sc;
        double m;
        if (gridSumLast(B.pa.massPos, B.p.N, B.redPartial, sc, &m, vb, vg))
        {
            sc->massNew = m;
            sc->sigma = (m > 1.0e-30) ? sc->massOld / m : 1.0;
        }
    });
    // 5: fixup
    run(std::integral_constant<int, 5>{}, [&](int vg, int vb) { k_fixup_body<T>(B.pa, B.p, vb, vg); });
    // 6: end-of-step mass
    run(std::integral_constant<int, 6>{}, [&](int vg, int vb) {
        StepScalars *sc = B.pa.sc;
        double m;
        if (gridSumLast(B.pa.massEnd, B.p.N, B.redPartial, sc, &m, vb, vg))
        {
            const double sigma = sc->sigma;
            sc->massEnd = sigma * m;
            sc->massOld = sc->massEnd;
            sc->scale = sigma;
            sc->steps += 1;
        }
    });
    // 7: sigma on the macros, moodCheck
    run(std::integral_constant<int, 7>{}, [&](int, int vb) {
        k_scale_mood_body(B.p, B.pa.boundary, B.pa.macNew, B.pa.minG, B.mood, B.pa.sc, vb);
    });
    // 8: second collision where moodCheck failed
    run(std::integral_constant<int, 8>{}, [&](int vg, int vb) { persistentRecollide<T>(B, vb, vg); });
    // 9: end mass after a second collision
    run(std::integral_constant<int, 9>{}, [&](int vg, int vb) {
        StepScalars *sc = B.pa.sc;
        double m;
        if (sc->moodfail != 0 &&
            gridSumLast(B.pa.massEnd, B.p.N, B.redPartial, sc, &m, vb, vg))
        {
            sc->massEnd = sc->sigma * m;
            sc->massOld = sc->massEnd;
        }
    });
    // 10: steady residual (1024-thread virtual blocks)
    run(std::integral_constant<int, 10>{}, [&](int, int) { persistentResidual<T>(B); });
}

#undef BATCH_CTX

template <typename T>
static cudaError_t buildBatchT(alebgk_ctx *const *cs, int n, double *const *resid,
                               BatchLaunch &bl)
{
    const int L = cs[0]->sp.L;
    std::vector<BatchCtx<T>> h[2];
    std::vector<int> off((size_t)kBatchStages * (n + 1), 0);
    size_t smemP = 0, smemR = 0;
    for (int i = 0; i < n; ++i)
    {
        alebgk_ctx *c = cs[i];
        const StepParams &p = c->sp;
        DeviceBuffers &d = c->d;
        const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
        // A batch has parallelism enough in its clouds: every particle block
        // holds as many particles as fit (the launch shape changes no result).
        const int wpb = particleWarpsPerBlock(p, sizeof(T));
        smemP = std::max(smemP, wpb * rowBytes);
        smemR = std::max(smemR, rowBytes);
        const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
        // the transport runs fused in the particle stage (stage 1 is empty)
        const int blocks[kBatchStages] = {1,
                                          0,
                                          (p.N + wpb - 1) / wpb,
                                          // the list stages mostly find empty
                                          // lists: few blocks per cloud (any
                                          // count gives the same results)
                                          std::min(p.N, 32),
                                          kRedBlocks,
                                          std::min(pBlocks, 16),
                                          kRedBlocks,
                                          (p.N + 255) / 256,
                                          p.limiter == 2 ? std::min(pBlocks, 64) : 0,
                                          p.limiter == 2 ? kRedBlocks : 0,
                                          1};
        for (int s = 0; s < kBatchStages; ++s)
            off[(size_t)s * (n + 1) + i + 1] = off[(size_t)s * (n + 1) + i] + blocks[s];
        for (int from = 0; from < 2; ++from)
        {
            BatchCtx<T> b{};
            ParticleArgs<T> &pa = b.pa;
            pa.g = static_cast<T *>(d.f[1 - from]);
            pa.fold = static_cast<const T *>(d.f[from]);
            pa.coefLin = static_cast<const T *>(d.coefLin);
            pa.coef = static_cast<const T *>(d.coef);
            pa.boundary = d.boundary; pa.cls = d.cls; pa.nslot = d.nslot; pa.slots = d.slots;
            pa.rowOrder = d.rowOrder;
            pa.wall = d.wall; pa.macPrev = d.macro[from]; pa.macNew = d.macro[1 - from];
            pa.massPos = d.massPos; pa.massEnd = d.massEnd; pa.minG = d.minG; pa.dpx = d.dpx;
            pa.flag = d.flag; pa.flagList = d.flagList; pa.degList = d.degList; pa.sc = d.sc;
            pa.nad = d.nad;
            b.p = p;
            b.mood = d.mood;
            b.redPartial = d.redPartial;
            b.resid = resid[i];
            b.wpb = wpb;
            h[from].push_back(b);
        }
    }
    for (int s = 0; s < kBatchStages; ++s) bl.blocks[s] = off[(size_t)s * (n + 1) + n];
    cudaError_t e = cudaSuccess;
    for (int from = 0; from < 2 && e == cudaSuccess; ++from)
    {
        e = cudaMalloc(&bl.desc[from], sizeof(BatchCtx<T>) * n);
        if (e == cudaSuccess)
            e = cudaMemcpy(bl.desc[from], h[from].data(), sizeof(BatchCtx<T>) * n,
                           cudaMemcpyHostToDevice);
    }
    // the persistent launch's virtual-block -> cloud tables: 16 stage
    // starts, then per stage one entry per virtual block
    std::vector<int> vm(16, 0);
    for (int s = 0; s < kBatchStages; ++s)
    {
        vm[s] = (int)vm.size();
        for (int i = 0; i < n; ++i)
            for (int b = off[(size_t)s * (n + 1) + i]; b < off[(size_t)s * (n + 1) + i + 1]; ++b)
                vm.push_back(i);
    }
    if (e == cudaSuccess) e = cudaMalloc(&bl.vmap, sizeof(int) * vm.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(bl.vmap, vm.data(), sizeof(int) * vm.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&bl.bar, kBarWords * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(bl.bar, 0, kBarWords * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMalloc(&bl.off, sizeof(int) * off.size());
    if (e == cudaSuccess)
        e = cudaMemcpy(bl.off, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice);
    bl.n = n;
    bl.L = L;
    bl.smemParticle = smemP;
    bl.smemRedo = smemR;
    return e;
}

cudaError_t buildBatchLaunch(alebgk_ctx *const *cs, int n, double *const *resid,
                             BatchLaunch &bl)
{
    bl = BatchLaunch();
    if (n < 1) return cudaErrorInvalidValue;
    alebgk_ctx *c0 = cs[0];
    for (int i = 0; i < n; ++i)
    {
        alebgk_ctx *c = cs[i];
        if (c->cfg.precision != c0->cfg.precision || c->sp.L != c0->sp.L || c->pStream ||
            c->march.enabled || c->cfg.device != c0->cfg.device)
            return cudaErrorNotSupported;
    }
    bl.f64 = c0->cfg.precision == 64;
    return bl.f64 ? buildBatchT<double>(cs, n, resid, bl) : buildBatchT<float>(cs, n, resid, bl);
}

template <typename T, int L>
static cudaError_t batchStepT(const BatchLaunch &bl, int from, cudaStream_t st)
{
    const BatchCtx<T> *ctx = static_cast<const BatchCtx<T> *>(bl.desc[from]);
    const int n = bl.n;
    const int *off = bl.off;
    auto go = [&](int s) { return bl.blocks[s] > 0; };
    if (go(0)) k_batch_begin<T><<<bl.blocks[0], kNT, 0, st>>>(ctx, off, n);
    if (go(2)) k_batch_particle<T, L><<<bl.blocks[2], kNT, bl.smemParticle, st>>>(ctx, off, n);
    if (go(3)) k_batch_redo<T, L><<<bl.blocks[3], kNT, bl.smemRedo, st>>>(ctx, off, n);
    if (go(4)) k_batch_sigma<T><<<bl.blocks[4], kRedThreads, 0, st>>>(ctx, off, n);
    if (go(5)) k_batch_fixup<T><<<bl.blocks[5], kNT, 0, st>>>(ctx, off, n);
    if (go(6)) k_batch_mass_sum<T><<<bl.blocks[6], kRedThreads, 0, st>>>(ctx, off, n);
    if (go(7)) k_batch_scale_mood<T><<<bl.blocks[7], 256, 0, st>>>(ctx, off, n);
    if (go(8)) k_batch_recollide<T><<<bl.blocks[8], kNT, 0, st>>>(ctx, off, n);
    if (go(9)) k_batch_mass_end<T><<<bl.blocks[9], kRedThreads, 0, st>>>(ctx, off, n);
    if (go(10)) k_batch_residual<T><<<bl.blocks[10], 1024, 0, st>>>(ctx, off, n);
    return cudaGetLastError();
}

template <typename T, int L>
static cudaError_t batchPrepareT(const BatchLaunch &bl)
{
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
        e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    auto set = [&](const void *fn, size_t bytes) {
        cudaFuncAttributes fa{};
        if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, fn);
        const size_t cap = (size_t)optin - fa.sharedSizeBytes;
        if (e == cudaSuccess && bytes > cap) e = cudaErrorInvalidValue;
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    };
    set((const void *)k_batch_particle<T, L>, bl.smemParticle);
    set((const void *)k_batch_redo<T, L>, bl.smemRedo);
    // the persistent form: as many blocks as are resident at once
    const size_t smemPersist = std::max(bl.smemParticle, bl.smemRedo);
    set((const void *)k_batch_persistent<T, L>, smemPersist);
    int occ = 0, sms = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_batch_persistent<T, L>, kNT,
                                                          smemPersist);
    const_cast<BatchLaunch &>(bl).pGrid = occ * sms;
    return e;
}

template <typename T, int L>
static cudaError_t batchPersistentT(const BatchLaunch &bl, int from, cudaStream_t st)
{
    int most = 0;
    for (int s = 0; s < kBatchStages; ++s) most = std::max(most, bl.blocks[s]);
    const int grid = std::min(bl.pGrid, most);
    if (grid < 1) return cudaErrorLaunchOutOfResources;
    const BatchCtx<T> *ctx = static_cast<const BatchCtx<T> *>(bl.desc[from]);
    cudaError_t e = cudaMemsetAsync(bl.bar, 0, kBarWords * sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kNT);
    cfg.dynamicSmemBytes = std::max(bl.smemParticle, bl.smemRedo);
    cfg.stream = st;
    // co-resident blocks (a cooperative launch); the barrier's poll limit
    // still ends the launch with an error if they ever were not
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_batch_persistent<T, L>, ctx, (const int *)bl.off,
                              (const int *)bl.vmap, bl.n, bl.bar, bl.spinCap);
}

cudaError_t prepareBatchLaunch(const BatchLaunch &bl)
{
    if (bl.f64) return bl.L == 2 ? batchPrepareT<double, 2>(bl) : batchPrepareT<double, 1>(bl);
    return bl.L == 2 ? batchPrepareT<float, 2>(bl) : batchPrepareT<float, 1>(bl);
}

cudaError_t launchBatchStep(const BatchLaunch &bl, int from, cudaStream_t st)
{
    if (bl.persistent)
    {
        if (bl.f64)
            return bl.L == 2 ? batchPersistentT<double, 2>(bl, from, st)
                             : batchPersistentT<double, 1>(bl, from, st);
        return bl.L == 2 ? batchPersistentT<float, 2>(bl, from, st)
                         : batchPersistentT<float, 1>(bl, from, st);
    }
    if (bl.f64) return bl.L == 2 ? batchStepT<double, 2>(bl, from, st)
                                 : batchStepT<double, 1>(bl, from, st);
    return bl.L == 2 ? batchStepT<float, 2>(bl, from, st) : batchStepT<float, 1>(bl, from, st);
}

void freeBatchLaunch(BatchLaunch &bl)
{
    for (void *p : {bl.desc[0], bl.desc[1], (void *)bl.off, (void *)bl.bar, (void *)bl.vmap})
        if (p) cudaFree(p);
    bl = BatchLaunch();
}

template <typename T>
static cudaError_t massInitT(alebgk_ctx *c)
{
    const StepParams &p = c->sp;
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    k_particle_mass<T><<<pBlocks, kNT, 0, c->stream>>>(
        static_cast<const T *>(c->d.f[c->cur]), p, c->d.massEnd);
    k_mass_init<<<kRedBlocks, kRedThreads, 0, c->stream>>>(c->d.massEnd, p.N, c->d.redPartial,
                                                            c->d.sc);
    return cudaGetLastError();
}

// One segment of the step of a slab, on stream st: the launches of stepT up
// to each global sum, with the sum restricted to the owned range.
template <typename T>
static cudaError_t slabSegT(alebgk_ctx *c, int from, int seg, cudaStream_t st)
{
    const StepParams &p = c->sp;
    DeviceBuffers &d = c->d;
    T *fa = static_cast<T *>(d.f[from]);
    T *fb = static_cast<T *>(d.f[1 - from]);
    double *macA = d.macro[from], *macB = d.macro[1 - from];
    ParticleArgs<T> pa;
    pa.g = fb; pa.fold = fa; pa.coefLin = static_cast<const T *>(d.coefLin);
    pa.coef = static_cast<const T *>(d.coef);
    pa.boundary = d.boundary; pa.cls = d.cls; pa.nslot = d.nslot; pa.slots = d.slots;
    pa.rowOrder = d.rowOrder;
    pa.wall = d.wall; pa.macPrev = macA; pa.macNew = macB;
    pa.massPos = d.massPos; pa.massEnd = d.massEnd; pa.minG = d.minG; pa.dpx = d.dpx;
    pa.flag = d.flag; pa.flagList = d.flagList; pa.degList = d.degList; pa.sc = d.sc;
    pa.nad = d.nad;
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    const int listBlocks = min(p.N, 296);
    const int lo = p.ownLo, n = p.ownHi - p.ownLo;
    const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
    if (seg == 0)
    {
        const bool nadOn = c->pStream && p.limiter == 2;
        const int nadBlocks = min((p.N + kNT / 32 - 1) / (kNT / 32), 1184);
        k_step_begin<<<nadOn ? nadBlocks : 1, kNT, 0, st>>>(
            d.sc, 1, macA, d.boundary, d.nslot, d.slots, p.S, p.N, nadOn ? d.nad : nullptr);
        const bool march = sizeof(T) == 4 && c->march.enabled;
        const bool fused = !march && !c->pStream && c->tune.transportThreads == 0;
        if (march)
        {
            cudaError_t e = launchMarch(c, from, reinterpret_cast<float *>(fb), st);
            if (e != cudaSuccess) return e;
        }
        else if (!fused)
        {
            const int tt = c->tune.transportThreads > 0 ? c->tune.transportThreads : kNT;
            dim3 gt(transportChunks(p.V), (p.N + tt / 32 - 1) / (tt / 32));
            k_transport<T><<<gt, tt, 0, st>>>(fa, fb, static_cast<const T *>(d.coef), d.cls,
                                               d.nslot, d.slots, p.S, p.N, p.V, p.L, p.ldf,
                                               d.sc);
        }
        const int wmax = particleWarpsPerBlock(p, sizeof(T));
        const int wpb = (c->tune.particleWarps > 0 && c->tune.particleWarps < wmax)
                            ? c->tune.particleWarps : wmax;
        const int ppBlocks = (p.N + wpb - 1) / wpb;
        if (c->pStream)
            launchParticleStream<T>(c, pa, p, st);
        else if (fused && p.L == 2)
            k_particle<T, 2, true><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
        else if (fused) k_particle<T, 1, true><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
        else if (p.L == 2)
            k_particle<T, 2, false><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
        else k_particle<T, 1, false><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
        if (p.L == 2) k_redo<T, 2><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
        else k_redo<T, 1><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
        k_sum_range<<<kRedBlocks, kRedThreads, 0, st>>>(d.massPos + lo, n, d.redPartial, d.sc,
                                                        0, 0);
    }
    else if (seg == 1)
    {
        k_fixup<T><<<min(pBlocks, 296), kNT, 0, st>>>(pa, p);
        k_sum_range<<<kRedBlocks, kRedThreads, 0, st>>>(d.massEnd + lo, n, d.redPartial, d.sc,
                                                        1, 0);
    }
    else if (seg == 2)
        k_scale_mood<<<(p.N + 255) / 256, 256, 0, st>>>(p, d.boundary, macB, d.minG, d.mood,
                                                         d.sc);
    else if (seg == 3 && p.limiter == 2)
    {
        k_recollide<T><<<min(pBlocks, 592), kNT, 0, st>>>(fb, p, d.boundary, macB, d.massEnd,
                                                         d.sc);
        k_sum_range<<<kRedBlocks, kRedThreads, 0, st>>>(d.massEnd + lo, n, d.redPartial, d.sc,
                                                        2, 1);
    }
    return cudaGetLastError();
}

cudaError_t launchSlabSegment(alebgk_ctx *c, int from, int seg, cudaStream_t st)
{
    return (c->cfg.precision == 64) ? slabSegT<double>(c, from, seg, st)
                                    : slabSegT<float>(c, from, seg, st);
}

cudaError_t launchSlabCombine(StepScalars *const *scs, int n, int phase, cudaStream_t st)
{
    k_slab_combine<<<1, 32, 0, st>>>(scs, n, phase);
    return cudaGetLastError();
}

cudaError_t launchRankCombine(alebgk_ctx *c, const double *allDev, int n, int phase,
                              cudaStream_t st)
{
    k_rank_combine<<<1, 32, 0, st>>>(c->d.sc, allDev, n, phase);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t slabInitT(alebgk_ctx *c, cudaStream_t st)
{
    const StepParams &p = c->sp;
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    k_particle_mass<T><<<pBlocks, kNT, 0, st>>>(static_cast<const T *>(c->d.f[c->cur]), p,
                                                c->d.massEnd);
    k_sum_range<<<kRedBlocks, kRedThreads, 0, st>>>(c->d.massEnd + p.ownLo, p.ownHi - p.ownLo,
                                                    c->d.redPartial, c->d.sc, 1, 0);
    return cudaGetLastError();
}

cudaError_t launchSlabInitSum(alebgk_ctx *c, cudaStream_t st)
{
    return (c->cfg.precision == 64) ? slabInitT<double>(c, st) : slabInitT<float>(c, st);
}

cudaError_t launchMassInit(alebgk_ctx *c)
{
    return (c->cfg.precision == 64) ? massInitT<double>(c) : massInitT<float>(c);
}

template <typename T>
static cudaError_t bodyLoadsT(alebgk_ctx *c, int nbodies, const double *centre,
                              const double *area)
{
    const StepParams &p = c->sp;
    k_body_contrib<T><<<p.N, kNT, 0, c->stream>>>(
        static_cast<const T *>(c->d.f[c->cur]), p, c->d.bodyId, c->d.boundary,
        c->d.pos, c->d.wall, centre, area, c->d.bodyTmp, c->d.sc);
    k_body_sum<<<1, 384, 0, c->stream>>>(c->d.bodyTmp, c->d.bodyId,
                                         c->d.boundary, p.N, nbodies,
                                         c->d.bodyOut);
    return cudaGetLastError();
}

cudaError_t launchBodyLoads(alebgk_ctx *c, int nbodies, const double *centre,
                            const double *area)
{
    return (c->cfg.precision == 64) ? bodyLoadsT<double>(c, nbodies, centre, area)
                                    : bodyLoadsT<float>(c, nbodies, centre, area);
}

cudaError_t launchSetSurfaceVelocity(alebgk_ctx *c, int nbodies,
                                     const double *centre, const double *state)
{
    (void)nbodies;
    const int N = c->sp.N;
    k_set_surface_velocity<<<(N + 255) / 256, 256, 0, c->stream>>>(
        N, c->sp.dim, c->d.bodyId, c->d.boundary, c->d.pos, c->d.wall, centre,
        state);
    return cudaGetLastError();
}

cudaError_t launchResidual(alebgk_ctx *c, double *out, cudaStream_t st)
{
    k_residual<<<1, 1024, 0, st>>>(c->d.macro[c->cur], c->d.macro[1 - c->cur], c->d.boundary,
                                   c->sp.N, c->sp.R, out, c->sp.resU);
    return cudaGetLastError();
}

cudaError_t launchConvertIn(alebgk_ctx *c, const double *src, int buf)
{
    const StepParams &p = c->sp;
    if (c->cfg.precision == 64)
        k_convert_in<double><<<1184, 256, 0, c->stream>>>(
            src, static_cast<double *>(c->d.f[buf]), p.N, p.gs, p.ldf);
    else
        k_convert_in<float><<<1184, 256, 0, c->stream>>>(
            src, static_cast<float *>(c->d.f[buf]), p.N, p.gs, p.ldf);
    return cudaGetLastError();
}

cudaError_t launchRowsBuild(alebgk_ctx *c, int n, const int *a, const int *b,
                            const double *fresh, double *out)
{
    const StepParams &p = c->sp;
    if (c->cfg.precision == 64)
        k_rows_build<double><<<1184, 256, 0, c->stream>>>(
            static_cast<const double *>(c->d.f[c->cur]), p.ldf, p.gs, n, a, b, fresh, c->d.sc,
            out);
    else
        k_rows_build<float><<<1184, 256, 0, c->stream>>>(
            static_cast<const float *>(c->d.f[c->cur]), p.ldf, p.gs, n, a, b, fresh, c->d.sc,
            out);
    return cudaGetLastError();
}

cudaError_t launchConvertOut(alebgk_ctx *c, double *dst, int buf)
{
    const StepParams &p = c->sp;
    if (c->cfg.precision == 64)
        k_convert_out<double><<<1184, 256, 0, c->stream>>>(
            static_cast<const double *>(c->d.f[buf]), dst, p.N, p.gs, p.ldf, c->d.sc);
    else
        k_convert_out<float><<<1184, 256, 0, c->stream>>>(
            static_cast<const float *>(c->d.f[buf]), dst, p.N, p.gs, p.ldf, c->d.sc);
    return cudaGetLastError();
}

}  // namespace alebgk
