// step.cu -- device kernels of the ALE-BGK time step for sm_100a.
//
// One step (the CPU step order of Solver/Solver.cpp:632-705):
//   k_step_begin      reset the step's counters
//   k_transport       gt[i][k] = scale * sum_s coef[class][s][k] * h[slot s][k]
//   k_particle        per particle (one warp): positivity repair, MOOD PAD/NAD
//                     screen with linear redo, diffuse wall or moments + BGK
//                     collision + moments, without the global rescale
//   k_sigma           deterministic mass sums -> global rescale sigma
//   k_scale_mood      sigma on the macros, moodCheck
//   k_recollide       second collision when moodCheck failed (else exits)
//   k_mass_end        end-of-step mass after a second collision (else exits)
// The stored state h is the true distribution divided by StepScalars::scale.
// All reductions are FP64 and in a fixed order, so a step is bitwise
// reproducible.  No kernel waits on another block, so none can hang.
#include <cuda_runtime.h>

#include <cmath>

#include "ctx.h"

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
// Transport: coefficient gather.  Thread = (particle, node); the node's
// coefficients are shared by both Chu layers in 2-D.  The output is scaled
// by the stored-state scale so that gt carries the true magnitude.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_transport(const T *__restrict__ f, T *__restrict__ g,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int V, int L, int ldf, const StepScalars *__restrict__ sc)
{
    const int i = blockIdx.x;
    const int k = blockIdx.y * blockDim.x + threadIdx.x;
    if (k >= V) return;
    const T scale = T(sc->scale);
    const int c = cls[i], ns = nslot[i];
    const T *cc = coef + (size_t)c * S * V + k;
    const int *sl = slots + (size_t)i * S;
    T a0 = T(0), a1 = T(0);
    if (L == 2)
    {
        for (int s = 0; s < ns; ++s)
        {
            const T cs = __ldg(cc + (size_t)s * V);
            const T *fr = f + (size_t)__ldg(sl + s) * ldf + k;
            a0 = fma(cs, __ldg(fr), a0);
            a1 = fma(cs, __ldg(fr + V), a1);
        }
        g[(size_t)i * ldf + k] = a0 * scale;
        g[(size_t)i * ldf + V + k] = a1 * scale;
    }
    else
    {
        for (int s = 0; s < ns; ++s)
        {
            const T cs = __ldg(cc + (size_t)s * V);
            a0 = fma(cs, __ldg(f + (size_t)__ldg(sl + s) * ldf + k), a0);
        }
        g[(size_t)i * ldf + k] = a0 * scale;
    }
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
    const T *coefLin;         // linear MLS tables (MOOD redo)
    const int *boundary, *cls, *nslot, *slots;
    const double *wall, *macPrev;
    double *macNew, *massPos, *massEnd, *minG, *dpx;
    int *flag, *flagList, *degList;
    StepScalars *sc;
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
template <typename T, int L>
__device__ void finishParticle(const ParticleArgs<T> &a, const StepParams &p, int i,
                               RowRegs<T, L> &r, const Positivity &pv, double (*tb)[kMaxNv])
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
        double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9;
        if (rn < lo - slack || rn > hi + slack) return 1;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Positivity + MOOD screen + finish, one warp per particle.  A particle the
// screen flags is listed for k_redo and left as is.
// ---------------------------------------------------------------------------
template <typename T, int L>
__global__ void __launch_bounds__(kNT)
k_particle(ParticleArgs<T> a, StepParams p, int warpsPerBlock)
{
    __shared__ double tab[kNT / 32][3][kMaxNv];
    extern __shared__ __align__(16) unsigned char rowSmem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp >= warpsPerBlock) return;
    const int i = blockIdx.x * warpsPerBlock + warp;
    if (i >= p.N) return;                        // warp-uniform
    T *buf = reinterpret_cast<T *>(rowSmem) + (size_t)warp * L * p.V;
    RowRegs<T, L> r(a.g + (size_t)i * p.ldf, buf, p, lane);
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
    finishParticle(a, p, i, r, pv, tab[warp]);
}

// ---------------------------------------------------------------------------
// Linear MLS redo of the flagged particles (Solver/Solver.cpp:641-646:
// mlsTransportCompute(..., 1, onlyFlagged=true)) from the pre-transport
// state, one block per particle, then positivity and finish on warp 0.
// ---------------------------------------------------------------------------
template <typename T, int L>
__global__ void __launch_bounds__(kNT)
k_redo(ParticleArgs<T> a, StepParams p)
{
    __shared__ double tab[3][kMaxNv];
    extern __shared__ __align__(16) unsigned char rowSmem[];
    const int nflag = a.sc->nflag;
    const T scale = T(a.sc->scale);
    for (int li = blockIdx.x; li < nflag; li += gridDim.x)
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

// Finishes the listed particles once sigma is known, on true magnitudes:
// moments (kept from the previous step when the row has no positive mass,
// Moments.cpp:89), collision, moments; stored as h = g / sigma with the
// macros' density and pressure divided by sigma, as k_scale_mood expects.
template <typename T>
__global__ void __launch_bounds__(kNT)
k_fixup(ParticleArgs<T> a, StepParams p)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ndeg = a.sc->ndeg;
    const double sigma = a.sc->sigma;
    const int V = p.V, dim = p.dim;
    for (int li = blockIdx.x * (kNT / 32) + warp; li < ndeg; li += gridDim.x * (kNT / 32))
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

// Deterministic single-block sums; thread t sums a contiguous chunk.
template <int K>
__device__ void blockReduceArrays(const double *const (&a)[K], int N, double (&out)[K],
                                  double *sh)
{
    const int t = threadIdx.x, nt = blockDim.x;
    const int chunk = (N + nt - 1) / nt;
    const int lo = t * chunk, hi = min(N, lo + chunk);
    double v[K];
#pragma unroll
    for (int q = 0; q < K; ++q)
    {
        double s = 0.0;
        for (int i = lo; i < hi; ++i) s += a[q][i];
        v[q] = s;
    }
    blockSums<K>(v, sh);
#pragma unroll
    for (int q = 0; q < K; ++q) out[q] = v[q];
}

// Global mass rescale (Solver/Solver.cpp:650-655): sigma = massOld/massNew.
__global__ void __launch_bounds__(1024)
k_sigma(const double *__restrict__ massPos, int N, StepScalars *sc)
{
    __shared__ double sh[32];
    const double *const a[1] = {massPos};
    double out[1];
    blockReduceArrays<1>(a, N, out, sh);
    if (threadIdx.x == 0)
    {
        sc->massNew = out[0];
        sc->sigma = (out[0] > 1.0e-30) ? sc->massOld / out[0] : 1.0;
    }
}

// Mass at the end of the step (the next step's massOld); the stored state
// now carries the scale sigma.
__global__ void __launch_bounds__(1024)
k_mass_sum(const double *__restrict__ massEnd, int N, StepScalars *sc)
{
    __shared__ double sh[32];
    const double *const a[1] = {massEnd};
    double out[1];
    blockReduceArrays<1>(a, N, out, sh);
    if (threadIdx.x == 0)
    {
        const double sigma = sc->sigma;
        sc->massEnd = sigma * out[0];
        sc->massOld = sc->massEnd;
        sc->scale = sigma;
        sc->steps += 1;
    }
}

// Applies sigma to the macros and runs moodCheck (Conservation.cpp:16-38,
// MLSBasis.hpp:208-222) on the true values.
__global__ void k_scale_mood(StepParams p, const int *__restrict__ boundary,
                             double *__restrict__ macNew, const double *__restrict__ minG,
                             int *__restrict__ mood, StepScalars *sc)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.N) return;
    const double sigma = sc->sigma;
    double *mac = macNew + 6 * (size_t)i;
    mac[0] *= sigma;
    mac[5] *= sigma;
    if (p.limiter != 2) return;
    if (boundary[i]) { mood[i] = 0; return; }
    const int fail = (mac[0] < 1.0e-10) || (mac[4] < 1.0e-6) || (sigma * minG[i] < -1.0e-14);
    mood[i] = fail;
    if (fail) atomicOr(&sc->moodfail, 1);
}

// Second collision + moments of every interior particle when moodCheck
// failed (Solver/Solver.cpp:685-693).  Exits at once otherwise.
template <typename T>
__global__ void __launch_bounds__(kNT)
k_recollide(T *__restrict__ g, StepParams p, const int *__restrict__ boundary,
            double *__restrict__ macNew, double *__restrict__ massEnd, StepScalars *sc)
{
    if (sc->moodfail == 0) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kNT / 32) + warp;
    if (i >= p.N || boundary[i]) return;
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

// Mass at the end of a step whose moodCheck failed (after k_recollide).
__global__ void __launch_bounds__(1024)
k_mass_end(const double *__restrict__ massEnd, int N, StepScalars *sc)
{
    if (sc->moodfail == 0) return;
    __shared__ double sh[32];
    const double *const a[1] = {massEnd};
    double out[1];
    blockReduceArrays<1>(a, N, out, sh);
    if (threadIdx.x == 0)
    {
        sc->massEnd = sc->sigma * out[0];
        sc->massOld = sc->massEnd;
    }
}

__global__ void k_step_begin(StepScalars *sc)
{
    sc->nflag = 0;
    sc->ndeg = 0;
    sc->nfix = 0;
    sc->moodfail = 0;
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

__global__ void __launch_bounds__(1024)
k_mass_init(const double *__restrict__ massEnd, int N, StepScalars *sc)
{
    __shared__ double sh[32];
    const double *const a[1] = {massEnd};
    double out[1];
    blockReduceArrays<1>(a, N, out, sh);
    if (threadIdx.x == 0)
    {
        sc->massOld = out[0];
        sc->massEnd = out[0];
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
    pa.boundary = d.boundary; pa.cls = d.cls; pa.nslot = d.nslot; pa.slots = d.slots;
    pa.wall = d.wall; pa.macPrev = macA; pa.macNew = macB;
    pa.massPos = d.massPos; pa.massEnd = d.massEnd; pa.minG = d.minG; pa.dpx = d.dpx;
    pa.flag = d.flag; pa.flagList = d.flagList; pa.degList = d.degList; pa.sc = d.sc;
    int q = 0;
    auto mark = [&]() { if (ev) cudaEventRecord(ev[q++], st); };
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    const int listBlocks = min(p.N, 1184);
    mark();
    k_step_begin<<<1, 1, 0, st>>>(d.sc);
    mark();
    if (sizeof(T) == 4 && c->march.enabled)
    {
        cudaError_t e = launchMarch(c, c->march.tmap[from], reinterpret_cast<float *>(fb), st);
        if (e != cudaSuccess) return e;
    }
    else
    {
        dim3 gt(p.N, (p.V + kNT - 1) / kNT);
        k_transport<T><<<gt, kNT, 0, st>>>(fa, fb, static_cast<const T *>(d.coef),
                                           d.cls, d.nslot, d.slots, p.S, p.V, p.L,
                                           p.ldf, d.sc);
    }
    mark();
    const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
    const int wpb = particleWarpsPerBlock(p, sizeof(T));
    const int ppBlocks = (p.N + wpb - 1) / wpb;
    if (p.L == 2) k_particle<T, 2><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
    else k_particle<T, 1><<<ppBlocks, kNT, wpb * rowBytes, st>>>(pa, p, wpb);
    mark();
    if (p.L == 2) k_redo<T, 2><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
    else k_redo<T, 1><<<listBlocks, kNT, rowBytes, st>>>(pa, p);
    mark();
    k_sigma<<<1, 1024, 0, st>>>(d.massPos, p.N, d.sc);
    mark();
    k_fixup<T><<<min(pBlocks, 296), kNT, 0, st>>>(pa, p);
    mark();
    k_mass_sum<<<1, 1024, 0, st>>>(d.massEnd, p.N, d.sc);
    mark();
    k_scale_mood<<<(p.N + 255) / 256, 256, 0, st>>>(p, d.boundary, macB, d.minG, d.mood, d.sc);
    mark();
    if (p.limiter == 2)
        k_recollide<T><<<pBlocks, kNT, 0, st>>>(fb, p, d.boundary, macB, d.massEnd, d.sc);
    mark();
    if (p.limiter == 2) k_mass_end<<<1, 1024, 0, st>>>(d.massEnd, p.N, d.sc);
    mark();
    return cudaGetLastError();
}

template <typename T>
static cudaError_t prepareT(alebgk_ctx *c)
{
    const StepParams &p = c->sp;
    const size_t rowBytes = (size_t)p.L * p.V * sizeof(T);
    const int wpb = particleWarpsPerBlock(p, sizeof(T));
    cudaError_t e = cudaSuccess;
    auto set = [&](const void *fn, size_t bytes) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    };
    set((const void *)k_particle<T, 1>, wpb * rowBytes);
    set((const void *)k_particle<T, 2>, wpb * rowBytes);
    set((const void *)k_redo<T, 1>, rowBytes);
    set((const void *)k_redo<T, 2>, rowBytes);
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

template <typename T>
static cudaError_t massInitT(alebgk_ctx *c)
{
    const StepParams &p = c->sp;
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    k_particle_mass<T><<<pBlocks, kNT, 0, c->stream>>>(
        static_cast<const T *>(c->d.f[c->cur]), p, c->d.massEnd);
    k_mass_init<<<1, 1024, 0, c->stream>>>(c->d.massEnd, p.N, c->d.sc);
    return cudaGetLastError();
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
