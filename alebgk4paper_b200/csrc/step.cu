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
    __device__ NodeWalk(int lane, int Nv_, int dim) : k(lane), Nv(Nv_)
    {
        iv = lane % Nv; jv = (lane / Nv) % Nv; kv = (dim == 3) ? lane / (Nv * Nv) : 0;
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

// ---------------------------------------------------------------------------
// Everything between transport and the global rescale, one warp per
// particle: positivity repair, MOOD PAD/NAD screen with the linear redo of a
// flagged particle (MLSTransport.cpp:189-200, 325-379; Solver/Solver.cpp:
// 641-646), diffuse wall (BoundaryConditions/DiffuseWall.cpp:19-154) or
// moments + implicit BGK collision + moments (Moments.cpp:17-97,
// Collision.cpp:70-139).  The global rescale sigma of the step is not known
// yet; every operation here is homogeneous of degree one in g, so the row is
// finished without it and sigma is applied afterwards (k_scale_mood).
// Maxwellians are evaluated as products of per-axis exponentials.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_particle(T *__restrict__ g, const T *__restrict__ fold,
           const T *__restrict__ coefLin, StepParams p,
           const int *__restrict__ boundary, const double *__restrict__ wall,
           const int *__restrict__ cls, const int *__restrict__ nslot,
           const int *__restrict__ slots, const double *__restrict__ macPrev,
           double *__restrict__ macNew, int *__restrict__ flag,
           double *__restrict__ massPos, double *__restrict__ massEnd,
           double *__restrict__ minG, double *__restrict__ dpx, StepScalars *sc)
{
    __shared__ double tab[kNT / 32][3][kMaxNv];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * (kNT / 32) + warp;
    if (i >= p.N) return;                        // warp-uniform
    T *row = g + (size_t)i * p.ldf;
    const int V = p.V, Nv = p.Nv, dim = p.dim;
    double (*tb)[kMaxNv] = tab[warp];

    double pos, neg;
    bool bad;
    rowSigns(row, V, lane, pos, neg, bad);
    double m = pos + neg;
    // positivity repairs of the first transport pass (the redo's own repair
    // is not counted, as in MLSTransport.cpp's counters)
    const bool fixFirst = Positivity(pos, neg).fix;
    int flagged = 0;
    const int bnd = boundary[i];
    if (p.limiter == 2 && !bnd)
    {
        if (bad || m <= 0.0) flagged = 1;
        else
        {
            const int ns = nslot[i];
            const int *sl = slots + (size_t)i * p.S;
            double lo = INFINITY, hi = -INFINITY;
            for (int s = 1 + lane; s < ns; s += 32)
            {
                double r = macPrev[6 * (size_t)sl[s]];
                lo = fmin(lo, r);
                hi = fmax(hi, r);
            }
            lo = warpMin(lo);
            hi = warpMax(hi);
            if (isfinite(lo) && isfinite(hi))
            {
                double rn = m * p.dvN;
                double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9;
                if (rn < lo - slack || rn > hi + slack) flagged = 1;
            }
        }
        if (flagged)
        {
            // Linear MLS from the pre-transport state (order 1 tables).
            const T scale = T(sc->scale);
            const int ns = nslot[i];
            const int *sl = slots + (size_t)i * p.S;
            const T *cl = coefLin + (size_t)cls[i] * p.S * V;
            for (int k = lane; k < V; k += 32)
            {
                T a0 = T(0), a1 = T(0);
                for (int s = 0; s < ns; ++s)
                {
                    const T cs = cl[(size_t)s * V + k];
                    const T *fr = fold + (size_t)sl[s] * p.ldf + k;
                    a0 = fma(cs, fr[0], a0);
                    if (p.L == 2) a1 = fma(cs, fr[V], a1);
                }
                row[k] = a0 * scale;
                if (p.L == 2) row[V + k] = a1 * scale;
            }
            __syncwarp();
            rowSigns(row, V, lane, pos, neg, bad);
            m = pos + neg;
            if (lane == 0) atomicAdd(&sc->nflag, 1);
        }
    }
    const Positivity pv(pos, neg);
    if (lane == 0)
    {
        flag[i] = flagged;
        massPos[i] = m * p.dvN;
        if (fixFirst) atomicAdd(&sc->nfix, 1);
    }
    double *mac = macNew + 6 * (size_t)i;
    const double *mp = macPrev + 6 * (size_t)i;

    if (bnd)
    {
        const double *w = wall + 7 * (size_t)i;
        const double Ux = w[3], Uy = w[4], Uz = w[5], Tw = w[6];
        const double RT2w = 2.0 * p.R * Tw;
        const double norm = (dim == 3) ? pow(kPi * RT2w, 1.5) : kPi * RT2w;
        for (int a = lane; a < Nv; a += 32)
        {
            double va = fma((double)a, p.dv, p.vmin);
            tb[0][a] = exp(-(va - Ux) * (va - Ux) / RT2w);
            tb[1][a] = exp(-(va - Uy) * (va - Uy) / RT2w);
            tb[2][a] = (dim == 3) ? exp(-(va - Uz) * (va - Uz) / RT2w) : 1.0;
        }
        __syncwarp();
        double iM = 0.0, iP = 0.0;
        NodeWalk nw(lane, Nv, dim);
        for (; nw.k < V; nw.next())
        {
            double vx = fma((double)nw.iv, p.dv, p.vmin);
            double vy = fma((double)nw.jv, p.dv, p.vmin);
            double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
            const double cn = bcCn(dim, vx, vy, vz, w);
            if (cn < 0.0) iM += cn * pv.v1((double)row[nw.k]) * p.dvN;
            else if (cn > 0.0)
                iP += cn * (tb[0][nw.iv] * tb[1][nw.jv] * tb[2][nw.kv] / norm) * p.dvN;
        }
        iM = warpSum(iM);
        iP = warpSum(iP);
        const double rhow = (iP > 1.0e-30) ? (-iM / iP) : 1.0;
        double dp = 0.0, ms = 0.0;
        NodeWalk nw2(lane, Nv, dim);
        for (; nw2.k < V; nw2.next())
        {
            const int k = nw2.k;
            double vx = fma((double)nw2.iv, p.dv, p.vmin);
            double vy = fma((double)nw2.jv, p.dv, p.vmin);
            double vz = (dim == 3) ? fma((double)nw2.kv, p.dv, p.vmin) : 0.0;
            const double cn = bcCn(dim, vx, vy, vz, w);
            const double g1 = (double)row[k];
            double h1 = pv.v1(g1);
            double h2 = (p.L == 2) ? pv.v2(g1, (double)row[V + k]) : 0.0;
            if (cn > 0.0)
            {
                double Mw = rhow * (tb[0][nw2.iv] * tb[1][nw2.jv] * tb[2][nw2.kv]) / norm;
                dp += vx * (Mw - h1) * p.dvN;
                h1 = Mw;
                h2 = 0.5 * p.R * Tw * Mw;
            }
            ms += h1;
            row[k] = T(h1);
            if (p.L == 2) row[V + k] = T(h2);
        }
        dp = warpSum(dp);
        ms = warpSum(ms);
        if (lane == 0)
        {
            mac[0] = rhow; mac[1] = Ux; mac[2] = Uy;
            mac[3] = (dim == 3) ? Uz : mp[3];
            mac[4] = Tw; mac[5] = rhow * p.R * Tw;
            dpx[i] = dp;
            massEnd[i] = ms * p.dvN;
            minG[i] = 0.0;
        }
        return;
    }

    // Interior: moments of the repaired row.
    double M0 = 0, Mx = 0, My = 0, Mz = 0, ME = 0;
    {
        NodeWalk nw(lane, Nv, dim);
        for (; nw.k < V; nw.next())
        {
            double vx = fma((double)nw.iv, p.dv, p.vmin);
            double vy = fma((double)nw.jv, p.dv, p.vmin);
            double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
            const double g1 = (double)row[nw.k];
            const double f1 = pv.v1(g1) * p.dvN;
            M0 += f1; Mx += vx * f1; My += vy * f1; Mz += vz * f1;
            ME += (vx * vx + vy * vy + vz * vz) * f1;
            if (p.L == 2) ME += 2.0 * pv.v2(g1, (double)row[V + nw.k]) * p.dvN;
        }
    }
    M0 = warpSum(M0); Mx = warpSum(Mx); My = warpSum(My); Mz = warpSum(Mz); ME = warpSum(ME);
    double rho = mp[0], ux = mp[1], uy = mp[2], uz = mp[3], Tt = mp[4];
    if (M0 > 1.0e-30)
    {
        rho = M0; ux = Mx / M0; uy = My / M0;
        uz = (dim == 3) ? Mz / M0 : mp[3];
        double u2 = ux * ux + uy * uy + uz * uz;
        Tt = fmax((ME / M0 - u2) / (3.0 * p.R), 1.0e-6);
    }
    // Implicit BGK toward the Maxwellian of these moments.
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
    for (int a = lane; a < Nv; a += 32)
    {
        double va = fma((double)a, p.dv, p.vmin);
        tb[0][a] = exp(-(va - ux) * (va - ux) / twoRT);
        tb[1][a] = exp(-(va - uy) * (va - uy) / twoRT);
        tb[2][a] = (dim == 3) ? exp(-(va - uz) * (va - uz) / twoRT) : 1.0;
    }
    __syncwarp();
    double N0 = 0, Nx = 0, Ny = 0, Nz = 0, NE = 0, mn = INFINITY;
    const double halfRT = 0.5 * p.R * Tt;
    {
        NodeWalk nw(lane, Nv, dim);
        for (; nw.k < V; nw.next())
        {
            const int k = nw.k;
            double vx = fma((double)nw.iv, p.dv, p.vmin);
            double vy = fma((double)nw.jv, p.dv, p.vmin);
            double vz = (dim == 3) ? fma((double)nw.kv, p.dv, p.vmin) : 0.0;
            const double g1 = (double)row[k];
            const double M = A * (tb[0][nw.iv] * tb[1][nw.jv] * tb[2][nw.kv]);
            const double h1 = c1 * (pv.v1(g1) + lam * M);
            const T h1s = T(h1);
            row[k] = h1s;
            const double f1 = (double)h1s * p.dvN;
            N0 += f1; Nx += vx * f1; Ny += vy * f1; Nz += vz * f1;
            NE += (vx * vx + vy * vy + vz * vz) * f1;
            mn = fmin(mn, (double)h1s);
            if (p.L == 2)
            {
                const double h2 = c1 * (pv.v2(g1, (double)row[V + k]) + lam * halfRT * M);
                const T h2s = T(h2);
                row[V + k] = h2s;
                NE += 2.0 * (double)h2s * p.dvN;
            }
        }
    }
    N0 = warpSum(N0); Nx = warpSum(Nx); Ny = warpSum(Ny); Nz = warpSum(Nz); NE = warpSum(NE);
    mn = warpMin(mn);
    if (lane == 0)
    {
        double r2 = rho, x2 = ux, y2 = uy, z2 = uz, T2 = Tt;
        if (N0 > 1.0e-30)
        {
            r2 = N0; x2 = Nx / N0; y2 = Ny / N0;
            z2 = (dim == 3) ? Nz / N0 : uz;
            double u2 = x2 * x2 + y2 * y2 + z2 * z2;
            T2 = fmax((NE / N0 - u2) / (3.0 * p.R), 1.0e-6);
        }
        mac[0] = r2; mac[1] = x2; mac[2] = y2; mac[3] = z2; mac[4] = T2;
        mac[5] = r2 * p.R * T2;
        dpx[i] = 0.0;
        massEnd[i] = N0;
        minG[i] = mn;
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

// Global mass rescale (Solver/Solver.cpp:650-655): sigma = massOld/massNew,
// and the mass at the end of the step, which is the next step's massOld.
__global__ void __launch_bounds__(1024)
k_sigma(const double *__restrict__ massPos, const double *__restrict__ massEnd, int N,
        StepScalars *sc)
{
    __shared__ double sh[2 * 32];
    const double *const a[2] = {massPos, massEnd};
    double out[2];
    blockReduceArrays<2>(a, N, out, sh);
    if (threadIdx.x == 0)
    {
        const double mOld = sc->massOld;
        const double sigma = (out[0] > 1.0e-30) ? mOld / out[0] : 1.0;
        sc->massNew = out[0];
        sc->sigma = sigma;
        sc->massEnd = sigma * out[1];
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
// Launches one step.  With ev != nullptr an event is recorded before each
// launch and after the last one (ev[0..8]), in launch order: step_begin,
// transport, particle, sigma, scale_mood, recollide, mass_end.
template <typename T>
static cudaError_t stepT(alebgk_ctx *c, int from, cudaEvent_t *ev)
{
    const StepParams &p = c->sp;
    DeviceBuffers &d = c->d;
    cudaStream_t st = c->stream;
    T *fa = static_cast<T *>(d.f[from]);
    T *fb = static_cast<T *>(d.f[1 - from]);
    double *macA = d.macro[from], *macB = d.macro[1 - from];
    int q = 0;
    auto mark = [&]() { if (ev) cudaEventRecord(ev[q++], st); };
    const int pBlocks = (p.N + kNT / 32 - 1) / (kNT / 32);
    mark();
    k_step_begin<<<1, 1, 0, st>>>(d.sc);
    mark();
    dim3 gt(p.N, (p.V + kNT - 1) / kNT);
    k_transport<T><<<gt, kNT, 0, st>>>(fa, fb, static_cast<const T *>(d.coef),
                                       d.cls, d.nslot, d.slots, p.S, p.V, p.L,
                                       p.ldf, d.sc);
    mark();
    k_particle<T><<<pBlocks, kNT, 0, st>>>(fb, fa, static_cast<const T *>(d.coefLin), p,
                                           d.boundary, d.wall, d.cls, d.nslot, d.slots,
                                           macA, macB, d.flag, d.massPos, d.massEnd,
                                           d.minG, d.dpx, d.sc);
    mark();
    k_sigma<<<1, 1024, 0, st>>>(d.massPos, d.massEnd, p.N, d.sc);
    mark();
    k_scale_mood<<<(p.N + 255) / 256, 256, 0, st>>>(p, d.boundary, macB, d.minG, d.mood, d.sc);
    mark();
    if (p.limiter == 2)
        k_recollide<T><<<pBlocks, kNT, 0, st>>>(fb, p, d.boundary, macB, d.massEnd, d.sc);
    mark();
    if (p.limiter == 2) k_mass_end<<<1, 1024, 0, st>>>(d.massEnd, p.N, d.sc);
    mark();
    mark();
    return cudaGetLastError();
}

template <typename T>
static cudaError_t prepareT(alebgk_ctx *c)
{
    (void)c;
    return cudaFuncSetCacheConfig(k_particle<T>, cudaFuncCachePreferL1);
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
