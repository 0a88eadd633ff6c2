// step.cu -- device kernels of the ALE-BGK time step for sm_100a.
//
// One step (the CPU step order of Solver/Solver.cpp:632-705):
//   k_transport        gt[i][k] = sum_s coef[class][s][k] * f[slot s][k]
//   k_post_transport   per-particle positivity repair + MOOD PAD/NAD screen
//   k_redo             flagged particles re-transported with linear MLS
//   k_mass_reduce      deterministic sum -> global rescale sigma
//   k_finalize         sigma, diffuse wall / moments + BGK collision +
//                      moments, moodCheck, per-particle mass
//   k_recollide        conditional second collision when moodCheck failed
//   k_mass_reduce      mass at the end of the step (next step's massOld)
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
// coefficients are shared by both Chu layers in 2-D.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_transport(const T *__restrict__ f, T *__restrict__ g,
            const T *__restrict__ coef, const int *__restrict__ cls,
            const int *__restrict__ nslot, const int *__restrict__ slots,
            int S, int V, int L, int ldf)
{
    const int i = blockIdx.x;
    const int k = blockIdx.y * blockDim.x + threadIdx.x;
    if (k >= V) return;
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
        g[(size_t)i * ldf + k] = a0;
        g[(size_t)i * ldf + V + k] = a1;
    }
    else
    {
        for (int s = 0; s < ns; ++s)
        {
            const T cs = __ldg(cc + (size_t)s * V);
            a0 = fma(cs, __ldg(f + (size_t)__ldg(sl + s) * ldf + k), a0);
        }
        g[(size_t)i * ldf + k] = a0;
    }
}

// Positivity repair on one particle row (MLSTransport.cpp:189-200 in 3-D,
// 283-309 in 2-D, where the g1 sign also zeroes g2).  Returns the mass-layer
// sum after the repair and whether any value was non-finite.
template <typename T>
__device__ void positivity(T *row, int V, int L, double *sh, int nfixAdd,
                           StepScalars *sc, double &m, bool &bad)
{
    double v3[3] = {0.0, 0.0, 0.0};
    for (int k = threadIdx.x; k < V; k += blockDim.x)
    {
        double v = (double)row[k];
        if (!isfinite(v)) v3[2] = 1.0;
        if (v >= 0.0) v3[0] += v; else v3[1] += v;
    }
    blockSums<3>(v3, sh);
    const double pos = v3[0], neg = v3[1];
    bad = v3[2] != 0.0;
    if (neg < -1.0e-30 && pos > 1.0e-30 && (pos + neg) > 0.0)
    {
        const double s = (pos + neg) / pos;
        for (int k = threadIdx.x; k < V; k += blockDim.x)
        {
            double v = (double)row[k];
            if (v < 0.0)
            {
                row[k] = T(0);
                if (L == 2) row[V + k] = T(0);
            }
            else
            {
                row[k] = T(v * s);
                if (L == 2) row[V + k] = T((double)row[V + k] * s);
            }
        }
        if (threadIdx.x == 0 && nfixAdd) atomicAdd(&sc->nfix, 1);
        __syncthreads();
    }
    m = pos + neg;
}

// ---------------------------------------------------------------------------
// Positivity + MOOD transport screen (MLSTransport.cpp:325-379).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_post_transport(T *g, int ldf, int V, int L, double dvN,
                 const int *__restrict__ boundary, const int *__restrict__ nslot,
                 const int *__restrict__ slots, int S,
                 const double *__restrict__ macro, int limiter, int *flag,
                 int *list, double *mass, StepScalars *sc)
{
    __shared__ double sh[3 * 32];
    const int i = blockIdx.x;
    T *row = g + (size_t)i * ldf;
    double m;
    bool bad;
    positivity(row, V, L, sh, 1, sc, m, bad);
    if (threadIdx.x == 0) mass[i] = m * dvN;
    int flagged = 0;
    if (limiter == 2 && !boundary[i])
    {
        if (bad || m <= 0.0) flagged = 1;
        else
        {
            // NAD against the neighbours' current (pre-transport) density.
            const int ns = nslot[i];
            double lo = INFINITY, hi = -INFINITY;
            for (int s = 1 + threadIdx.x; s < ns; s += blockDim.x)
            {
                double r = macro[6 * (size_t)slots[(size_t)i * S + s]];
                lo = fmin(lo, r);
                hi = fmax(hi, r);
            }
            lo = warpMin(lo);
            hi = warpMax(hi);
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            if (lane == 0) { sh[wid] = lo; sh[32 + wid] = hi; }
            __syncthreads();
            lo = INFINITY; hi = -INFINITY;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            {
                lo = fmin(lo, sh[w]);
                hi = fmax(hi, sh[32 + w]);
            }
            if (isfinite(lo) && isfinite(hi))
            {
                double rn = m * dvN;
                double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9;
                if (rn < lo - slack || rn > hi + slack) flagged = 1;
            }
        }
    }
    if (threadIdx.x == 0)
    {
        flag[i] = flagged;
        if (flagged) list[atomicAdd(&sc->nflag, 1)] = i;
    }
}

// Partial-pivot elimination with the |pivot| < 1e-30 skip rule for one or
// two right-hand sides (MLSTransport.cpp:20-62), P <= 4.
__device__ void solveSmall(double *A, double *b1, double *b2, int P)
{
    for (int col = 0; col < P; ++col)
    {
        int piv = col;
        double mx = fabs(A[col * P + col]);
        for (int row = col + 1; row < P; ++row)
            if (fabs(A[row * P + col]) > mx) { mx = fabs(A[row * P + col]); piv = row; }
        if (piv != col)
        {
            for (int j = 0; j < P; ++j)
            {
                double t = A[col * P + j]; A[col * P + j] = A[piv * P + j]; A[piv * P + j] = t;
            }
            double t = b1[col]; b1[col] = b1[piv]; b1[piv] = t;
            t = b2[col]; b2[col] = b2[piv]; b2[piv] = t;
        }
        double d = A[col * P + col];
        if (fabs(d) < 1.0e-30) continue;
        for (int row = col + 1; row < P; ++row)
        {
            double fct = A[row * P + col] / d;
            for (int j = col; j < P; ++j) A[row * P + j] -= fct * A[col * P + j];
            b1[row] -= fct * b1[col];
            b2[row] -= fct * b2[col];
        }
    }
    for (int i = P - 1; i >= 0; --i)
    {
        double s1 = b1[i], s2 = b2[i];
        for (int j = i + 1; j < P; ++j) { s1 -= A[i * P + j] * b1[j]; s2 -= A[i * P + j] * b2[j]; }
        bool ok = fabs(A[i * P + i]) > 1.0e-30;
        b1[i] = ok ? s1 / A[i * P + i] : 0.0;
        b2[i] = ok ? s2 / A[i * P + i] : 0.0;
    }
}

// ---------------------------------------------------------------------------
// Linear MLS redo of MOOD-flagged particles (Solver/Solver.cpp:641-646 with
// mlsTransportCompute(..., 1, onlyFlagged=true)): direct FP64 solve per node
// from the pre-transport f.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_redo(const T *__restrict__ f, T *g, int ldf, StepParams p,
       const double *__restrict__ pos, const double *__restrict__ meshv,
       const int *__restrict__ nslot, const int *__restrict__ slots,
       const int *__restrict__ list, double *mass, StepScalars *sc)
{
    __shared__ double sh[3 * 32];
    const int nflag = sc->nflag;
    const int P = (p.dim == 3) ? 4 : 3;
    for (int li = blockIdx.x; li < nflag; li += gridDim.x)
    {
        const int i = list[li];
        const int ns = nslot[i];
        const int *sl = slots + (size_t)i * p.S;
        const T *fo = f + (size_t)i * p.ldf;
        T *row = g + (size_t)i * p.ldf;
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            double vx, vy, vz;
            nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
            double xf = pos[3 * i] - (vx - meshv[3 * i]) * p.dt;
            double yf = pos[3 * i + 1] - (vy - meshv[3 * i + 1]) * p.dt;
            double zf = pos[3 * i + 2] - (vz - meshv[3 * i + 2]) * p.dt;
            double A[16], b1[4], b2[4];
            for (int q = 0; q < 16; ++q) A[q] = 0.0;
            for (int q = 0; q < 4; ++q) b1[q] = b2[q] = 0.0;
            bool any = false;
            for (int s = 1; s < ns; ++s)
            {
                const int j = sl[s];
                double dx = pos[3 * j] - xf, dy = pos[3 * j + 1] - yf;
                double dz = (p.dim == 3) ? pos[3 * j + 2] - zf : 0.0;
                if (p.periodic[0]) dx = minImage(dx, p.Lp[0]);
                if (p.periodic[1]) dy = minImage(dy, p.Lp[1]);
                if (p.dim == 3 && p.periodic[2]) dz = minImage(dz, p.Lp[2]);
                double q2 = (dx * dx + dy * dy + dz * dz) / (p.h * p.h);
                if (q2 >= 1.0) continue;
                double w = (1.0 - q2) * (1.0 - q2);
                if (w < 1.0e-30) continue;
                double b[4] = {1.0, dx / p.h, dy / p.h, dz / p.h};
                for (int p1 = 0; p1 < P; ++p1)
                    for (int p2 = 0; p2 < P; ++p2) A[p1 * P + p2] += w * b[p1] * b[p2];
                double g1 = (double)f[(size_t)j * p.ldf + k];
                double g2 = (p.L == 2) ? (double)f[(size_t)j * p.ldf + p.V + k] : 0.0;
                for (int q = 0; q < P; ++q) { b1[q] += w * b[q] * g1; b2[q] += w * b[q] * g2; }
                any = true;
            }
            if (!any)
            {
                row[k] = fo[k];
                if (p.L == 2) row[p.V + k] = fo[p.V + k];
                continue;
            }
            solveSmall(A, b1, b2, P);
            row[k] = T(b1[0]);
            if (p.L == 2) row[p.V + k] = T(b2[0]);
        }
        __syncthreads();
        double m;
        bool bad;
        positivity(row, p.V, p.L, sh, 0, sc, m, bad);
        if (threadIdx.x == 0) mass[i] = m * p.dvN;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Deterministic mass reduction, one block: contiguous chunks per thread,
// then a fixed-shape tree.  mode 0: after transport -> sigma; mode 1: end of
// step -> massOld of the next step.  mode 2: initial mass only.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024)
k_mass_reduce(const double *__restrict__ mass, int N, StepScalars *sc, int mode)
{
    __shared__ double sh[32];
    const int t = threadIdx.x, nt = blockDim.x;
    const int chunk = (N + nt - 1) / nt;
    const int lo = t * chunk, hi = min(N, lo + chunk);
    double s = 0.0;
    for (int i = lo; i < hi; ++i) s += mass[i];
    double v[1] = {s};
    blockSums<1>(v, sh);
    if (t == 0)
    {
        if (mode == 0)
        {
            sc->massNew = v[0];
            sc->sigma = (v[0] > 1.0e-30) ? sc->massOld / v[0] : 1.0;
        }
        else
        {
            sc->massOld = v[0];
            sc->massEnd = v[0];
            if (mode == 1) sc->steps += 1;
        }
    }
}

__global__ void k_step_begin(StepScalars *sc)
{
    sc->nflag = 0;
    sc->nfix = 0;
    sc->moodfail = 0;
}

// Moments of one particle row (MomentCalculations/Moments.cpp:17-97):
// writes rho, u, T, p into mac when rho > 1e-30.
__device__ void rowMoments(const double *row, const StepParams &p, double *mac,
                           double *sh)
{
    double v[5] = {0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < p.V; k += blockDim.x)
    {
        double vx, vy, vz;
        nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
        double f1 = row[k] * p.dvN;
        v[0] += f1;
        v[1] += vx * f1;
        v[2] += vy * f1;
        v[3] += vz * f1;
        v[4] += (vx * vx + vy * vy + vz * vz) * f1;
        if (p.L == 2) v[4] += 2.0 * row[p.V + k] * p.dvN;
    }
    blockSums<5>(v, sh);
    if (v[0] > 1.0e-30)
    {
        double rho = v[0];
        double ux = v[1] / rho, uy = v[2] / rho;
        double uz = (p.dim == 3) ? v[3] / rho : mac[3];
        double u2 = ux * ux + uy * uy + uz * uz;
        double T = fmax((v[4] / rho - u2) / (3.0 * p.R), 1.0e-6);
        if (threadIdx.x == 0)
        {
            mac[0] = rho; mac[1] = ux; mac[2] = uy; mac[3] = uz;
            mac[4] = T; mac[5] = rho * p.R * T;
        }
    }
    __syncthreads();
}

// Implicit BGK relaxation of one row (MomentCalculations/Collision.cpp:70-139).
__device__ void rowCollide(double *row, const StepParams &p, const double *mac)
{
    double lam = p.dt / p.tau;
    if (p.tauVar)
    {
        const double kB = 1.380649e-23;
        double l = kB / (sqrt(2.0) * kPi * mac[0] * p.R * p.dHS * p.dHS);
        double cbar = sqrt(8.0 * p.R * mac[4] / kPi);
        double tp = 4.0 * l / (kPi * cbar);
        lam = p.dt / tp;
    }
    const double coeff = 1.0 / (1.0 + lam);
    const double rho = mac[0], ux = mac[1], uy = mac[2], uz = mac[3], T = mac[4];
    const double twoRT = 2.0 * p.R * T;
    if (p.dim == 3)
    {
        const double norm = pow(kPi * twoRT, 1.5);
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            double vx, vy, vz;
            nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
            double e = -((vx - ux) * (vx - ux) + (vy - uy) * (vy - uy) +
                         (vz - uz) * (vz - uz)) / twoRT;
            double M = rho / norm * exp(e);
            row[k] = coeff * (row[k] + lam * M);
        }
    }
    else
    {
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            double vx, vy, vz;
            nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
            double e = -((vx - ux) * (vx - ux) + (vy - uy) * (vy - uy)) / twoRT;
            double M1 = rho / (kPi * twoRT) * exp(e);
            double M2 = 0.5 * p.R * T * M1;
            row[k] = coeff * (row[k] + lam * M1);
            row[p.V + k] = coeff * (row[p.V + k] + lam * M2);
        }
    }
    __syncthreads();
}

__device__ double rowMass(const double *row, const StepParams &p, double *sh)
{
    double v[1] = {0.0};
    for (int k = threadIdx.x; k < p.V; k += blockDim.x) v[0] += row[k];
    blockSums<1>(v, sh);
    return v[0] * p.dvN;
}

// ---------------------------------------------------------------------------
// Finalize: global rescale, diffuse wall (BoundaryConditions/DiffuseWall.cpp
// :19-154) or moments + collision + moments (Moments.cpp, Collision.cpp),
// moodCheck (Conservation.cpp:16-38, MLSBasis.hpp:208-222), particle mass.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kNT)
k_finalize(T *g, StepParams p, const int *__restrict__ boundary,
           const double *__restrict__ wall, double *macro, int *mood,
           double *mass, double *dpx, StepScalars *sc)
{
    extern __shared__ double row[];
    __shared__ double sh[5 * 32];
    const int i = blockIdx.x;
    const double sigma = sc->sigma;
    T *gr = g + (size_t)i * p.ldf;
    for (int k = threadIdx.x; k < p.gs; k += blockDim.x) row[k] = (double)gr[k] * sigma;
    __syncthreads();
    double *mac = macro + 6 * (size_t)i;
    if (boundary[i])
    {
        const double *w = wall + 7 * (size_t)i;
        const double Ux = w[3], Uy = w[4], Uz = w[5], Tw = w[6];
        const double RT2w = 2.0 * p.R * Tw;
        const double norm = (p.dim == 3) ? pow(kPi * RT2w, 1.5) : kPi * RT2w;
        double v[2] = {0.0, 0.0};
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            double vx, vy, vz;
            nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
            const double cn = bcCn(p.dim, vx, vy, vz, w);
            double e2 = (vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy);
            if (p.dim == 3) e2 += (vz - Uz) * (vz - Uz);
            if (cn < 0.0) v[0] += cn * row[k] * p.dvN;
            else if (cn > 0.0) v[1] += cn * (exp(-e2 / RT2w) / norm) * p.dvN;
        }
        blockSums<2>(v, sh);
        const double rhow = (v[1] > 1.0e-30) ? (-v[0] / v[1]) : 1.0;
        double dp[1] = {0.0};
        for (int k = threadIdx.x; k < p.V; k += blockDim.x)
        {
            double vx, vy, vz;
            nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
            const double cn = bcCn(p.dim, vx, vy, vz, w);
            double e2 = (vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy);
            if (p.dim == 3) e2 += (vz - Uz) * (vz - Uz);
            if (cn > 0.0)
            {
                double Mw = rhow * exp(-e2 / RT2w) / norm;
                dp[0] += vx * (Mw - row[k]) * p.dvN;
                row[k] = Mw;
                if (p.L == 2) row[p.V + k] = 0.5 * p.R * Tw * Mw;
            }
        }
        blockSums<1>(dp, sh);
        if (threadIdx.x == 0)
        {
            mac[0] = rhow; mac[1] = Ux; mac[2] = Uy;
            if (p.dim == 3) mac[3] = Uz;
            mac[4] = Tw; mac[5] = rhow * p.R * Tw;
            mood[i] = 0;
            dpx[i] = dp[0];
        }
        __syncthreads();
    }
    else
    {
        rowMoments(row, p, mac, sh);
        rowCollide(row, p, mac);
        rowMoments(row, p, mac, sh);
        if (threadIdx.x == 0) dpx[i] = 0.0;
        if (p.limiter == 2)
        {
            double mn = INFINITY;
            for (int k = threadIdx.x; k < p.V; k += blockDim.x) mn = fmin(mn, row[k]);
            mn = warpMin(mn);
            const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
            if (lane == 0) sh[wid] = mn;
            __syncthreads();
            if (threadIdx.x == 0)
            {
                double m2 = INFINITY;
                for (int q = 0; q < (int)(blockDim.x >> 5); ++q) m2 = fmin(m2, sh[q]);
                int fail = (mac[0] < 1.0e-10) || (mac[4] < 1.0e-6) || (m2 < -1.0e-14);
                mood[i] = fail;
                if (fail) atomicOr(&sc->moodfail, 1);
            }
            __syncthreads();
        }
    }
    double m = rowMass(row, p, sh);
    if (threadIdx.x == 0) mass[i] = m;
    for (int k = threadIdx.x; k < p.gs; k += blockDim.x) gr[k] = T(row[k]);
}

// Second collision + moments of every interior particle when moodCheck
// failed (Solver/Solver.cpp:685-693).  Exits at once otherwise.
template <typename T>
__global__ void __launch_bounds__(kNT)
k_recollide(T *g, StepParams p, const int *__restrict__ boundary, double *macro,
            double *mass, StepScalars *sc)
{
    if (sc->moodfail == 0) return;
    extern __shared__ double row[];
    __shared__ double sh[5 * 32];
    const int i = blockIdx.x;
    if (boundary[i]) return;
    T *gr = g + (size_t)i * p.ldf;
    for (int k = threadIdx.x; k < p.gs; k += blockDim.x) row[k] = (double)gr[k];
    __syncthreads();
    double *mac = macro + 6 * (size_t)i;
    rowCollide(row, p, mac);
    rowMoments(row, p, mac, sh);
    double m = rowMass(row, p, sh);
    if (threadIdx.x == 0) mass[i] = m;
    for (int k = threadIdx.x; k < p.gs; k += blockDim.x) gr[k] = T(row[k]);
}

// Initial particle masses (sumMass of the uploaded state).
template <typename T>
__global__ void __launch_bounds__(kNT)
k_particle_mass(const T *g, StepParams p, double *mass)
{
    __shared__ double sh[32];
    const int i = blockIdx.x;
    const T *gr = g + (size_t)i * p.ldf;
    double v[1] = {0.0};
    for (int k = threadIdx.x; k < p.V; k += blockDim.x) v[0] += (double)gr[k];
    blockSums<1>(v, sh);
    if (threadIdx.x == 0) mass[i] = v[0] * p.dvN;
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
               const double *__restrict__ area, double *tmp)
{
    __shared__ double sh[6 * 32];
    const int i = blockIdx.x;
    const int b = bodyId[i];
    if (!boundary[i] || b < 0) return;
    const T *gr = g + (size_t)i * p.ldf;
    const double *w = wall + 7 * (size_t)i;
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int k = threadIdx.x; k < p.V; k += blockDim.x)
    {
        double vx, vy, vz;
        nodeVel(k, p.Nv, p.dim, p.vmin, p.dv, vx, vy, vz);
        double cx = vx - w[3], cy = vy - w[4], cz = vz - w[5];
        double f = (double)gr[k] * p.dvN;
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
__global__ void k_convert_out(const T *src, double *dst, int N, int gs, int ldf)
{
    size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    size_t tot = (size_t)N * gs;
    for (; idx < tot; idx += (size_t)gridDim.x * blockDim.x)
    {
        size_t i = idx / gs, k = idx % gs;
        dst[idx] = (double)src[i * ldf + k];
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
// Launches one step.  With ev != nullptr an event is recorded before each
// stage and after the last one (ev[0..8]), in the stage order
// step_begin, transport, post_transport, redo, mass, finalize, recollide,
// mass_end.
template <typename T>
static cudaError_t stepT(alebgk_ctx *c, int from, cudaEvent_t *ev)
{
    const StepParams &p = c->sp;
    DeviceBuffers &d = c->d;
    cudaStream_t st = c->stream;
    T *fa = static_cast<T *>(d.f[from]);
    T *fb = static_cast<T *>(d.f[1 - from]);
    const size_t rowBytes = (size_t)p.gs * sizeof(double);
    int q = 0;
    auto mark = [&]() { if (ev) cudaEventRecord(ev[q++], st); };
    mark();
    k_step_begin<<<1, 1, 0, st>>>(d.sc);
    mark();
    dim3 gt(p.N, (p.V + kNT - 1) / kNT);
    k_transport<T><<<gt, kNT, 0, st>>>(fa, fb, static_cast<const T *>(d.coef),
                                       d.cls, d.nslot, d.slots, p.S, p.V, p.L,
                                       p.ldf);
    mark();
    k_post_transport<T><<<p.N, kNT, 0, st>>>(fb, p.ldf, p.V, p.L, p.dvN,
                                             d.boundary, d.nslot, d.slots, p.S,
                                             d.macro, p.limiter, d.flag, d.list,
                                             d.mass, d.sc);
    mark();
    if (p.limiter == 2)
        k_redo<T><<<min(p.N, 1024), kNT, 0, st>>>(fa, fb, p.ldf, p, d.pos,
                                                   d.meshv, d.nslot, d.slots,
                                                   d.list, d.mass, d.sc);
    mark();
    k_mass_reduce<<<1, 1024, 0, st>>>(d.mass, p.N, d.sc, 0);
    mark();
    k_finalize<T><<<p.N, kNT, rowBytes, st>>>(fb, p, d.boundary, d.wall,
                                              d.macro, d.mood, d.mass, d.dpx,
                                              d.sc);
    mark();
    if (p.limiter == 2)
        k_recollide<T><<<p.N, kNT, rowBytes, st>>>(fb, p, d.boundary, d.macro,
                                                   d.mass, d.sc);
    mark();
    k_mass_reduce<<<1, 1024, 0, st>>>(d.mass, p.N, d.sc, 1);
    mark();
    return cudaGetLastError();
}

template <typename T>
static cudaError_t prepareT(alebgk_ctx *c)
{
    const int rowBytes = c->sp.gs * (int)sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_finalize<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         rowBytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_recollide<T>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, rowBytes);
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
    k_particle_mass<T><<<p.N, kNT, 0, c->stream>>>(
        static_cast<const T *>(c->d.f[c->cur]), p, c->d.mass);
    k_mass_reduce<<<1, 1024, 0, c->stream>>>(c->d.mass, p.N, c->d.sc, 2);
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
        c->d.pos, c->d.wall, centre, area, c->d.bodyTmp);
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
            static_cast<const double *>(c->d.f[buf]), dst, p.N, p.gs, p.ldf);
    else
        k_convert_out<float><<<1184, 256, 0, c->stream>>>(
            static_cast<const float *>(c->d.f[buf]), dst, p.N, p.gs, p.ldf);
    return cudaGetLastError();
}

}  // namespace alebgk
