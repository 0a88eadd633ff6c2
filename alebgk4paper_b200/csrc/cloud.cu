// cloud.cu -- cloud management around moving bodies
// (RigidBody/CloudManagement.cpp:17-275) with its all-particle tests on the
// device.
//
// The reference runs, after the body motion of a step (Solver.cpp:381-395):
//   manageRemove        drop fluid particles inside a body or within 0.4 dx
//                       of a body-surface particle;
//   neighbour rebuild;
//   mergeCloseParticles two interior neighbours closer than minDist become
//                       one at the mean position with the mean distribution;
//   (rebuild if merged)
//   manageRefill        initial-lattice sites in a 3.5 dx margin around the
//                       bodies with no particle within 0.8 dx, outside the
//                       bodies and 0.6 dx clear of the surface particles, get
//                       a Maxwellian particle with the weight-averaged moments
//                       of the particles within the MLS radius;
//   (rebuild if refilled)
// Its cost is in the all-particle loops: the hug test against the surface
// particles, the hole test of every margin site against the whole cloud, the
// pair scan of the merge, and the neighbour rebuilds.  Those run here as
// device kernels (one thread per particle or site); the host keeps the
// order-dependent bookkeeping of the few hits -- stable compaction, the
// merge sweep (only when the device found a close pair), and the moment
// averages and Maxwellian rows of the accepted refill sites, summed in the
// reference's particle order -- so the managed cloud equals the reference's
// bitwise.  Distances use the FMA form of the reference's compiled build,
// fma(dz, dz, fma(dx, dx, dy * dy)).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "alebgk.h"
#include "cases.h"
#include "ctx.h"

namespace alebgk {

namespace {

__device__ __forceinline__ double dist2(double dx, double dy, double dz)
{
    return fma(dz, dz, fma(dx, dx, __dmul_rn(dy, dy)));
}

// manageRemove's hug test: fluid particle within sqrt(hug2) of a surface point.
__global__ void k_hug(const double *__restrict__ xyz, const int *__restrict__ boundary, int N,
                      const double *__restrict__ surf, int nsurf, double hug2, int d3,
                      int *__restrict__ hug)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    int h = 0;
    if (!boundary[i])
    {
        const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1],
                     z = xyz[3 * (size_t)i + 2];
        for (int q = 0; q < nsurf && !h; ++q)
        {
            const double dx = x - surf[3 * q], dy = y - surf[3 * q + 1];
            const double dz = d3 ? z - surf[3 * q + 2] : 0.0;
            if (dist2(dx, dy, dz) < hug2) h = 1;
        }
    }
    hug[i] = h;
}

// mergeCloseParticles: does any interior particle have a later interior
// neighbour closer than minDist?  (Only then does the host sweep run.)
__global__ void k_merge_pairs(const double *__restrict__ xyz, const int *__restrict__ boundary,
                              const int *__restrict__ nnb, const int *__restrict__ nbr, int N,
                              double min2, int d3, int *__restrict__ any)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || boundary[i]) return;
    const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    for (int s = 0; s < nnb[i]; ++s)
    {
        const int j = nbr[(size_t)i * kMaxNeigh + s];
        if (j <= i || boundary[j]) continue;
        const double dx = x - xyz[3 * (size_t)j], dy = y - xyz[3 * (size_t)j + 1];
        const double dz = d3 ? z - xyz[3 * (size_t)j + 2] : 0.0;
        if (dist2(dx, dy, dz) < min2)
        {
            atomicOr(any, 1);
            return;
        }
    }
}

// manageRefill's hole test: no particle within sqrt(hole2) of the site.
__global__ void k_hole(const double *__restrict__ sites, int nsites,
                       const double *__restrict__ xyz, int N, double hole2, int d3,
                       int *__restrict__ hole)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsites) return;
    const double xm = sites[3 * s], ym = sites[3 * s + 1], zm = sites[3 * s + 2];
    int h = 1;
    for (int q = 0; q < N && h; ++q)
    {
        const double dx = xyz[3 * (size_t)q] - xm, dy = xyz[3 * (size_t)q + 1] - ym;
        const double dz = d3 ? xyz[3 * (size_t)q + 2] - zm : 0.0;
        if (dist2(dx, dy, dz) < hole2) h = 0;
    }
    hole[s] = h;
}

inline double hostDist2(double dx, double dy, double dz)
{
    return std::fma(dz, dz, std::fma(dx, dx, dy * dy));
}

// Core/MLSBasis.hpp:142-148
inline double weightSq(double r2, double h)
{
    double q2 = r2 / (h * h);
    if (q2 >= 1.0) return 0.0;
    double w = 1.0 - q2;
    return w * w;
}

struct Cloud2
{
    int N = 0, gs = 0;
    std::vector<double> xyz, meshv, wall, g, macro;
    std::vector<int> boundary, bodyId, nnb, nbr;
    // Plan mode (the distribution stays on the device): the origin of every
    // row instead of the row.  originA >= 0: the input row originA (and, when
    // originB >= 0, the mean of the input rows originA and originB, a merge);
    // originA < 0: row -1 - originA of fresh (a refill Maxwellian, gsFresh
    // values each).
    bool plan = false;
    int gsFresh = 0;
    std::vector<int> originA, originB;
    std::vector<double> fresh;

    void keep(const std::vector<char> &k)
    {
        int n = 0;
        for (int i = 0; i < N; ++i)
        {
            if (!k[i]) continue;
            if (n != i)
            {
                std::copy_n(&xyz[3 * (size_t)i], 3, &xyz[3 * (size_t)n]);
                std::copy_n(&meshv[3 * (size_t)i], 3, &meshv[3 * (size_t)n]);
                std::copy_n(&wall[7 * (size_t)i], 7, &wall[7 * (size_t)n]);
                std::copy_n(&g[(size_t)gs * i], gs, &g[(size_t)gs * n]);
                std::copy_n(&macro[7 * (size_t)i], 7, &macro[7 * (size_t)n]);
                boundary[n] = boundary[i];
                bodyId[n] = bodyId[i];
                if (plan)
                {
                    originA[n] = originA[i];
                    originB[n] = originB[i];
                }
            }
            ++n;
        }
        N = n;
        xyz.resize(3 * (size_t)N); meshv.resize(3 * (size_t)N); wall.resize(7 * (size_t)N);
        g.resize((size_t)gs * N); macro.resize(7 * (size_t)N);
        boundary.resize(N); bodyId.resize(N);
        if (plan) { originA.resize(N); originB.resize(N); }
    }
};

struct DevScratch
{
    double *xyz = nullptr, *aux = nullptr;
    int *flag = nullptr, *boundary = nullptr;
    LatticeDev nb;
    size_t cap = 0, auxCap = 0;
    ~DevScratch()
    {
        for (void *p : {(void *)xyz, (void *)aux, (void *)flag, (void *)boundary,
                        (void *)nb.voxel, (void *)nb.voxCount, (void *)nb.voxStart,
                        (void *)nb.voxCursor, (void *)nb.voxList, (void *)nb.nnb, (void *)nb.nbr})
            if (p) cudaFree(p);
    }
};

}  // namespace

struct ManageParams
{
    int dim, Nv, nbh, nbv, nbw;
    double dx, minDist, radius, xleft, xright, ybottom, ytop, zfront, zback, vmin, dv, R;
    double hBox, vBox, wBox;
};

struct ManagedCloud
{
    Cloud2 c;
    int counts[3] = {0, 0, 0};
    bool needState = false;   // geometry-only run: the particle set would change
};

// The whole cloud-management block.  Returns a CUDA error or cudaSuccess;
// *bad gets a message for bad input.
cudaError_t manageCloud(const ManageParams &mp, const std::vector<Body> &bodies,
                        const alebgk_cloud &in, int N, int gs, ManagedCloud &out,
                        std::string *bad)
{
    Cloud2 &c = out.c;
    // Without g and macros the run only decides: it stops with needState as
    // soon as the particle set would change.
    // Plan mode: macros without g -- the run decides as with the state and
    // records where every row of the result comes from.
    c.plan = !in.g && in.macro;
    const bool haveState = (in.g && in.macro) || c.plan;
    c.N = N; c.gs = (in.g && in.macro) ? gs : 0;
    c.gsFresh = gs;
    if (c.plan)
    {
        c.originA.resize(N);
        c.originB.assign(N, -1);
        for (int i = 0; i < N; ++i) c.originA[i] = i;
    }
    c.xyz.assign(in.xyz, in.xyz + 3 * (size_t)N);
    c.meshv.assign(in.meshv, in.meshv + 3 * (size_t)N);
    c.wall.assign(in.wall, in.wall + 7 * (size_t)N);
    if (haveState)
    {
        if (c.gs) c.g.assign(in.g, in.g + (size_t)gs * N);
        c.macro.assign(in.macro, in.macro + 7 * (size_t)N);
    }
    else
        c.macro.assign(7 * (size_t)N, 0.0);
    c.boundary.assign(in.boundary, in.boundary + N);
    c.bodyId.assign(in.body_id, in.body_id + N);
    const bool d3 = mp.dim == 3;
    const int maxN = N + 4096;
    DevScratch ds;
    cudaError_t e = cudaSuccess;
    auto reserve = [&](size_t n) -> cudaError_t {
        if (n <= ds.cap) return cudaSuccess;
        for (void **p : {(void **)&ds.xyz, (void **)&ds.flag, (void **)&ds.boundary,
                         (void **)&ds.nb.voxel, (void **)&ds.nb.voxList, (void **)&ds.nb.nnb,
                         (void **)&ds.nb.nbr})
            if (*p) { cudaFree(*p); *p = nullptr; }
        cudaError_t r = cudaMalloc(&ds.xyz, 24 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.flag, 4 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.boundary, 4 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.nb.voxel, 4 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.nb.voxList, 4 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.nb.nnb, 4 * n);
        if (r == cudaSuccess) r = cudaMalloc(&ds.nb.nbr, 4 * n * kMaxNeigh);
        ds.cap = n;
        return r;
    };
    const size_t nvox = (size_t)mp.nbh * mp.nbv * mp.nbw;
    e = reserve(maxN);
    if (e == cudaSuccess) e = cudaMalloc(&ds.nb.voxCount, 4 * nvox);
    if (e == cudaSuccess) e = cudaMalloc(&ds.nb.voxStart, 4 * (nvox + 1));
    if (e == cudaSuccess) e = cudaMalloc(&ds.nb.voxCursor, 4 * nvox);
    if (e != cudaSuccess) return e;
    NeighbourGrid grid;
    grid.dim = mp.dim;
    grid.x0 = mp.xleft; grid.y0 = mp.ybottom; grid.z0 = mp.zfront;
    grid.hx = mp.hBox; grid.hy = mp.vBox; grid.hz = mp.wBox; grid.radius = mp.radius;
    grid.nx = mp.nbh; grid.ny = mp.nbv; grid.nz = mp.nbw;

    auto upload = [&]() -> cudaError_t {
        cudaError_t r = reserve((size_t)c.N);
        if (r == cudaSuccess)
            r = cudaMemcpy(ds.xyz, c.xyz.data(), 24 * (size_t)c.N, cudaMemcpyHostToDevice);
        if (r == cudaSuccess)
            r = cudaMemcpy(ds.boundary, c.boundary.data(), 4 * (size_t)c.N,
                           cudaMemcpyHostToDevice);
        return r;
    };
    auto rebuild = [&]() -> cudaError_t {
        cudaError_t r = upload();
        if (r == cudaSuccess) r = buildNeighboursDevice(grid, ds.xyz, c.N, ds.nb, nullptr);
        if (r == cudaSuccess) r = cudaDeviceSynchronize();
        c.nnb.resize(c.N);
        c.nbr.resize((size_t)c.N * kMaxNeigh);
        if (r == cudaSuccess)
            r = cudaMemcpy(c.nnb.data(), ds.nb.nnb, 4 * (size_t)c.N, cudaMemcpyDeviceToHost);
        if (r == cudaSuccess)
            r = cudaMemcpy(c.nbr.data(), ds.nb.nbr, 4 * (size_t)c.N * kMaxNeigh,
                           cudaMemcpyDeviceToHost);
        return r;
    };

    // surface points, in particle order
    auto surfacePoints = [&]() {
        std::vector<double> s;
        for (int i = 0; i < c.N; ++i)
            if (c.boundary[i] && c.bodyId[i] >= 0)
                s.insert(s.end(), {c.xyz[3 * (size_t)i], c.xyz[3 * (size_t)i + 1],
                                   c.xyz[3 * (size_t)i + 2]});
        return s;
    };

    // ---- manageRemove (CloudManagement.cpp:17-72)
    if (!bodies.empty())
    {
        const double hug2 = std::pow(0.4 * std::fabs(mp.dx), 2);
        std::vector<double> surf = surfacePoints();
        double *surfDev = nullptr;
        e = upload();
        if (e == cudaSuccess) e = cudaMalloc(&surfDev, 8 * std::max<size_t>(surf.size(), 3));
        if (e == cudaSuccess && !surf.empty())
            e = cudaMemcpy(surfDev, surf.data(), 8 * surf.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
        {
            k_hug<<<(c.N + 255) / 256, 256>>>(ds.xyz, ds.boundary, c.N, surfDev,
                                              (int)surf.size() / 3, hug2, d3 ? 1 : 0, ds.flag);
            e = cudaGetLastError();
        }
        std::vector<int> hug(c.N);
        if (e == cudaSuccess)
            e = cudaMemcpy(hug.data(), ds.flag, 4 * (size_t)c.N, cudaMemcpyDeviceToHost);
        if (surfDev) cudaFree(surfDev);
        if (e != cudaSuccess) return e;
        std::vector<char> keep(c.N, 1);
        int removed = 0;
        for (int i = 0; i < c.N; ++i)
        {
            if (c.boundary[i]) continue;
            bool drop = false;
            for (const Body &b : bodies)
                if (b.inside(c.xyz[3 * (size_t)i], c.xyz[3 * (size_t)i + 1],
                             d3 ? c.xyz[3 * (size_t)i + 2] : b.cz))
                {
                    drop = true;
                    break;
                }
            if (drop || hug[i]) { keep[i] = 0; ++removed; }
        }
        out.counts[0] = removed;
        if (removed && !haveState)
        {
            out.needState = true;
            return cudaSuccess;
        }
        c.keep(keep);
    }
    e = rebuild();
    if (e != cudaSuccess) return e;

    // ---- mergeCloseParticles (CloudManagement.cpp:80-120)
    const double min2 = mp.minDist * mp.minDist;
    if (min2 > 0.0)
    {
        int *anyDev = nullptr, any = 0;
        e = cudaMalloc(&anyDev, 4);
        if (e == cudaSuccess) e = cudaMemset(anyDev, 0, 4);
        if (e == cudaSuccess)
        {
            k_merge_pairs<<<(c.N + 255) / 256, 256>>>(ds.xyz, ds.boundary, ds.nb.nnb, ds.nb.nbr,
                                                      c.N, min2, d3 ? 1 : 0, anyDev);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpy(&any, anyDev, 4, cudaMemcpyDeviceToHost);
        if (anyDev) cudaFree(anyDev);
        if (e != cudaSuccess) return e;
        if (any && !haveState)
        {
            out.needState = true;
            return cudaSuccess;
        }
        if (any)
        {
            std::vector<char> dead(c.N, 0);
            int merged = 0;
            for (int i = 0; i < c.N; ++i)
            {
                if (dead[i] || c.boundary[i]) continue;
                for (int s = 0; s < c.nnb[i]; ++s)
                {
                    const int j = c.nbr[(size_t)i * kMaxNeigh + s];
                    if (j <= i || j >= c.N || dead[j]) continue;
                    if (c.boundary[j]) continue;
                    double *pi = &c.xyz[3 * (size_t)i];
                    const double *pj = &c.xyz[3 * (size_t)j];
                    const double dx = pi[0] - pj[0], dy = pi[1] - pj[1];
                    const double dz = d3 ? pi[2] - pj[2] : 0.0;
                    if (hostDist2(dx, dy, dz) < min2)
                    {
                        pi[0] = 0.5 * (pi[0] + pj[0]);
                        pi[1] = 0.5 * (pi[1] + pj[1]);
                        if (d3) pi[2] = 0.5 * (pi[2] + pj[2]);
                        if (c.plan)
                            c.originB[i] = c.originA[j];
                        else
                        {
                            double *gi = &c.g[(size_t)gs * i];
                            const double *gj = &c.g[(size_t)gs * j];
                            for (int k = 0; k < gs; ++k) gi[k] = 0.5 * (gi[k] + gj[k]);
                        }
                        dead[j] = 1;
                        ++merged;
                        break;
                    }
                }
            }
            if (merged)
            {
                std::vector<char> keep(c.N);
                for (int i = 0; i < c.N; ++i) keep[i] = !dead[i];
                c.keep(keep);
                e = rebuild();
                if (e != cudaSuccess) return e;
            }
            out.counts[1] = merged;
        }
    }

    // ---- manageRefill (CloudManagement.cpp:122-275)
    if (!bodies.empty())
    {
        const double dxl = std::fabs(mp.dx);
        const double hole2 = std::pow(0.8 * dxl, 2);
        double bx0 = 1e300, bx1 = -1e300, by0 = 1e300, by1 = -1e300, bz0 = 1e300, bz1 = -1e300;
        bool anySurf = false;
        for (int i = 0; i < c.N; ++i)
        {
            if (!c.boundary[i] || c.bodyId[i] < 0) continue;
            const double *p = &c.xyz[3 * (size_t)i];
            bx0 = std::min(bx0, p[0]); bx1 = std::max(bx1, p[0]);
            by0 = std::min(by0, p[1]); by1 = std::max(by1, p[1]);
            if (d3) { bz0 = std::min(bz0, p[2]); bz1 = std::max(bz1, p[2]); }
            anySurf = true;
        }
        if (anySurf)
        {
            const double margin = 3.5 * dxl;
            bx0 -= margin; bx1 += margin; by0 -= margin; by1 += margin;
            if (d3) { bz0 -= margin; bz1 += margin; }
            const int nxs = (int)std::llround((mp.xright - mp.xleft) / dxl);
            const int nys = (int)std::llround((mp.ytop - mp.ybottom) / dxl);
            const int nzs = d3 ? (int)std::llround((mp.zback - mp.zfront) / dxl) : 0;
            const int i0 = std::max(1, (int)std::ceil((bx0 - mp.xleft) / dxl));
            const int i1 = std::min(nxs - 1, (int)std::floor((bx1 - mp.xleft) / dxl));
            const int j0 = std::max(1, (int)std::ceil((by0 - mp.ybottom) / dxl));
            const int j1 = std::min(nys - 1, (int)std::floor((by1 - mp.ybottom) / dxl));
            const int k0 = d3 ? std::max(1, (int)std::ceil((bz0 - mp.zfront) / dxl)) : 0;
            const int k1 = d3 ? std::min(nzs - 1, (int)std::floor((bz1 - mp.zfront) / dxl)) : 0;
            std::vector<double> sites;
            for (int vk = k0; vk <= k1; ++vk)
                for (int vj = j0; vj <= j1; ++vj)
                    for (int vi = i0; vi <= i1; ++vi)
                        sites.insert(sites.end(),
                                     {std::fma((double)vi, dxl, mp.xleft),
                                      std::fma((double)vj, dxl, mp.ybottom),
                                      d3 ? std::fma((double)vk, dxl, mp.zfront) : 0.0});
            const int nsites = (int)sites.size() / 3;
            // Hole test of every site against the cloud before the refill: a
            // refilled particle sits on another lattice site, at least dx from
            // any other site, so it never fills a hole of a later site.
            std::vector<int> hole(nsites, 0);
            if (nsites > 0)
            {
                double *sitesDev = nullptr;
                int *holeDev = nullptr;
                e = upload();
                if (e == cudaSuccess) e = cudaMalloc(&sitesDev, 8 * sites.size());
                if (e == cudaSuccess) e = cudaMalloc(&holeDev, 4 * (size_t)nsites);
                if (e == cudaSuccess)
                    e = cudaMemcpy(sitesDev, sites.data(), 8 * sites.size(), cudaMemcpyHostToDevice);
                if (e == cudaSuccess)
                {
                    k_hole<<<(nsites + 127) / 128, 128>>>(sitesDev, nsites, ds.xyz, c.N, hole2,
                                                          d3 ? 1 : 0, holeDev);
                    e = cudaGetLastError();
                }
                if (e == cudaSuccess)
                    e = cudaMemcpy(hole.data(), holeDev, 4 * (size_t)nsites, cudaMemcpyDeviceToHost);
                if (sitesDev) cudaFree(sitesDev);
                if (holeDev) cudaFree(holeDev);
                if (e != cudaSuccess) return e;
            }
            const double clr2 = std::pow(0.6 * dxl, 2);
            const double r2 = mp.radius * mp.radius;
            std::vector<double> surf = surfacePoints();
            int added = 0;
            const int nv2 = mp.Nv * mp.Nv;
            for (int s = 0; s < nsites; ++s)
            {
                if (!hole[s]) continue;
                const double xm = sites[3 * s], ym = sites[3 * s + 1], zm = sites[3 * s + 2];
                bool inBody = false;
                for (const Body &b : bodies)
                    if (b.inside(xm, ym, d3 ? zm : b.cz)) { inBody = true; break; }
                if (inBody) continue;
                bool hugs = false;
                for (size_t q = 0; q < surf.size() / 3; ++q)
                {
                    const double dx = surf[3 * q] - xm, dy = surf[3 * q + 1] - ym;
                    const double dz = d3 ? surf[3 * q + 2] - zm : 0.0;
                    if (hostDist2(dx, dy, dz) < clr2) { hugs = true; break; }
                }
                if (hugs) continue;
                double wsum = 0, rho = 0, ux = 0, uy = 0, uz = 0, T = 0;
                for (int q = 0; q < c.N; ++q)
                {
                    const double dx = c.xyz[3 * (size_t)q] - xm, dy = c.xyz[3 * (size_t)q + 1] - ym;
                    const double dz = d3 ? c.xyz[3 * (size_t)q + 2] - zm : 0.0;
                    const double d2 = hostDist2(dx, dy, dz);
                    if (d2 >= r2) continue;
                    const double w = weightSq(d2, mp.radius);
                    const double *m = &c.macro[7 * (size_t)q];
                    wsum += w;
                    rho = std::fma(w, m[0], rho);
                    ux = std::fma(w, m[1], ux);
                    uy = std::fma(w, m[2], uy);
                    uz = std::fma(w, m[3], uz);
                    T = std::fma(w, m[4], T);
                }
                if (wsum < 1e-30) continue;
                if (!haveState)
                {
                    out.needState = true;
                    return cudaSuccess;
                }
                rho /= wsum; ux /= wsum; uy /= wsum; uz /= wsum; T /= wsum;
                const double p = rho * mp.R * T;
                c.xyz.insert(c.xyz.end(), {xm, ym, zm});
                c.meshv.insert(c.meshv.end(), {0.0, 0.0, 0.0});
                c.wall.insert(c.wall.end(), 7, 0.0);
                c.boundary.push_back(0);
                c.bodyId.push_back(-1);
                c.macro.insert(c.macro.end(), {rho, ux, uy, d3 ? uz : 0.0, T, p, 0.0});
                std::vector<double> &rows = c.plan ? c.fresh : c.g;
                if (c.plan)
                {
                    c.originA.push_back(-1 - (int)(c.fresh.size() / gs));
                    c.originB.push_back(-1);
                }
                const size_t base = rows.size();
                rows.resize(base + gs);
                double *row = &rows[base];
                if (d3)
                {
                    for (int kv = 0; kv < mp.Nv; ++kv)
                    {
                        const double vz = std::fma((double)kv, mp.dv, mp.vmin);
                        for (int jv = 0; jv < mp.Nv; ++jv)
                        {
                            const double vy = std::fma((double)jv, mp.dv, mp.vmin);
                            for (int iv = 0; iv < mp.Nv; ++iv)
                            {
                                const double vx = std::fma((double)iv, mp.dv, mp.vmin);
                                row[iv + mp.Nv * (jv + mp.Nv * kv)] =
                                    maxwellian3(vx, vy, vz, ux, uy, uz, T, rho, mp.R);
                            }
                        }
                    }
                }
                else
                {
                    for (int jv = 0; jv < mp.Nv; ++jv)
                    {
                        const double vy = std::fma((double)jv, mp.dv, mp.vmin);
                        for (int iv = 0; iv < mp.Nv; ++iv)
                        {
                            const double vx = std::fma((double)iv, mp.dv, mp.vmin);
                            const double m1 = maxwellianG1(vx, vy, ux, uy, T, rho, mp.R);
                            row[iv + mp.Nv * jv] = m1;
                            row[iv + mp.Nv * jv + nv2] = 0.5 * mp.R * T * m1;
                        }
                    }
                }
                ++c.N;
                ++added;
            }
            out.counts[2] = added;
            if (added)
            {
                e = rebuild();
                if (e != cudaSuccess) return e;
            }
        }
    }
    (void)bad;
    return cudaSuccess;
}

}  // namespace alebgk

// ---------------------------------------------------------------------------
using namespace alebgk;

struct alebgk_managed
{
    ManagedCloud m;
    std::string err;
};

extern "C" {

int alebgk_manage_cloud(int device, const double *prm, const int *iprm, int nbodies,
                        const alebgk_body *bodies, int N, int gstride,
                        const alebgk_cloud *cloud, alebgk_managed **out)
{
    if (!prm || !iprm || !cloud || !out || N <= 0 || gstride <= 0 || nbodies < 0 ||
        (nbodies > 0 && !bodies))
        return ALEBGK_EINVAL;
    // g without macros is the one combination without a meaning
    if (!cloud->xyz || !cloud->meshv || !cloud->wall || !cloud->boundary || !cloud->body_id ||
        (cloud->g && !cloud->macro))
        return ALEBGK_EINVAL;
    *out = nullptr;
    ManageParams mp;
    mp.dim = iprm[0]; mp.Nv = iprm[1]; mp.nbh = iprm[2]; mp.nbv = iprm[3]; mp.nbw = iprm[4];
    mp.dx = prm[0]; mp.minDist = prm[1]; mp.radius = prm[2];
    mp.xleft = prm[3]; mp.xright = prm[4]; mp.ybottom = prm[5]; mp.ytop = prm[6];
    mp.zfront = prm[7]; mp.zback = prm[8]; mp.vmin = prm[9]; mp.dv = prm[10]; mp.R = prm[11];
    mp.hBox = prm[12]; mp.vBox = prm[13]; mp.wBox = prm[14];
    if ((mp.dim != 2 && mp.dim != 3) || mp.Nv < 2 || mp.nbh < 1 || mp.nbv < 1 || mp.nbw < 1)
        return ALEBGK_EINVAL;
    const int expect = (mp.dim == 3) ? mp.Nv * mp.Nv * mp.Nv : 2 * mp.Nv * mp.Nv;
    if (gstride != expect) return ALEBGK_EINVAL;
    std::vector<Body> bs(nbodies);
    for (int b = 0; b < nbodies; ++b)
    {
        Body &o = bs[b];
        const double *st = bodies[b].state;
        o.kind = bodies[b].kind;
        o.dim = mp.dim;
        o.size = bodies[b].size;
        o.cx = st[0]; o.cy = st[1]; o.cz = st[2];
        o.ox = st[17]; o.oy = st[18];
        for (int k = 0; k < 9; ++k) o.Rm[k] = st[22 + k];
    }
    if (cudaSetDevice(device) != cudaSuccess) return ALEBGK_ECUDA;
    auto *m = new alebgk_managed();
    std::string bad;
    cudaError_t e = manageCloud(mp, bs, *cloud, N, gstride, m->m, &bad);
    if (e != cudaSuccess)
    {
        delete m;
        return ALEBGK_ECUDA;
    }
    *out = m;
    return ALEBGK_OK;
}

int alebgk_managed_info(const alebgk_managed *m, int *info)
{
    if (!m || !info) return ALEBGK_EINVAL;
    info[0] = m->m.c.N;
    info[1] = m->m.counts[0];
    info[2] = m->m.counts[1];
    info[3] = m->m.counts[2];
    info[4] = m->m.needState ? 1 : 0;
    return ALEBGK_OK;
}

int alebgk_managed_cloud(alebgk_managed *m, alebgk_cloud *view)
{
    if (!m || !view) return ALEBGK_EINVAL;
    Cloud2 &c = m->m.c;
    view->xyz = c.xyz.data(); view->meshv = c.meshv.data(); view->wall = c.wall.data();
    view->boundary = c.boundary.data(); view->body_id = c.bodyId.data();
    view->nnb = c.nnb.data(); view->nbr = c.nbr.data();
    view->g = c.gs ? c.g.data() : nullptr;
    view->macro = c.macro.data();
    return ALEBGK_OK;
}

void alebgk_managed_free(alebgk_managed *m) { delete m; }

int alebgk_managed_plan(const alebgk_managed *m, int *a, int *b, double *fresh)
{
    if (!m) return ALEBGK_EINVAL;
    const Cloud2 &c = m->m.c;
    if (!c.plan) return ALEBGK_ESTATE;
    if (a) std::copy(c.originA.begin(), c.originA.end(), a);
    if (b) std::copy(c.originB.begin(), c.originB.end(), b);
    if (fresh) std::copy(c.fresh.begin(), c.fresh.end(), fresh);
    return ALEBGK_OK;
}

}  // extern "C"
