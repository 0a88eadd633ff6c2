// setup.cu -- the lattice set-up of a box cavity on the device: positions,
// wall flags and wall state, voxel bins and neighbour lists.
//
// Restates, thread per particle, the host set-up of cases.cpp (itself the
// reference's Initialization/ParticleGeneration.cpp:30-200,
// Initialization/NeighbourSearch.cpp:17-99 and the wall state of
// Core/MLSBasis.hpp:228-287 with TestCases/TestCases.cpp:230-249) with the
// same floating-point operations in the same order, so every array comes out
// bitwise equal to the host's.  No expression here is a product feeding a sum
// except where the host itself writes fma(), so contraction cannot change a
// result; products and sums that must stay separate use __dmul_rn/__dadd_rn.
//
// Voxel lists keep the host's order (particles ascending within a voxel):
// particles are counted and scattered per voxel, then each voxel's list is
// sorted.  The neighbour scan then visits voxels and particles exactly as the
// reference does, with the same 128-neighbour cap.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cases.h"
#include "ctx.h"

namespace alebgk {

namespace {

struct LatticeArgs
{
    int dim, Nx, Ny, Nz, N;
    double dx, dy, dz, xleft, xright, ybottom, ytop, zfront, zback;
    double hBox, vBox, wBox, r2max, Tw, lidSpeed;
    int nbh, nbv, nbw, lidKind;
    double lid[6][3];
};

__global__ void k_lattice(LatticeArgs a, double *__restrict__ xyz, int *__restrict__ boundary,
                          int *__restrict__ bodyId, double *__restrict__ wall,
                          double *__restrict__ meshv, int *__restrict__ voxel,
                          int *__restrict__ voxCount)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    const int ix = i % a.Nx, r = i / a.Nx, jy = r % a.Ny, kz = r / a.Ny;
    const double x = fma((double)ix, a.dx, a.xleft);
    const double y = fma((double)jy, a.dy, a.ybottom);
    const double z = (a.dim == 3) ? fma((double)kz, a.dz, a.zfront) : 0.0;
    xyz[3 * (size_t)i] = x;
    xyz[3 * (size_t)i + 1] = y;
    xyz[3 * (size_t)i + 2] = z;
    const bool bx = (ix == 0 || ix == a.Nx - 1);
    const bool by = (jy == 0 || jy == a.Ny - 1);
    const bool bz = (a.dim == 3) && (kz == 0 || kz == a.Nz - 1);
    const int b = (bx || by || bz) ? 1 : 0;
    boundary[i] = b;
    bodyId[i] = -1;
    meshv[3 * (size_t)i] = 0.0;
    meshv[3 * (size_t)i + 1] = 0.0;
    meshv[3 * (size_t)i + 2] = 0.0;

    // wall state: normal, wall velocity, wall temperature
    double w[7] = {0, 0, 0, 0, 0, 0, 0};
    if (b)
    {
        constexpr double eps = 1.0e-13;
        double n[3] = {0, 0, 0}, U[3] = {0, 0, 0}, Tsum = 0;
        int nHit = 0;
        auto hit = [&](double ax, double ay, double az, int face) {
            n[0] = __dadd_rn(n[0], ax);
            n[1] = __dadd_rn(n[1], ay);
            n[2] = __dadd_rn(n[2], az);
            U[0] = __dadd_rn(U[0], a.lid[face][0]);
            U[1] = __dadd_rn(U[1], a.lid[face][1]);
            U[2] = __dadd_rn(U[2], a.lid[face][2]);
            Tsum = __dadd_rn(Tsum, a.Tw);
            ++nHit;
        };
        if (fabs(x - a.xleft) < eps) hit(1, 0, 0, 0);
        if (fabs(x - a.xright) < eps) hit(-1, 0, 0, 1);
        if (fabs(y - a.ytop) < eps) hit(0, -1, 0, 2);
        if (fabs(y - a.ybottom) < eps) hit(0, 1, 0, 3);
        if (fabs(z - a.zfront) < eps) hit(0, 0, -1, 4);
        if (fabs(z - a.zback) < eps) hit(0, 0, 1, 5);
        if (nHit == 0)
            w[6] = a.Tw;
        else if (nHit == 1)
        {
            for (int q = 0; q < 3; ++q) { w[q] = n[q]; w[3 + q] = U[q]; }
            w[6] = Tsum;
        }
        else
        {
            const double nlen = sqrt(fma(n[2], n[2], fma(n[0], n[0], __dmul_rn(n[1], n[1]))));
            if (nlen > eps)
            {
                n[0] = n[0] / nlen;
                n[1] = n[1] / nlen;
                n[2] = n[2] / nlen;
            }
            for (int q = 0; q < 3; ++q) { w[q] = n[q]; w[3 + q] = U[q] / nHit; }
            w[6] = Tsum / nHit;
        }
        if (a.lidKind == 2 && !(fabs(y - a.ytop) > 1e-13))
        {
            const double s = x / (a.xright - a.xleft);
            const double t = fma(-2.0, s, 2.0);
            const double s2 = __dmul_rn(2.0, s);
            w[3] = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(a.lidSpeed, s2), s2), t), t);
        }
    }
    for (int q = 0; q < 7; ++q) wall[7 * (size_t)i + q] = w[q];

    // voxel bin
    const int vi = max(0, min(a.nbh - 1, (int)floor((x - a.xleft) / a.hBox)));
    const int vj = max(0, min(a.nbv - 1, (int)floor((y - a.ybottom) / a.vBox)));
    const int vk = (a.dim == 3) ? max(0, min(a.nbw - 1, (int)floor((z - a.zfront) / a.wBox))) : 0;
    const int v = vi + a.nbh * (vj + a.nbv * vk);
    voxel[i] = v;
    atomicAdd(voxCount + v, 1);
}

// Voxel bin of arbitrary positions (NeighbourSearch.cpp:24-37).
__global__ void k_voxel_assign(LatticeArgs a, const double *__restrict__ xyz, int N,
                               int *__restrict__ voxel, int *__restrict__ voxCount)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    const int vi = max(0, min(a.nbh - 1, (int)floor((x - a.xleft) / a.hBox)));
    const int vj = max(0, min(a.nbv - 1, (int)floor((y - a.ybottom) / a.vBox)));
    const int vk = (a.dim == 3) ? max(0, min(a.nbw - 1, (int)floor((z - a.zfront) / a.wBox))) : 0;
    const int v = vi + a.nbh * (vj + a.nbv * vk);
    voxel[i] = v;
    atomicAdd(voxCount + v, 1);
}

// Exclusive scan of the voxel counts (one thread: a few thousand voxels).
__global__ void k_voxel_scan(const int *__restrict__ count, int nvox, int *start, int *cursor)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int s = 0;
    for (int v = 0; v < nvox; ++v)
    {
        start[v] = s;
        cursor[v] = s;
        s += count[v];
    }
    start[nvox] = s;
}

__global__ void k_voxel_fill(const int *__restrict__ voxel, int N, int *cursor, int *list)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    list[atomicAdd(cursor + voxel[i], 1)] = i;
}

// Sorts each voxel's list ascending, as the host's push_back in index order.
__global__ void k_voxel_sort(const int *__restrict__ start, int nvox, int *list)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    const int a = start[v], b = start[v + 1];
    for (int p = a + 1; p < b; ++p)
    {
        const int key = list[p];
        int q = p - 1;
        while (q >= a && list[q] > key)
        {
            list[q + 1] = list[q];
            --q;
        }
        list[q + 1] = key;
    }
}

__global__ void k_neighbours(LatticeArgs a, const double *__restrict__ xyz,
                             const int *__restrict__ voxel, const int *__restrict__ start,
                             const int *__restrict__ list, int *__restrict__ nnb,
                             int *__restrict__ nbr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.N) return;
    int *out = nbr + (size_t)i * kMaxNeigh;
    const double xi = xyz[3 * (size_t)i], yi = xyz[3 * (size_t)i + 1],
                 zi = xyz[3 * (size_t)i + 2];
    const int vi = voxel[i] % a.nbh, t = voxel[i] / a.nbh, vj = t % a.nbv, vk = t / a.nbv;
    const int dkmax = (a.dim == 3) ? 1 : 0;
    int cnt = 0;
    bool done = false;
    for (int dk = -dkmax; dk <= dkmax && !done; dk++)
        for (int dj = -1; dj <= 1 && !done; dj++)
            for (int di = -1; di <= 1 && !done; di++)
            {
                const int ni = vi + di, nj = vj + dj, nk = vk + dk;
                if (ni < 0 || ni >= a.nbh) continue;
                if (nj < 0 || nj >= a.nbv) continue;
                if (nk < 0 || nk >= a.nbw) continue;
                const int v = ni + a.nbh * (nj + a.nbv * nk);
                for (int p = start[v]; p < start[v + 1]; ++p)
                {
                    const int j = list[p];
                    if (j == i) continue;
                    const double ddx = xyz[3 * (size_t)j] - xi;
                    const double ddy = xyz[3 * (size_t)j + 1] - yi;
                    const double ddz = (a.dim == 3) ? xyz[3 * (size_t)j + 2] - zi : 0.0;
                    if (fma(ddz, ddz, fma(ddx, ddx, __dmul_rn(ddy, ddy))) < a.r2max)
                    {
                        out[cnt++] = j;
                        if (cnt >= kMaxNeigh) { done = true; break; }
                    }
                }
            }
    nnb[i] = cnt;
    for (int s = cnt; s < kMaxNeigh; ++s) out[s] = -1;
}

// Every particle's row from one rest-state row; macros (rho, 0, 0, 0, T, p).
template <typename T>
__global__ void k_rest_state(const double *__restrict__ row, int gs, int ldf, int N, double rho,
                             double T0, double R, T *__restrict__ f, double *__restrict__ macro,
                             int *__restrict__ mood)
{
    const size_t tot = (size_t)N * gs;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tot;
         q += (size_t)gridDim.x * blockDim.x)
    {
        const size_t i = q / gs, k = q % gs;
        f[i * ldf + k] = (T)row[k];
        if (k == 0)
        {
            double *m = macro + 6 * i;
            m[0] = rho; m[1] = 0.0; m[2] = 0.0; m[3] = 0.0; m[4] = T0;
            m[5] = __dmul_rn(__dmul_rn(rho, R), T0);
            mood[i] = 0;
        }
    }
}

// ---------------------------------------------------------------------------
// Body embedding (Initialization/BodyEmbedding.cpp:18-104): drop the lattice
// particles inside a body or within 0.4 dx of one of its surface points,
// keep the rest in order, append the surface particles.  The surface points
// and their wall state come from the host (bodySurface in cases.cpp, the
// same records the host set-up appends).
// ---------------------------------------------------------------------------
struct EmbedBody
{
    int kind, s0, s1;   // surface points [s0, s1)
    double cx, cy, cz, size, ox, oy;
    double Rm[9];
};

// Body::inside of cases.cpp (RigidBody/Geometry.hpp) with the host's
// operations: explicit fma where the host writes one, separately rounded
// products and sums elsewhere.
__device__ bool insideBody(const EmbedBody &b, double x, double y, double z)
{
    switch (b.kind)
    {
    case 0:
    {
        const double xC = __dsub_rn(x, b.cx), yC = __dsub_rn(y, b.cy);
        const double D = __dadd_rn(__dmul_rn(b.ox, b.ox), __dmul_rn(b.oy, b.oy));
        const double xp = __dadd_rn(__dmul_rn(b.ox, xC), __dmul_rn(b.oy, yC)) / D;
        const double yp = __dsub_rn(__dmul_rn(b.oy, xC), __dmul_rn(b.ox, yC)) / D;
        return fabs(xp) <= b.size / 2 && fabs(yp) <= b.size / 2;
    }
    case 1:
    {
        const double dx = __dsub_rn(x, b.cx), dy = __dsub_rn(y, b.cy);
        return fma(dx, dx, __dmul_rn(dy, dy)) <= __dmul_rn(b.size, b.size);
    }
    case 2:
    {
        const double dx = __dsub_rn(x, b.cx), dy = __dsub_rn(y, b.cy), dz = __dsub_rn(z, b.cz);
        return fma(dz, dz, fma(dx, dx, __dmul_rn(dy, dy))) <= __dmul_rn(b.size, b.size);
    }
    default:
    {
        const double dx = __dsub_rn(x, b.cx), dy = __dsub_rn(y, b.cy), dz = __dsub_rn(z, b.cz);
        const double bx = fma(b.Rm[6], dz, fma(b.Rm[0], dx, __dmul_rn(b.Rm[3], dy)));
        const double by = fma(b.Rm[7], dz, fma(b.Rm[1], dx, __dmul_rn(b.Rm[4], dy)));
        const double bz = fma(b.Rm[8], dz, fma(b.Rm[2], dx, __dmul_rn(b.Rm[5], dy)));
        const double h = b.size / 2;
        return fabs(bx) <= h && fabs(by) <= h && fabs(bz) <= h;
    }
    }
}

__global__ void k_embed_mark(const double *__restrict__ xyz, int N, int dim,
                             const EmbedBody *__restrict__ bodies, int nb,
                             const double *__restrict__ surf, double hug2, int *__restrict__ keep)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const double x = xyz[3 * (size_t)i], y = xyz[3 * (size_t)i + 1], z = xyz[3 * (size_t)i + 2];
    bool drop = false;
    for (int b = 0; b < nb && !drop; ++b)
    {
        const EmbedBody &B = bodies[b];
        if (insideBody(B, x, y, dim == 3 ? z : B.cz)) { drop = true; break; }
        for (int q = B.s0; q < B.s1; ++q)
        {
            const double dx = __dsub_rn(x, surf[3 * q]), dy = __dsub_rn(y, surf[3 * q + 1]);
            double d2 = fma(dx, dx, __dmul_rn(dy, dy));
            if (dim == 3)
            {
                const double dz = __dsub_rn(z, surf[3 * q + 2]);
                d2 = fma(dz, dz, d2);
            }
            if (d2 < hug2) { drop = true; break; }
        }
    }
    keep[i] = drop ? 0 : 1;
}

// Exclusive scan of keep[0..n) in one 1024-thread block; *count = the total.
__global__ void __launch_bounds__(1024)
k_embed_scan(const int *__restrict__ keep, int n, int *__restrict__ pos, int *count)
{
    __shared__ int part[1024];
    const int t = threadIdx.x, per = (n + 1023) / 1024;
    const int lo = min(n, t * per), hi = min(n, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += keep[i];
    part[t] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1)
    {
        const int v = (t >= off) ? part[t - off] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    int run = (t > 0) ? part[t - 1] : 0;
    for (int i = lo; i < hi; ++i)
    {
        pos[i] = run;
        run += keep[i];
    }
    if (t == 1023) *count = part[1023];
}

__global__ void k_embed_scatter(LatticeDev in, const int *__restrict__ keep,
                                const int *__restrict__ pos, int N, LatticeDev out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N || !keep[i]) return;
    const size_t j = pos[i];
    for (int q = 0; q < 3; ++q)
    {
        out.xyz[3 * j + q] = in.xyz[3 * (size_t)i + q];
        out.meshv[3 * j + q] = in.meshv[3 * (size_t)i + q];
    }
    for (int q = 0; q < 7; ++q) out.wall[7 * j + q] = in.wall[7 * (size_t)i + q];
    out.boundary[j] = in.boundary[i];
    out.bodyId[j] = in.bodyId[i];
}

__global__ void k_embed_append(const double *__restrict__ surf, const double *__restrict__ wall,
                               const int *__restrict__ body, int nsurf,
                               const int *__restrict__ kept, LatticeDev out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nsurf) return;
    const size_t j = (size_t)*kept + q;
    for (int k = 0; k < 3; ++k)
    {
        out.xyz[3 * j + k] = surf[3 * (size_t)q + k];
        out.meshv[3 * j + k] = 0.0;
    }
    for (int k = 0; k < 7; ++k) out.wall[7 * j + k] = wall[7 * (size_t)q + k];
    out.boundary[j] = 1;
    out.bodyId[j] = body[q];
}

}  // namespace

cudaError_t embedLatticeDevice(const CaseParams &p, const std::vector<Body> &bodies,
                               const std::vector<double> &surfXyz,
                               const std::vector<double> &surfWall,
                               const std::vector<int> &surfStart, const LatticeDev &raw, int NL,
                               const LatticeDev &out, int *nOut, cudaStream_t st)
{
    const int nb = (int)bodies.size(), nsurf = (int)(surfXyz.size() / 3);
    std::vector<EmbedBody> eb(nb);
    std::vector<int> bodyOf(nsurf);
    for (int b = 0; b < nb; ++b)
    {
        const Body &B = bodies[b];
        EmbedBody &e = eb[b];
        e.kind = B.kind; e.s0 = surfStart[b]; e.s1 = surfStart[b + 1];
        e.cx = B.cx; e.cy = B.cy; e.cz = B.cz; e.size = B.size; e.ox = B.ox; e.oy = B.oy;
        for (int k = 0; k < 9; ++k) e.Rm[k] = B.Rm[k];
        for (int q = e.s0; q < e.s1; ++q) bodyOf[q] = b;
    }
    EmbedBody *dB = nullptr;
    double *dSurf = nullptr, *dWall = nullptr;
    int *dBody = nullptr, *keep = nullptr, *pos = nullptr, *count = nullptr;
    const size_t nsa = std::max(nsurf, 1);
    cudaError_t e = cudaMalloc(&dB, sizeof(EmbedBody) * std::max(nb, 1));
    if (e == cudaSuccess) e = cudaMalloc(&dSurf, 24 * nsa);
    if (e == cudaSuccess) e = cudaMalloc(&dWall, 56 * nsa);
    if (e == cudaSuccess) e = cudaMalloc(&dBody, 4 * nsa);
    if (e == cudaSuccess) e = cudaMalloc(&keep, 4 * (size_t)NL);
    if (e == cudaSuccess) e = cudaMalloc(&pos, 4 * (size_t)NL);
    if (e == cudaSuccess) e = cudaMalloc(&count, 4);
    if (e == cudaSuccess && nb)
        e = cudaMemcpyAsync(dB, eb.data(), sizeof(EmbedBody) * nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nsurf)
        e = cudaMemcpyAsync(dSurf, surfXyz.data(), 24 * (size_t)nsurf, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nsurf)
        e = cudaMemcpyAsync(dWall, surfWall.data(), 56 * (size_t)nsurf, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nsurf)
        e = cudaMemcpyAsync(dBody, bodyOf.data(), 4 * (size_t)nsurf, cudaMemcpyHostToDevice, st);
    const double hug = 0.4 * std::fabs(p.dx);
    const double hug2 = std::pow(hug, 2);
    int kept = 0;
    if (e == cudaSuccess)
    {
        k_embed_mark<<<(NL + 127) / 128, 128, 0, st>>>(raw.xyz, NL, p.dim, dB, nb, dSurf, hug2,
                                                       keep);
        k_embed_scan<<<1, 1024, 0, st>>>(keep, NL, pos, count);
        k_embed_scatter<<<(NL + 255) / 256, 256, 0, st>>>(raw, keep, pos, NL, out);
        if (nsurf)
            k_embed_append<<<(nsurf + 127) / 128, 128, 0, st>>>(dSurf, dWall, dBody, nsurf,
                                                                count, out);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&kept, count, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    const int N = kept + nsurf;
    if (e == cudaSuccess && out.nnb)
    {
        NeighbourGrid g;
        g.dim = p.dim;
        g.x0 = p.xleft; g.y0 = p.ybottom; g.z0 = p.zfront;
        g.hx = p.hBox; g.hy = p.vBox; g.hz = p.wBox;
        g.nx = p.nbhBox; g.ny = p.nbvBox; g.nz = p.nbwBox;
        g.radius = p.radius;
        e = buildNeighboursDevice(g, out.xyz, N, out, st);
    }
    for (void *q : {(void *)dB, (void *)dSurf, (void *)dWall, (void *)dBody, (void *)keep,
                    (void *)pos, (void *)count})
        if (q) cudaFree(q);
    if (nOut) *nOut = N;
    return e;
}

cudaError_t buildLatticeDevice(const CaseParams &p, const LatticeDev &o, cudaStream_t st,
                               bool neighbours)
{
    LatticeArgs a{};
    a.dim = p.dim; a.Nx = p.Nx; a.Ny = p.Ny; a.Nz = (p.dim == 3) ? p.Nz : 1;
    a.N = a.Nx * a.Ny * a.Nz;
    a.dx = p.dx; a.dy = p.dy; a.dz = p.dz;
    a.xleft = p.xleft; a.xright = p.xright; a.ybottom = p.ybottom; a.ytop = p.ytop;
    a.zfront = p.zfront; a.zback = p.zback;
    a.hBox = p.hBox; a.vBox = p.vBox; a.wBox = p.wBox;
    a.nbh = p.nbhBox; a.nbv = p.nbvBox; a.nbw = p.nbwBox;
    a.r2max = p.radius * p.radius;
    a.Tw = p.Tw;
    a.lidKind = p.lidKind;
    a.lidSpeed = p.lidSpeed;
    for (int f = 0; f < 6; ++f)
        for (int q = 0; q < 3; ++q) a.lid[f][q] = 0.0;
    if (p.lidKind == 0) a.lid[2][0] = p.lidSpeed;
    if (p.lidKind == 1) a.lid[4][0] = p.lidSpeed;
    const int nvox = a.nbh * a.nbv * a.nbw;
    const int nb = (a.N + 255) / 256;
    cudaError_t e = cudaMemsetAsync(o.voxCount, 0, sizeof(int) * nvox, st);
    if (e != cudaSuccess) return e;
    k_lattice<<<nb, 256, 0, st>>>(a, o.xyz, o.boundary, o.bodyId, o.wall, o.meshv, o.voxel,
                                  o.voxCount);
    if (!neighbours) return cudaGetLastError();
    k_voxel_scan<<<1, 32, 0, st>>>(o.voxCount, nvox, o.voxStart, o.voxCursor);
    k_voxel_fill<<<nb, 256, 0, st>>>(o.voxel, a.N, o.voxCursor, o.voxList);
    k_voxel_sort<<<(nvox + 127) / 128, 128, 0, st>>>(o.voxStart, nvox, o.voxList);
    k_neighbours<<<(a.N + 127) / 128, 128, 0, st>>>(a, o.xyz, o.voxel, o.voxStart, o.voxList,
                                                    o.nnb, o.nbr);
    return cudaGetLastError();
}

cudaError_t buildNeighboursDevice(const NeighbourGrid &gr, const double *xyz, int N,
                                  const LatticeDev &o, cudaStream_t st)
{
    LatticeArgs a{};
    a.dim = gr.dim; a.N = N;
    a.xleft = gr.x0; a.ybottom = gr.y0; a.zfront = gr.z0;
    a.hBox = gr.hx; a.vBox = gr.hy; a.wBox = gr.hz;
    a.nbh = gr.nx; a.nbv = gr.ny; a.nbw = gr.nz;
    a.r2max = gr.radius * gr.radius;
    const int nvox = a.nbh * a.nbv * a.nbw;
    const int nb = (N + 255) / 256;
    cudaError_t e = cudaMemsetAsync(o.voxCount, 0, sizeof(int) * nvox, st);
    if (e != cudaSuccess) return e;
    k_voxel_assign<<<nb, 256, 0, st>>>(a, xyz, N, o.voxel, o.voxCount);
    k_voxel_scan<<<1, 32, 0, st>>>(o.voxCount, nvox, o.voxStart, o.voxCursor);
    k_voxel_fill<<<nb, 256, 0, st>>>(o.voxel, N, o.voxCursor, o.voxList);
    k_voxel_sort<<<(nvox + 127) / 128, 128, 0, st>>>(o.voxStart, nvox, o.voxList);
    k_neighbours<<<(N + 127) / 128, 128, 0, st>>>(a, xyz, o.voxel, o.voxStart, o.voxList,
                                                  o.nnb, o.nbr);
    return cudaGetLastError();
}

cudaError_t launchRestState(alebgk_ctx *c, const double *rowDev, double rho, double T0)
{
    const StepParams &p = c->sp;
    if (c->cfg.precision == 64)
        k_rest_state<double><<<1184, 256, 0, c->stream>>>(
            rowDev, p.gs, p.ldf, p.N, rho, T0, p.R, static_cast<double *>(c->d.f[c->cur]),
            c->d.macro[c->cur], c->d.mood);
    else
        k_rest_state<float><<<1184, 256, 0, c->stream>>>(
            rowDev, p.gs, p.ldf, p.N, rho, T0, p.R, static_cast<float *>(c->d.f[c->cur]),
            c->d.macro[c->cur], c->d.mood);
    return cudaGetLastError();
}

}  // namespace alebgk
