// classes_dev.cu -- stencil classes on the device.
//
// The class of a particle is the exact key of coeffs.cpp's buildClasses
// (the MLS set-up of MLSTransport/MLSTransport.cpp:88-311 depends on nothing
// else): wall flag, MLS order, neighbour count, the bit patterns of the
// mesh velocity (and of the wall state for wall particles), and the
// neighbour displacements quantised on a grid of h 2^-32, sorted by
// (dz, dy, dx) then neighbour index.  One warp per particle computes the
// displacements with the host's operations (x_j - x_i, the minimum image
// unfused, division by the quantum, round half away from zero), ranks them,
// writes the particle's slot list in that order and its key, and folds the
// key into a 64-bit hash.  The host groups the hashes (first particle of
// each hash), the device compares every key with its group's first key in
// full, and the class ids follow in order of first appearance, as the host
// builder numbers them.  Two different keys with one hash would need the
// host builder: the caller falls back to it when the comparison reports one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <vector>

#include "coeffs.h"
#include "ctx.h"

namespace alebgk {

namespace {

constexpr int kCW = 4;   // warps per block (two 4 KB entry arrays per warp)

struct NbEntry
{
    long long k2, k1, k0;
    int j, pad;
};

__device__ __forceinline__ bool entryLess(const NbEntry &a, const NbEntry &b)
{
    if (a.k2 != b.k2) return a.k2 < b.k2;
    if (a.k1 != b.k1) return a.k1 < b.k1;
    if (a.k0 != b.k0) return a.k0 < b.k0;
    return a.j < b.j;
}

__device__ __forceinline__ unsigned long long foldKey(unsigned long long h, long long x)
{
    h ^= (unsigned long long)x + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
    return h * 1099511628211ULL;
}

struct KeyArgs
{
    int N, dim, S, maxNeigh, mlsOrder;
    double q;
    int periodic[3];
    double L[3];
};

__global__ void __launch_bounds__(kCW * 32)
k_class_keys(KeyArgs a, const double *__restrict__ xyz, const double *__restrict__ meshv,
             const double *__restrict__ wall, const int *__restrict__ boundary,
             const int *__restrict__ nnb, const int *__restrict__ nbr,
             const long long *__restrict__ koff, long long *__restrict__ keys,
             unsigned long long *__restrict__ hashes, int *__restrict__ nslot,
             int *__restrict__ slots)
{
    __shared__ NbEntry ent[kCW][ALEBGK_MAX_NEIGH];
    __shared__ NbEntry srt[kCW][ALEBGK_MAX_NEIGH];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kCW + warp;
    if (i >= a.N) return;                      // warp-uniform
    const int nn = nnb[i];
    const double xi[3] = {xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]};
    for (int s = lane; s < nn; s += 32)
    {
        const int j = nbr[(size_t)i * a.maxNeigh + s];
        long long kq[3];
        for (int c = 0; c < 3; ++c)
        {
            double d = 0.0;
            if (c < a.dim)
            {
                d = __dsub_rn(xyz[3 * (size_t)j + c], xi[c]);
                if (a.periodic[c]) d = __dsub_rn(d, __dmul_rn(a.L[c], round(__ddiv_rn(d, a.L[c]))));
            }
            kq[c] = llround(__ddiv_rn(d, a.q));
        }
        ent[warp][s] = NbEntry{kq[2], kq[1], kq[0], j, 0};
    }
    __syncwarp();
    // rank of each entry: the entries before it in sorted order (equal
    // entries, which distinct neighbours never give, in list order), so the
    // ranks are a permutation of 0..nn-1
    for (int s = lane; s < nn; s += 32)
    {
        const NbEntry e = ent[warp][s];
        int r = 0;
        for (int t = 0; t < nn; ++t)
        {
            const NbEntry &f = ent[warp][t];
            r += (entryLess(f, e) || (t < s && !entryLess(e, f))) ? 1 : 0;
        }
        srt[warp][r] = e;
    }
    __syncwarp();
    int *sl = slots + (size_t)i * a.S;
    for (int s = lane; s < a.S; s += 32) sl[s] = (s >= 1 && s <= nn) ? srt[warp][s - 1].j : i;
    const int bnd = boundary[i];
    const int head = 6 + (bnd ? 7 : 0);
    long long *k = keys + koff[i];
    if (lane == 0)
    {
        nslot[i] = 1 + nn;
        k[0] = bnd;
        k[1] = bnd ? 1 : a.mlsOrder;
        k[2] = nn;
        for (int c = 0; c < 3; ++c) k[3 + c] = __double_as_longlong(meshv[3 * (size_t)i + c]);
        if (bnd)
            for (int c = 0; c < 7; ++c) k[6 + c] = __double_as_longlong(wall[7 * (size_t)i + c]);
    }
    for (int s = lane; s < nn; s += 32)
    {
        const NbEntry &e = srt[warp][s];
        k[head + 3 * s] = e.k2;
        k[head + 3 * s + 1] = e.k1;
        k[head + 3 * s + 2] = e.k0;
    }
    __syncwarp();
    if (lane == 0)
    {
        unsigned long long h = 1469598103934665603ULL;
        for (int w = 0; w < head; ++w) h = foldKey(h, k[w]);
        for (int s = 0; s < nn; ++s)
        {
            const NbEntry &e = srt[warp][s];
            h = foldKey(h, e.k2);
            h = foldKey(h, e.k1);
            h = foldKey(h, e.k0);
        }
        hashes[i] = h;
    }
}

// same[i] = 1 when particle i's key equals the key of particle first[i].
__global__ void __launch_bounds__(kCW * 32)
k_class_same(int N, const long long *__restrict__ koff, const long long *__restrict__ keys,
             const int *__restrict__ first, int *__restrict__ same)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kCW + warp;
    if (i >= N) return;
    const int f = first[i];
    const long long li = koff[i + 1] - koff[i], lf = koff[f + 1] - koff[f];
    int eq = li == lf;
    if (eq && f != i)
    {
        const long long *a = keys + koff[i], *b = keys + koff[f];
        for (long long w = lane; w < li; w += 32) eq &= a[w] == b[w];
        eq = __all_sync(0xffffffffu, eq);
    }
    if (lane == 0) same[i] = eq;
}

// Slot rows and slot counts of the class representatives, packed.
__global__ void k_class_rep_rows(int ncls, int S, const int *__restrict__ rep,
                                 const int *__restrict__ nslot, const int *__restrict__ slots,
                                 int *__restrict__ repSlots, int *__restrict__ repNslot)
{
    const int c = blockIdx.x;
    const int r = rep[c];
    for (int s = threadIdx.x; s < S; s += blockDim.x)
        repSlots[(size_t)c * S + s] = slots[(size_t)r * S + s];
    if (threadIdx.x == 0) repNslot[c] = nslot[r];
}

template <typename P>
cudaError_t grow(P **p, size_t &cap, size_t n)
{
    if (n <= cap && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(P));
    if (e == cudaSuccess) cap = std::max<size_t>(n, 1);
    return e;
}

}  // namespace

void freeClassScratch(ClassScratch &s)
{
    for (void *p : {(void *)s.nnb, (void *)s.nbr, (void *)s.koff, (void *)s.keys,
                    (void *)s.hashes, (void *)s.first, (void *)s.same, (void *)s.rep,
                    (void *)s.repSlots, (void *)s.repNslot})
        if (p) cudaFree(p);
    s = ClassScratch();
}

cudaError_t buildClassesDevice(const CoeffInput &in, const double *dXyz, const double *dMeshv,
                               const double *dWall, const int *dBoundary, int *dCls,
                               int *dNslot, int *dSlots, size_t slotsCap, ClassScratch &scr,
                               CoeffTables &out, bool &collision, cudaStream_t st)
{
    collision = false;
    const int N = in.N;
    const int V = (in.dim == 3) ? in.Nv * in.Nv * in.Nv : in.Nv * in.Nv;
    int maxnn = 0;
    for (int i = 0; i < N; ++i)
    {
        if (in.nnb[i] < 0 || in.nnb[i] > in.maxNeigh || in.maxNeigh > ALEBGK_MAX_NEIGH)
            return cudaErrorInvalidValue;
        maxnn = std::max(maxnn, in.nnb[i]);
    }
    const int S = 1 + maxnn;
    if ((size_t)N * S > slotsCap) return cudaErrorInvalidValue;
    std::vector<long long> koff((size_t)N + 1, 0);
    for (int i = 0; i < N; ++i)
        koff[i + 1] = koff[i] + 6 + (in.boundary[i] ? 7 : 0) + 3 * (long long)in.nnb[i];
    cudaError_t e = grow(&scr.nnb, scr.capN, (size_t)N);
    if (e == cudaSuccess) e = grow(&scr.hashes, scr.capHash, (size_t)N);
    if (e == cudaSuccess) e = grow(&scr.first, scr.capFirst, (size_t)N);
    if (e == cudaSuccess) e = grow(&scr.same, scr.capSame, (size_t)N);
    if (e == cudaSuccess) e = grow(&scr.koff, scr.capKoff, (size_t)N + 1);
    if (e == cudaSuccess) e = grow(&scr.nbr, scr.capNbr, (size_t)N * in.maxNeigh);
    if (e == cudaSuccess) e = grow(&scr.keys, scr.capKeys, (size_t)koff[N]);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr.nnb, in.nnb, 4 * (size_t)N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr.nbr, in.nbr, 4 * (size_t)N * in.maxNeigh, cudaMemcpyHostToDevice,
                            st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr.koff, koff.data(), 8 * koff.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    KeyArgs a{};
    a.N = N; a.dim = in.dim; a.S = S; a.maxNeigh = in.maxNeigh; a.mlsOrder = in.mlsOrder;
    a.q = in.h * std::ldexp(1.0, -32);
    for (int c = 0; c < 3; ++c) { a.periodic[c] = in.periodic[c] ? 1 : 0; a.L[c] = in.L[c]; }
    const int blocks = (N + kCW - 1) / kCW;
    k_class_keys<<<blocks, kCW * 32, 0, st>>>(a, dXyz, dMeshv, dWall, dBoundary, scr.nnb,
                                              scr.nbr, scr.koff, scr.keys, scr.hashes, dNslot,
                                              dSlots);
    e = cudaGetLastError();
    std::vector<unsigned long long> hashes(N);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(hashes.data(), scr.hashes, 8 * (size_t)N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    // first particle of every hash
    std::vector<int> first(N);
    {
        std::unordered_map<unsigned long long, int> firstOf;
        firstOf.reserve(4096);
        for (int i = 0; i < N; ++i) first[i] = firstOf.emplace(hashes[i], i).first->second;
    }
    e = cudaMemcpyAsync(scr.first, first.data(), 4 * (size_t)N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
    {
        k_class_same<<<blocks, kCW * 32, 0, st>>>(N, scr.koff, scr.keys, scr.first, scr.same);
        e = cudaGetLastError();
    }
    std::vector<int> same(N);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(same.data(), scr.same, 4 * (size_t)N, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    for (int i = 0; i < N; ++i)
        if (!same[i])
        {
            collision = true;
            return cudaSuccess;
        }
    // class ids in order of first appearance
    out = CoeffTables();
    out.S = S; out.V = V;
    out.cls.assign(N, 0);
    for (int i = 0; i < N; ++i)
    {
        if (first[i] == i)
        {
            out.cls[i] = (int)out.rep.size();
            out.rep.push_back(i);
        }
        else
            out.cls[i] = out.cls[first[i]];
    }
    const int ncls = (int)out.rep.size();
    out.ncls = ncls;
    out.members.assign(ncls, 0);
    out.order.assign(ncls, 0);
    out.degenerate.assign(ncls, 0);
    for (int i = 0; i < N; ++i) out.members[out.cls[i]]++;
    for (int c = 0; c < ncls; ++c) out.order[c] = in.boundary[out.rep[c]] ? 1 : in.mlsOrder;
    // the representatives' slot rows for the table builder
    e = grow(&scr.rep, scr.capRep, (size_t)ncls);
    if (e == cudaSuccess) e = grow(&scr.repSlots, scr.capRepSlots, (size_t)ncls * S);
    if (e == cudaSuccess) e = grow(&scr.repNslot, scr.capRepNslot, (size_t)ncls);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr.rep, out.rep.data(), 4 * (size_t)ncls, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
    {
        k_class_rep_rows<<<ncls, 128, 0, st>>>(ncls, S, scr.rep, dNslot, dSlots, scr.repSlots,
                                               scr.repNslot);
        e = cudaGetLastError();
    }
    out.repSlots.resize((size_t)ncls * S);
    out.repNslot.resize(ncls);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out.repSlots.data(), scr.repSlots, 4 * (size_t)ncls * S,
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out.repNslot.data(), scr.repNslot, 4 * (size_t)ncls,
                            cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dCls, out.cls.data(), 4 * (size_t)N, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e;
}

}  // namespace alebgk
