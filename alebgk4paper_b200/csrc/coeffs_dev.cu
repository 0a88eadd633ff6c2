// coeffs_dev.cu -- the MLS transport coefficient tables built on the device,
// one thread per (stencil class, velocity node), equal bitwise to the host
// builder of coeffs.cpp (and so to the reference's MLS solve that the host
// builder restates, MLSTransport/MLSTransport.cpp:88-311 with the basis and
// weight of Core/MLSBasis.hpp:142-202 and the pivot-skip elimination of
// MLSTransport.cpp:20-62).
//
// The host builder is compiled without floating-point contraction, so this
// file is compiled with -fmad=false and follows the host's operations and
// loop orders one for one: foot point, per-slot weight and basis, the
// normal-equation matrix summed slot by slot, elimination with unit
// right-hand sides, and the coefficients w_s * (row 0 of the inverse . b_s).
// The stencil classes themselves (a hash of each particle's neighbour
// offsets) are still built on the host.
#include <cuda_runtime.h>

#include <vector>

#include "coeffs.h"
#include "ctx.h"

namespace alebgk {

namespace {

struct ClassArgs
{
    int dim, Nv, V, S, mlsOrder;
    double dt, h, vmin, dv;
    int periodic[3];
    double L[3];
};

__device__ __forceinline__ double minImageD(double d, double L)
{
    return d - L * round(d / L);
}

__device__ __forceinline__ double weightSqD(double r2, double h)
{
    double q2 = r2 / (h * h);
    if (q2 >= 1.0) return 0.0;
    double w = 1.0 - q2;
    return w * w;
}

__device__ __forceinline__ int basisD(double dx, double dy, double dz, int ndim, double h,
                                      double *b, int order)
{
    double sx = dx / h, sy = dy / h, sz = dz / h;
    b[0] = 1.0; b[1] = sx; b[2] = sy;
    if (ndim == 2)
    {
        if (order >= 2)
        {
            b[3] = sx * sx; b[4] = sx * sy; b[5] = sy * sy;
            return 6;
        }
        return 3;
    }
    b[3] = sz;
    if (order >= 2)
    {
        b[4] = sx * sx; b[5] = sy * sy; b[6] = sz * sz;
        b[7] = sx * sy; b[8] = sx * sz; b[9] = sy * sz;
        return 10;
    }
    return 4;
}

__device__ int solveSkipGED(double *A, double *B, int n, int nrhs)
{
    int skipped = 0;
    for (int col = 0; col < n; ++col)
    {
        int piv = col;
        double mx = fabs(A[col * n + col]);
        for (int row = col + 1; row < n; ++row)
            if (fabs(A[row * n + col]) > mx)
            {
                mx = fabs(A[row * n + col]);
                piv = row;
            }
        if (piv != col)
        {
            for (int j = 0; j < n; ++j)
            {
                double t = A[col * n + j]; A[col * n + j] = A[piv * n + j]; A[piv * n + j] = t;
            }
            for (int j = 0; j < nrhs; ++j)
            {
                double t = B[col * nrhs + j]; B[col * nrhs + j] = B[piv * nrhs + j];
                B[piv * nrhs + j] = t;
            }
        }
        double d = A[col * n + col];
        if (fabs(d) < 1.0e-30) { ++skipped; continue; }
        for (int row = col + 1; row < n; ++row)
        {
            double f = A[row * n + col] / d;
            for (int j = col; j < n; ++j) A[row * n + j] -= f * A[col * n + j];
            for (int j = 0; j < nrhs; ++j) B[row * nrhs + j] -= f * B[col * nrhs + j];
        }
    }
    for (int i = n - 1; i >= 0; --i)
    {
        bool ok = fabs(A[i * n + i]) > 1.0e-30;
        for (int r = 0; r < nrhs; ++r)
        {
            double s = B[i * nrhs + r];
            for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * B[j * nrhs + r];
            B[i * nrhs + r] = ok ? s / A[i * n + i] : 0.0;
        }
    }
    return skipped;
}

// Per class: rep position (3), mesh velocity (3), wall state (7), then the
// positions of slots 1..nsl-1 (3 each) at [c][S][3].
template <typename T>
__global__ void k_class_tables(ClassArgs a, int order0, const int *__restrict__ boundary,
                               const int *__restrict__ nsl, const double *__restrict__ rep,
                               const double *__restrict__ slotPos, T *__restrict__ table,
                               int *__restrict__ degen)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (k >= a.V) return;
    const int ndim = a.dim, Nv = a.Nv, V = a.V;
    const bool bnd = boundary[c] != 0;
    const int order = bnd ? 1 : order0;
    const double *rp = rep + 13 * (size_t)c;
    const double *wl = rp + 6;
    T *cc = table + (size_t)c * a.S * V;
    const int iv = k % Nv, jv = (k / Nv) % Nv, kv = (ndim == 3) ? k / (Nv * Nv) : 0;
    const double vx = fma((double)iv, a.dv, a.vmin);
    const double vy = fma((double)jv, a.dv, a.vmin);
    const double vz = fma((double)kv, a.dv, a.vmin);
    if (bnd)
    {
        const double ca = vx - wl[3], cb = vy - wl[4];
        const double cn = (ndim == 3) ? fma(vz - wl[5], wl[2], fma(ca, wl[0], cb * wl[1]))
                                      : fma(ca, wl[0], cb * wl[1]);
        if (cn >= 0.0) { cc[k] = (T)1.0; return; }
    }
    const double xf = rp[0] - (vx - rp[3]) * a.dt;
    const double yf = rp[1] - (vy - rp[4]) * a.dt;
    const double zf = rp[2] - (vz - rp[5]) * a.dt;
    const int n = nsl[c];
    const double *sp = slotPos + (size_t)c * a.S * 3;
    auto offset = [&](int s, double &dx, double &dy, double &dz) {
        dx = sp[3 * s] - xf;
        dy = sp[3 * s + 1] - yf;
        dz = (ndim == 3) ? sp[3 * s + 2] - zf : 0.0;
        if (a.periodic[0]) dx = minImageD(dx, a.L[0]);
        if (a.periodic[1]) dy = minImageD(dy, a.L[1]);
        if (ndim == 3 && a.periodic[2]) dz = minImageD(dz, a.L[2]);
    };
    int P = 0;
    double A[100];
    for (int q = 0; q < 100; ++q) A[q] = 0.0;
    bool any = false;
    double b[10];
    for (int s = 1; s < n; ++s)
    {
        double dx, dy, dz;
        offset(s, dx, dy, dz);
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double ws = weightSqD(r2, a.h);
        if (ws < 1.0e-30) continue;
        P = basisD(dx, dy, dz, ndim, a.h, b, order);
        for (int p1 = 0; p1 < P; ++p1)
            for (int p2 = 0; p2 < P; ++p2) A[p1 * P + p2] += ws * b[p1] * b[p2];
        any = true;
    }
    if (!any) { cc[k] = (T)1.0; return; }
    double B[100];
    for (int q = 0; q < 100; ++q) B[q] = 0.0;
    for (int m = 0; m < P; ++m) B[m * P + m] = 1.0;
    if (solveSkipGED(A, B, P, P) > 0) atomicAdd(degen + c, 1);
    // FP32 tables: the largest coefficient takes the rounding of the node's
    // sum, as roundCoefFP32 does on the host (same order, same operations).
    double s64 = 0.0, s32 = 0.0, big = -1.0;
    int smax = 0;
    for (int s = 1; s < n; ++s)
    {
        double dx, dy, dz;
        offset(s, dx, dy, dz);
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double ws = weightSqD(r2, a.h);
        if (ws < 1.0e-30) continue;
        basisD(dx, dy, dz, ndim, a.h, b, order);
        double acc = 0.0;
        for (int m = 0; m < P; ++m) acc += B[m] * b[m];
        const double c = ws * acc;
        cc[(size_t)s * V + k] = (T)c;
        if (sizeof(T) == 4)
        {
            s64 += c;
            s32 += (double)(T)c;
            if (fabs(c) > big) { big = fabs(c); smax = s; }
        }
    }
    if (sizeof(T) == 4 && big > 0.0)
    {
        const size_t q = (size_t)smax * V + k;
        cc[q] = (T)((double)cc[q] + (s64 - s32));
    }
}

}  // namespace

cudaError_t buildTablesDevice(const CoeffInput &in, const CoeffTables &cls, int order,
                              void *table, bool f64, std::vector<int> &degenerate,
                              cudaStream_t st)
{
    const int ncls = cls.ncls, S = cls.S, V = cls.V;
    std::vector<int> bnd(ncls), nsl(ncls);
    std::vector<double> rep(13 * (size_t)ncls), pos((size_t)ncls * S * 3, 0.0);
    for (int c = 0; c < ncls; ++c)
    {
        const int r = cls.rep[c];
        bnd[c] = in.boundary[r];
        const bool packed = cls.slots.empty();
        nsl[c] = packed ? cls.repNslot[c] : cls.nslot[r];
        double *o = &rep[13 * (size_t)c];
        for (int q = 0; q < 3; ++q) { o[q] = in.xyz[3 * (size_t)r + q]; o[3 + q] = in.meshv[3 * (size_t)r + q]; }
        for (int q = 0; q < 7; ++q) o[6 + q] = in.wall[7 * (size_t)r + q];
        const int *sl = packed ? &cls.repSlots[(size_t)c * S] : &cls.slots[(size_t)r * S];
        for (int s = 1; s < nsl[c]; ++s)
            for (int q = 0; q < 3; ++q) pos[((size_t)c * S + s) * 3 + q] = in.xyz[3 * (size_t)sl[s] + q];
    }
    ClassArgs a{};
    a.dim = in.dim; a.Nv = in.Nv; a.V = V; a.S = S; a.mlsOrder = order;
    a.dt = in.dt; a.h = in.h; a.vmin = in.vmin; a.dv = in.dv;
    for (int q = 0; q < 3; ++q) { a.periodic[q] = in.periodic[q] ? 1 : 0; a.L[q] = in.L[q]; }
    int *dBnd = nullptr, *dNsl = nullptr, *dDeg = nullptr;
    double *dRep = nullptr, *dPos = nullptr;
    auto freeAll = [&]() {
        for (void *p : {(void *)dBnd, (void *)dNsl, (void *)dDeg, (void *)dRep, (void *)dPos})
            if (p) cudaFree(p);
    };
    cudaError_t e = cudaMalloc(&dBnd, 4 * (size_t)ncls);
    if (e == cudaSuccess) e = cudaMalloc(&dNsl, 4 * (size_t)ncls);
    if (e == cudaSuccess) e = cudaMalloc(&dDeg, 4 * (size_t)ncls);
    if (e == cudaSuccess) e = cudaMalloc(&dRep, 8 * rep.size());
    if (e == cudaSuccess) e = cudaMalloc(&dPos, 8 * pos.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(dBnd, bnd.data(), 4 * (size_t)ncls, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dNsl, nsl.data(), 4 * (size_t)ncls, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dDeg, 0, 4 * (size_t)ncls, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dRep, rep.data(), 8 * rep.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dPos, pos.data(), 8 * pos.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(table, 0, (size_t)ncls * S * V * (f64 ? 8 : 4), st);
    if (e == cudaSuccess)
    {
        dim3 grid((V + 127) / 128, ncls);
        if (f64)
            k_class_tables<double><<<grid, 128, 0, st>>>(a, order, dBnd, dNsl, dRep, dPos,
                                                         static_cast<double *>(table), dDeg);
        else
            k_class_tables<float><<<grid, 128, 0, st>>>(a, order, dBnd, dNsl, dRep, dPos,
                                                        static_cast<float *>(table), dDeg);
        e = cudaGetLastError();
    }
    degenerate.assign(ncls, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(degenerate.data(), dDeg, 4 * (size_t)ncls, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    freeAll();
    return e;
}

}  // namespace alebgk
