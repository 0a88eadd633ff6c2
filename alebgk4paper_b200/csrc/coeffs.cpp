// coeffs.cpp -- FP64 MLS stencil classes and transport coefficients.
#include "coeffs.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <unordered_map>

namespace alebgk {

int solveSkipGE(double *A, double *B, int n, int nrhs)
{
    // Forward elimination with partial pivoting; a pivot below 1e-30 leaves
    // its column un-eliminated (MLSTransport.cpp:29-54).
    int skipped = 0;
    for (int col = 0; col < n; ++col)
    {
        int piv = col;
        double mx = std::fabs(A[col * n + col]);
        for (int row = col + 1; row < n; ++row)
            if (std::fabs(A[row * n + col]) > mx)
            {
                mx = std::fabs(A[row * n + col]);
                piv = row;
            }
        if (piv != col)
        {
            for (int j = 0; j < n; ++j) std::swap(A[col * n + j], A[piv * n + j]);
            for (int j = 0; j < nrhs; ++j) std::swap(B[col * nrhs + j], B[piv * nrhs + j]);
        }
        double d = A[col * n + col];
        if (std::fabs(d) < 1.0e-30) { ++skipped; continue; }
        for (int row = col + 1; row < n; ++row)
        {
            double f = A[row * n + col] / d;
            for (int j = col; j < n; ++j) A[row * n + j] -= f * A[col * n + j];
            for (int j = 0; j < nrhs; ++j) B[row * nrhs + j] -= f * B[col * nrhs + j];
        }
    }
    // Back substitution; an unknown whose pivot is not above 1e-30 is 0
    // (MLSTransport.cpp:56-61).
    for (int i = n - 1; i >= 0; --i)
    {
        bool ok = std::fabs(A[i * n + i]) > 1.0e-30;
        for (int r = 0; r < nrhs; ++r)
        {
            double s = B[i * nrhs + r];
            for (int j = i + 1; j < n; ++j) s -= A[i * n + j] * B[j * nrhs + r];
            B[i * nrhs + r] = ok ? s / A[i * n + i] : 0.0;
        }
    }
    return skipped;
}

namespace {

// Core/MLSBasis.hpp:46-49
inline double minImage(double d, double L) { return d - L * std::round(d / L); }

// Core/MLSBasis.hpp:142-148
inline double weightSq(double r2, double h)
{
    double q2 = r2 / (h * h);
    if (q2 >= 1.0) return 0.0;
    double w = 1.0 - q2;
    return w * w;
}

// Core/MLSBasis.hpp:158-202 -- basis ordering [1,sx,sy,(sz),quadratic...]
inline int basis(double dx, double dy, double dz, int ndim, double h,
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

struct KeyHash
{
    size_t operator()(const int64_t *v, size_t n) const
    {
        uint64_t h = 1469598103934665603ULL;
        for (size_t q = 0; q < n; ++q)
        {
            h ^= (uint64_t)v[q] + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2);
            h *= 1099511628211ULL;
        }
        return (size_t)h;
    }
};

inline int64_t bitsOf(double d)
{
    int64_t b;
    std::memcpy(&b, &d, sizeof b);
    return b;
}

}  // namespace

bool buildClasses(const CoeffInput &in, CoeffTables &out, std::string *err)
{
    const int N = in.N, ndim = in.dim, Nv = in.Nv;
    if (N <= 0 || Nv < 2 || (ndim != 2 && ndim != 3) || in.h <= 0)
    {
        if (err) *err = "buildCoefficients: bad sizes";
        return false;
    }
    const int V = (ndim == 3) ? Nv * Nv * Nv : Nv * Nv;
    int maxnn = 0;
    for (int i = 0; i < N; ++i)
    {
        if (in.nnb[i] < 0 || in.nnb[i] > in.maxNeigh)
        {
            if (err) *err = "buildCoefficients: neighbour count out of range";
            return false;
        }
        maxnn = std::max(maxnn, in.nnb[i]);
    }
    const int S = 1 + maxnn;
    out = CoeffTables();
    out.S = S; out.V = V;
    out.cls.assign(N, 0);
    out.nslot.assign(N, 0);
    out.slots.assign((size_t)N * S, 0);

    // Displacements are quantised on a grid of h * 2^-32, far below any
    // geometric difference between distinct stencils and far above the
    // rounding of x_j - x_i, so translated copies of a stencil compare equal.
    const double q = in.h * std::ldexp(1.0, -32);
    // Every particle's key (boundary flag, order, count, mesh velocity bits,
    // wall bits for wall particles, quantised sorted displacements) in one
    // flat array; keys are hashed in parallel and compared in full on a hash
    // hit.
    std::vector<size_t> koff((size_t)N + 1, 0);
    for (int i = 0; i < N; ++i)
        koff[i + 1] = koff[i] + 6 + (in.boundary[i] ? 7 : 0) + 3 * (size_t)in.nnb[i];
    // (uninitialised: every entry is written below, in parallel)
    std::unique_ptr<int64_t[]> keys(new int64_t[std::max<size_t>(koff[N], 1)]);
    std::vector<uint64_t> hashes(N);
#pragma omp parallel
    {
        std::vector<std::pair<std::array<int64_t, 3>, int>> nb(std::max(maxnn, 1));
#pragma omp for schedule(static)
        for (int i = 0; i < N; ++i)
        {
            const int nn = in.nnb[i];
            for (int s = 0; s < nn; ++s)
            {
                int j = in.nbr[(size_t)i * in.maxNeigh + s];
                double d[3];
                for (int a = 0; a < 3; ++a)
                {
                    d[a] = (a < ndim) ? in.xyz[3 * j + a] - in.xyz[3 * i + a] : 0.0;
                    if (a < ndim && in.periodic[a]) d[a] = minImage(d[a], in.L[a]);
                }
                nb[s].first = {std::llround(d[2] / q), std::llround(d[1] / q),
                               std::llround(d[0] / q)};
                nb[s].second = j;
            }
            std::sort(nb.begin(), nb.begin() + nn);
            int *sl = &out.slots[(size_t)i * S];
            sl[0] = i;
            for (int s = 0; s < nn; ++s) sl[1 + s] = nb[s].second;
            for (int s = 1 + nn; s < S; ++s) sl[s] = i;   // padding, coefficient 0
            out.nslot[i] = 1 + nn;
            int64_t *k = &keys[koff[i]];
            size_t w = 0;
            const int order = in.boundary[i] ? 1 : in.mlsOrder;
            k[w++] = in.boundary[i];
            k[w++] = order;
            k[w++] = nn;
            for (int a = 0; a < 3; ++a) k[w++] = bitsOf(in.meshv[3 * i + a]);
            if (in.boundary[i])
                for (int a = 0; a < 7; ++a) k[w++] = bitsOf(in.wall[7 * i + a]);
            for (int s = 0; s < nn; ++s)
                for (int a = 0; a < 3; ++a) k[w++] = nb[s].first[a];
            hashes[i] = KeyHash()(k, w);
        }
    }
    // Class ids in order of first appearance.
    auto sameKey = [&](int x, int y) {
        const size_t lx = koff[x + 1] - koff[x], ly = koff[y + 1] - koff[y];
        return lx == ly && std::memcmp(&keys[koff[x]], &keys[koff[y]], lx * 8) == 0;
    };
    std::unordered_map<uint64_t, std::vector<int>> byHash;
    byHash.reserve(1024);
    for (int i = 0; i < N; ++i)
    {
        std::vector<int> &cand = byHash[hashes[i]];
        int id = -1;
        for (int c : cand)
            if (sameKey(out.rep[c], i)) { id = c; break; }
        if (id < 0)
        {
            id = (int)out.rep.size();
            cand.push_back(id);
            out.rep.push_back(i);
        }
        out.cls[i] = id;
    }
    const int ncls = (int)out.rep.size();
    out.ncls = ncls;
    out.degenerate.assign(ncls, 0);
    out.order.assign(ncls, 0);
    out.members.assign(ncls, 0);
    for (int i = 0; i < N; ++i) out.members[out.cls[i]]++;
    for (int c = 0; c < ncls; ++c) out.order[c] = in.boundary[out.rep[c]] ? 1 : in.mlsOrder;
    return true;
}

bool buildCoefficients(const CoeffInput &in, CoeffTables &out, std::string *err)
{
    if (!buildClasses(in, out, err)) return false;
    const int N = in.N, ndim = in.dim, Nv = in.Nv;
    (void)N;
    const int V = out.V, S = out.S, ncls = out.ncls;
    out.coef.assign((size_t)ncls * S * V, 0.0);
#pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < ncls; ++c)
    {
        const int r = out.rep[c];
        const int order = in.boundary[r] ? 1 : in.mlsOrder;
        out.order[c] = order;
        const int nsl = out.nslot[r];
        const int *sl = &out.slots[(size_t)r * S];
        const double xr = in.xyz[3 * r], yr = in.xyz[3 * r + 1], zr = in.xyz[3 * r + 2];
        const double *mv = &in.meshv[3 * r];
        const double *wl = &in.wall[7 * r];
        double *cc = &out.coef[(size_t)c * S * V];
        std::vector<double> w(nsl), bas((size_t)nsl * 10);
        int degen = 0;
        for (int k = 0; k < V; ++k)
        {
            int iv = k % Nv, jv = (k / Nv) % Nv, kv = (ndim == 3) ? k / (Nv * Nv) : 0;
            double vx = std::fma((double)iv, in.dv, in.vmin);
            double vy = std::fma((double)jv, in.dv, in.vmin);
            double vz = std::fma((double)kv, in.dv, in.vmin);
            if (in.boundary[r])
            {
                // Wall particles transport incoming nodes only
                // (MLSTransport.cpp:144-150 in 3-D, 213-218 with wallCN in 2-D).
                // cn is evaluated in the FMA-contracted form the reference's
                // -O3 -march=native build uses, which decides the exact ties
                // cn = 0 of edge and corner particles.
                double a = vx - wl[3], b = vy - wl[4];
                double cn = (ndim == 3) ? std::fma(vz - wl[5], wl[2], std::fma(a, wl[0], b * wl[1]))
                                        : std::fma(a, wl[0], b * wl[1]);
                if (cn >= 0.0) { cc[k] = 1.0; continue; }
            }
            double xf = xr - (vx - mv[0]) * in.dt;
            double yf = yr - (vy - mv[1]) * in.dt;
            double zf = zr - (vz - mv[2]) * in.dt;
            int P = 0;
            double A[100] = {0};
            bool any = false;
            for (int s = 1; s < nsl; ++s)
            {
                int j = sl[s];
                double dx = in.xyz[3 * j] - xf;
                double dy = in.xyz[3 * j + 1] - yf;
                double dz = (ndim == 3) ? in.xyz[3 * j + 2] - zf : 0.0;
                if (in.periodic[0]) dx = minImage(dx, in.L[0]);
                if (in.periodic[1]) dy = minImage(dy, in.L[1]);
                if (ndim == 3 && in.periodic[2]) dz = minImage(dz, in.L[2]);
                double r2 = dx * dx + dy * dy + dz * dz;
                double ws = weightSq(r2, in.h);
                if (ws < 1.0e-30) { w[s] = 0.0; continue; }
                w[s] = ws;
                double *b = &bas[(size_t)s * 10];
                P = basis(dx, dy, dz, ndim, in.h, b, order);
                for (int p1 = 0; p1 < P; ++p1)
                    for (int p2 = 0; p2 < P; ++p2) A[p1 * P + p2] += ws * b[p1] * b[p2];
                any = true;
            }
            if (!any) { cc[k] = 1.0; continue; }   // no neighbour: keep old g
            // Row 0 of the elimination's linear map: solve with unit
            // right-hand sides, sol_m[0] = l0[m].
            double B[100] = {0};
            for (int m = 0; m < P; ++m) B[m * P + m] = 1.0;
            if (solveSkipGE(A, B, P, P) > 0) ++degen;
            for (int s = 1; s < nsl; ++s)
            {
                if (w[s] == 0.0) continue;
                const double *b = &bas[(size_t)s * 10];
                double acc = 0.0;
                for (int m = 0; m < P; ++m) acc += B[m] * b[m];
                cc[(size_t)s * V + k] = w[s] * acc;
            }
        }
        out.degenerate[c] = degen;
    }
    return true;
}

void roundCoefFP32(const double *src, float *dst, int S, int V)
{
    for (int k = 0; k < V; ++k)
    {
        double s64 = 0.0, s32 = 0.0, big = -1.0;
        int smax = 0;
        for (int s = 0; s < S; ++s)
        {
            const double c = src[(size_t)s * V + k];
            const float c32 = (float)c;
            dst[(size_t)s * V + k] = c32;
            s64 += c;
            s32 += (double)c32;
            if (std::fabs(c) > big) { big = std::fabs(c); smax = s; }
        }
        const size_t q = (size_t)smax * V + k;
        dst[q] = (float)((double)dst[q] + (s64 - s32));
    }
}

}  // namespace alebgk
