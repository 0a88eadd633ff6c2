// march_plan.cpp -- lattice detection, canonical coefficient tables and work
// units for the marching transport (see march.h).
#include "march.h"

#include <algorithm>
#include <cmath>
#include <map>

namespace alebgk {

int templateIndex(int dx, int dy, int dz)
{
    int n = 0;
    for (int z = -2; z <= 2; ++z)
        for (int y = -2; y <= 2; ++y)
            for (int x = -2; x <= 2; ++x)
            {
                if (x * x + y * y + z * z > 6) continue;
                if (x == dx && y == dy && z == dz) return n;
                ++n;
            }
    return -1;
}

namespace {

// Cluster the values of one axis: returns the number of distinct values and
// each particle's rank among them (ascending).
int axisRanks(const double *xyz, int N, int axis, std::vector<int> &rank)
{
    std::vector<double> v(N);
    for (int i = 0; i < N; ++i) v[i] = xyz[3 * i + axis];
    std::vector<double> s(v);
    std::sort(s.begin(), s.end());
    const double span = s.back() - s.front();
    const double tol = 1e-9 * (span > 0 ? span : 1.0);
    std::vector<double> u;
    for (double x : s)
        if (u.empty() || x - u.back() > tol) u.push_back(x);
    rank.resize(N);
    for (int i = 0; i < N; ++i)
    {
        auto it = std::lower_bound(u.begin(), u.end(), v[i] - tol);
        rank[i] = (int)(it - u.begin());
    }
    return (int)u.size();
}

}  // namespace

void buildMarchPlan(const double *xyz, int N, int dim, const int *nnb, const int *nbr,
                    int maxNeigh, const CoeffTables &tb, const CoeffTables *tl,
                    MarchPlan &plan)
{
    plan = MarchPlan();
    if (dim != 3 || N < 8) return;
    std::vector<int> rx, ry, rz;
    const int nx = axisRanks(xyz, N, 0, rx);
    const int ny = axisRanks(xyz, N, 1, ry);
    const int nz = axisRanks(xyz, N, 2, rz);
    if ((long long)nx * ny * nz != N || nx < 2 || ny < 2 || nz < 2) return;
    // Generation order: x and y ascend; z ascends or descends (the reference
    // builds z from zfront with a negative spacing).
    const bool zdesc = rz[0] > rz[(size_t)nx * ny];
    for (int i = 0; i < N; ++i)
    {
        const int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
        const int ez = zdesc ? nz - 1 - iz : iz;
        if (rx[i] != ix || ry[i] != iy || rz[i] != ez) return;
    }
    // Lattice coordinates in index space: (ix, iy, iz) with i = ix + nx (iy + ny iz).
    auto coord = [&](int i, int &x, int &y, int &z) {
        x = i % nx; y = (i / nx) % ny; z = i / (nx * ny);
    };
    for (int i = 0; i < N; ++i)
    {
        int xi, yi, zi;
        coord(i, xi, yi, zi);
        for (int s = 0; s < nnb[i]; ++s)
        {
            int xj, yj, zj;
            coord(nbr[(size_t)i * maxNeigh + s], xj, yj, zj);
            if (templateIndex(xj - xi, yj - yi, zj - zi) < 0) return;
        }
    }

    // Canonical tables [class][81][Vpad].
    const int V = tb.V, ncls = tb.ncls, S = tb.S;
    const int Vpad = (V + kMarchChunk - 1) / kMarchChunk * kMarchChunk;
    plan.Nx = nx; plan.Ny = ny; plan.Nz = nz; plan.ncls = ncls; plan.Vpad = Vpad;
    plan.coefT.assign((size_t)ncls * kTmplOffsets * Vpad, 0.0f);
    if (tl) plan.coefTLin.assign((size_t)ncls * kTmplOffsets * Vpad, 0.0f);
    for (int c = 0; c < ncls; ++c)
    {
        const int r = tb.rep[c];
        int xr, yr, zr;
        coord(r, xr, yr, zr);
        const int *sl = &tb.slots[(size_t)r * S];
        for (int s = 0; s < tb.nslot[r]; ++s)
        {
            int xj, yj, zj;
            coord(sl[s], xj, yj, zj);
            const int o = templateIndex(xj - xr, yj - yr, zj - zr);
            const double *src = &tb.coef[((size_t)c * S + s) * V];
            float *dst = &plan.coefT[((size_t)c * kTmplOffsets + o) * Vpad];
            for (int k = 0; k < V; ++k) dst[k] = (float)src[k];
            if (tl)
            {
                const double *sl2 = &tl->coef[((size_t)c * S + s) * V];
                float *d2 = &plan.coefTLin[((size_t)c * kTmplOffsets + o) * Vpad];
                for (int k = 0; k < V; ++k) d2[k] = (float)sl2[k];
            }
        }
    }

    // z-segments: output planes between which no column changes class.
    auto cls = [&](int x, int y, int z) { return tb.cls[x + nx * (y + (size_t)ny * z)]; };
    std::vector<int> cuts = {0};
    for (int z = 1; z < nz; ++z)
    {
        bool change = false;
        for (int y = 0; y < ny && !change; ++y)
            for (int x = 0; x < nx && !change; ++x)
                change = cls(x, y, z) != cls(x, y, z - 1);
        if (change) cuts.push_back(z);
    }
    cuts.push_back(nz);

    // Work units: per segment and 8x4 column tile, the tile's columns are
    // covered by class-uniform warp blocks: whole 2x2 blocks first, then
    // 1x4 strips along y (one column x), then 4x1 strips along x, and what
    // is left by 2x2 blocks split per class (masked).  The strips cover the
    // columns next to the tile's x and y walls, whose classes change from
    // column to column.  At most kMarchWarps blocks per unit.
    for (size_t sgi = 0; sgi + 1 < cuts.size(); ++sgi)
    {
        const int za = cuts[sgi], zb = cuts[sgi + 1];
        for (int y0 = 0; y0 < ny; y0 += kMarchTileY)
            for (int x0 = 0; x0 < nx; x0 += kMarchTileX)
            {
                // class of tile column (bx, by), or -1 outside the lattice
                int tc[kMarchTileY][kMarchTileX];
                for (int by = 0; by < kMarchTileY; ++by)
                    for (int bx = 0; bx < kMarchTileX; ++bx)
                    {
                        const int x = x0 + bx, y = y0 + by;
                        tc[by][bx] = (x < nx && y < ny) ? cls(x, y, za) : -1;
                    }
                std::vector<int> subs;
                auto take = [&](int bx, int by, int shape, const int (&cx)[4],
                                const int (&cy)[4]) {
                    const int k = tc[by + cy[0]][bx + cx[0]];
                    if (k < 0) return;
                    for (int q = 1; q < 4; ++q)
                        if (tc[by + cy[q]][bx + cx[q]] != k) return;
                    for (int q = 0; q < 4; ++q) tc[by + cy[q]][bx + cx[q]] = -1;
                    subs.push_back(bx | by << 4 | 15 << 8 | shape << 12 | k << 14);
                };
                const int bX[4] = {0, 1, 0, 1}, bY[4] = {0, 0, 1, 1};     // 2x2
                const int vX[4] = {0, 0, 0, 0}, vY[4] = {0, 1, 2, 3};     // 1x4
                const int hX[4] = {0, 1, 2, 3}, hY[4] = {0, 0, 0, 0};     // 4x1
                for (int by = 0; by < kMarchTileY; by += 2)
                    for (int bx = 0; bx < kMarchTileX; bx += 2) take(bx, by, kShapeBlock, bX, bY);
                for (int bx = 0; bx < kMarchTileX; ++bx) take(bx, 0, kShapeColumn, vX, vY);
                for (int by = 0; by < kMarchTileY; ++by)
                    for (int bx = 0; bx < kMarchTileX; bx += 4) take(bx, by, kShapeRow, hX, hY);
                for (int by = 0; by < kMarchTileY; by += 2)
                    for (int bx = 0; bx < kMarchTileX; bx += 2)
                    {
                        std::map<int, int> masks;   // class -> column mask
                        for (int q = 0; q < 4; ++q)
                        {
                            const int k = tc[by + (q >> 1)][bx + (q & 1)];
                            if (k >= 0) masks[k] |= 1 << q;
                        }
                        for (auto &m : masks)
                            subs.push_back(bx | by << 4 | m.second << 8 | kShapeBlock << 12 |
                                           m.first << 14);
                    }
                for (size_t a = 0; a < subs.size(); a += kMarchWarps)
                {
                    MarchUnit u{};
                    u.x0 = x0; u.y0 = y0; u.za = za; u.zb = zb;
                    u.nsub = (int)std::min<size_t>(kMarchWarps, subs.size() - a);
                    for (int w = 0; w < u.nsub; ++w) u.sub[w] = subs[a + w];
                    plan.units.push_back(u);
                }
            }
    }
    plan.ok = ncls < (1 << 17);
}

}  // namespace alebgk
