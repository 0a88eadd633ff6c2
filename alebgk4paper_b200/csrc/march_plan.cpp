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

bool marchEligible(const double *xyz, int N, int dim, const int *nnb, const int *nbr,
                   int maxNeigh)
{
    if (dim != 3 || N < 8) return false;
    std::vector<int> rx, ry, rz;
    const int nx = axisRanks(xyz, N, 0, rx);
    const int ny = axisRanks(xyz, N, 1, ry);
    const int nz = axisRanks(xyz, N, 2, rz);
    if ((long long)nx * ny * nz != N || nx < 2 || ny < 2 || nz < 2) return false;
    const bool zdesc = rz[0] > rz[(size_t)nx * ny];
    for (int i = 0; i < N; ++i)
    {
        const int ix = i % nx, iy = (i / nx) % ny, iz = i / (nx * ny);
        const int ez = zdesc ? nz - 1 - iz : iz;
        if (rx[i] != ix || ry[i] != iy || rz[i] != ez) return false;
    }
    for (int i = 0; i < N; ++i)
    {
        const int xi = i % nx, yi = (i / nx) % ny, zi = i / (nx * ny);
        for (int s = 0; s < nnb[i]; ++s)
        {
            const int j = nbr[(size_t)i * maxNeigh + s];
            if (templateIndex(j % nx - xi, (j / nx) % ny - yi, j / (nx * ny) - zi) < 0)
                return false;
        }
    }
    return true;
}

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
    // Rows padded to whole chunks of the widest march (two velocities per lane).
    const int Vpad = (V + 2 * kMarchChunk - 1) / (2 * kMarchChunk) * (2 * kMarchChunk);
    plan.Nx = nx; plan.Ny = ny; plan.Nz = nz; plan.ncls = ncls; plan.Vpad = Vpad;
    plan.coefT.assign((size_t)ncls * kTmplOffsets * Vpad, 0.0f);
    if (tl) plan.coefTLin.assign((size_t)ncls * kTmplOffsets * Vpad, 0.0f);
    // FP32 images of the class tables (roundCoefFP32), re-laid by offset.
    std::vector<float> img((size_t)S * V), imgLin(tl ? (size_t)S * V : 0);
    for (int c = 0; c < ncls; ++c)
    {
        const int r = tb.rep[c];
        int xr, yr, zr;
        coord(r, xr, yr, zr);
        const int *sl = &tb.slots[(size_t)r * S];
        roundCoefFP32(&tb.coef[(size_t)c * S * V], img.data(), S, V);
        if (tl) roundCoefFP32(&tl->coef[(size_t)c * S * V], imgLin.data(), S, V);
        for (int s = 0; s < tb.nslot[r]; ++s)
        {
            int xj, yj, zj;
            coord(sl[s], xj, yj, zj);
            const int o = templateIndex(xj - xr, yj - yr, zj - zr);
            const float *src = &img[(size_t)s * V];
            float *dst = &plan.coefT[((size_t)c * kTmplOffsets + o) * Vpad];
            for (int k = 0; k < V; ++k) dst[k] = src[k];
            if (tl)
            {
                const float *sl2 = &imgLin[(size_t)s * V];
                float *d2 = &plan.coefTLin[((size_t)c * kTmplOffsets + o) * Vpad];
                for (int k = 0; k < V; ++k) d2[k] = sl2[k];
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

    // A z-segment shorter than kThinSegment (the wall layers next to the z
    // walls) is marched along y instead where it can be: within such a
    // plane the column classes stay constant along y except next to the y
    // walls, so the plane's lines along y form long segments.  y-segments
    // are cut where any column (x, z) of a thin plane changes class.
    std::vector<char> thin(nz, 0);
    for (size_t sgi = 0; sgi + 1 < cuts.size(); ++sgi)
        if (cuts[sgi + 1] - cuts[sgi] < kThinSegment)
            for (int z = cuts[sgi]; z < cuts[sgi + 1]; ++z) thin[z] = 1;
    std::vector<int> ycuts = {0};
    for (int y = 1; y < ny; ++y)
    {
        bool change = false;
        for (int z = 0; z < nz && !change; ++z)
            for (int x = 0; x < nx && !change && thin[z]; ++x)
                change = cls(x, y, z) != cls(x, y - 1, z);
        if (change) ycuts.push_back(y);
    }
    ycuts.push_back(ny);
    std::vector<char> yLong(ny, 0);      // y lies in a long y-segment
    for (size_t s = 0; s + 1 < ycuts.size(); ++s)
        if (ycuts[s + 1] - ycuts[s] >= kThinSegment)
            for (int y = ycuts[s]; y < ycuts[s + 1]; ++y) yLong[y] = 1;

    // Covers the columns of one tile (class of column (bx, by) in tc, -1 if
    // not the unit's) by class-uniform warp blocks: whole 2x2 blocks first,
    // then 1x4 strips along the tile's y, then 4x1 strips along its x, and
    // what is left by 2x2 blocks split per class (masked).  The strips cover
    // the columns next to walls, whose classes change from column to column.
    auto coverTile = [&](int (&tc)[kMarchTileY][kMarchTileX], std::vector<int> &subs) {
        auto take = [&](int bx, int by, int shape, const int (&cx)[4], const int (&cy)[4]) {
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
    };
    auto emit = [&](std::vector<MarchUnit> &out, int x0, int y0, int za, int zb,
                    const std::vector<int> &subs) {
        for (size_t a = 0; a < subs.size(); a += kMarchWarps)
        {
            MarchUnit u{};
            u.x0 = x0; u.y0 = y0; u.za = za; u.zb = zb;
            u.yMarch = (&out == &plan.unitsY) ? 1 : 0;
            u.nsub = (int)std::min<size_t>(kMarchWarps, subs.size() - a);
            for (int w = 0; w < u.nsub; ++w) u.sub[w] = subs[a + w];
            out.push_back(u);
        }
    };

    // z-march units: every long z-segment; in thin planes only the columns
    // whose y is next to a y wall (the rest go to the y-march).
    for (size_t sgi = 0; sgi + 1 < cuts.size(); ++sgi)
    {
        const int za = cuts[sgi], zb = cuts[sgi + 1];
        const bool isThin = zb - za < kThinSegment;
        for (int y0 = 0; y0 < ny; y0 += kMarchTileY)
            for (int x0 = 0; x0 < nx; x0 += kMarchTileX)
            {
                int tc[kMarchTileY][kMarchTileX];
                for (int by = 0; by < kMarchTileY; ++by)
                    for (int bx = 0; bx < kMarchTileX; ++bx)
                    {
                        const int x = x0 + bx, y = y0 + by;
                        tc[by][bx] = (x < nx && y < ny && !(isThin && yLong[y]))
                                         ? cls(x, y, za) : -1;
                    }
                std::vector<int> subs;
                coverTile(tc, subs);
                emit(plan.units, x0, y0, za, zb, subs);
            }
    }
    // y-march units: the thin planes' columns along long y-segments.  In the
    // y-march frame a unit's tile spans lattice x (8) and lattice z (4) and
    // marches through lattice y; only the thin planes' rows are outputs.
    for (size_t s = 0; s + 1 < ycuts.size(); ++s)
    {
        const int ya = ycuts[s], yb = ycuts[s + 1];
        if (yb - ya < kThinSegment) continue;
        for (int z0 = 0; z0 < nz; z0 += kMarchTileY)
            for (int x0 = 0; x0 < nx; x0 += kMarchTileX)
            {
                int tc[kMarchTileY][kMarchTileX];
                bool any = false;
                for (int bz = 0; bz < kMarchTileY; ++bz)
                    for (int bx = 0; bx < kMarchTileX; ++bx)
                    {
                        const int x = x0 + bx, z = z0 + bz;
                        const bool out = x < nx && z < nz && thin[z];
                        tc[bz][bx] = out ? cls(x, ya, z) : -1;
                        any = any || out;
                    }
                if (!any) continue;
                std::vector<int> subs;
                coverTile(tc, subs);
                emit(plan.unitsY, x0, z0, ya, yb, subs);
            }
    }
    // Coefficients in the y-march frame (x, lattice z, lattice y): the
    // kernel's offset (ox, oy, oz) is the lattice offset (ox, oz, oy).
    if (!plan.unitsY.empty())
    {
        plan.coefTy.assign(plan.coefT.size(), 0.0f);
        for (int c = 0; c < ncls; ++c)
            for (int oz = -2; oz <= 2; ++oz)
                for (int oy = -2; oy <= 2; ++oy)
                    for (int ox = -2; ox <= 2; ++ox)
                    {
                        const int tk = templateIndex(ox, oy, oz);
                        if (tk < 0) continue;
                        const int tl = templateIndex(ox, oz, oy);
                        std::copy_n(&plan.coefT[((size_t)c * kTmplOffsets + tl) * Vpad], Vpad,
                                    &plan.coefTy[((size_t)c * kTmplOffsets + tk) * Vpad]);
                    }
    }
    plan.ok = ncls < (1 << 17);
}

}  // namespace alebgk
