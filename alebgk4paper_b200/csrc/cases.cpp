// cases.cpp -- host-side case set-up (see cases.h).
//
// Each function restates one piece of the reference's set-up so that the
// cloud built here is the cloud the reference builds for the same case:
// same particle order, positions, wall flags, wall state, neighbour sets and
// initial distribution.  The reference is built with -march=native, and GCC
// contracts a*b + c into one rounding (an FMA) on any FMA-capable x86-64;
// the expressions below spell those contractions out with std::fma so that
// positions, voxel bins (floor at exact multiples of the box size) and hence
// neighbour order come out bitwise identical to the reference's build.
#include "cases.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace alebgk {

namespace {

constexpr double kPi = 3.14159265358979323846;

// TestCases/TestCases.cpp:24-54 -- per-family constants.
constexpr double kUniformLid = 1.0, kParabolicPeak = 10.0;
constexpr double kWallTemp = 270.0, kHSDiam = 0.368e-9;
constexpr double kBodyDensityRatio = 10.0;
constexpr double kSquareSide = 7.5e-8, kCircleRadius = kSquareSide / 2.0;
constexpr double kCubeSide = 1.5e-7, kSphereRadius = kCubeSide / 2.0;
constexpr int kSquarePts = 16, kCirclePts = 32, kSpherePts = 48, kCubePts = 96;

struct CaseRow
{
    const char *name;
    int dim;
    bool hasBody;
    int lidKind;        // 0 UniformTop, 1 UniformFront, 2 ParabolicTop
    double lidSpeed;
};

// TestCases/TestCases.cpp:56-75
const CaseRow kCases[6] = {
    {"cavity2d", 2, false, 0, kUniformLid},
    {"cavity3d", 3, false, 1, kUniformLid},
    {"cavity2d-square", 2, true, 2, kParabolicPeak},
    {"cavity2d-circle", 2, true, 2, kParabolicPeak},
    {"cavity3d-sphere", 3, true, 2, kParabolicPeak},
    {"cavity3d-cube", 3, true, 2, kParabolicPeak},
};

}  // namespace

// Core/MLSBasis.hpp:112-122 (3-D Maxwellian, Theta = 2RT)
double maxwellian3(double vx, double vy, double vz, double ux, double uy,
                   double uz, double T, double rho, double R)
{
    double twoRT = 2.0 * R * T;
    double ax = vx - ux, ay = vy - uy, az = vz - uz;
    double e = -std::fma(az, az, std::fma(ax, ax, ay * ay)) / twoRT;
    double norm = std::pow(kPi * twoRT, 1.5);
    return rho / norm * std::exp(e);
}

// Core/MLSBasis.hpp:87-94 (Chu-reduced G1)
double maxwellianG1(double vx, double vy, double ux, double uy, double T,
                    double rho, double R)
{
    double twoRT = 2.0 * R * T;
    double ax = vx - ux, ay = vy - uy;
    double e = -std::fma(ax, ax, ay * ay) / twoRT;
    return rho / (kPi * twoRT) * std::exp(e);
}


// ---------------------------------------------------------------------------
// Bodies: RigidBody/Geometry.hpp:84-362
// ---------------------------------------------------------------------------
double Body::inertia() const
{
    switch (kind)
    {
    case 0: return mass * size * size / 6.0;          // Geometry.hpp:158
    case 1: return mass * size * size / 2.0;          // Geometry.hpp:222
    case 2: return 0.4 * mass * size * size;          // Geometry.hpp:98
    default: return mass * size * size / 6.0;         // Geometry.hpp:272
    }
}

double Body::surfaceArea() const
{
    switch (kind)
    {
    case 0: return 4.0 * size / npts;                 // Geometry.hpp:159
    case 1: return 2.0 * kPi * size / npts;           // Geometry.hpp:223
    case 2: return 4.0 * kPi * size * size / npts;    // Geometry.hpp:99
    default: return 6.0 * size * size / npts;         // Geometry.hpp:273
    }
}

bool Body::inside(double x, double y, double z) const
{
    switch (kind)
    {
    case 0:
    {   // Geometry.hpp:179-186
        double xC = x - cx, yC = y - cy;
        double D = ox * ox + oy * oy;
        double xp = (ox * xC + oy * yC) / D;
        double yp = (oy * xC - ox * yC) / D;
        return (std::fabs(xp) <= size / 2) && (std::fabs(yp) <= size / 2);
    }
    case 1:
    {   // Geometry.hpp:233-237
        double dx = x - cx, dy = y - cy;
        return std::fma(dx, dx, dy * dy) <= size * size;
    }
    case 2:
    {   // Geometry.hpp:105-109
        double dx = x - cx, dy = y - cy, dz = z - cz;
        return std::fma(dz, dz, std::fma(dx, dx, dy * dy)) <= size * size;
    }
    default:
    {   // Geometry.hpp:275-293 (R^T applied to the offset)
        double dx = x - cx, dy = y - cy, dz = z - cz;
        double bx = std::fma(Rm[6], dz, std::fma(Rm[0], dx, Rm[3] * dy));
        double by = std::fma(Rm[7], dz, std::fma(Rm[1], dx, Rm[4] * dy));
        double bz = std::fma(Rm[8], dz, std::fma(Rm[2], dx, Rm[5] * dy));
        return std::fabs(bx) <= size / 2 && std::fabs(by) <= size / 2 &&
               std::fabs(bz) <= size / 2;
    }
    }
}

void Body::normal(double x, double y, double z, double *nx, double *ny,
                  double *nz) const
{
    switch (kind)
    {
    case 0:
    {   // Geometry.hpp:161-177: side whose outward normal is closest
        double xp = x - cx, yp = y - cy;
        double n = std::sqrt(std::fma(xp, xp, yp * yp));
        double d1 = std::fma(xp, ox, yp * oy), d2 = std::fma(xp, oy, -(yp * ox));
        double dots[4][3] = {
            {d1 / n, ox, oy},
            {-d1 / n, -ox, -oy},
            {d2 / n, oy, -ox},
            {-d2 / n, -oy, ox},
        };
        int best = 0;
        for (int i = 1; i < 4; ++i)
            if (dots[i][0] > dots[best][0]) best = i;
        *nx = dots[best][1]; *ny = dots[best][2]; *nz = 0.0;
        return;
    }
    case 1:
    {   // Geometry.hpp:225-231
        double dx = x - cx, dy = y - cy;
        double n = std::sqrt(std::fma(dx, dx, dy * dy));
        *nx = dx / n; *ny = dy / n; *nz = 0.0;
        return;
    }
    case 2:
    {   // Geometry.hpp:117-123
        double dx = x - cx, dy = y - cy, dz = z - cz;
        double n = std::sqrt(std::fma(dz, dz, std::fma(dx, dx, dy * dy)));
        *nx = dx / n; *ny = dy / n; *nz = dz / n;
        return;
    }
    default:
    {   // Geometry.hpp:298-309: dominant body-frame axis, column of Rm
        double dx = x - cx, dy = y - cy, dz = z - cz;
        double b[3] = {std::fma(Rm[6], dz, std::fma(Rm[0], dx, Rm[3] * dy)),
                       std::fma(Rm[7], dz, std::fma(Rm[1], dx, Rm[4] * dy)),
                       std::fma(Rm[8], dz, std::fma(Rm[2], dx, Rm[5] * dy))};
        int f = 0;
        for (int i = 1; i < 3; ++i)
            if (std::fabs(b[i]) > std::fabs(b[f])) f = i;
        double s = (b[f] >= 0.0) ? 1.0 : -1.0;
        *nx = s * Rm[0 + f]; *ny = s * Rm[3 + f]; *nz = s * Rm[6 + f];
        return;
    }
    }
}

void Body::surfacePoints(std::vector<double> &v) const
{
    switch (kind)
    {
    case 0:
    {   // Geometry.hpp:188-211
        double t = std::atan2(oy, ox);
        double c = std::cos(t), s = std::sin(t);
        int nSide = npts / 4;
        double dl = size / nSide;
        double tlx = cx + size * (c - s) / 2, tly = cy + size * (s + c) / 2;
        double brx = cx + size * (s - c) / 2, bry = cy - size * (s + c) / 2;
        for (int i = 0; i < nSide; ++i)
            v.insert(v.end(), {std::fma(dl * (i + 0.5), c, brx),
                               std::fma(dl * (i + 0.5), s, bry), 0.0});
        for (int i = 0; i < nSide; ++i)
            v.insert(v.end(), {std::fma(-(dl * (i + 0.5)), c, tlx),
                               std::fma(-(dl * (i + 0.5)), s, tly), 0.0});
        for (int i = 0; i < nSide; ++i)
            v.insert(v.end(), {std::fma(-(dl * (i + 0.5)), s, brx),
                               std::fma(dl * (i + 0.5), c, bry), 0.0});
        for (int i = 0; i < nSide; ++i)
            v.insert(v.end(), {std::fma(dl * (i + 0.5), s, tlx),
                               std::fma(-(dl * (i + 0.5)), c, tly), 0.0});
        return;
    }
    case 1:
    {   // Geometry.hpp:239-246
        double dth = 2.0 * kPi / npts;
        for (int i = 0; i < npts; ++i)
            v.insert(v.end(), {std::fma(size, std::cos(i * dth), cx),
                               std::fma(size, std::sin(i * dth), cy), 0.0});
        return;
    }
    case 2:
    {   // Geometry.hpp:129-143: Fibonacci lattice
        const double ga = kPi * (3.0 - std::sqrt(5.0));
        for (int i = 0; i < npts; ++i)
        {
            double zf = 1.0 - 2.0 * (i + 0.5) / npts;
            double rf = std::sqrt(std::fma(-zf, zf, 1.0));
            double th = ga * i;
            v.insert(v.end(), {std::fma(size * rf, std::cos(th), cx),
                               std::fma(size * rf, std::sin(th), cy),
                               std::fma(size, zf, cz)});
        }
        return;
    }
    default:
    {   // Geometry.hpp:315-333: n x n points per face
        int n = std::max(1, (int)std::lround(std::sqrt(npts / 6.0)));
        double dl = size / n;
        for (int f = 0; f < 3; ++f)
            for (int sgn = -1; sgn <= 1; sgn += 2)
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j)
                    {
                        double b[3];
                        b[f] = sgn * size / 2.0;
                        b[(f + 1) % 3] = std::fma(i + 0.5, dl, -(size / 2.0));
                        b[(f + 2) % 3] = std::fma(j + 0.5, dl, -(size / 2.0));
                        v.insert(v.end(),
                                 {std::fma(Rm[2], b[2], std::fma(Rm[1], b[1], std::fma(Rm[0], b[0], cx))),
                                  std::fma(Rm[5], b[2], std::fma(Rm[4], b[1], std::fma(Rm[3], b[0], cy))),
                                  std::fma(Rm[8], b[2], std::fma(Rm[7], b[1], std::fma(Rm[6], b[0], cz)))});
                    }
        return;
    }
    }
}

// Geometry.hpp:335-361: Rodrigues increment, then Gram-Schmidt on the rows.
void Body::rotate3(double wx, double wy, double wz, double dt)
{
    if (kind != 3) return;
    double w = std::sqrt(wx * wx + wy * wy + wz * wz);
    if (w < 1e-300) return;
    double ax = wx / w, ay = wy / w, az = wz / w;
    double th = w * dt, c = std::cos(th), s = std::sin(th), C = 1.0 - c;
    double D[9] = {c + ax * ax * C, ax * ay * C - az * s, ax * az * C + ay * s,
                   ay * ax * C + az * s, c + ay * ay * C, ay * az * C - ax * s,
                   az * ax * C - ay * s, az * ay * C + ax * s, c + az * az * C};
    double Rn[9];
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col)
            Rn[3 * r + col] = D[3 * r + 0] * Rm[0 + col] +
                              D[3 * r + 1] * Rm[3 + col] +
                              D[3 * r + 2] * Rm[6 + col];
    auto nrm = [&](int r) {
        double m = std::sqrt(Rn[3 * r] * Rn[3 * r] + Rn[3 * r + 1] * Rn[3 * r + 1] +
                             Rn[3 * r + 2] * Rn[3 * r + 2]);
        for (int k = 0; k < 3; ++k) Rn[3 * r + k] /= m;
    };
    nrm(0);
    double d = Rn[0] * Rn[3] + Rn[1] * Rn[4] + Rn[2] * Rn[5];
    for (int k = 0; k < 3; ++k) Rn[3 + k] -= d * Rn[k];
    nrm(1);
    Rn[6] = Rn[1] * Rn[5] - Rn[2] * Rn[4];
    Rn[7] = Rn[2] * Rn[3] - Rn[0] * Rn[5];
    Rn[8] = Rn[0] * Rn[4] - Rn[1] * Rn[3];
    for (int k = 0; k < 9; ++k) Rm[k] = Rn[k];
}

// ---------------------------------------------------------------------------
// Case table: TestCases/TestCases.cpp:84-228 and TestCases/main.cpp:193-205
// ---------------------------------------------------------------------------
bool caseByName(const std::string &token, int *caseId)
{
    if (!token.empty() && token.find_first_not_of("0123456789") == std::string::npos)
    {
        int n = std::atoi(token.c_str());
        if (n >= 1 && n <= 6) { *caseId = n; return true; }
        return false;
    }
    for (int i = 0; i < 6; ++i)
        if (token == kCases[i].name) { *caseId = i + 1; return true; }
    return false;
}

bool configureCase(int caseId, int Nx, int Nv, double dt, int mlsOrder,
                   bool fixedBody, CaseParams &p)
{
    if (caseId < 1 || caseId > 6) return false;
    const CaseRow &row = kCases[caseId - 1];
    p = CaseParams();
    p.name = row.name;
    p.caseId = caseId;
    p.dim = row.dim;
    p.Tw = kWallTemp;
    p.dHS = kHSDiam;
    p.hasBody = row.hasBody;
    p.movingBodies = row.hasBody && !fixedBody;
    p.lidKind = row.lidKind;
    p.lidSpeed = row.lidSpeed;
    p.xleft = 0; p.xright = 1e-6; p.ytop = 1e-6; p.ybottom = 0;
    if (row.dim == 3) { p.zfront = 1e-6; p.zback = 0; }
    else { p.zfront = 0; p.zback = 0; }
    switch (caseId)
    {
    case 1:   // TestCases.cpp:151-160
        p.rho0 = 1.0; p.tau = 3.7142e-10; p.Nx = p.Ny = 100; p.Nz = 1;
        p.Nv = 44; p.VMax = 1303; p.VMin = -1303; p.dt = 1e-13;
        p.tfinal = 5e-9; p.saveEvery = 500;
        break;
    case 2:   // TestCases.cpp:164-173
        p.rho0 = 1.0; p.tau = 3.7142e-10; p.Nx = p.Ny = p.Nz = 31;
        p.Nv = 20; p.VMax = 1303; p.VMin = -1303; p.dt = 1e-11;
        p.tfinal = 5e-9; p.saveEvery = 500;
        break;
    case 3: case 4:   // TestCases.cpp:185-195
        p.rho0 = 11.0; p.tau = 3.37e-11; p.Nx = p.Ny = 60; p.Nz = 1;
        p.Nv = 30; p.VMax = 1500; p.VMin = -1500; p.dt = 1.5e-11;
        p.tfinal = 1e-6; p.saveEvery = 200;
        break;
    default:  // TestCases.cpp:214-224
        p.rho0 = 4.4; p.tau = 8.425e-11; p.Nx = p.Ny = p.Nz = 40;
        p.Nv = 10; p.VMax = 1303; p.VMin = -1303; p.dt = 1.5e-11;
        p.tfinal = 1.8e-7; p.saveEvery = 500;
        break;
    }
    if (Nx > 0) { p.Nx = p.Ny = Nx; if (row.dim == 3) p.Nz = Nx; }
    if (row.dim == 2) p.Nz = 1;
    if (Nv > 0) p.Nv = Nv;
    if (dt > 0) p.dt = dt;
    p.dtRequested = p.dt;
    p.mlsOrder = mlsOrder > 0 ? mlsOrder : 1;
    return true;
}

// Initialization/ParticleGeneration.cpp:30-200 (non-periodic, Fixed grid):
// lattice spacings, support radius and voxel boxes.
void latticeParams(CaseParams &p)
{
    int ndim = p.dim;
    int Nx = p.Nx, Ny = p.Ny, Nz = (ndim == 3) ? p.Nz : 1;
    double Lx = p.xright - p.xleft;
    double Ly = p.ytop - p.ybottom;
    double Lz = (ndim == 3) ? (p.zback - p.zfront) : 1.0;
    p.dx = Lx / (Nx - 1);
    p.dy = Ly / (Ny - 1);
    p.dz = (ndim == 3 && Nz > 1) ? Lz / (Nz - 1) : 1.0;
    p.radius = 2.5 * std::max({std::fabs(p.dx), std::fabs(p.dy),
                               (ndim == 3 ? std::fabs(p.dz) : std::fabs(p.dx))});
    p.minDist = 0.5 * std::min({std::fabs(p.dx), std::fabs(p.dy),
                                (ndim == 3 ? std::fabs(p.dz) : std::fabs(p.dy))});
    p.dv = (p.VMax - p.VMin) / (p.Nv - 1);
    p.hBox = 3.0 * p.dx;
    p.nbhBox = static_cast<int>(std::ceil(Lx / p.hBox)) + 1;
    p.vBox = 3.0 * p.dy;
    p.nbvBox = static_cast<int>(std::ceil(Ly / p.vBox)) + 1;
    if (ndim == 3)
    {
        p.wBox = 3.0 * p.dz;
        p.nbwBox = static_cast<int>(std::ceil(Lz / p.wBox)) + 1;
    }
    else { p.wBox = 1.0; p.nbwBox = 1; }
}

// Initialization/ParticleGeneration.cpp:30-200 (non-periodic, Fixed grid)
static void generateLattice(Cloud &c)
{
    CaseParams &p = c.prm;
    latticeParams(p);
    int ndim = p.dim;
    int Nx = p.Nx, Ny = p.Ny, Nz = (ndim == 3) ? p.Nz : 1;
    for (int k = 0; k < Nz; k++)
    {
        double z = (ndim == 3) ? std::fma((double)k, p.dz, p.zfront) : 0.0;
        for (int j = 0; j < Ny; j++)
        {
            double y = std::fma((double)j, p.dy, p.ybottom);
            for (int i = 0; i < Nx; i++)
            {
                double x = std::fma((double)i, p.dx, p.xleft);
                c.x.push_back(x); c.y.push_back(y); c.z.push_back(z);
                bool bx = (i == 0 || i == Nx - 1);
                bool by = (j == 0 || j == Ny - 1);
                bool bz = (ndim == 3) && (k == 0 || k == Nz - 1);
                c.boundary.push_back((bx || by || bz) ? 1 : 0);
                c.bodyId.push_back(-1);
                c.wall.insert(c.wall.end(), {0, 0, 0, 0, 0, 0, 0});
            }
        }
    }
    c.N = (int)c.x.size();
}

// TestCases/TestCases.cpp:251-294
static void makeBodies(Cloud &c, double bodyScale)
{
    const CaseParams &p = c.prm;
    if (!p.hasBody) return;
    const double rhoBody = p.rho0 * kBodyDensityRatio;
    constexpr double cx = 6e-7, cy = 7e-7, cz = 5e-7;
    Body b;
    b.cx = cx; b.cy = cy; b.T = kWallTemp;
    switch (p.caseId)
    {
    case 3:
        b.kind = 0; b.npts = kSquarePts; b.dim = 2;
        b.size = kSquareSide * bodyScale;
        b.mass = rhoBody * b.size * b.size;
        b.ox = 0.0; b.oy = 1.0;
        {
            double n = std::sqrt(b.ox * b.ox + b.oy * b.oy);
            b.ox /= n; b.oy /= n;
        }
        break;
    case 4:
        b.kind = 1; b.npts = kCirclePts; b.dim = 2;
        b.size = kCircleRadius * bodyScale;
        b.mass = rhoBody * kPi * b.size * b.size;
        break;
    case 5:
        b.kind = 2; b.npts = kSpherePts; b.dim = 3; b.cz = cz;
        b.size = kSphereRadius * bodyScale;
        b.mass = rhoBody * 4.0 / 3.0 * kPi * b.size * b.size * b.size;
        break;
    default:
        b.kind = 3; b.npts = kCubePts; b.dim = 3; b.cz = cz;
        b.size = kCubeSide * bodyScale;
        b.mass = rhoBody * b.size * b.size * b.size;
        break;
    }
    c.bodies.push_back(b);
}

void caseBodies(const CaseParams &p, double bodyScale, std::vector<Body> &bodies)
{
    Cloud c;
    c.prm = p;
    makeBodies(c, bodyScale > 0 ? bodyScale : 1.0);
    bodies = c.bodies;
}

void bodySurface(const CaseParams &p, const std::vector<Body> &bodies,
                 std::vector<double> &xyz, std::vector<double> &wall, std::vector<int> &start)
{
    const int ndim = p.dim;
    xyz.clear(); wall.clear(); start.assign(1, 0);
    for (const Body &B : bodies)
    {
        std::vector<double> s;
        B.surfacePoints(s);
        for (size_t q = 0; q + 2 < s.size(); q += 3)
        {
            const double px = s[q], py = s[q + 1], pz = (ndim == 3) ? s[q + 2] : 0.0;
            double nx, ny, nz;
            B.normal(px, py, (ndim == 3) ? pz : B.cz, &nx, &ny, &nz);
            if (ndim != 3) nz = 0.0;
            xyz.insert(xyz.end(), {px, py, pz});
            wall.insert(wall.end(), {nx, ny, nz, B.velx, B.vely, B.velz, B.T});
        }
        start.push_back((int)(xyz.size() / 3));
    }
}

// Initialization/BodyEmbedding.cpp:18-104
static void embedBodies(Cloud &c)
{
    if (c.bodies.empty()) return;
    const CaseParams &p = c.prm;
    int ndim = p.dim;
    std::vector<std::vector<double>> surf(c.bodies.size());
    for (size_t b = 0; b < c.bodies.size(); ++b) c.bodies[b].surfacePoints(surf[b]);
    double hug2 = std::pow(0.4 * std::fabs(p.dx), 2);
    std::vector<int> keep;
    for (int i = 0; i < c.N; ++i)
    {
        bool drop = false;
        for (size_t b = 0; b < c.bodies.size() && !drop; ++b)
        {
            if (c.bodies[b].inside(c.x[i], c.y[i], ndim == 3 ? c.z[i] : c.bodies[b].cz))
            { drop = true; break; }
            const std::vector<double> &s = surf[b];
            for (size_t q = 0; q + 2 < s.size(); q += 3)
            {
                double dx = c.x[i] - s[q], dy = c.y[i] - s[q + 1];
                double d2 = std::fma(dx, dx, dy * dy);
                if (ndim == 3) { double dz = c.z[i] - s[q + 2]; d2 = std::fma(dz, dz, d2); }
                if (d2 < hug2) { drop = true; break; }
            }
        }
        if (!drop) keep.push_back(i);
    }
    Cloud o;
    o.prm = c.prm;
    for (int i : keep)
    {
        o.x.push_back(c.x[i]); o.y.push_back(c.y[i]); o.z.push_back(c.z[i]);
        o.boundary.push_back(c.boundary[i]); o.bodyId.push_back(c.bodyId[i]);
        o.wall.insert(o.wall.end(), c.wall.begin() + 7 * i, c.wall.begin() + 7 * i + 7);
    }
    for (size_t b = 0; b < c.bodies.size(); ++b)
    {
        const Body &B = c.bodies[b];
        const std::vector<double> &s = surf[b];
        for (size_t q = 0; q + 2 < s.size(); q += 3)
        {
            double px = s[q], py = s[q + 1], pz = (ndim == 3) ? s[q + 2] : 0.0;
            double nx, ny, nz;
            B.normal(px, py, (ndim == 3) ? pz : B.cz, &nx, &ny, &nz);
            if (ndim != 3) nz = 0.0;
            o.x.push_back(px); o.y.push_back(py); o.z.push_back(pz);
            o.boundary.push_back(1); o.bodyId.push_back((int)b);
            o.wall.insert(o.wall.end(), {nx, ny, nz, B.velx, B.vely, B.velz, B.T});
        }
    }
    o.N = (int)o.x.size();
    o.bodies = c.bodies;
    c = std::move(o);
}

// Initialization/NeighbourSearch.cpp:17-99 (non-periodic axes)
void rebuildNeighbours(Cloud &c)
{
    const CaseParams &p = c.prm;
    int N = c.N, ndim = p.dim;
    int nvox = p.nbhBox * p.nbvBox * p.nbwBox;
    std::vector<std::vector<int>> vox(nvox);
    c.voxel.assign(N, 0);
    for (int i = 0; i < N; i++)
    {
        int vi = std::max(0, std::min(p.nbhBox - 1,
                 static_cast<int>(std::floor((c.x[i] - p.xleft) / p.hBox))));
        int vj = std::max(0, std::min(p.nbvBox - 1,
                 static_cast<int>(std::floor((c.y[i] - p.ybottom) / p.vBox))));
        int vk = (ndim == 3)
               ? std::max(0, std::min(p.nbwBox - 1,
                 static_cast<int>(std::floor((c.z[i] - p.zfront) / p.wBox))))
               : 0;
        c.voxel[i] = vi + p.nbhBox * (vj + p.nbvBox * vk);
        if (c.voxel[i] < nvox) vox[c.voxel[i]].push_back(i);
    }
    double r2max = p.radius * p.radius;
    int dkmax = (ndim == 3) ? 1 : 0;
    c.nnb.assign(N, 0);
    c.nbr.assign((size_t)N * kMaxNeigh, -1);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < N; i++)
    {
        int cnt = 0;
        int *out = &c.nbr[(size_t)i * kMaxNeigh];
        int vi = c.voxel[i] % p.nbhBox;
        int tmp = c.voxel[i] / p.nbhBox;
        int vj = tmp % p.nbvBox;
        int vk = tmp / p.nbvBox;
        bool done = false;
        for (int dk = -dkmax; dk <= dkmax && !done; dk++)
            for (int dj = -1; dj <= 1 && !done; dj++)
                for (int di = -1; di <= 1 && !done; di++)
                {
                    int ni = vi + di, nj = vj + dj, nk = vk + dk;
                    if (ni < 0 || ni >= p.nbhBox) continue;
                    if (nj < 0 || nj >= p.nbvBox) continue;
                    if (nk < 0 || nk >= p.nbwBox) continue;
                    int v = ni + p.nbhBox * (nj + p.nbvBox * nk);
                    for (int j : vox[v])
                    {
                        if (j == i) continue;
                        double ddx = c.x[j] - c.x[i];
                        double ddy = c.y[j] - c.y[i];
                        double ddz = (ndim == 3) ? c.z[j] - c.z[i] : 0.0;
                        if (std::fma(ddz, ddz, std::fma(ddx, ddx, ddy * ddy)) < r2max)
                        {
                            out[cnt++] = j;
                            if (cnt >= kMaxNeigh) { done = true; break; }
                        }
                    }
                }
        c.nnb[i] = cnt;
    }
}

// Core/MLSBasis.hpp:228-287 (getWallNormal) via BoundaryConditions/
// WallState.cpp:16-26, then TestCases/TestCases.cpp:230-249.
static void wallState(Cloud &c)
{
    const CaseParams &p = c.prm;
    constexpr double eps = 1.0e-13;
    double lid[6][3] = {{0}};      // left right top bottom front back
    if (p.lidKind == 0) lid[2][0] = p.lidSpeed;
    if (p.lidKind == 1) lid[4][0] = p.lidSpeed;
    for (int i = 0; i < c.N; ++i)
    {
        if (!c.boundary[i] || c.bodyId[i] >= 0) continue;
        double n[3] = {0, 0, 0}, U[3] = {0, 0, 0}, Tsum = 0;
        int nHit = 0;
        auto hit = [&](double ax, double ay, double az, int face) {
            n[0] += ax; n[1] += ay; n[2] += az;
            U[0] += lid[face][0]; U[1] += lid[face][1]; U[2] += lid[face][2];
            Tsum += p.Tw; ++nHit;
        };
        if (std::fabs(c.x[i] - p.xleft) < eps) hit(1, 0, 0, 0);
        if (std::fabs(c.x[i] - p.xright) < eps) hit(-1, 0, 0, 1);
        if (std::fabs(c.y[i] - p.ytop) < eps) hit(0, -1, 0, 2);
        if (std::fabs(c.y[i] - p.ybottom) < eps) hit(0, 1, 0, 3);
        if (std::fabs(c.z[i] - p.zfront) < eps) hit(0, 0, -1, 4);
        if (std::fabs(c.z[i] - p.zback) < eps) hit(0, 0, 1, 5);
        double *w = &c.wall[7 * i];
        if (nHit == 0) { w[6] = p.Tw; continue; }
        if (nHit == 1)
        {
            for (int a = 0; a < 3; ++a) { w[a] = n[a]; w[3 + a] = U[a]; }
            w[6] = Tsum;
            continue;
        }
        double nlen = std::sqrt(std::fma(n[2], n[2], std::fma(n[0], n[0], n[1] * n[1])));
        if (nlen > eps) { n[0] /= nlen; n[1] /= nlen; n[2] /= nlen; }
        for (int a = 0; a < 3; ++a) { w[a] = n[a]; w[3 + a] = U[a] / nHit; }
        w[6] = Tsum / nHit;
    }
    if (p.lidKind == 2)
    {
        const double L = p.xright - p.xleft;
        for (int i = 0; i < c.N; ++i)
        {
            if (!c.boundary[i] || c.bodyId[i] >= 0) continue;
            if (std::fabs(c.y[i] - p.ytop) > 1e-13) continue;
            const double s = c.x[i] / L;
            const double t = std::fma(-2.0, s, 2.0);
            c.wall[7 * i + 3] = p.lidSpeed * (2.0 * s) * (2.0 * s) * t * t;
        }
    }
}

// Initialization/InitialConditions.cpp:18-80 -- the row of the uniform
// Maxwellian at rest that every particle starts from.
void restRow(const CaseParams &p, std::vector<double> &row)
{
    int Nv = p.Nv, Nv2 = Nv * Nv;
    row.assign((p.dim == 3) ? Nv * Nv * Nv : 2 * Nv2, 0.0);
    const double rho = p.rho0, T = 270.0, R = p.R;
    if (p.dim == 3)
    {
        for (int kv = 0; kv < Nv; ++kv)
            for (int jv = 0; jv < Nv; ++jv)
                for (int iv = 0; iv < Nv; ++iv)
                    row[iv + Nv * (jv + Nv * kv)] =
                        maxwellian3(std::fma((double)iv, p.dv, p.VMin),
                                    std::fma((double)jv, p.dv, p.VMin),
                                    std::fma((double)kv, p.dv, p.VMin), 0, 0, 0, T, rho, R);
    }
    else
    {
        for (int jv = 0; jv < Nv; ++jv)
            for (int iv = 0; iv < Nv; ++iv)
            {
                double m = maxwellianG1(std::fma((double)iv, p.dv, p.VMin),
                                        std::fma((double)jv, p.dv, p.VMin), 0, 0, T, rho, R);
                row[iv + Nv * jv] = m;
                row[iv + Nv * jv + Nv2] = 0.5 * R * T * m;
            }
    }
}

static void initialState(Cloud &c)
{
    const CaseParams &p = c.prm;
    int Nv = p.Nv, Nv2 = Nv * Nv;
    c.gStride = (p.dim == 3) ? Nv * Nv * Nv : 2 * Nv2;
    c.g.assign((size_t)c.N * c.gStride, 0.0);
    c.macro.assign((size_t)c.N * 7, 0.0);
    c.meshv.assign((size_t)c.N * 3, 0.0);
    const double rho = p.rho0, T = 270.0, R = p.R;
    std::vector<double> row;
    restRow(p, row);
    for (int i = 0; i < c.N; ++i)
    {
        std::copy(row.begin(), row.end(), c.g.begin() + (size_t)i * c.gStride);
        double *m = &c.macro[7 * i];
        m[0] = rho; m[1] = m[2] = m[3] = 0.0; m[4] = T; m[5] = rho * R * T; m[6] = 0;
    }
}

bool buildCloud(const CaseParams &prmIn, double bodyScale, Cloud &c,
                std::string *err)
{
    c = Cloud();
    c.prm = prmIn;
    if (c.prm.Nx < 3 || c.prm.Nv < 2)
    {
        if (err) *err = "Nx must be >= 3 and Nv >= 2";
        return false;
    }
    if (bodyScale <= 0) bodyScale = 1.0;
    makeBodies(c, bodyScale);
    generateLattice(c);
    embedBodies(c);
    rebuildNeighbours(c);
    wallState(c);
    initialState(c);
    clampDt(c.prm);
    return true;
}

// Foot-point clamp, Solver/Solver.cpp:167-205.
void clampDt(CaseParams &p)
{
    double vmax = std::max(std::fabs(p.VMax), std::fabs(p.VMin));
    double dxmin = std::fabs(p.dx);
    if (std::fabs(p.dy) < dxmin) dxmin = std::fabs(p.dy);
    if (p.dim == 3 && std::fabs(p.dz) < dxmin) dxmin = std::fabs(p.dz);
    if (vmax * p.dt / dxmin > 1.5) p.dt = 0.75 * dxmin / vmax;
}

}  // namespace alebgk
