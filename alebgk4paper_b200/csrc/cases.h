// cases.h -- host-side case set-up for the ALE-BGK step (internal header).
//
// Builds the point cloud of one of the reference's six lid-driven-cavity
// cases as plain structure-of-arrays: lattice positions, wall flags and wall
// state, neighbour lists, rigid bodies and the initial Maxwellian.  Every
// routine restates the reference's set-up code, cited per function; the cloud
// it produces is what alebgk_upload() consumes.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace alebgk {

constexpr int kMaxNeigh = 128;  // Core/Types.hpp:22 (MAX_NEIGH)

// One rigid body, the union of the reference's Square/Circle/Sphere/Cube
// (RigidBody/Geometry.hpp:19-362).  kind: 0 square, 1 circle, 2 sphere, 3 cube.
struct Body
{
    int kind = 0;
    int npts = 0;
    int dim = 2;
    double cx = 0, cy = 0, cz = 0;
    double mass = 0, T = 270.0;
    double ox = 1.0, oy = 0.0;          // 2-D orientation
    double size = 0;                    // side (square, cube) or radius
    double velx = 0, vely = 0, velz = 0;
    double angularVel = 0, omx = 0, omy = 0, omz = 0;
    double forcex = 0, forcey = 0, forcez = 0;
    double torque = 0, tqx = 0, tqy = 0, tqz = 0;
    bool rotates = true;
    double Rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};

    double inertia() const;
    double surfaceArea() const;
    bool inside(double x, double y, double z) const;
    void normal(double x, double y, double z, double *nx, double *ny,
                double *nz) const;
    void surfacePoints(std::vector<double> &xyz) const;  // 3 per point
    void rotate3(double wx, double wy, double wz, double dt);
};

// Case parameters (TestCases/TestCases.cpp:113-228 plus main.cpp overrides).
struct CaseParams
{
    std::string name;
    int caseId = 1;
    int dim = 2;
    int Nx = 0, Ny = 0, Nz = 1, Nv = 0;
    double VMin = 0, VMax = 0, dv = 0;
    double tau = 0, dt = 0, dtRequested = 0, tfinal = 0;
    double rho0 = 1.0, Tw = 270.0, R = 208.0, dHS = 0.368e-9;
    double xleft = 0, xright = 1e-6, ybottom = 0, ytop = 1e-6,
           zfront = 0, zback = 0;
    double dx = 0, dy = 0, dz = 0, radius = 0, minDist = 0;
    double hBox = 0, vBox = 0, wBox = 0;
    int nbhBox = 1, nbvBox = 1, nbwBox = 1;
    int mlsOrder = 2;
    bool hasBody = false, movingBodies = false;
    int lidKind = 0;            // 0 uniform y=L, 1 uniform z=L, 2 parabolic y=L
    double lidSpeed = 1.0;
    int saveEvery = 500;
};

// The cloud in structure-of-arrays form.  g is FP64 in the reference's
// per-particle layout (Nv^3 values in 3-D, g1[Nv^2] then g2[Nv^2] in 2-D).
struct Cloud
{
    CaseParams prm;
    int N = 0;
    int gStride = 0;
    std::vector<double> x, y, z;
    std::vector<double> xyz;       // interleaved copy for the C-ABI view
    std::vector<double> meshv;     // 3 per particle
    std::vector<double> wall;      // 7 per particle: n, U_w, T_w
    std::vector<int> boundary, bodyId, voxel;
    std::vector<int> nnb;          // neighbour count
    std::vector<int> nbr;          // kMaxNeigh per particle
    std::vector<double> g;         // N * gStride
    std::vector<double> macro;     // 7 per particle: rho ux uy uz T p mood
    std::vector<Body> bodies;
};

// Resolves a case by number ("1".."6") or name; false if unknown.
bool caseByName(const std::string &token, int *caseId);

// Fills prm for a case with optional overrides (<= 0 keeps the default).
bool configureCase(int caseId, int Nx, int Nv, double dt, int mlsOrder,
                   bool fixedBody, CaseParams &prm);

// Full set-up as TestCases/main.cpp:335-345 + Solver/Solver.cpp:154-205.
bool buildCloud(const CaseParams &prmIn, double bodyScale, Cloud &c,
                std::string *err);

// The bodies of a configured case (TestCases/TestCases.cpp:251-294), and
// the surface particles embedBodies appends for them
// (Initialization/BodyEmbedding.cpp:66-96): positions (3 per point), wall
// state (7 per point: n, U_w, T_w), and per body the first point
// (start[b] .. start[b + 1]).
void caseBodies(const CaseParams &p, double bodyScale, std::vector<Body> &bodies);
void bodySurface(const CaseParams &p, const std::vector<Body> &bodies,
                 std::vector<double> &xyz, std::vector<double> &wall, std::vector<int> &start);

// Lattice spacings, support radius and voxel boxes of a configured case
// (the scalar part of Initialization/ParticleGeneration.cpp:30-200).
void latticeParams(CaseParams &p);

// The rest-state Maxwellian row every particle starts from
// (Initialization/InitialConditions.cpp:18-80).
void restRow(const CaseParams &p, std::vector<double> &row);

// The reference's Maxwellians (Core/MLSBasis.hpp:87-122), in the FMA form of
// its compiled build.
double maxwellian3(double vx, double vy, double vz, double ux, double uy, double uz,
                   double T, double rho, double R);
double maxwellianG1(double vx, double vy, double ux, double uy, double T, double rho,
                    double R);

// Foot-point clamp of dt (Solver/Solver.cpp:167-205).
void clampDt(CaseParams &p);

// Rebuilds voxel bins and neighbour lists from the positions
// (Initialization/NeighbourSearch.cpp:17-99).
void rebuildNeighbours(Cloud &c);

}  // namespace alebgk
