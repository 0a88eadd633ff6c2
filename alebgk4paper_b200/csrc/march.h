// march.h -- lattice-marching transport plan (internal header).
//
// When the cloud is a complete Cartesian lattice in the reference's particle
// order (i = x + Nx (y + Ny z), Initialization/ParticleGeneration.cpp:119-184)
// and every neighbour lies within two lattice steps, the transport is a
// stencil over lattice positions: gt(x,y,z;k) = sum_o C[class][o][k] f(x+o;k)
// over the 81 offsets |o|^2 <= 6 (self included).  The plan groups lattice
// columns into work units of class-uniform four-column blocks (2x2, 1x4 or
// 4x1) that march through z.
#pragma once
#include <cstdint>
#include <vector>

#include "coeffs.h"

namespace alebgk {

constexpr int kTmplOffsets = 81;    // (dx,dy,dz) in [-2,2]^3 with |d|^2 <= 6
constexpr int kMarchTileX = 8;      // CTA column tile
constexpr int kMarchTileY = 4;
constexpr int kMarchWarps = 8;      // one 2x2 column block per warp
constexpr int kMarchChunk = 32;     // velocities per CTA (one per lane)
constexpr int kThinSegment = 4;     // segments shorter than this are marched across

// Canonical template offset index of (dx, dy, dz), or -1 if outside.
int templateIndex(int dx, int dy, int dz);

// Warp block shapes: the four columns c = 0..3 of a block at (bx, by) are
// (bx + (c & 1), by + (c >> 1)) for kShapeBlock, (bx, by + c) for
// kShapeColumn and (bx + c, by) for kShapeRow.
constexpr int kShapeBlock = 0;    // 2 x 2
constexpr int kShapeColumn = 1;   // 1 x 4 (one lattice x, four y)
constexpr int kShapeRow = 2;      // 4 x 1 (four x, one lattice y)

struct MarchUnit
{
    int x0, y0, za, zb;   // tile origin (columns) and output planes [za, zb)
    int yMarch;           // 0: lattice (x, y) columns through z; 1: (x, z) through y
    int nsub;             // active warps
    int sub[kMarchWarps]; // bx | by << 4 | mask << 8 | shape << 12 | class << 14
};

struct MarchPlan
{
    bool ok = false;
    int Nx = 0, Ny = 0, Nz = 0;
    int ncls = 0, Vpad = 0;
    std::vector<MarchUnit> units;    // marching through z
    std::vector<MarchUnit> unitsY;   // thin z-planes, marching through y
    std::vector<float> coefT;        // [class][81][Vpad]
    std::vector<float> coefTy;       // the same in the y-march frame
    std::vector<float> coefTLin;     // same, linear MLS
};

// Detects the lattice and builds the plan; plan.ok is false when the cloud
// is not a complete lattice with two-step stencils.
// Whether a cloud is a complete lattice in generation order with every
// neighbour within the march's 81-offset template (the test of buildMarchPlan).
bool marchEligible(const double *xyz, int N, int dim, const int *nnb, const int *nbr,
                   int maxNeigh);

void buildMarchPlan(const double *xyz, int N, int dim, const int *nnb,
                    const int *nbr, int maxNeigh, const CoeffTables &tb,
                    const CoeffTables *tl, MarchPlan &plan);

}  // namespace alebgk
