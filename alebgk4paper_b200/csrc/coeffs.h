// coeffs.h -- FP64 MLS stencil classes and transport coefficients (internal).
//
// The MLS transport of MLSTransport/MLSTransport.cpp:88-311 solves, for every
// particle i and velocity node k, the weighted normal equations A(i,k) sol =
// sum_j w_j b_j f_j[k] and keeps gt = sol[0].  The matrix, the weights and
// the basis depend only on the geometry (neighbour offsets, foot point
// x_i - (v_k - meshV_i) dt, support h), never on f; partial-pivot Gaussian
// elimination with the reference's skip rule is a linear map of the
// right-hand side once the pivots are chosen from A.  Hence
//     gt[i][k] = sum_s c[class(i)][k][s] * f[nbr(i,s)][k]
// with coefficients computed once in FP64.  Particles whose neighbour
// offsets, wall state, mesh velocity and MLS order coincide share a class.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace alebgk {

struct CoeffInput
{
    int dim = 3, N = 0, Nv = 0, mlsOrder = 2;
    double dt = 0, h = 0, vmin = 0, dv = 0;
    bool periodic[3] = {false, false, false};
    double L[3] = {0, 0, 0};
    const double *xyz = nullptr;    // N*3
    const double *meshv = nullptr;  // N*3
    const double *wall = nullptr;   // N*7
    const int *boundary = nullptr;  // N
    const int *nnb = nullptr;       // N
    const int *nbr = nullptr;       // N*maxNeigh
    int maxNeigh = 128;
};

struct CoeffTables
{
    int S = 0;                      // slot stride: 1 (self) + max neighbours
    int V = 0;                      // velocity nodes per layer
    int ncls = 0;
    std::vector<int> cls;           // N: class of each particle
    std::vector<int> nslot;         // N: 1 + neighbour count
    std::vector<int> slots;         // N*S: slot 0 = self, then canonical order
    std::vector<int> rep;           // ncls: representative particle
    std::vector<double> coef;       // ncls*S*V, layout [class][slot][node]
    std::vector<int> degenerate;    // ncls: nodes with a skipped pivot
    std::vector<int> order;         // ncls: MLS order used
    std::vector<int> members;       // ncls: particles in the class
    // Set by the device class builder instead of nslot/slots (which stay
    // on the device): the slot count and slot row of each representative.
    std::vector<int> repNslot;      // ncls
    std::vector<int> repSlots;      // ncls*S
};

// Builds classes and coefficients.  Returns false with *err on bad input.
bool buildCoefficients(const CoeffInput &in, CoeffTables &out, std::string *err);

// FP32 image of the FP64 coefficients of one class, [S slots][V nodes]: each
// node's coefficients are rounded to nearest, then the largest of them (in
// magnitude, the first in slot order on a tie) takes the FP64 difference
// between the FP64 sum and the sum of the rounded values.  The FP32
// stencil then reproduces a constant field to within half an FP32 ulp of
// its largest coefficient, instead of to the accumulated rounding of all of
// them; a uniform state transports without a systematic density bias of
// order 1e-7, which would otherwise swamp the 1e-9 slack of the MOOD NAD
// screen (MLSTransport.cpp:370).  The device table builder does the same.
void roundCoefFP32(const double *src, float *dst, int S, int V);

// The class part alone (cls, nslot, slots, rep, members, order; no coef).
bool buildClasses(const CoeffInput &in, CoeffTables &out, std::string *err);

// Partial-pivot Gaussian elimination with the reference's |pivot| < 1e-30
// skip rule (MLSTransport/MLSTransport.cpp:20-62), applied to nrhs
// right-hand sides at once: A is n x n row-major, B is n x nrhs row-major and
// is overwritten with the solutions.  Returns the number of skipped pivots.
int solveSkipGE(double *A, double *B, int n, int nrhs);

}  // namespace alebgk
