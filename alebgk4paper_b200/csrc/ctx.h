// ctx.h -- device context of the ALE-BGK step (internal header).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/alebgk.h"

namespace alebgk {

struct MarchUnit;

// Device state of the lattice-marching transport (march.cu).
struct MarchState
{
    bool enabled = false;
    int nunits = 0, nunitsY = 0, Vpad = 0, Nx = 0, Ny = 0, Nz = 0;
    int vpl = 2;                              // velocities per lane (1 or 2)
    MarchUnit *units = nullptr;               // y-march units first, then z-march
    float *coefT = nullptr, *coefTy = nullptr;
    alignas(64) unsigned char tmap[2][128];   // CUtensorMap per source buffer
    alignas(64) unsigned char tmapY[2][128];  // the same with the y-march box
};

// Per-step scalars kept on the device so that a step needs no host
// synchronisation (the reference reads three masses back per step,
// Solver/CudaBackend.cu:1384-1395).
//
// The stored distribution h is the true one divided by `scale`: the global
// mass rescale of a step (Solver/Solver.cpp:650-655) is a uniform factor, and
// everything after it in the step is homogeneous of degree one in g, so the
// factor is applied to the macros at once and to h lazily, by the next
// transport (which is linear) and by every download.
struct StepScalars
{
    double massOld;        // true sumMass at the start of the step
    double massNew;        // true sumMass after transport + positivity + redo
    double sigma;          // massOld / massNew of the last step
    double massEnd;        // true sumMass at the end of the step
    double scale;          // true g = scale * stored h
    int nflag;             // transport MOOD flags (length of the redo list)
    int ndeg;              // particles finished after sigma (k_fixup list)
    int nfix;              // positivity repairs
    int moodfail;          // post-collision moodCheck failed
    int err;               // device error bits
    unsigned redCount;     // ticket of the grid sums (zero between kernels)
    long long steps;
    double slabPart[3];    // slab group: this slab's owned-range partial sums
};

struct DeviceBuffers
{
    void *f[2] = {nullptr, nullptr};   // ping-pong distribution, N x ldf
    void *coef = nullptr;              // [class][slot][node], MLS order of the cloud
    void *coefLin = nullptr;           // same, linear MLS (MOOD redo)
    double *pos = nullptr, *meshv = nullptr, *wall = nullptr;
    int *boundary = nullptr, *bodyId = nullptr;
    int *cls = nullptr, *nslot = nullptr, *slots = nullptr;
    double *macro[2] = {nullptr, nullptr};   // N x 6: rho ux uy uz T p (true)
    int *mood = nullptr, *flag = nullptr;
    int *flagList = nullptr, *degList = nullptr;
    double *massPos = nullptr;         // per particle: mass after positivity (true)
    double *massEnd = nullptr;         // per particle: mass of h at step end
    double *minG = nullptr;            // per particle: min of h over the mass layer
    double *nad = nullptr;             // per particle: NAD neighbour density range (lo, hi)
    double *redPartial = nullptr;      // per-block partials of the grid sums
    double *dpx = nullptr;
    double *bodyTmp = nullptr;         // N x 6 per-particle load contributions
    double *bodyOut = nullptr;         // up to 64 bodies x 6
    double *stage = nullptr;           // N x gs FP64 host-transfer staging
    int *surfList = nullptr;           // body-surface particles (boundary, bodyId >= 0)
    int *rowOrder = nullptr;           // the row kernel's visiting order: interior
                                       // particles, then wall particles
    double *bodyIO = nullptr;          // body-step staging: kBodyIOHead + 13 per surface particle
    double *rankAll = nullptr;         // multi-process slab: every rank's 4 combine words
    int rankAllCap = 0;                // ranks rankAll holds
    StepScalars *sc = nullptr;
};

struct StepParams
{
    int N = 0, dim = 3, Nv = 0, V = 0, L = 1, gs = 0, ldf = 0, S = 0;
    // Slab group: particles [ownLo, ownHi) are this slab's own, the rest are
    // ghost copies of the neighbouring slabs' rows (ownHi <= ownLo: no slab).
    int ownLo = 0, ownHi = 0;
    int limiter = 2, tauVar = 0, mlsOrder = 2;
    int periodic[3] = {0, 0, 0};
    double Lp[3] = {0, 0, 0};
    double R = 208, tau = 1, dHS = 0, vmin = 0, dv = 0, dvN = 0, h = 0, dt = 0;
    double lam = 0, c1 = 1, inv3R = 0;   // dt/tau, 1/(1+lam), 1/(3R) for this dt
    // Relative rounding floor added to the NAD slack (MLSTransport.cpp:370):
    // 0 in FP64; in FP32 the transported density carries rounding of a few
    // ulp of FP32, far above the reference's 1e-9 absolute slack near a
    // uniform state, so the screen would flag rounding noise.
    double nadNoise = 0;
    double resU = 0;      // momentum speed scale of the steady residual (0: thermal)
};

}  // namespace alebgk

namespace alebgk {
// Device scratch of the stencil-class builder (classes_dev.cu), kept by a
// context between geometry refreshes; caps in elements.
struct ClassScratch
{
    int *nnb = nullptr, *nbr = nullptr, *first = nullptr, *same = nullptr, *rep = nullptr;
    int *repSlots = nullptr, *repNslot = nullptr;
    long long *koff = nullptr, *keys = nullptr;
    unsigned long long *hashes = nullptr;
    size_t capN = 0, capNbr = 0, capFirst = 0, capSame = 0, capRep = 0, capRepSlots = 0;
    size_t capRepNslot = 0, capKoff = 0, capKeys = 0, capHash = 0;
};
}  // namespace alebgk

struct alebgk_ctx
{
    alebgk_config cfg{};
    alebgk::StepParams sp;
    alebgk::DeviceBuffers d;
    alebgk::MarchState march;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;          // side stream of the step graph
    cudaEvent_t evFork = nullptr, evJoin = nullptr;
    // Pinned host staging of the state transfers (alebgk_upload_state,
    // alebgk_download_moments), allocated on first use: the macro rows, then
    // a ring of kPinChunks chunks of FP32 rows; one event per ring chunk.
    static constexpr int kPinChunks = 4;
    void *pin = nullptr;
    size_t pinBytes = 0;
    cudaEvent_t pinEv[kPinChunks] = {};
    int cur = 0;                 // buffer holding the current h and macros
    bool uploaded = false;
    int ncls = 0;
    int degenerateParticles = 0;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // Launch shapes of the general kernels (alebgk_set_launch / autotune).
    struct
    {
        int transportThreads = 0;     // coefficient-gather transport per block; 0 fused
        int particleWarps = 0;        // warp-per-particle kernel; 0 = as many as fit
        int marchVpl = 2;             // lattice march: velocities per lane (1 or 2)
    } tune;
    // Streamed particle kernel: on, warps per block, blocks, dynamic smem.
    bool pStream = false;
    int pStreamWpb = 0, pStreamBlocks = 0;
    size_t pStreamSmem = 0;
    // Register-row form of the streamed stages (FP32, Nv <= 10): on, blocks.
    bool pRows = false;
    int pRowsBlocks = 0;
    std::string err;
    std::vector<int> bodyIdHost;
    int maxBodyId = -1;          // largest entry of bodyIdHost (-1: no body particle)
    std::vector<int> boundaryHost;
    std::vector<int> surfHost;   // body-surface particle indices, ascending
    bool geometryDirty = false;  // a body step moved the surface since the upload
    long long hostSteps = 0;     // steps enqueued since the upload
    double *macSnap = nullptr;   // macros at the last interval residual (N x 6)
    long long snapSteps = -1;    // hostSteps of that snapshot (-1: none)
    // Allocated elements of the buffers that a geometry refresh may resize:
    // each MLS table, the slot lists, the surface list.
    size_t coefCap = 0, slotsCap = 0, surfCap = 0;
    alebgk::ClassScratch clsScratch;
    // Counts the uploads and geometry refreshes: captured batch graphs and
    // stage descriptors hold device pointers and slot strides of one epoch.
    unsigned long long epoch = 0;
};

namespace alebgk {

// Launch wrappers (step.cu).
cudaError_t prepareKernels(alebgk_ctx *c);
cudaError_t launchStep(alebgk_ctx *c, int from, cudaEvent_t *ev = nullptr);
cudaError_t launchMassInit(alebgk_ctx *c);
// Slab groups (slab.cpp): one segment of the split step (0..3) on stream st,
// the cross-slab combine of a segment's partial sums (phase 0..3, 4 = set-up
// mass), and the owned-range mass of a freshly uploaded slab into slabPart[1].
// Batches of clouds stepped by one launch per stage (step.cu): per-parity
// device descriptors, per-stage block offsets, launch sizes.
struct BatchLaunch
{
    void *desc[2] = {nullptr, nullptr};
    int *off = nullptr;
    int n = 0, L = 1;
    bool f64 = false;
    size_t smemParticle = 0, smemRedo = 0;
    int blocks[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    // One persistent launch per step instead of one launch per stage: its
    // grid (co-resident blocks), the grid barrier's words and poll limit.
    bool persistent = false;
    int pGrid = 0;
    unsigned *bar = nullptr;
    int *vmap = nullptr;      // virtual block -> cloud, per stage
    long long spinCap = 1ll << 24;
};
// cudaErrorNotSupported when the clouds cannot share launches (mixed
// precision or layers, the streamed particle kernel or the lattice march).
cudaError_t buildBatchLaunch(alebgk_ctx *const *cs, int n, double *const *resid,
                             BatchLaunch &bl);
cudaError_t prepareBatchLaunch(const BatchLaunch &bl);
cudaError_t launchBatchStep(const BatchLaunch &bl, int from, cudaStream_t st);
void freeBatchLaunch(BatchLaunch &bl);
cudaError_t launchSlabSegment(alebgk_ctx *c, int from, int seg, cudaStream_t st);
cudaError_t launchSlabCombine(StepScalars *const *scs, int n, int phase, cudaStream_t st);
cudaError_t launchSlabInitSum(alebgk_ctx *c, cudaStream_t st);
// One slab of a multi-process run: the combine of the slab group for this
// slab alone, from every rank's words all[4 r + q] (slabPart[q], q < 3, and
// moodfail at q = 3) in rank order (step.cu).
cudaError_t launchRankCombine(alebgk_ctx *c, const double *allDev, int n, int phase,
                              cudaStream_t st);
struct CaseParams;
// Device arrays of the lattice set-up (setup.cu).
struct LatticeDev
{
    double *xyz = nullptr, *wall = nullptr, *meshv = nullptr;
    int *boundary = nullptr, *bodyId = nullptr, *voxel = nullptr, *voxCount = nullptr;
    int *voxStart = nullptr, *voxCursor = nullptr, *voxList = nullptr;
    int *nnb = nullptr, *nbr = nullptr;
};
// The lattice of a box cavity (positions, flags, wall state), and unless
// neighbours is false its voxel bins and neighbour lists.
cudaError_t buildLatticeDevice(const CaseParams &p, const LatticeDev &o, cudaStream_t st,
                               bool neighbours = true);
// Voxel grid of the neighbour search: origin, box sizes, box counts, radius.
struct NeighbourGrid
{
    int dim = 3;
    double x0 = 0, y0 = 0, z0 = 0, hx = 1, hy = 1, hz = 1, radius = 0;
    int nx = 1, ny = 1, nz = 1;
};
cudaError_t buildNeighboursDevice(const NeighbourGrid &g, const double *xyz, int N,
                                  const LatticeDev &o, cudaStream_t st);
cudaError_t launchRestState(alebgk_ctx *c, const double *rowDev, double rho, double T0);
// The distribution of a managed cloud from a row plan (step.cu k_rows_build).
cudaError_t launchRowsBuild(alebgk_ctx *c, int n, const int *a, const int *b,
                            const double *fresh, double *out);
struct Body;
// Body embedding of a lattice set-up on the device (setup.cu): raw holds
// the whole lattice (NL particles, from buildLatticeDevice); out receives the
// kept lattice particles in order, then the surface particles, and (when
// out.nnb is set) the neighbour lists of the result; *nOut is its count.
cudaError_t embedLatticeDevice(const CaseParams &p, const std::vector<Body> &bodies,
                               const std::vector<double> &surfXyz,
                               const std::vector<double> &surfWall,
                               const std::vector<int> &surfStart, const LatticeDev &raw, int NL,
                               const LatticeDev &out, int *nOut, cudaStream_t st);
struct CoeffInput;
struct CoeffTables;
// MLS tables of the classes `cls` built on the device (coeffs_dev.cu).
cudaError_t buildTablesDevice(const CoeffInput &in, const CoeffTables &cls, int order,
                              void *table, bool f64, std::vector<int> &degenerate,
                              cudaStream_t st);
// Stencil classes of a cloud whose geometry is on the device (classes_dev.cu):
// writes the slot counts, slot lists (stride 1 + max neighbours) and class
// ids on the device and fills `out` as buildClasses does (with the
// representatives' slot rows in repSlots/repNslot instead of slots/nslot).
// `collision` set: two different keys share a hash; use buildClasses.
cudaError_t buildClassesDevice(const CoeffInput &in, const double *dXyz, const double *dMeshv,
                               const double *dWall, const int *dBoundary, int *dCls,
                               int *dNslot, int *dSlots, size_t slotsCap, ClassScratch &scr,
                               CoeffTables &out, bool &collision, cudaStream_t st);
void freeClassScratch(ClassScratch &s);
cudaError_t launchSeedGrad13(alebgk_ctx *c, const float *net, int ldnet, const double *scale,
                             const double *shift);
cudaError_t launchMoments13(alebgk_ctx *c, double *out);
cudaError_t launchBodyLoads(alebgk_ctx *c, int nbodies, const double *centreDev,
                            const double *areaDev);
cudaError_t launchSetSurfaceVelocity(alebgk_ctx *c, int nbodies,
                                     const double *centreDev,
                                     const double *stateDev);
// Heun Newton-Euler step of the rigid bodies (body_step.cu).
constexpr int kMaxBodyIO = 64;                 // bodies per body call
constexpr int kBodyIOHead = 13 * kMaxBodyIO;   // doubles before the surface rows
cudaError_t bodyStep(alebgk_ctx *c, int nbodies, alebgk_body *bodies, const double *box,
                     double dx, double dt, std::string *err);
// Restart files in the reference's checkpoint layout (checkpoint.cpp).
int checkpointHeader(const char *path, alebgk_ckpt_header *out, std::string *err);
int checkpointRead(const char *path, const alebgk_ckpt_header *expect, alebgk_cloud *cl,
                   int *voxel, alebgk_body *bodies, std::string *err);
int checkpointSave(alebgk_ctx *c, const char *path, int64_t step, double t, const double *vgrid,
                   const int *voxel, int nbodies, const alebgk_body *bodies, std::string *err);
// Body loads on the fixed device scratch of body_noalloc.cu (no allocation).
constexpr int kNoAllocMaxBodies = ALEBGK_NOALLOC_MAX_BODIES;
cudaError_t bodyLoadsNoAlloc(alebgk_ctx *c, int nbodies, const double *centre,
                             const double *area, double *out, std::string *err);
cudaError_t launchResidual(alebgk_ctx *c, double *out, cudaStream_t st);
cudaError_t launchConvertIn(alebgk_ctx *c, const double *src, int buf);
cudaError_t launchConvertOut(alebgk_ctx *c, double *dst, int buf);
cudaError_t launchMarch(alebgk_ctx *c, int from, float *outBuf, cudaStream_t st);
cudaError_t prepareMarch();
bool encodeMarchMap(void *tmapOut, void *f, int V, int Nx, int Ny, int Nz, int ldf,
                    bool yMarch, int vpl, std::string *err);

}  // namespace alebgk
