// ref_driver.cpp -- test infrastructure, NOT product code.
//
// A thin C-ABI driver around the UNMODIFIED reference CPU sources of
// panchiittp/ALEBGK4Paper.  The recipe in oracle/Makefile compiles this file
// together with the reference's own Initialization/, MLSTransport/,
// MomentCalculations/, BoundaryConditions/, RigidBody/ and TestCases/
// translation units, straight from where they lie, into oracle/_ref/.
// Nothing here re-implements the reference's arithmetic: it reproduces the
// set-up sequence of TestCases/main.cpp:193-345 and the CPU step order of
// Solver/Solver.cpp:632-766 by calling the reference's own functions, and it
// adds two knobs the reference CLI cannot reach (mlsOrder, exact step count).
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
// legs load the resulting library, and only as the checker or as the timed
// reference implementation.
#include "Config.hpp"
#include "Types.hpp"
#include "MLSBasis.hpp"
#include "Geometry.hpp"
#include "Initialization.hpp"
#include "BoundaryConditions.hpp"
#include "Moments.hpp"
#include "MLSTransport.hpp"
#include "RigidBody.hpp"
#include "TestCases.hpp"
#include "Checkpoint.hpp"
#include "Output.hpp"

#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct RefCase
{
    TestCase tc;
    SimParameters sp;
    DomainBoundary dom;
    BoundaryConditions BC;
    GasConstants gc;
    CalcParameters cp{};
    std::vector<Particle> P;
    std::vector<std::unique_ptr<RigidBody>> bodies;
    double dt = 0.0;
    double t = 0.0;
    long step = 0;
    int lastTransportFlags = 0;
    int lastMoodFail = 0;
};

}  // namespace

extern "C" {

// Build a case exactly as TestCases/main.cpp:186-345 does, then apply the
// initial state as Solver/Solver.cpp:154 does and the foot-point clamp of
// Solver/Solver.cpp:167-205.  Nx/Nv/dt <= 0 keep the case defaults.
// fixedBody != 0 is the CLI's --fixed.
void *ref_create(const char *name, int Nx, int Nv, double dt, int mlsOrder,
                 int fixedBody, double bodyScale)
{
    auto *c = new RefCase();
    if (!parseCaseName(name, &c->tc)) { delete c; return nullptr; }
    BodyMotion motion = fixedBody ? BodyMotion::Fixed : BodyMotion::Free;
    const CaseInfo &info = caseInfo(c->tc);
    configureCase(c->tc, motion, c->sp, c->dom, c->BC, c->gc);
    c->sp.problem = ProblemID::DrivenCavity;
    if (Nx > 0) { c->sp.Nx = c->sp.Ny = Nx; if (info.dim == 3) c->sp.Nz = Nx; }
    if (Nv > 0) c->sp.Nv = c->sp.NvMin = c->sp.NvMax = Nv;
    if (dt > 0) c->sp.dt = dt;
    c->sp.mlsOrder = mlsOrder;
    if (bodyScale <= 0) bodyScale = 1.0;

    c->bodies = makeBodies(c->tc, motion, c->BC.rho, bodyScale);
    generateParticles(c->P, c->sp, c->dom, c->cp);
    embedRigidBodies(c->P, c->bodies, c->sp, c->cp);
    updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
    initWallData(c->P, c->dom, c->BC);
    applyLidProfile(c->tc, c->P, c->dom);

    int ndim = c->cp.dim;
    double Lx = c->dom.xright - c->dom.xleft;
    double Ly = c->dom.ytop - c->dom.ybottom;
    double Lz = (ndim == 3) ? (c->dom.zback - c->dom.zfront) : 1.0;
    applyIC(c->P, c->BC.rho, c->gc.R, Lx, Ly, Lz);

    double d = c->sp.dt;
    double vmax = std::max(std::fabs(c->sp.VMax), std::fabs(c->sp.VMin));
    double dxmin = std::fabs(c->cp.dx);
    if (std::fabs(c->cp.dy) < dxmin) dxmin = std::fabs(c->cp.dy);
    if (ndim == 3 && std::fabs(c->cp.dz) < dxmin) dxmin = std::fabs(c->cp.dz);
    if (vmax * d / dxmin > 1.5) d = 0.75 * dxmin / vmax;
    c->dt = d;
    return c;
}

void ref_destroy(void *h) { delete static_cast<RefCase *>(h); }

void ref_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int ref_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// dims[0..5] = N, dim, Nv, gStride, nBodies, mlsOrder
void ref_dims(void *h, int *dims)
{
    auto *c = static_cast<RefCase *>(h);
    dims[0] = (int)c->P.size();
    dims[1] = c->cp.dim;
    dims[2] = c->sp.Nv;
    dims[3] = c->P.empty() ? 0 : (int)c->P[0].g.size();
    dims[4] = (int)c->bodies.size();
    dims[5] = c->sp.mlsOrder;
}

// p[0..23]: dt, tau, R, dx, dy, dz, radius, minDist, dv, vlo, vhi, rho0, Tw,
//           xleft, xright, ybottom, ytop, zfront, zback, t, step, dHS,
//           tauVariable, movingBodies
void ref_params(void *h, double *p)
{
    auto *c = static_cast<RefCase *>(h);
    p[0] = c->dt; p[1] = c->sp.tao; p[2] = c->gc.R;
    p[3] = c->cp.dx; p[4] = c->cp.dy; p[5] = c->cp.dz;
    p[6] = c->cp.radius; p[7] = c->cp.minDist; p[8] = c->cp.dv;
    p[9] = c->sp.VMin; p[10] = c->sp.VMax; p[11] = c->BC.rho; p[12] = c->BC.Tw;
    p[13] = c->dom.xleft; p[14] = c->dom.xright; p[15] = c->dom.ybottom;
    p[16] = c->dom.ytop; p[17] = c->dom.zfront; p[18] = c->dom.zback;
    p[19] = c->t; p[20] = (double)c->step; p[21] = c->sp.d;
    p[22] = c->sp.tauVariable ? 1.0 : 0.0;
    p[23] = c->sp.movingBodies ? 1.0 : 0.0;
}

// Per particle: xyz[3], mesh velocity[3], wall state[7] (n, U_w, T_w),
// ints[3] (boundary, bodyId, neighbour count), neighbour indices (cap 128).
void ref_get_cloud(void *h, double *xyz, double *meshv, double *wall,
                   int *ints, int *nbr)
{
    auto *c = static_cast<RefCase *>(h);
    size_t N = c->P.size();
    for (size_t i = 0; i < N; ++i)
    {
        const Particle &p = c->P[i];
        xyz[3 * i] = p.x; xyz[3 * i + 1] = p.y; xyz[3 * i + 2] = p.z;
        meshv[3 * i] = p.meshVx; meshv[3 * i + 1] = p.meshVy; meshv[3 * i + 2] = p.meshVz;
        double *w = wall + 7 * i;
        w[0] = p.wnx; w[1] = p.wny; w[2] = p.wnz;
        w[3] = p.wUx; w[4] = p.wUy; w[5] = p.wUz; w[6] = p.wT;
        ints[3 * i] = p.boundary ? 1 : 0;
        ints[3 * i + 1] = p.bodyId;
        ints[3 * i + 2] = (int)p.neighindex.size();
        for (int s = 0; s < MAX_NEIGH; ++s)
            nbr[(size_t)MAX_NEIGH * i + s] =
                s < (int)p.neighindex.size() ? p.neighindex[s] : -1;
    }
}

void ref_get_g(void *h, double *g)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t i = 0; i < c->P.size(); ++i)
        std::memcpy(g + i * c->P[i].g.size(), c->P[i].g.data(),
                    c->P[i].g.size() * sizeof(double));
}

void ref_set_g(void *h, const double *g)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t i = 0; i < c->P.size(); ++i)
        std::memcpy(c->P[i].g.data(), g + i * c->P[i].g.size(),
                    c->P[i].g.size() * sizeof(double));
}

void ref_get_gt(void *h, double *gt)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t i = 0; i < c->P.size(); ++i)
        std::memcpy(gt + i * c->P[i].gt.size(), c->P[i].gt.data(),
                    c->P[i].gt.size() * sizeof(double));
}

// Per particle: rho, ux, uy, uz, T, p, moodFlag
void ref_get_macros(void *h, double *m)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t i = 0; i < c->P.size(); ++i)
    {
        const Particle &p = c->P[i];
        double *o = m + 7 * i;
        o[0] = p.rho; o[1] = p.ux; o[2] = p.uy; o[3] = p.uz;
        o[4] = p.T; o[5] = p.p; o[6] = p.moodFlag ? 1.0 : 0.0;
    }
}

void ref_set_macros(void *h, const double *m)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t i = 0; i < c->P.size(); ++i)
    {
        Particle &p = c->P[i];
        const double *o = m + 7 * i;
        p.rho = o[0]; p.ux = o[1]; p.uy = o[2]; p.uz = o[3];
        p.T = o[4]; p.p = o[5]; p.moodFlag = o[6] != 0.0;
    }
}

// One stage at a time, for stage-level parity (Solver/Solver.cpp:639-650):
// transport + MOOD screen + linear redo, leaving the result in gt (no commit).
int ref_transport(void *h)
{
    auto *c = static_cast<RefCase *>(h);
    mlsTransportCompute(c->P, c->dt, c->cp, c->dom, c->BC, c->sp.mlsOrder);
    int nf = 0;
    if (c->sp.limiter == LimiterMode::MOOD)
    {
        nf = checkTransportPAD(c->P);
        if (nf > 0)
            mlsTransportCompute(c->P, c->dt, c->cp, c->dom, c->BC, 1, true);
    }
    return nf;
}

double ref_sum_mass(void *h) { return sumMass(static_cast<RefCase *>(h)->P); }

// Single stages of Solver/Solver.cpp:632-705, for stage-level parity:
// 0 commit, 1 scaleG(s), 2 applyBoundaryBC, 3 computeMoments,
// 4 bgkCollision, 5 moodCheck (returns 1 on failure).
int ref_stage(void *h, int stage, double s)
{
    auto *c = static_cast<RefCase *>(h);
    switch (stage)
    {
    case 0: mlsTransportCommit(c->P); return 0;
    case 1: scaleG(c->P, s); return 0;
    case 2: applyBoundaryBC(c->P, c->gc.R, c->dom, c->BC); return 0;
    case 3: computeMoments(c->P, c->gc.R); return 0;
    case 4: bgkCollision(c->P, c->dt, c->sp.tao, c->gc.R, c->sp.tauVariable, c->sp.d);
            return 0;
    case 5: return moodCheck(c->P) ? 1 : 0;
    default: return -1;
    }
}

// The full CPU step sequence of Solver/Solver.cpp:632-766, nsteps times,
// with dt fixed (no tfinal truncation).  Returns the number of steps run.
int ref_step(void *h, int nsteps)
{
    auto *c = static_cast<RefCase *>(h);
    for (int n = 0; n < nsteps; ++n)
    {
        double dt = c->dt;
        double massOld = sumMass(c->P);
        mlsTransportCompute(c->P, dt, c->cp, c->dom, c->BC, c->sp.mlsOrder);
        int nf = 0;
        if (c->sp.limiter == LimiterMode::MOOD)
        {
            nf = checkTransportPAD(c->P);
            if (nf > 0)
                mlsTransportCompute(c->P, dt, c->cp, c->dom, c->BC, 1, true);
        }
        c->lastTransportFlags = nf;
        mlsTransportCommit(c->P);
        double massNew = sumMass(c->P);
        if (massNew > 1.0e-30) scaleG(c->P, massOld / massNew);
        applyGravity(c->P, c->sp.gravityY, dt);
        applyBoundaryBC(c->P, c->gc.R, c->dom, c->BC);
        computeMoments(c->P, c->gc.R);
        bgkCollision(c->P, dt, c->sp.tao, c->gc.R, c->sp.tauVariable, c->sp.d);
        computeMoments(c->P, c->gc.R);
        c->lastMoodFail = 0;
        if (c->sp.limiter == LimiterMode::MOOD)
        {
            if (moodCheck(c->P))
            {
                c->lastMoodFail = 1;
                bgkCollision(c->P, dt, c->sp.tao, c->gc.R, c->sp.tauVariable,
                             c->sp.d);
                computeMoments(c->P, c->gc.R);
            }
        }
        if (c->sp.movingBodies && !c->bodies.empty())
        {
            moveRigidBodies(c->P, c->bodies, dt, c->dom, c->cp);
            manageRemove(c->P, c->bodies, c->cp);
            updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
            int mergedN = mergeCloseParticles(c->P, c->cp);
            if (mergedN > 0) updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
            int added = manageRefill(c->P, c->bodies, c->sp, c->cp, c->dom,
                                     c->gc.R);
            if (added > 0) updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
            c->cp.N = static_cast<int>(c->P.size());
        }
        c->t += dt;
        c->step++;
    }
    return nsteps;
}

// last[0] = particles flagged by the transport MOOD screen in the last step,
// last[1] = 1 if the post-collision moodCheck failed in the last step.
void ref_last_flags(void *h, int *last)
{
    auto *c = static_cast<RefCase *>(h);
    last[0] = c->lastTransportFlags;
    last[1] = c->lastMoodFail;
}

// Body state: per body 32 doubles: cx cy cz velx vely velz angularVel omx omy
// omz forcex forcey forcez torque tqx tqy tqz ox oy mass I T Rm[9] area
void ref_get_bodies(void *h, double *out)
{
    auto *c = static_cast<RefCase *>(h);
    for (size_t b = 0; b < c->bodies.size(); ++b)
    {
        const RigidBody &r = *c->bodies[b];
        double *o = out + 32 * b;
        o[0] = r.cx; o[1] = r.cy; o[2] = r.cz;
        o[3] = r.velx; o[4] = r.vely; o[5] = r.velz;
        o[6] = r.angularVel; o[7] = r.omx; o[8] = r.omy; o[9] = r.omz;
        o[10] = r.forcex; o[11] = r.forcey; o[12] = r.forcez;
        o[13] = r.torque; o[14] = r.tqx; o[15] = r.tqy; o[16] = r.tqz;
        o[17] = r.ox; o[18] = r.oy; o[19] = r.mass;
        o[20] = r.getMomentOfInertia(); o[21] = r.T;
        const double *Rm = r.orientation();
        for (int k = 0; k < 9; ++k)
            o[22 + k] = Rm ? Rm[k] : ((k % 4) == 0 ? 1.0 : 0.0);
        o[31] = r.getSurfaceArea();
    }
}

// Test hook: shifts body b and its surface particles by (dx, dy, dz), as a
// body motion larger than one step would, so that the cloud management below
// has work to do.
void ref_shift_body(void *h, int b, double dx, double dy, double dz)
{
    auto *c = static_cast<RefCase *>(h);
    if (b < 0 || b >= (int)c->bodies.size()) return;
    RigidBody &r = *c->bodies[b];
    r.cx += dx; r.cy += dy; r.cz += dz;
    for (Particle &p : c->P)
        if (p.boundary && p.bodyId == b)
        {
            p.x += dx; p.y += dy;
            if (c->cp.dim == 3) p.z += dz;
        }
}

// Test hook: sets body b's velocity.
void ref_set_body_velocity(void *h, int b, double vx, double vy, double vz)
{
    auto *c = static_cast<RefCase *>(h);
    if (b < 0 || b >= (int)c->bodies.size()) return;
    RigidBody &r = *c->bodies[b];
    r.velx = vx; r.vely = vy; r.velz = vz;
}

// Test hook: moves particle i to (x, y, z).
void ref_set_position(void *h, int i, double x, double y, double z)
{
    auto *c = static_cast<RefCase *>(h);
    if (i < 0 || i >= (int)c->P.size()) return;
    c->P[i].x = x; c->P[i].y = y; c->P[i].z = z;
}

// The cloud-management block of the moving-body step (Solver.cpp:381-395,
// ref_step above): remove, rebuild, merge (+ rebuild), refill (+ rebuild).
// counts = removed, merged, added.
void ref_manage(void *h, int *counts)
{
    auto *c = static_cast<RefCase *>(h);
    int removed = manageRemove(c->P, c->bodies, c->cp);
    updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
    int mergedN = mergeCloseParticles(c->P, c->cp);
    if (mergedN > 0) updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
    int added = manageRefill(c->P, c->bodies, c->sp, c->cp, c->dom, c->gc.R);
    if (added > 0) updateVoxelsAndNeighbours(c->P, c->cp, c->dom);
    c->cp.N = static_cast<int>(c->P.size());
    counts[0] = removed;
    counts[1] = mergedN;
    counts[2] = added;
}

// Test hook: resizes the particle array to n (new particles default-built),
// so that ckpt::restore, which requires the file's particle count, can load
// the restart file of a moving-body run whose count has changed since the
// set-up.  The restore then overwrites every particle.
void ref_resize(void *h, int n)
{
    auto *c = static_cast<RefCase *>(h);
    c->P.resize((size_t)n, Particle(c->sp.Nv, c->cp.dim));
    c->cp.N = n;
}

// The reference's own restart files (Core/Checkpoint.hpp): save the case's
// state, restore into it, and the record sizes of the format.
int ref_checkpoint_save(void *h, const char *path)
{
    auto *c = static_cast<RefCase *>(h);
    return ckpt::save(path, c->step, c->t, c->P, c->bodies) ? 1 : 0;
}

int ref_checkpoint_load(void *h, const char *path, long *step, double *t)
{
    auto *c = static_cast<RefCase *>(h);
    const bool ok = ckpt::restore(path, step, t, c->P, c->bodies);
    if (ok) { c->step = *step; c->t = *t; }
    return ok ? 1 : 0;
}

// The reference's own save-cycle output (Core/Output.hpp): the VTK frame of
// the case's particles, the interior diagnostics, one timeseries row (the
// first call in the process writes the column line) and the step line on
// stdout.
void ref_write_vtk(void *h, const char *outdir, int step, double time)
{
    writeVTK(static_cast<RefCase *>(h)->P, outdir, step, time);
}

void ref_diagnostics(void *h, double *out)
{
    const Diagnostics d = computeDiagnostics(static_cast<RefCase *>(h)->P);
    out[0] = d.rho_avg; out[1] = d.KE; out[2] = d.T_avg; out[3] = d.p_avg;
    out[4] = d.moodCount; out[5] = d.n;
}

void ref_write_timeseries(void *h, const char *path, double t)
{
    writeTimeseries(path, t, computeDiagnostics(static_cast<RefCase *>(h)->P));
}

void ref_print_step(void *h, int step, double t, double dt)
{
    printStep(step, t, dt, computeDiagnostics(static_cast<RefCase *>(h)->P));
    std::fflush(stdout);
}

void ref_checkpoint_sizes(int *out)
{
    out[0] = (int)sizeof(ckpt::Header);
    out[1] = (int)sizeof(ckpt::PRec);
    out[2] = (int)sizeof(ckpt::BRec);
}

#ifdef ALEBGK_REF_CUDA
// The reference's own CUDA backend (Solver/CudaBackend.cu, compiled
// unmodified for sm_100a by oracle/Makefile's refcuda recipe), declared as
// Solver/Solver.cpp:67-89 declares it.  Built only into
// libalebgk_refcuda.so: the reference GPU path timed on the same case.
}  // extern "C"
void cudaUploadCloud(const std::vector<Particle> &P, const SimParameters &sp);
void cudaStep(const SimParameters &sp, const CalcParameters &cp, double dt, double R);
void cudaDownloadMoments(std::vector<Particle> &P);
void cudaFreeCloud();
extern "C" int cudaDeviceSynchronize(void);
extern "C" {

// Uploads the case's current state to the reference's device cloud, runs
// `warmup` untimed steps and then `steps` timed steps of cudaStep (the
// reference's GPU time loop body, Solver/Solver.cpp:301-303), with the
// device synchronised on both sides of the timed region; the mean wall
// time per step in *ms.  Downloads the moments (cudaDownloadMoments) into
// the case afterwards, so that ref_get_macros reads the device result.
int ref_cuda_run(void *h, int warmup, int steps, double *ms)
{
    auto *c = static_cast<RefCase *>(h);
    cudaUploadCloud(c->P, c->sp);
    for (int s = 0; s < warmup; ++s) cudaStep(c->sp, c->cp, c->dt, c->gc.R);
    if (cudaDeviceSynchronize() != 0) return -1;
    const auto t0 = std::chrono::high_resolution_clock::now();
    for (int s = 0; s < steps; ++s) cudaStep(c->sp, c->cp, c->dt, c->gc.R);
    if (cudaDeviceSynchronize() != 0) return -1;
    const auto t1 = std::chrono::high_resolution_clock::now();
    *ms = steps > 0 ? std::chrono::duration<double, std::milli>(t1 - t0).count() / steps : 0.0;
    cudaDownloadMoments(c->P);
    c->step += warmup + steps;
    c->t += (warmup + steps) * c->dt;
    cudaFreeCloud();
    return 0;
}
#endif

}  // extern "C"
