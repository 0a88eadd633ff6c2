// cuda_backend_shim.cpp -- the reference's CUDA-backend API on the B200
// C-ABI.
//
// The reference's time loop (Solver/Solver.cpp:253-578, built with
// ALEBGK_WITH_CUDA) calls 13 C++ functions declared at Solver/Solver.cpp:
// 67-89 and defined in Solver/CudaBackend.cu.  This file defines the same 13
// functions with the same signatures on top of include/alebgk.h, so that the
// reference's Solver.cpp and TestCases/main.cpp build and run unchanged with
// this file in place of CudaBackend.cu and libalebgk_b200.so on the link line.
//
// Precision: FP32 f storage (the default), or FP64 throughout with
// ALEBGK_B200_PRECISION=64 in the environment (the reference's loop reads its
// other run options from the environment the same way).
//
// Errors: the reference's CUCHECK prints and exits (CudaBackend.cu:58-66);
// the library returns a status from every call, and check() restores the
// print-and-exit behaviour in one place.
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

#include "Types.hpp"
#include "RigidBody.hpp"      // RigidBody, DomainBoundary, moveRigidBodies
#include "alebgk.h"

namespace {

alebgk_ctx *g_ctx = nullptr;
alebgk_config g_cfg{};
double g_dt = -1.0;                 // dt the device tables were built for
int g_N = 0, g_gs = 0, g_dim = 3;
std::vector<Particle> *g_host = nullptr;   // cloud of the last upload

void check(int rc, const char *what)
{
    if (rc == ALEBGK_OK) return;
    char msg[512];
    alebgk_last_error(g_ctx, msg, sizeof msg);
    std::fprintf(stderr, "[alebgk] %s failed (%d): %s\n", what, rc, msg);
    std::exit(1);
}

// Particle AoS -> the SoA arrays of alebgk_cloud (kept alive while uploading).
struct Soa
{
    std::vector<double> xyz, meshv, wall, g, macro;
    std::vector<int> boundary, bodyId, nnb, nbr;
    alebgk_cloud view{};

    explicit Soa(const std::vector<Particle> &P)
    {
        const size_t N = P.size(), gs = P.empty() ? 0 : P[0].g.size();
        xyz.resize(3 * N); meshv.resize(3 * N); wall.resize(7 * N);
        g.resize(N * gs); macro.resize(7 * N);
        boundary.resize(N); bodyId.resize(N); nnb.resize(N);
        nbr.assign(N * ALEBGK_MAX_NEIGH, 0);
        for (size_t i = 0; i < N; ++i)
        {
            const Particle &p = P[i];
            double *x = &xyz[3 * i], *m = &meshv[3 * i], *w = &wall[7 * i];
            x[0] = p.x; x[1] = p.y; x[2] = p.z;
            m[0] = p.meshVx; m[1] = p.meshVy; m[2] = p.meshVz;
            w[0] = p.wnx; w[1] = p.wny; w[2] = p.wnz;
            w[3] = p.wUx; w[4] = p.wUy; w[5] = p.wUz; w[6] = p.wT;
            boundary[i] = p.boundary;
            bodyId[i] = p.bodyId;
            nnb[i] = (int)std::min<size_t>(p.neighindex.size(), ALEBGK_MAX_NEIGH);
            for (int s = 0; s < nnb[i]; ++s) nbr[i * ALEBGK_MAX_NEIGH + s] = p.neighindex[s];
            std::copy(p.g.begin(), p.g.end(), g.begin() + i * gs);
            double *q = &macro[7 * i];
            q[0] = p.rho; q[1] = p.ux; q[2] = p.uy; q[3] = p.uz;
            q[4] = p.T; q[5] = p.p; q[6] = p.moodFlag ? 1.0 : 0.0;
        }
        view = {xyz.data(), meshv.data(), wall.data(), boundary.data(), bodyId.data(),
                nnb.data(), nbr.data(), g.data(), macro.data()};
    }
};

void fillConfig(const SimParameters &sp, const CalcParameters &cp, double R,
                const std::vector<Particle> &P)
{
    g_cfg = alebgk_config{};
    g_cfg.dim = cp.dim;
    g_cfg.N = (int)P.size();
    g_cfg.Nv = sp.Nv;
    g_cfg.mls_order = sp.mlsOrder;
    const char *prec = std::getenv("ALEBGK_B200_PRECISION");
    g_cfg.precision = (prec && std::atoi(prec) == 64) ? 64 : 32;
    g_cfg.limiter = (sp.limiter == LimiterMode::MOOD) ? 2 : 0;
    g_cfg.tau_variable = sp.tauVariable;
    g_cfg.device = 0;
    g_cfg.R = R;
    g_cfg.tau = sp.tao;
    g_cfg.dHS = sp.d;
    g_cfg.vmin = P.empty() ? sp.VMin : P[0].vlo;
    g_cfg.dv = cp.dv;
    g_cfg.radius = cp.radius;
    g_cfg.periodic[0] = cp.periodicX; g_cfg.periodic[1] = cp.periodicY;
    g_cfg.periodic[2] = cp.periodicZ;
    g_cfg.L[0] = cp.Lx; g_cfg.L[1] = cp.Ly; g_cfg.L[2] = cp.Lz;
}

void upload(const std::vector<Particle> &P, double dt)
{
    Soa s(P);
    check(alebgk_upload(g_ctx, &s.view, dt), "alebgk_upload");
    g_dt = dt;
}

void scatter(std::vector<Particle> &P, const std::vector<double> &macro,
             const std::vector<double> *g)
{
    for (size_t i = 0; i < P.size(); ++i)
    {
        Particle &p = P[i];
        const double *q = &macro[7 * i];
        p.rho = q[0]; p.ux = q[1]; p.uy = q[2]; p.uz = q[3];
        p.T = q[4]; p.p = q[5]; p.moodFlag = q[6] != 0.0;
        if (g) std::copy(g->begin() + i * g_gs, g->begin() + (i + 1) * g_gs, p.g.begin());
    }
}

}  // namespace

void cudaUploadCloud(const std::vector<Particle> &P, const SimParameters &)
{
    // The context needs CalcParameters and dt, which arrive with the first
    // cudaStep; until then the cloud is only remembered.
    g_host = const_cast<std::vector<Particle> *>(&P);
    if (g_ctx && (int)P.size() == g_N) upload(P, g_dt);
    else if (g_ctx) { alebgk_destroy(g_ctx); g_ctx = nullptr; }
}

void cudaStep(const SimParameters &sp, const CalcParameters &cp, double dt, double R)
{
    if (!g_ctx)
    {
        fillConfig(sp, cp, R, *g_host);
        check(alebgk_create(&g_cfg, &g_ctx), "alebgk_create");
        g_N = g_cfg.N;
        g_dim = g_cfg.dim;
        g_gs = (g_dim == 3) ? g_cfg.Nv * g_cfg.Nv * g_cfg.Nv : 2 * g_cfg.Nv * g_cfg.Nv;
        upload(*g_host, dt);
    }
    else if (dt != g_dt)
    {
        std::vector<double> g((size_t)g_N * g_gs), macro(7 * (size_t)g_N);
        check(alebgk_download_full(g_ctx, g.data(), macro.data()), "alebgk_download_full");
        scatter(*g_host, macro, &g);
        upload(*g_host, dt);          // tables for the new dt
    }
    check(alebgk_step(g_ctx, 1), "alebgk_step");
}

void cudaDownloadMoments(std::vector<Particle> &P)
{
    std::vector<double> macro(7 * P.size());
    check(alebgk_download_moments(g_ctx, macro.data()), "alebgk_download_moments");
    scatter(P, macro, nullptr);
}

void cudaDownloadFull(std::vector<Particle> &P)
{
    std::vector<double> g(P.size() * g_gs), macro(7 * P.size());
    check(alebgk_download_full(g_ctx, g.data(), macro.data()), "alebgk_download_full");
    scatter(P, macro, &g);
}

void cudaSyncBodies(std::vector<Particle> &P, std::vector<std::unique_ptr<RigidBody>> &bodies,
                    double dt, const DomainBoundary &dom, const CalcParameters &cp)
{
    cudaDownloadFull(P);
    moveRigidBodies(P, bodies, dt, dom, cp);   // the reference's own host update
    upload(P, dt);                             // new wall state and surface positions
}

void cudaLimiterCounts(int *nPositivity, int *nNAD)
{
    alebgk_counters c{};
    check(alebgk_get_counters(g_ctx, &c), "alebgk_get_counters");
    *nPositivity = c.positivity_fixes;
    *nNAD = c.transport_flags;
}

void cudaMlsCounts(int *nDegenerate, int *nExtrapolate)
{
    alebgk_counters c{};
    check(alebgk_get_counters(g_ctx, &c), "alebgk_get_counters");
    *nDegenerate = c.mls_degenerate;
    *nExtrapolate = 0;
}

void cudaMlsOvershoot(double *sum, double *worst) { *sum = 0.0; *worst = 0.0; }
void cudaMlsOvershootNow(double *sum, double *worst) { *sum = 0.0; *worst = 0.0; }

double cudaTotalMass()
{
    double m = 0.0;
    check(alebgk_total_mass(g_ctx, &m), "alebgk_total_mass");
    return m;
}

void cudaMassBudget(double *afterCorrection, double *afterCollision)
{
    alebgk_counters c{};
    check(alebgk_get_counters(g_ctx, &c), "alebgk_get_counters");
    *afterCorrection = c.mass_after_transport * c.mass_scale;
    *afterCollision = c.mass_end;
}

void cudaWallMomentum(std::vector<double> &out)
{
    out.assign(g_N, 0.0);
    check(alebgk_wall_momentum(g_ctx, out.data()), "alebgk_wall_momentum");
}

void cudaFreeCloud()
{
    if (g_ctx) alebgk_destroy(g_ctx);
    g_ctx = nullptr;
    g_dt = -1.0;
}
