// body_step.cu -- one Heun Newton-Euler step of the rigid bodies
// (moveRigidBodies, RigidBody/BodyDynamics.cpp:352-638).
//
// The surface-stress loads are device reductions over the current
// distribution (k_body_contrib / k_body_sum in step.cu).  The rest is a
// handful of FP64 operations per body and per surface particle, done on the
// host in the reference's order:
//   1. loads L0 at the stored wall state;
//   2. predicted (V*, w*) = (V, w) + L0 dt / (m, I);
//   3. loads L1 with the surface moving at (V*, w*), same frozen g;
//   4. rigid motion of the surface particles with the OLD (V, w)
//      (Rodrigues rotation in 3-D, planar rotation in 2-D);
//   5. centre and orientation advance with the OLD (V, w); (V, w) advance
//      with the Heun average (L0 + L1) / 2;
//   6. box-wall contact: one rigid shift that keeps the surface a gap of
//      0.4 dx inside the box, and zero normal velocity into the wall;
//   7. surface wall state from the new pose: normal, U_w = V + w x r,
//      mesh velocity = U_w.
// The surface particles' rows of position, wall state and mesh velocity go
// to the host and back through one gather/scatter each.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cases.h"
#include "ctx.h"

namespace alebgk {

namespace {

constexpr int kRowDoubles = 13;   // x y z | n(3) U_w(3) T_w | meshV(3)

__global__ void k_gather_surface(const int *__restrict__ list, int n,
                                 const double *__restrict__ pos,
                                 const double *__restrict__ wall,
                                 const double *__restrict__ meshv, double *__restrict__ out)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = list[t];
    double *o = out + (size_t)kRowDoubles * t;
    for (int q = 0; q < 3; ++q) o[q] = pos[3 * (size_t)i + q];
    for (int q = 0; q < 7; ++q) o[3 + q] = wall[7 * (size_t)i + q];
    for (int q = 0; q < 3; ++q) o[10 + q] = meshv[3 * (size_t)i + q];
}

__global__ void k_scatter_surface(const int *__restrict__ list, int n,
                                  const double *__restrict__ in, double *__restrict__ pos,
                                  double *__restrict__ wall, double *__restrict__ meshv)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = list[t];
    const double *r = in + (size_t)kRowDoubles * t;
    for (int q = 0; q < 3; ++q) pos[3 * (size_t)i + q] = r[q];
    for (int q = 0; q < 7; ++q) wall[7 * (size_t)i + q] = r[3 + q];
    for (int q = 0; q < 3; ++q) meshv[3 * (size_t)i + q] = r[10 + q];
}

// Device loads of every body: out[6 b + {Fx, Fy, Fz, Tx, Ty, Tz}].
cudaError_t loads(alebgk_ctx *c, int nb, const std::vector<Body> &B,
                  const std::vector<double> &area, double *out)
{
    double *io = c->d.bodyIO;
    std::vector<double> h(4 * kMaxBodyIO, 0.0);
    for (int b = 0; b < nb; ++b)
    {
        h[3 * b] = B[b].cx; h[3 * b + 1] = B[b].cy; h[3 * b + 2] = B[b].cz;
        h[3 * kMaxBodyIO + b] = area[b];
    }
    cudaError_t e = cudaMemcpyAsync(io, h.data(), h.size() * 8, cudaMemcpyHostToDevice,
                                    c->stream);
    if (e == cudaSuccess) e = launchBodyLoads(c, nb, io, io + 3 * kMaxBodyIO);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(out, c->d.bodyOut, 48 * (size_t)nb, cudaMemcpyDeviceToHost,
                            c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    return e;
}

}  // namespace

cudaError_t bodyStep(alebgk_ctx *c, int nb, alebgk_body *desc, const double *box, double dx,
                     double dt, std::string *err)
{
    const int dim = c->sp.dim;
    const bool d3 = dim == 3;
    std::vector<Body> B(nb);
    std::vector<double> I(nb), area(nb);   // given moment of inertia, area per point
    for (int b = 0; b < nb; ++b)
    {
        Body &r = B[b];
        const double *s = desc[b].state;
        r.kind = desc[b].kind;
        r.dim = (r.kind >= 2) ? 3 : 2;
        r.size = desc[b].size;
        r.rotates = desc[b].rotates != 0;
        r.cx = s[0]; r.cy = s[1]; r.cz = s[2];
        r.velx = s[3]; r.vely = s[4]; r.velz = s[5];
        r.angularVel = s[6]; r.omx = s[7]; r.omy = s[8]; r.omz = s[9];
        r.forcex = s[10]; r.forcey = s[11]; r.forcez = s[12];
        r.torque = s[13]; r.tqx = s[14]; r.tqy = s[15]; r.tqz = s[16];
        r.ox = s[17]; r.oy = s[18]; r.mass = s[19]; I[b] = s[20]; r.T = s[21];
        for (int k = 0; k < 9; ++k) r.Rm[k] = s[22 + k];
        area[b] = s[31];
    }

    // 1. loads at the current wall state
    std::vector<double> L0(6 * nb), L1(6 * nb);
    cudaError_t e = loads(c, nb, B, area, L0.data());
    if (e != cudaSuccess) { if (err) *err = "body loads L0"; return e; }

    // 2. predictor; 2-D spin lives in the z-component
    std::vector<double> pred(6 * kMaxBodyIO, 0.0);
    for (int b = 0; b < nb; ++b)
    {
        const Body &r = B[b];
        const double *F = &L0[6 * b];
        double *p = &pred[6 * b];
        p[0] = r.velx + F[0] * dt / r.mass;
        p[1] = r.vely + F[1] * dt / r.mass;
        p[2] = d3 ? r.velz + F[2] * dt / r.mass : 0.0;
        if (r.rotates)
        {
            if (d3)
            {
                p[3] = r.omx + F[3] * dt / I[b];
                p[4] = r.omy + F[4] * dt / I[b];
                p[5] = r.omz + F[5] * dt / I[b];
            }
            else
            {
                p[3] = 0.0; p[4] = 0.0;
                p[5] = r.angularVel + F[5] * dt / I[b];
            }
        }
        else
        {
            p[3] = d3 ? r.omx : 0.0;
            p[4] = d3 ? r.omy : 0.0;
            p[5] = d3 ? r.omz : r.angularVel;
        }
    }

    // 3. corrector loads with the surface at the predicted velocities
    double *io = c->d.bodyIO;
    std::vector<double> cen(3 * kMaxBodyIO, 0.0);
    for (int b = 0; b < nb; ++b)
    {
        cen[3 * b] = B[b].cx; cen[3 * b + 1] = B[b].cy; cen[3 * b + 2] = B[b].cz;
    }
    e = cudaMemcpyAsync(io + 4 * kMaxBodyIO, cen.data(), cen.size() * 8,
                        cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(io + 7 * kMaxBodyIO, pred.data(), pred.size() * 8,
                            cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess)
        e = launchSetSurfaceVelocity(c, nb, io + 4 * kMaxBodyIO, io + 7 * kMaxBodyIO);
    if (e == cudaSuccess) e = loads(c, nb, B, area, L1.data());
    if (e != cudaSuccess) { if (err) *err = "body loads L1"; return e; }

    // surface rows to the host
    const int ns = (int)c->surfHost.size();
    std::vector<double> rows((size_t)kRowDoubles * ns);
    double *rowsDev = io + kBodyIOHead;
    if (ns > 0)
    {
        k_gather_surface<<<(ns + 127) / 128, 128, 0, c->stream>>>(
            c->d.surfList, ns, c->d.pos, c->d.wall, c->d.meshv, rowsDev);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(rows.data(), rowsDev, rows.size() * 8, cudaMemcpyDeviceToHost,
                                c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { if (err) *err = "surface gather"; return e; }
    }
    auto bodyOf = [&](int t) { return c->bodyIdHost[c->surfHost[t]]; };

    // 4. rigid motion of the surface particles with the OLD body state
    for (int t = 0; t < ns; ++t)
    {
        const Body &r = B[bodyOf(t)];
        double *x = &rows[(size_t)kRowDoubles * t];
        const double rx = x[0] - r.cx, ry = x[1] - r.cy, rz = x[2] - r.cz;
        if (d3)
        {
            const double wmag = std::sqrt(r.omx * r.omx + r.omy * r.omy + r.omz * r.omz);
            double nxr = rx, nyr = ry, nzr = rz;
            if (wmag > 1e-300)
            {
                const double ax = r.omx / wmag, ay = r.omy / wmag, az = r.omz / wmag;
                const double th = wmag * dt, cs = std::cos(th), sn = std::sin(th);
                const double adotr = ax * rx + ay * ry + az * rz;
                const double crx = ay * rz - az * ry;
                const double cry = az * rx - ax * rz;
                const double crz = ax * ry - ay * rx;
                nxr = rx * cs + crx * sn + ax * adotr * (1.0 - cs);
                nyr = ry * cs + cry * sn + ay * adotr * (1.0 - cs);
                nzr = rz * cs + crz * sn + az * adotr * (1.0 - cs);
            }
            x[0] = r.cx + dt * r.velx + nxr;
            x[1] = r.cy + dt * r.vely + nyr;
            x[2] = r.cz + dt * r.velz + nzr;
        }
        else
        {
            const double th = r.angularVel * dt;
            x[0] = r.cx + dt * r.velx + std::cos(th) * rx - std::sin(th) * ry;
            x[1] = r.cy + dt * r.vely + std::sin(th) * rx + std::cos(th) * ry;
        }
    }

    // 5. Newton-Euler with the Heun-averaged loads
    for (int b = 0; b < nb; ++b)
    {
        Body &r = B[b];
        const double *F0 = &L0[6 * b], *F1 = &L1[6 * b];
        r.cx += dt * r.velx;
        r.cy += dt * r.vely;
        if (d3) r.cz += dt * r.velz;
        if (d3)
            r.rotate3(r.omx, r.omy, r.omz, dt);
        else
        {
            const double th = r.angularVel * dt;
            const double ox2 = r.ox, oy2 = r.oy;
            r.ox = std::cos(th) * ox2 - std::sin(th) * oy2;
            r.oy = std::sin(th) * ox2 + std::cos(th) * oy2;
        }
        r.forcex = 0.5 * (F0[0] + F1[0]);
        r.forcey = 0.5 * (F0[1] + F1[1]);
        r.forcez = 0.5 * (F0[2] + F1[2]);
        r.tqx = 0.5 * (F0[3] + F1[3]);
        r.tqy = 0.5 * (F0[4] + F1[4]);
        r.tqz = 0.5 * (F0[5] + F1[5]);
        r.torque = r.tqz;
        r.velx += r.forcex * dt / r.mass;
        r.vely += r.forcey * dt / r.mass;
        if (d3) r.velz += r.forcez * dt / r.mass;
        if (r.rotates)
        {
            if (d3)
            {
                r.omx += r.tqx * dt / I[b];
                r.omy += r.tqy * dt / I[b];
                r.omz += r.tqz * dt / I[b];
            }
            else
                r.angularVel += r.tqz * dt / I[b];
        }
        if (d3) r.angularVel = r.omz;
    }

    // 6. box-wall contact, from the body's own surface extent
    {
        const double gap = 0.4 * std::fabs(dx);
        const double xlo = std::min(box[0], box[1]), xhi = std::max(box[0], box[1]);
        const double ylo = std::min(box[2], box[3]), yhi = std::max(box[2], box[3]);
        const double zlo = std::min(box[4], box[5]), zhi = std::max(box[4], box[5]);
        for (int b = 0; b < nb; ++b)
        {
            double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
            int n = 0;
            for (int t = 0; t < ns; ++t)
            {
                if (bodyOf(t) != b) continue;
                const double *x = &rows[(size_t)kRowDoubles * t];
                for (int q = 0; q < 3; ++q)
                {
                    lo[q] = std::min(lo[q], x[q]);
                    hi[q] = std::max(hi[q], x[q]);
                }
                ++n;
            }
            if (n == 0) continue;
            const double sx = std::max(0.0, (xlo + gap) - lo[0]) - std::max(0.0, hi[0] - (xhi - gap));
            const double sy = std::max(0.0, (ylo + gap) - lo[1]) - std::max(0.0, hi[1] - (yhi - gap));
            const double sz = d3 ? std::max(0.0, (zlo + gap) - lo[2]) -
                                       std::max(0.0, hi[2] - (zhi - gap))
                                 : 0.0;
            if (sx == 0.0 && sy == 0.0 && sz == 0.0) continue;
            Body &r = B[b];
            r.cx += sx; r.cy += sy; r.cz += sz;
            for (int t = 0; t < ns; ++t)
            {
                if (bodyOf(t) != b) continue;
                double *x = &rows[(size_t)kRowDoubles * t];
                x[0] += sx; x[1] += sy; x[2] += sz;
            }
            if (sx > 0.0 && r.velx < 0.0) r.velx = 0.0;
            if (sx < 0.0 && r.velx > 0.0) r.velx = 0.0;
            if (sy > 0.0 && r.vely < 0.0) r.vely = 0.0;
            if (sy < 0.0 && r.vely > 0.0) r.vely = 0.0;
            if (d3)
            {
                if (sz > 0.0 && r.velz < 0.0) r.velz = 0.0;
                if (sz < 0.0 && r.velz > 0.0) r.velz = 0.0;
            }
        }
    }

    // 7. surface wall state from the new pose
    for (int t = 0; t < ns; ++t)
    {
        const Body &r = B[bodyOf(t)];
        double *x = &rows[(size_t)kRowDoubles * t];
        double *w = x + 3, *mv = x + 10;
        const double rx = x[0] - r.cx, ry = x[1] - r.cy, rz = x[2] - r.cz;
        double nz = 0.0;
        if (d3)
        {
            r.normal(x[0], x[1], x[2], &w[0], &w[1], &nz);
            w[2] = nz;
            w[3] = r.velx + r.omy * rz - r.omz * ry;
            w[4] = r.vely + r.omz * rx - r.omx * rz;
            w[5] = r.velz + r.omx * ry - r.omy * rx;
            mv[2] = w[5];
        }
        else
        {
            r.normal(x[0], x[1], r.cz, &w[0], &w[1], &nz);
            w[3] = r.velx - r.angularVel * ry;
            w[4] = r.vely + r.angularVel * rx;
        }
        mv[0] = w[3];
        mv[1] = w[4];
    }
    if (ns > 0)
    {
        e = cudaMemcpyAsync(rowsDev, rows.data(), rows.size() * 8, cudaMemcpyHostToDevice,
                            c->stream);
        if (e == cudaSuccess)
        {
            k_scatter_surface<<<(ns + 127) / 128, 128, 0, c->stream>>>(
                c->d.surfList, ns, rowsDev, c->d.pos, c->d.wall, c->d.meshv);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) { if (err) *err = "surface scatter"; return e; }
    }

    for (int b = 0; b < nb; ++b)
    {
        const Body &r = B[b];
        double *s = desc[b].state;
        const double v[22] = {r.cx, r.cy, r.cz, r.velx, r.vely, r.velz, r.angularVel,
                              r.omx, r.omy, r.omz, r.forcex, r.forcey, r.forcez,
                              r.torque, r.tqx, r.tqy, r.tqz, r.ox, r.oy, r.mass,
                              I[b], r.T};
        std::copy(v, v + 22, s);
        for (int k = 0; k < 9; ++k) s[22 + k] = r.Rm[k];
        s[31] = area[b];
    }
    return cudaSuccess;
}

}  // namespace alebgk
