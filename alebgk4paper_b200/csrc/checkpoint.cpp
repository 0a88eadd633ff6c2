// checkpoint.cpp -- restart files in the reference's checkpoint layout
// (Core/Checkpoint.hpp:37-236: magic "ALEBGK01", version 1).
//
// File: one header, one record per particle (geometry, macros, wall state),
// N * gStride FP64 values of g in particle order, one record per rigid body;
// raw little-endian POD with the natural alignment of the records.  The
// layout is a format, so the records below mirror the reference's field
// for field; the code around them is this library's.
//
// Saving streams g off the device: the FP64 image of the distribution is
// made on the device (k_convert_out applies the stored-state scale), then
// copied in chunks through two pinned host buffers so that the copy of one
// chunk overlaps the file write of the previous one.  The file is written
// to path.tmp and renamed, so an interrupted save never replaces the last
// good checkpoint.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"

namespace alebgk {

namespace {

constexpr uint64_t kMagic = 0x414c4542474b3031ULL;   // "ALEBGK01"
constexpr uint32_t kVersion = 1;

struct Header
{
    uint64_t magic;
    uint32_t version;
    uint32_t dim;
    uint64_t N;
    uint64_t gStride;
    uint64_t step;
    double t;
    uint32_t nBodies;
    uint32_t pad;
};

struct PRec
{
    double x, y, z;
    double ux, uy, uz, T, rho, p;
    double meshVx, meshVy, meshVz;
    double wnx, wny, wnz, wUx, wUy, wUz, wT;
    double vlo, vhi, dv_local;
    int32_t Nv_local, dim, bodyId, voxel;
    uint8_t boundary, validg, moodFlag, pad;
};

struct BRec
{
    double cx, cy, cz;
    double velx, vely, velz;
    double angularVel, omx, omy, omz;
    double forcex, forcey, forcez;
    double torque, tqx, tqy, tqz;
    double ox, oy;
    double Rm[9];
    int32_t dim;
    uint8_t rotates, pad[3];
};

static_assert(sizeof(Header) == 56, "checkpoint header layout");
static_assert(sizeof(PRec) == 200, "checkpoint particle record layout");
static_assert(sizeof(BRec) == 232, "checkpoint body record layout");

struct File
{
    FILE *f = nullptr;
    explicit File(FILE *f_) : f(f_) {}
    ~File() { if (f) std::fclose(f); }
};

bool readHeader(FILE *f, Header &h, std::string *err)
{
    if (std::fread(&h, sizeof h, 1, f) != 1 || h.magic != kMagic || h.version != kVersion)
    {
        if (err) *err = "not a version-1 ALEBGK01 checkpoint";
        return false;
    }
    return true;
}

}  // namespace

int checkpointHeader(const char *path, alebgk_ckpt_header *out, std::string *err)
{
    File fh(std::fopen(path, "rb"));
    if (!fh.f) { if (err) *err = std::string("cannot open ") + path; return ALEBGK_EINVAL; }
    Header h{};
    if (!readHeader(fh.f, h, err)) return ALEBGK_EINVAL;
    out->N = h.N; out->gstride = h.gStride; out->step = h.step; out->t = h.t;
    out->dim = h.dim; out->nbodies = h.nBodies;
    return ALEBGK_OK;
}

int checkpointRead(const char *path, const alebgk_ckpt_header *expect, alebgk_cloud *cl,
                   int *voxel, alebgk_body *bodies, std::string *err)
{
    File fh(std::fopen(path, "rb"));
    if (!fh.f) { if (err) *err = std::string("cannot open ") + path; return ALEBGK_EINVAL; }
    Header h{};
    if (!readHeader(fh.f, h, err)) return ALEBGK_EINVAL;
    // Refuse a file of another shape rather than read past a buffer.
    if (h.N != expect->N || h.gStride != expect->gstride || h.dim != expect->dim ||
        h.nBodies != expect->nbodies)
    {
        if (err)
            *err = "checkpoint shape N=" + std::to_string(h.N) + " gStride=" +
                   std::to_string(h.gStride) + " dim=" + std::to_string(h.dim) + " bodies=" +
                   std::to_string(h.nBodies) + " differs from the expected one";
        return ALEBGK_EINVAL;
    }
    const size_t N = h.N, gs = h.gStride;
    std::vector<PRec> pr(N);
    if (std::fread(pr.data(), sizeof(PRec), N, fh.f) != N)
    {
        if (err) *err = "truncated particle records";
        return ALEBGK_EINVAL;
    }
    for (size_t i = 0; i < N; ++i)
    {
        const PRec &r = pr[i];
        if (cl->xyz) { cl->xyz[3 * i] = r.x; cl->xyz[3 * i + 1] = r.y; cl->xyz[3 * i + 2] = r.z; }
        if (cl->meshv)
        {
            cl->meshv[3 * i] = r.meshVx; cl->meshv[3 * i + 1] = r.meshVy;
            cl->meshv[3 * i + 2] = r.meshVz;
        }
        if (cl->wall)
        {
            double *w = cl->wall + 7 * i;
            w[0] = r.wnx; w[1] = r.wny; w[2] = r.wnz;
            w[3] = r.wUx; w[4] = r.wUy; w[5] = r.wUz; w[6] = r.wT;
        }
        if (cl->boundary) cl->boundary[i] = r.boundary != 0;
        if (cl->body_id) cl->body_id[i] = r.bodyId;
        if (cl->macro)
        {
            double *q = cl->macro + 7 * i;
            q[0] = r.rho; q[1] = r.ux; q[2] = r.uy; q[3] = r.uz;
            q[4] = r.T; q[5] = r.p; q[6] = r.moodFlag ? 1.0 : 0.0;
        }
        if (voxel) voxel[i] = r.voxel;
    }
    if (cl->g)
    {
        if (std::fread(cl->g, sizeof(double), N * gs, fh.f) != N * gs)
        {
            if (err) *err = "truncated distribution";
            return ALEBGK_EINVAL;
        }
    }
    else if (std::fseek(fh.f, (long)(N * gs * sizeof(double)), SEEK_CUR) != 0)
    {
        if (err) *err = "truncated distribution";
        return ALEBGK_EINVAL;
    }
    if (h.nBodies)
    {
        std::vector<BRec> br(h.nBodies);
        if (std::fread(br.data(), sizeof(BRec), h.nBodies, fh.f) != h.nBodies)
        {
            if (err) *err = "truncated body records";
            return ALEBGK_EINVAL;
        }
        for (size_t b = 0; bodies && b < h.nBodies; ++b)
        {
            const BRec &r = br[b];
            double *s = bodies[b].state;
            const double v[19] = {r.cx, r.cy, r.cz, r.velx, r.vely, r.velz, r.angularVel,
                                  r.omx, r.omy, r.omz, r.forcex, r.forcey, r.forcez,
                                  r.torque, r.tqx, r.tqy, r.tqz, r.ox, r.oy};
            std::memcpy(s, v, sizeof v);
            std::memcpy(s + 22, r.Rm, sizeof r.Rm);
            bodies[b].rotates = r.rotates != 0;
        }
    }
    return ALEBGK_OK;
}

int checkpointSave(alebgk_ctx *c, const char *path, int64_t step, double t, const double *vgrid,
                   const int *voxel, int nbodies, const alebgk_body *bodies, std::string *err)
{
    const StepParams &p = c->sp;
    const size_t N = p.N, gs = p.gs;
    const std::string tmp = std::string(path) + ".tmp";
    File fh(std::fopen(tmp.c_str(), "wb"));
    if (!fh.f) { if (err) *err = "cannot open " + tmp; return ALEBGK_EINVAL; }

    // Per-particle state from the device.
    std::vector<double> pos(3 * N), mv(3 * N), wall(7 * N), mac(7 * N);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(pos.data(), c->d.pos, 24 * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(mv.data(), c->d.meshv, 24 * N, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(wall.data(), c->d.wall, 56 * N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { if (err) *err = cudaGetErrorString(e); return ALEBGK_ECUDA; }
    if (int rc = alebgk_download_moments(c, mac.data())) { if (err) *err = c->err; return rc; }

    Header h{};
    h.magic = kMagic; h.version = kVersion;
    h.dim = (uint32_t)p.dim; h.N = N; h.gStride = gs;
    h.step = (uint64_t)step; h.t = t; h.nBodies = (uint32_t)nbodies;
    const double vlo = vgrid ? vgrid[0] : p.vmin;
    const double vhi = vgrid ? vgrid[1] : p.vmin + (p.Nv - 1) * p.dv;
    const double dvl = vgrid ? vgrid[2] : p.dv;
    std::vector<PRec> pr(N);
    for (size_t i = 0; i < N; ++i)
    {
        PRec &r = pr[i];
        std::memset(&r, 0, sizeof r);
        r.x = pos[3 * i]; r.y = pos[3 * i + 1]; r.z = pos[3 * i + 2];
        const double *q = &mac[7 * i];
        r.rho = q[0]; r.ux = q[1]; r.uy = q[2]; r.uz = q[3]; r.T = q[4]; r.p = q[5];
        r.meshVx = mv[3 * i]; r.meshVy = mv[3 * i + 1]; r.meshVz = mv[3 * i + 2];
        const double *w = &wall[7 * i];
        r.wnx = w[0]; r.wny = w[1]; r.wnz = w[2];
        r.wUx = w[3]; r.wUy = w[4]; r.wUz = w[5]; r.wT = w[6];
        r.vlo = vlo; r.vhi = vhi; r.dv_local = dvl;
        r.Nv_local = p.Nv; r.dim = p.dim;
        r.bodyId = c->bodyIdHost[i];
        r.voxel = voxel ? voxel[i] : 0;
        r.boundary = c->boundaryHost[i] ? 1 : 0;
        r.validg = 1;
        r.moodFlag = q[6] != 0.0 ? 1 : 0;
    }
    bool ok = std::fwrite(&h, sizeof h, 1, fh.f) == 1 &&
              std::fwrite(pr.data(), sizeof(PRec), N, fh.f) == N;

    // g: FP64 image on the device, then chunked copies through two pinned
    // buffers, each copy overlapping the write of the other buffer.
    if (ok)
    {
        e = launchConvertOut(c, c->d.stage, c->cur);
        const size_t chunkRows = std::max<size_t>(1, (size_t)(8u << 20) / (gs * 8));
        double *pin[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        for (int b = 0; b < 2 && e == cudaSuccess; ++b)
        {
            e = cudaMallocHost(&pin[b], chunkRows * gs * 8);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming);
        }
        const size_t nChunks = (N + chunkRows - 1) / chunkRows;
        auto issue = [&](size_t ch) {
            const size_t r0 = ch * chunkRows, rows = std::min(chunkRows, N - r0);
            cudaError_t ee = cudaMemcpyAsync(pin[ch & 1], c->d.stage + r0 * gs, rows * gs * 8,
                                             cudaMemcpyDeviceToHost, c->stream);
            if (ee == cudaSuccess) ee = cudaEventRecord(done[ch & 1], c->stream);
            return ee;
        };
        if (e == cudaSuccess && nChunks > 0) e = issue(0);
        for (size_t ch = 0; ch < nChunks && e == cudaSuccess && ok; ++ch)
        {
            if (ch + 1 < nChunks) e = issue(ch + 1);
            if (e == cudaSuccess) e = cudaEventSynchronize(done[ch & 1]);
            if (e != cudaSuccess) break;
            const size_t rows = std::min(chunkRows, N - ch * chunkRows);
            ok = std::fwrite(pin[ch & 1], 8, rows * gs, fh.f) == rows * gs;
            // the buffer just written is reused by chunk ch + 2, issued next round
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        for (int b = 0; b < 2; ++b)
        {
            if (pin[b]) cudaFreeHost(pin[b]);
            if (done[b]) cudaEventDestroy(done[b]);
        }
        if (e != cudaSuccess)
        {
            if (err) *err = std::string("checkpoint g: ") + cudaGetErrorString(e);
            std::fclose(fh.f); fh.f = nullptr;
            std::remove(tmp.c_str());
            return ALEBGK_ECUDA;
        }
    }
    if (ok && nbodies > 0)
    {
        std::vector<BRec> br(nbodies);
        for (int b = 0; b < nbodies; ++b)
        {
            BRec &r = br[b];
            std::memset(&r, 0, sizeof r);
            const double *s = bodies[b].state;
            r.cx = s[0]; r.cy = s[1]; r.cz = s[2];
            r.velx = s[3]; r.vely = s[4]; r.velz = s[5];
            r.angularVel = s[6]; r.omx = s[7]; r.omy = s[8]; r.omz = s[9];
            r.forcex = s[10]; r.forcey = s[11]; r.forcez = s[12];
            r.torque = s[13]; r.tqx = s[14]; r.tqy = s[15]; r.tqz = s[16];
            r.ox = s[17]; r.oy = s[18];
            std::memcpy(r.Rm, s + 22, sizeof r.Rm);
            r.dim = bodies[b].kind >= 2 ? 3 : 2;
            r.rotates = bodies[b].rotates ? 1 : 0;
        }
        ok = std::fwrite(br.data(), sizeof(BRec), nbodies, fh.f) == (size_t)nbodies;
    }
    ok = ok && std::fflush(fh.f) == 0;
    std::fclose(fh.f);
    fh.f = nullptr;
    if (!ok)
    {
        std::remove(tmp.c_str());
        if (err) *err = "write failed for " + tmp;
        return ALEBGK_EINVAL;
    }
    std::remove(path);
    if (std::rename(tmp.c_str(), path) != 0)
    {
        if (err) *err = std::string("rename failed for ") + path;
        return ALEBGK_EINVAL;
    }
    return ALEBGK_OK;
}

}  // namespace alebgk
