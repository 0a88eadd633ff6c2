// fields.cpp -- field output: the reference's ASCII VTK frames, interior
// diagnostics, timeseries rows and step line (Core/Output.hpp:17-115), and a
// full-precision binary field dump.
//
// The VTK frame is text: 12 numbers per particle, each printed as the
// reference's output stream prints a double once std::scientific is set
// (six decimals, printf's %.6e).  The numbers are formatted in parallel, in
// chunks of particles per section, and the chunks written in order, so the
// file is the reference's byte for byte for the same data.
#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "ctx.h"

using namespace alebgk;

namespace {

int failc(alebgk_ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

constexpr int kChunk = 4096;   // particles per formatting chunk

// Formats rows [0, N) of one section into per-chunk strings in parallel.
// row(i, buf) writes particle i's line into buf and returns its length.
template <typename Row>
std::vector<std::string> formatRows(int N, Row row)
{
    const int nch = (N + kChunk - 1) / kChunk;
    std::vector<std::string> out(nch);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ch = 0; ch < nch; ++ch)
    {
        std::string &s = out[ch];
        const int lo = ch * kChunk, hi = std::min(N, lo + kChunk);
        s.reserve((size_t)(hi - lo) * 48);
        char buf[128];
        for (int i = lo; i < hi; ++i)
        {
            const int n = row(i, buf);
            s.append(buf, (size_t)n);
        }
    }
    return out;
}

bool putAll(FILE *f, const std::vector<std::string> &parts)
{
    for (const std::string &s : parts)
        if (!s.empty() && std::fwrite(s.data(), 1, s.size(), f) != s.size()) return false;
    return true;
}

// Host copies of the context's positions and moments (N*3, N*7).
int downloadFields(alebgk_ctx *c, std::vector<double> &xyz, std::vector<double> &macro)
{
    const size_t N = c->sp.N;
    xyz.resize(3 * N);
    macro.resize(7 * N);
    cudaError_t e = cudaSetDevice(c->cfg.device);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e == cudaSuccess) e = cudaMemcpy(xyz.data(), c->d.pos, 24 * N, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return failc(c, ALEBGK_ECUDA, std::string("field download: ") + cudaGetErrorString(e));
    return alebgk_download_moments(c, macro.data());
}

constexpr char kFieldsMagic[8] = {'A', 'L', 'B', 'G', 'K', 'F', 'L', 'D'};
constexpr uint32_t kFieldsVersion = 1;

}  // namespace

extern "C" {

int alebgk_vtk_write_host(const char *path, int N, const double *xyz, const double *macro,
                          const int *boundary, int Nv, double time)
{
    if (!path || N < 0 || (N > 0 && (!xyz || !macro || !boundary))) return ALEBGK_EINVAL;
    FILE *f = std::fopen(path, "wb");
    if (!f) return ALEBGK_EIO;
    // Header lines (Output.hpp:27-31); the title's time is the first number
    // printed in scientific form.
    bool ok = std::fprintf(f,
                           "# vtk DataFile Version 3.0\nALEBGK t=%.6e\nASCII\n"
                           "DATASET UNSTRUCTURED_GRID\nPOINTS %d double\n",
                           time, N) > 0;
    if (ok)
        ok = putAll(f, formatRows(N, [&](int i, char *b) {
                        return std::snprintf(b, 128, "%.6e %.6e %.6e\n", xyz[3 * (size_t)i],
                                             xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]);
                    }));
    if (ok) ok = std::fprintf(f, "CELLS 0 0\nCELL_TYPES 0\nPOINT_DATA %d\n", N) > 0;
    // Scalars in the reference's order (Output.hpp:40-45): rho, T, p,
    // Nv_local, moodFlag, boundary.
    struct Scalar { const char *name; int kind; };
    const Scalar scalars[6] = {{"rho", 0}, {"T", 4}, {"p", 5}, {"Nv_local", -1},
                               {"moodFlag", 6}, {"boundary", -2}};
    for (const Scalar &sc : scalars)
    {
        if (!ok) break;
        ok = std::fprintf(f, "SCALARS %s double 1\nLOOKUP_TABLE default\n", sc.name) > 0;
        if (!ok) break;
        ok = putAll(f, formatRows(N, [&](int i, char *b) {
                        // moodFlag and boundary are the reference's bools
                        const double v = sc.kind == 6 ? (macro[7 * (size_t)i + 6] != 0.0 ? 1.0 : 0.0)
                                         : sc.kind >= 0 ? macro[7 * (size_t)i + sc.kind]
                                         : sc.kind == -1 ? (double)Nv
                                                         : (boundary[i] ? 1.0 : 0.0);
                        return std::snprintf(b, 128, "%.6e\n", v);
                    }));
    }
    if (ok) ok = std::fprintf(f, "VECTORS velocity double\n") > 0;
    if (ok)
        ok = putAll(f, formatRows(N, [&](int i, char *b) {
                        const double *m = macro + 7 * (size_t)i;
                        return std::snprintf(b, 128, "%.6e %.6e %.6e\n", m[1], m[2], m[3]);
                    }));
    if (std::fclose(f) != 0) ok = false;
    return ok ? ALEBGK_OK : ALEBGK_EIO;
}

int alebgk_write_vtk(alebgk_ctx *c, const char *outdir, int step, double time)
{
    if (!c || !outdir) return failc(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    std::vector<double> xyz, macro;
    const int rc = downloadFields(c, xyz, macro);
    if (rc != ALEBGK_OK) return rc;
    // the reference's frame name (Output.hpp:20-22)
    char name[32];
    std::snprintf(name, sizeof name, "/output_%06d.vtk", step);
    const std::string path = std::string(outdir) + name;
    const int w = alebgk_vtk_write_host(path.c_str(), c->sp.N, xyz.data(), macro.data(),
                                        c->boundaryHost.data(), c->cfg.Nv, time);
    return w == ALEBGK_OK ? ALEBGK_OK : failc(c, w, "cannot write " + path);
}

int alebgk_diagnostics_host(int N, const double *macro, const int *boundary, alebgk_diag *out)
{
    if (!out || N < 0 || (N > 0 && (!macro || !boundary))) return ALEBGK_EINVAL;
    // Interior particles in particle order (Output.hpp:66-85).
    alebgk_diag d{};
    for (int i = 0; i < N; ++i)
    {
        if (boundary[i]) continue;
        const double *m = macro + 7 * (size_t)i;
        d.rho_avg += m[0];
        d.KE += 0.5 * m[0] * (m[1] * m[1] + m[2] * m[2] + m[3] * m[3]);
        d.T_avg += m[4];
        d.p_avg += m[5];
        d.mood_count += m[6] != 0.0 ? 1 : 0;
        d.n++;
    }
    if (d.n > 0)
    {
        const double n = d.n;
        d.rho_avg /= n;
        d.KE /= n;
        d.T_avg /= n;
        d.p_avg /= n;
    }
    *out = d;
    return ALEBGK_OK;
}

int alebgk_diagnostics(alebgk_ctx *c, alebgk_diag *out)
{
    if (!c || !out) return failc(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    std::vector<double> macro(7 * (size_t)c->sp.N);
    const int rc = alebgk_download_moments(c, macro.data());
    if (rc != ALEBGK_OK) return rc;
    return alebgk_diagnostics_host(c->sp.N, macro.data(), c->boundaryHost.data(), out);
}

int alebgk_write_timeseries(const char *path, double t, const alebgk_diag *d, int header)
{
    if (!path || !d) return ALEBGK_EINVAL;
    FILE *f = std::fopen(path, header ? "w" : "a");
    if (!f) return ALEBGK_EIO;
    bool ok = true;
    if (header) ok = std::fputs("t,rho_avg,KE,T_avg,p_avg,mood_count\n", f) >= 0;
    // Output.hpp:101-106: the doubles in scientific form, the count as an integer
    if (ok)
        ok = std::fprintf(f, "%.6e,%.6e,%.6e,%.6e,%.6e,%d\n", t, d->rho_avg, d->KE, d->T_avg,
                          d->p_avg, d->mood_count) > 0;
    if (std::fclose(f) != 0) ok = false;
    return ok ? ALEBGK_OK : ALEBGK_EIO;
}

int alebgk_format_step(char *buf, size_t len, int step, double t, double dt,
                       const alebgk_diag *d)
{
    if (!buf || !d || len == 0) return ALEBGK_EINVAL;
    // the columns of printStep (Output.hpp:111-115)
    const int n = std::snprintf(buf, len, "Step%6d|t=%9.3e|dt=%7.2e|rho=%7.4f|T=%7.4f|KE=%7.3e|MOOD=%3d\n",
                                step, t, dt, d->rho_avg, d->T_avg, d->KE, d->mood_count);
    return (n >= 0 && (size_t)n < len) ? ALEBGK_OK : ALEBGK_EINVAL;
}

int alebgk_write_fields(alebgk_ctx *c, const char *path, int64_t step, double t)
{
    if (!c || !path) return failc(c, ALEBGK_EINVAL, "null argument");
    if (!c->uploaded) return failc(c, ALEBGK_ESTATE, "upload the cloud first");
    std::vector<double> xyz, macro;
    const int rc = downloadFields(c, xyz, macro);
    if (rc != ALEBGK_OK) return rc;
    alebgk_fields_header h{};
    std::memcpy(h.magic, kFieldsMagic, 8);
    h.version = kFieldsVersion;
    h.dim = (uint32_t)c->cfg.dim;
    h.N = (uint64_t)c->sp.N;
    h.step = step;
    h.t = t;
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return failc(c, ALEBGK_EIO, "cannot open " + tmp);
    const size_t N = h.N;
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
              std::fwrite(xyz.data(), 8, 3 * N, f) == 3 * N &&
              std::fwrite(macro.data(), 8, 7 * N, f) == 7 * N &&
              std::fwrite(c->boundaryHost.data(), 4, N, f) == N;
    if (std::fclose(f) != 0) ok = false;
    if (!ok || std::rename(tmp.c_str(), path) != 0)
    {
        std::remove(tmp.c_str());
        return failc(c, ALEBGK_EIO, std::string("cannot write ") + path);
    }
    return ALEBGK_OK;
}

int alebgk_read_fields(const char *path, alebgk_fields_header *out, double *xyz, double *macro,
                       int *boundary)
{
    if (!path || !out) return ALEBGK_EINVAL;
    FILE *f = std::fopen(path, "rb");
    if (!f) return ALEBGK_EIO;
    alebgk_fields_header h{};
    bool ok = std::fread(&h, sizeof h, 1, f) == 1 && std::memcmp(h.magic, kFieldsMagic, 8) == 0 &&
              h.version == kFieldsVersion;
    if (ok) *out = h;
    const size_t N = ok ? (size_t)h.N : 0;
    auto section = [&](void *dst, size_t elem, size_t count) {
        if (!ok) return;
        if (dst) ok = std::fread(dst, elem, count, f) == count;
        else ok = std::fseek(f, (long)(elem * count), SEEK_CUR) == 0;
    };
    section(xyz, 8, 3 * N);
    section(macro, 8, 7 * N);
    section(boundary, 4, N);
    std::fclose(f);
    return ok ? ALEBGK_OK : ALEBGK_EIO;
}

}  // extern "C"
