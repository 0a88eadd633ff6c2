/*
 * alebgk_oracle.c -- TEST INFRASTRUCTURE ONLY (see alebgk_oracle.h).
 *
 * FP64 CPU restatement of the reference's step, function by function, each
 * citing the reference file:line it follows.  Arithmetic is kept in the same
 * order as the reference wherever that is cheap, so that the oracle agrees
 * with the compiled reference to rounding.
 */
#include "alebgk_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.14159265358979323846
#define MLS_MAX_N 10

void ora_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* The reference is built with -march=native (CMakeLists.txt:169-174), and
 * GCC contracts its expressions into FMAs on any FMA-capable x86-64.  Where
 * an exact tie decides a branch -- the wall-normal velocity cn of an edge or
 * corner particle, whose 45-degree normal makes cn vanish in plain
 * arithmetic -- the contracted form decides, so it is written out here:
 *   vlo + i*dv                 -> fma(i, dv, vlo)
 *   a*b + c*d                  -> fma(a, b, c*d)
 *   a*b + c*d + e*f            -> fma(e, f, fma(a, b, c*d))   (transport)
 * In the diffuse-wall loops (DiffuseWall.cpp:58,83) the wall state sits in
 * locals, so the z-term is hoisted out of the inner loop before contraction
 * and only the x-term is fused:
 *   a*b + c*d + e*f            -> fma(a, b, c*d) + e*f        (wall BC)
 * (both checked against the compiled reference, g++ 13 -O3 -march=x86-64-v4,
 * by comparing every wall particle's BC output). */
static double node_v(int i, double dv, double vlo) { return fma((double)i, dv, vlo); }

static double wall_cn(int ndim, double vx, double vy, double vz, const double *w)
{
    double a = vx - w[3], c = vy - w[4];
    if (ndim == 3) return fma(vz - w[5], w[2], fma(a, w[0], c * w[1]));
    return fma(a, w[0], c * w[1]);
}

static double bc_cn(int ndim, double vx, double vy, double vz, const double *w)
{
    double a = vx - w[3], c = vy - w[4];
    if (ndim == 3) return fma(a, w[0], c * w[1]) + (vz - w[5]) * w[2];
    return fma(a, w[0], c * w[1]);
}

/* Core/MLSBasis.hpp:46-49 */
static double min_image(double d, double L) { return d - L * round(d / L); }

/* Core/MLSBasis.hpp:142-148 */
static double weight_sq(double r2, double h)
{
    double q2 = r2 / (h * h);
    if (q2 >= 1.0) return 0.0;
    double w = 1.0 - q2;
    return w * w;
}

/* Core/MLSBasis.hpp:158-195 */
static int fill_basis(double dx, double dy, double dz, int ndim, double h,
                      double *b, int order)
{
    double sx = dx / h, sy = dy / h, sz = dz / h;
    b[0] = 1.0; b[1] = sx; b[2] = sy;
    if (ndim == 2)
    {
        if (order >= 2) { b[3] = sx * sx; b[4] = sx * sy; b[5] = sy * sy; return 6; }
        return 3;
    }
    b[3] = sz;
    if (order >= 2)
    {
        b[4] = sx * sx; b[5] = sy * sy; b[6] = sz * sz;
        b[7] = sx * sy; b[8] = sx * sz; b[9] = sy * sz;
        return 10;
    }
    return 4;
}

static int basis_size(int ndim, int order)
{
    if (ndim == 2) return order >= 2 ? 6 : 3;
    return order >= 2 ? 10 : 4;
}

/* MLSTransport/MLSTransport.cpp:20-62 -- partial-pivot elimination on the
 * augmented matrix, |pivot| < 1e-30 columns skipped, their unknowns 0. */
static void solve_linear(const double *A, const double *b, double *sol, int n)
{
    double aug[MLS_MAX_N][MLS_MAX_N + 1];
    for (int i = 0; i < n; ++i)
    {
        for (int j = 0; j < n; ++j) aug[i][j] = A[i * n + j];
        aug[i][n] = b[i];
    }
    for (int col = 0; col < n; ++col)
    {
        int piv = col;
        double mx = fabs(aug[col][col]);
        for (int row = col + 1; row < n; ++row)
            if (fabs(aug[row][col]) > mx) { mx = fabs(aug[row][col]); piv = row; }
        if (piv != col)
            for (int j = 0; j <= n; ++j)
            {
                double t = aug[col][j]; aug[col][j] = aug[piv][j]; aug[piv][j] = t;
            }
        double d = aug[col][col];
        if (fabs(d) < 1.0e-30) continue;
        for (int row = col + 1; row < n; ++row)
        {
            double f = aug[row][col] / d;
            for (int j = col; j <= n; ++j) aug[row][j] -= f * aug[col][j];
        }
    }
    for (int i = n - 1; i >= 0; --i)
    {
        double s = aug[i][n];
        for (int j = i + 1; j < n; ++j) s -= aug[i][j] * sol[j];
        sol[i] = (fabs(aug[i][i]) > 1.0e-30) ? s / aug[i][i] : 0.0;
    }
}

/* MLSTransport/MLSTransport.cpp:88-311 -- compute pass (writes gt from g). */
void ora_transport(ora_cloud *c, int mls_order, int only_flagged, int *nfix)
{
    const int N = c->N, ndim = c->dim, Nv = c->Nv, Nv2 = Nv * Nv;
    const double h = c->h, dt = c->dt;
    int fixes = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : fixes)
    for (int i = 0; i < N; ++i)
    {
        if (only_flagged && !c->flag[i]) continue;
        const int bnd = c->boundary[i];
        const int order = (bnd || only_flagged) ? 1 : mls_order;
        const int poly = basis_size(ndim, order);
        const int nn = c->nnb[i];
        const int *nb = c->nbr + (size_t)i * ORA_MAX_NEIGH;
        const double *w = c->wall + 7 * (size_t)i;
        const double *mv = c->meshv + 3 * (size_t)i;
        const double xi = c->xyz[3 * i], yi = c->xyz[3 * i + 1], zi = c->xyz[3 * i + 2];
        double *gti = c->gt + (size_t)i * c->gs;
        const double *gi = c->g + (size_t)i * c->gs;
        memcpy(gti, gi, sizeof(double) * c->gs);
        double A[MLS_MAX_N * MLS_MAX_N], b1[MLS_MAX_N], b2[MLS_MAX_N];
        double s1[MLS_MAX_N], s2[MLS_MAX_N], bas[MLS_MAX_N];
        const int nk = (ndim == 3) ? Nv * Nv * Nv : Nv2;
        for (int k = 0; k < nk; ++k)
        {
            const int iv = k % Nv, jv = (k / Nv) % Nv, kv = (ndim == 3) ? k / Nv2 : 0;
            const double vx = node_v(iv, c->dv, c->vmin);
            const double vy = node_v(jv, c->dv, c->vmin);
            const double vz = node_v(kv, c->dv, c->vmin);
            if (bnd)
            {
                /* 3-D: MLSTransport.cpp:144-150; 2-D wallCN: :73-78, 213-218 */
                if (wall_cn(ndim, vx, vy, vz, w) >= 0.0) continue;
            }
            const double xf = xi - (vx - mv[0]) * dt;
            const double yf = yi - (vy - mv[1]) * dt;
            const double zf = zi - (vz - mv[2]) * dt;
            for (int q = 0; q < poly * poly; ++q) A[q] = 0.0;
            for (int q = 0; q < poly; ++q) b1[q] = b2[q] = 0.0;
            int has = 0;
            for (int s = 0; s < nn; ++s)
            {
                const int j = nb[s];
                double dx = c->xyz[3 * j] - xf, dy = c->xyz[3 * j + 1] - yf;
                double dz = (ndim == 3) ? c->xyz[3 * j + 2] - zf : 0.0;
                if (c->periodic[0]) dx = min_image(dx, c->L[0]);
                if (c->periodic[1]) dy = min_image(dy, c->L[1]);
                if (ndim == 3 && c->periodic[2]) dz = min_image(dz, c->L[2]);
                double r2 = (ndim == 3) ? dx * dx + dy * dy + dz * dz : dx * dx + dy * dy;
                double wt = weight_sq(r2, h);
                if (wt < 1.0e-30) continue;
                fill_basis(dx, dy, dz, ndim, h, bas, order);
                for (int p1 = 0; p1 < poly; ++p1)
                    for (int p2 = 0; p2 < poly; ++p2) A[p1 * poly + p2] += wt * bas[p1] * bas[p2];
                const double *gj = c->g + (size_t)j * c->gs;
                const double f1 = gj[k];
                for (int q = 0; q < poly; ++q) b1[q] += wt * bas[q] * f1;
                if (ndim == 2)
                {
                    const double f2 = gj[k + Nv2];
                    for (int q = 0; q < poly; ++q) b2[q] += wt * bas[q] * f2;
                }
                has = 1;
            }
            if (!has) continue;
            solve_linear(A, b1, s1, poly);
            gti[k] = s1[0];
            if (ndim == 2)
            {
                solve_linear(A, b2, s2, poly);
                gti[k + Nv2] = s2[0];
            }
        }
        /* positivity: 3-D :189-201, 2-D :283-309 */
        const int nm = (ndim == 3) ? nk : Nv2;
        double mp = 0.0, mn = 0.0;
        for (int k = 0; k < nm; ++k)
        {
            double v = gti[k];
            if (v >= 0.0) mp += v; else mn += v;
        }
        if (mn < -1.0e-30 && mp > 1.0e-30 && (mp + mn) > 0.0)
        {
            double s = (mp + mn) / mp;
            ++fixes;
            for (int k = 0; k < nm; ++k)
            {
                if (gti[k] < 0.0)
                {
                    gti[k] = 0.0;
                    if (ndim == 2) gti[k + Nv2] = 0.0;
                }
                else
                {
                    gti[k] *= s;
                    if (ndim == 2) gti[k + Nv2] *= s;
                }
            }
        }
    }
    if (nfix) *nfix = fixes;
}

/* MLSTransport/MLSTransport.cpp:325-379 */
int ora_check_pad(ora_cloud *c)
{
    int nfail = 0;
    const int Nv = c->Nv;
    const int nm = (c->dim == 3) ? Nv * Nv * Nv : Nv * Nv;
    const double dvN = (c->dim == 3) ? c->dv * c->dv * c->dv : c->dv * c->dv;
    for (int i = 0; i < c->N; ++i)
    {
        c->flag[i] = 0;
        c->macro[7 * (size_t)i + 6] = 0.0;
        if (c->boundary[i]) continue;
        const double *gt = c->gt + (size_t)i * c->gs;
        double m = 0.0;
        int bad = 0;
        for (int k = 0; k < nm; ++k)
        {
            if (!isfinite(gt[k])) { bad = 1; break; }
            m += gt[k];
        }
        if (bad || m <= 0.0) { c->flag[i] = 1; nfail++; continue; }
        double rn = m * dvN, lo = INFINITY, hi = -INFINITY;
        for (int s = 0; s < c->nnb[i]; ++s)
        {
            double r = c->macro[7 * (size_t)c->nbr[(size_t)i * ORA_MAX_NEIGH + s]];
            lo = fmin(lo, r);
            hi = fmax(hi, r);
        }
        if (isfinite(lo) && isfinite(hi))
        {
            double slack = 0.1 * fmax(hi - lo, 1.0e-12) + 1.0e-9;
            if (rn < lo - slack || rn > hi + slack) { c->flag[i] = 1; nfail++; }
        }
    }
    return nfail;
}

/* MLSTransport/MLSTransport.cpp:384-400 */
void ora_commit(ora_cloud *c)
{
    memcpy(c->g, c->gt, sizeof(double) * (size_t)c->N * c->gs);
}

/* MomentCalculations/Conservation.cpp:48-87 -- serial, particle order. */
double ora_sum_mass(const ora_cloud *c)
{
    const int Nv = c->Nv;
    double total = 0.0;
    for (int i = 0; i < c->N; ++i)
    {
        const double *g = c->g + (size_t)i * c->gs;
        double m = 0.0;
        if (c->dim == 3)
        {
            double dv3 = c->dv * c->dv * c->dv;
            for (int k = 0; k < Nv * Nv * Nv; ++k) m += g[k] * dv3;
        }
        else
        {
            double dv2 = c->dv * c->dv;
            for (int k = 0; k < Nv * Nv; ++k) m += g[k] * dv2;
        }
        total += m;
    }
    return total;
}

/* MomentCalculations/Conservation.cpp:92-109 */
void ora_scale(ora_cloud *c, double s)
{
    size_t n = (size_t)c->N * c->gs;
    for (size_t q = 0; q < n; ++q) c->g[q] *= s;
}

/* BoundaryConditions/DiffuseWall.cpp:19-154 */
void ora_boundary(ora_cloud *c)
{
    const int Nv = c->Nv, Nv2 = Nv * Nv;
    const double R = c->R, dv = c->dv, vlo = c->vmin;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < c->N; ++i)
    {
        if (!c->boundary[i]) continue;
        const double *w = c->wall + 7 * (size_t)i;
        const double Ux = w[3], Uy = w[4], Uz = w[5], Tw = w[6];
        const double RT2w = 2.0 * R * Tw;
        double *g = c->g + (size_t)i * c->gs;
        double *mac = c->macro + 7 * (size_t)i;
        if (c->dim == 3)
        {
            double dv3 = dv * dv * dv, norm = pow(PI * RT2w, 1.5);
            double intM = 0.0, intP = 0.0;
            for (int kv = 0; kv < Nv; ++kv)
                for (int jv = 0; jv < Nv; ++jv)
                    for (int iv = 0; iv < Nv; ++iv)
                    {
                        double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo), vz = node_v(kv, dv, vlo);
                        double cn = bc_cn(3, vx, vy, vz, w);
                        int lin = iv + Nv * (jv + Nv * kv);
                        if (cn < 0.0) intM += cn * g[lin] * dv3;
                        else if (cn > 0.0)
                        {
                            double Mw = exp(-((vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy) +
                                              (vz - Uz) * (vz - Uz)) / RT2w) / norm;
                            intP += cn * Mw * dv3;
                        }
                    }
            double rw = (intP > 1.0e-30) ? (-intM / intP) : 1.0;
            for (int kv = 0; kv < Nv; ++kv)
                for (int jv = 0; jv < Nv; ++jv)
                    for (int iv = 0; iv < Nv; ++iv)
                    {
                        double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo), vz = node_v(kv, dv, vlo);
                        double cn = bc_cn(3, vx, vy, vz, w);
                        if (cn > 0.0)
                            g[iv + Nv * (jv + Nv * kv)] =
                                rw * exp(-((vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy) +
                                           (vz - Uz) * (vz - Uz)) / RT2w) / norm;
                    }
            mac[0] = rw; mac[1] = Ux; mac[2] = Uy; mac[3] = Uz;
            mac[4] = Tw; mac[5] = rw * R * Tw;
            continue;
        }
        double dv2 = dv * dv, intM = 0.0, intP = 0.0;
        for (int jv = 0; jv < Nv; ++jv)
            for (int iv = 0; iv < Nv; ++iv)
            {
                double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo);
                double cn = bc_cn(2, vx, vy, 0.0, w);
                int lin = iv + Nv * jv;
                if (cn < 0.0) intM += cn * g[lin] * dv2;
                if (cn > 0.0)
                {
                    double Mw = exp(-((vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy)) / RT2w) /
                                (PI * RT2w);
                    intP += cn * Mw * dv2;
                }
            }
        double rw = (intP > 1.0e-30) ? (-intM / intP) : 1.0;
        for (int jv = 0; jv < Nv; ++jv)
            for (int iv = 0; iv < Nv; ++iv)
            {
                double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo);
                double cn = bc_cn(2, vx, vy, 0.0, w);
                int lin = iv + Nv * jv;
                if (cn > 0.0)
                {
                    double Mw = rw * exp(-((vx - Ux) * (vx - Ux) + (vy - Uy) * (vy - Uy)) / RT2w) /
                                (PI * RT2w);
                    g[lin] = Mw;
                    g[lin + Nv2] = 0.5 * R * Tw * Mw;
                }
            }
        mac[0] = rw; mac[1] = Ux; mac[2] = Uy; mac[4] = Tw; mac[5] = rw * R * Tw;
    }
}

/* MomentCalculations/Moments.cpp:17-97 (interior particles only) */
void ora_moments(ora_cloud *c)
{
    const int Nv = c->Nv, Nv2 = Nv * Nv;
    const double dv = c->dv, vlo = c->vmin, R = c->R;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < c->N; ++i)
    {
        if (c->boundary[i]) continue;
        const double *g = c->g + (size_t)i * c->gs;
        double *mac = c->macro + 7 * (size_t)i;
        double rs = 0, rux = 0, ruy = 0, ruz = 0, E = 0;
        if (c->dim == 3)
        {
            double dv3 = dv * dv * dv;
            for (int kv = 0; kv < Nv; ++kv)
                for (int jv = 0; jv < Nv; ++jv)
                    for (int iv = 0; iv < Nv; ++iv)
                    {
                        double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo), vz = node_v(kv, dv, vlo);
                        double f = g[iv + Nv * (jv + Nv * kv)];
                        rs += f * dv3; rux += vx * f * dv3; ruy += vy * f * dv3;
                        ruz += vz * f * dv3; E += (vx * vx + vy * vy + vz * vz) * f * dv3;
                    }
        }
        else
        {
            double dv2 = dv * dv;
            for (int jv = 0; jv < Nv; ++jv)
                for (int iv = 0; iv < Nv; ++iv)
                {
                    double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo);
                    double g1 = g[iv + Nv * jv], g2 = g[iv + Nv * jv + Nv2];
                    rs += g1 * dv2; rux += vx * g1 * dv2; ruy += vy * g1 * dv2;
                    E += (vx * vx + vy * vy) * g1 * dv2 + 2.0 * g2 * dv2;
                }
        }
        if (rs > 1.0e-30)
        {
            mac[0] = rs;
            mac[1] = rux / rs;
            mac[2] = ruy / rs;
            if (c->dim == 3) mac[3] = ruz / rs;
            double u2 = mac[1] * mac[1] + mac[2] * mac[2] + mac[3] * mac[3];
            mac[4] = fmax((E / rs - u2) / (3.0 * R), 1.0e-6);
            mac[5] = rs * R * mac[4];
        }
    }
}

/* MomentCalculations/Collision.cpp:70-139 (interior particles only) */
void ora_collision(ora_cloud *c)
{
    const int Nv = c->Nv, Nv2 = Nv * Nv;
    const double dv = c->dv, vlo = c->vmin, R = c->R;
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < c->N; ++i)
    {
        if (c->boundary[i]) continue;
        double lam = c->dt / c->tau;
        double *mac = c->macro + 7 * (size_t)i;
        if (c->tau_variable)
        {
            const double kB = 1.380649e-23;
            double l = kB / (sqrt(2.0) * PI * mac[0] * R * c->dHS * c->dHS);
            double cbar = sqrt(8.0 * R * mac[4] / PI);
            double tp = 4.0 * l / (PI * cbar);
            lam = c->dt / tp;
        }
        double coeff = 1.0 / (1.0 + lam);
        double *g = c->g + (size_t)i * c->gs;
        double twoRT = 2.0 * R * mac[4];
        if (c->dim == 3)
        {
            double norm = pow(PI * twoRT, 1.5);
            for (int kv = 0; kv < Nv; ++kv)
                for (int jv = 0; jv < Nv; ++jv)
                    for (int iv = 0; iv < Nv; ++iv)
                    {
                        double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo), vz = node_v(kv, dv, vlo);
                        double e = -((vx - mac[1]) * (vx - mac[1]) + (vy - mac[2]) * (vy - mac[2]) +
                                     (vz - mac[3]) * (vz - mac[3])) / twoRT;
                        double M = mac[0] / norm * exp(e);
                        int lin = iv + Nv * (jv + Nv * kv);
                        g[lin] = coeff * (g[lin] + lam * M);
                    }
        }
        else
        {
            for (int jv = 0; jv < Nv; ++jv)
                for (int iv = 0; iv < Nv; ++iv)
                {
                    double vx = node_v(iv, dv, vlo), vy = node_v(jv, dv, vlo);
                    double e = -((vx - mac[1]) * (vx - mac[1]) + (vy - mac[2]) * (vy - mac[2])) / twoRT;
                    double M1 = mac[0] / (PI * twoRT) * exp(e);
                    double M2 = 0.5 * R * mac[4] * M1;
                    int lin = iv + Nv * jv;
                    g[lin] = coeff * (g[lin] + lam * M1);
                    g[lin + Nv2] = coeff * (g[lin + Nv2] + lam * M2);
                }
        }
    }
}

/* MomentCalculations/Conservation.cpp:16-38 with padCheck, MLSBasis.hpp:208-222 */
int ora_mood_check(ora_cloud *c)
{
    int any = 0;
    const int Nv = c->Nv;
    const int nm = (c->dim == 3) ? Nv * Nv * Nv : Nv * Nv;
    for (int i = 0; i < c->N; ++i)
    {
        if (c->boundary[i]) continue;
        double *mac = c->macro + 7 * (size_t)i;
        int ok = 1;
        if (mac[0] < 1.0e-10) ok = 0;
        else if (mac[4] < 1.0e-6) ok = 0;
        else
        {
            const double *g = c->g + (size_t)i * c->gs;
            for (int k = 0; k < nm; ++k)
                if (g[k] < -1.0e-14) { ok = 0; break; }
        }
        mac[6] = ok ? 0.0 : 1.0;
        if (!ok) any = 1;
    }
    return any;
}

/* Solver/Solver.cpp:632-705 with dt fixed (no gravity, no exchange). */
void ora_step(ora_cloud *c, int nsteps, ora_stats *st)
{
    for (int n = 0; n < nsteps; ++n)
    {
        ora_stats s;
        memset(&s, 0, sizeof s);
        s.mass_old = ora_sum_mass(c);
        ora_transport(c, c->mls_order, 0, &s.positivity_fixes);
        if (c->limiter == 2)
        {
            s.transport_flags = ora_check_pad(c);
            if (s.transport_flags > 0) ora_transport(c, 1, 1, NULL);
        }
        ora_commit(c);
        s.mass_new = ora_sum_mass(c);
        if (s.mass_new > 1.0e-30) ora_scale(c, s.mass_old / s.mass_new);
        ora_boundary(c);
        ora_moments(c);
        ora_collision(c);
        ora_moments(c);
        if (c->limiter == 2)
        {
            if (ora_mood_check(c))
            {
                s.mood_fail = 1;
                ora_collision(c);
                ora_moments(c);
            }
        }
        s.mass_end = ora_sum_mass(c);
        if (st) *st = s;
    }
}

/* RigidBody/BodyDynamics.cpp:17-97 -- out: nbodies*6 (Fx Fy Fz Tx Ty Tz). */
void ora_body_loads(const ora_cloud *c, int nbodies, const double *centre,
                    const double *area, double *out)
{
    const int Nv = c->Nv;
    const double dv = c->dv, vlo = c->vmin;
    for (int q = 0; q < 6 * nbodies; ++q) out[q] = 0.0;
    for (int i = 0; i < c->N; ++i)
    {
        const int b = c->body_id[i];
        if (!c->boundary[i] || b < 0 || b >= nbodies) continue;
        const double *w = c->wall + 7 * (size_t)i;
        const double *g = c->g + (size_t)i * c->gs;
        const double cdx = c->xyz[3 * i] - centre[3 * b];
        const double cdy = c->xyz[3 * i + 1] - centre[3 * b + 1];
        const double cdz = c->xyz[3 * i + 2] - centre[3 * b + 2];
        double *o = out + 6 * b;
        if (c->dim == 3)
        {
            double dv3 = dv * dv * dv;
            double pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
            for (int kv = 0; kv < Nv; ++kv)
            {
                double cz = node_v(kv, dv, vlo) - w[5];
                for (int jv = 0; jv < Nv; ++jv)
                {
                    double cy = node_v(jv, dv, vlo) - w[4];
                    for (int iv = 0; iv < Nv; ++iv)
                    {
                        double cx = node_v(iv, dv, vlo) - w[3];
                        double f = g[iv + Nv * (jv + Nv * kv)] * dv3;
                        pxx += f * cx * cx; pyy += f * cy * cy; pzz += f * cz * cz;
                        pxy += f * cx * cy; pxz += f * cx * cz; pyz += f * cy * cz;
                    }
                }
            }
            double tx = -(w[0] * pxx + w[1] * pxy + w[2] * pxz);
            double ty = -(w[0] * pxy + w[1] * pyy + w[2] * pyz);
            double tz = -(w[0] * pxz + w[1] * pyz + w[2] * pzz);
            o[0] += area[b] * tx; o[1] += area[b] * ty; o[2] += area[b] * tz;
            o[3] += area[b] * (cdy * tz - cdz * ty);
            o[4] += area[b] * (cdz * tx - cdx * tz);
            o[5] += area[b] * (cdx * ty - cdy * tx);
        }
        else
        {
            double dv2 = dv * dv, phiX = 0, phiY = 0, phiXY = 0;
            for (int jv = 0; jv < Nv; ++jv)
            {
                double cy = node_v(jv, dv, vlo) - w[4];
                for (int iv = 0; iv < Nv; ++iv)
                {
                    double cx = node_v(iv, dv, vlo) - w[3];
                    double g1 = g[iv + Nv * jv];
                    phiX += g1 * dv2 * cx * cx;
                    phiY += g1 * dv2 * cy * cy;
                    phiXY += g1 * dv2 * cx * cy;
                }
            }
            double valX = -w[0] * phiX - w[1] * phiXY;
            double valY = -w[0] * phiXY - w[1] * phiY;
            o[0] += area[b] * valX;
            o[1] += area[b] * valY;
            o[5] += area[b] * (cdx * valY - cdy * valX);
        }
    }
}
