/*
 * alebgk_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, FP64, CPU restatement of the reference's ALE-BGK step (the CPU
 * contract of panchiittp/ALEBGK4Paper, Solver/Solver.cpp:632-705).  It is the
 * checker for the CUDA library: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it.  The product never calls it.
 *
 * Parity pin: the oracle is checked against the reference's own CPU code,
 * compiled unmodified into oracle/_ref/ (tests/test_oracle_pin.py), and
 * against committed fixtures generated from that build (tests/golden/).
 */
#ifndef ALEBGK_ORACLE_H
#define ALEBGK_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_MAX_NEIGH 128

typedef struct ora_cloud
{
    int dim, N, Nv, gs;         /* gs = Nv^3 (3-D) or 2 Nv^2 (2-D)          */
    int mls_order, limiter, tau_variable;
    double dt, tau, R, dHS, vmin, dv, h;
    int periodic[3];
    double L[3];
    double *xyz, *meshv, *wall; /* N*3, N*3, N*7                           */
    int *boundary, *body_id, *nnb, *nbr;   /* nbr: N*ORA_MAX_NEIGH         */
    double *g, *gt;             /* N*gs each                                */
    double *macro;              /* N*7: rho ux uy uz T p moodFlag           */
    int *flag;                  /* N scratch: transport MOOD flags          */
} ora_cloud;

/* Per-step outputs: last[0] transport flags, last[1] moodCheck failed,
 * mass[0..2] = massOld, massNew (after transport), mass at step end. */
typedef struct ora_stats
{
    int transport_flags;
    int mood_fail;
    int positivity_fixes;
    double mass_old, mass_new, mass_end;
} ora_stats;

void ora_transport(ora_cloud *c, int order, int only_flagged, int *nfix);
int ora_check_pad(ora_cloud *c);
void ora_commit(ora_cloud *c);
double ora_sum_mass(const ora_cloud *c);
void ora_scale(ora_cloud *c, double s);
void ora_boundary(ora_cloud *c);
void ora_moments(ora_cloud *c);
void ora_collision(ora_cloud *c);
int ora_mood_check(ora_cloud *c);
void ora_step(ora_cloud *c, int nsteps, ora_stats *st);
void ora_body_loads(const ora_cloud *c, int nbodies, const double *centre,
                    const double *area, double *out);
void ora_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
