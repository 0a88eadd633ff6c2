/*
 * alebgk.h -- C-ABI of the B200-native ALE-BGK time step.
 *
 * This is the drop-in boundary for the solver-step interface of
 * panchiittp/ALEBGK4Paper.  The reference's time loop (Solver/Solver.cpp:
 * 253-578) drives its GPU backend through the C++ functions declared at
 * Solver/Solver.cpp:67-89 and defined in Solver/CudaBackend.cu:1199-2082; they
 * take std::vector<Particle> (Core/Types.hpp:213-261).  Each entry point below
 * replaces one of them with plain pointers, sizes and an int status, so that
 * a C, C++, Python (ctypes) or any other FFI caller can bind it; the
 * reference-side C++ shim that maps the original symbols onto these calls is
 * alebgk4paper_b200/shim/cuda_backend_shim.cpp.
 *
 * Conventions
 *   - Every call returns ALEBGK_OK (0) or a negative ALEBGK_E* code; the
 *     library never calls exit().  alebgk_last_error() returns the message.
 *   - A context owns one device, one non-default CUDA stream and its device
 *     buffers.  Calls on one context are not thread-safe; distinct contexts
 *     are independent.  Work is enqueued on the context's stream; the
 *     download_* calls synchronise that stream.
 *   - Host arrays are plain, densely packed, row-major FP64/int32 arrays in
 *     the reference's per-particle order.
 */
#ifndef ALEBGK_H
#define ALEBGK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALEBGK_OK 0
#define ALEBGK_EINVAL (-1)   /* bad argument or configuration            */
#define ALEBGK_ECUDA (-2)    /* a CUDA runtime call failed                */
#define ALEBGK_ESTATE (-3)   /* call out of order (e.g. step before upload) */
#define ALEBGK_ENOMEM (-4)   /* host or device allocation failed          */
#define ALEBGK_EDEVICE (-5)  /* a device-side check failed (error word)   */
#define ALEBGK_EIO (-6)      /* a field file could not be opened, read or written */

#define ALEBGK_MAX_NEIGH 128 /* Core/Types.hpp:22 (MAX_NEIGH)             */

typedef struct alebgk_ctx alebgk_ctx;
typedef struct alebgk_case alebgk_case;

/* Solver configuration: the subset of SimParameters / CalcParameters /
 * GasConstants (Core/Types.hpp:110-208) that the step reads. */
typedef struct alebgk_config
{
    int dim;          /* 2 (Chu-reduced g1/g2) or 3                          */
    int N;            /* particles                                           */
    int Nv;           /* velocity points per axis (uniform Fixed grid)       */
    int mls_order;    /* 1 linear or 2 quadratic MLS for interior particles   */
    int precision;    /* 32: FP32 f storage + FP32 reconstruction; 64: all FP64 */
    int limiter;      /* 0 none, 2 MOOD (Core/Types.hpp:56-61)                */
    int tau_variable; /* hard-sphere tau(rho,T) (MomentCalculations/Collision.cpp:87-96) */
    int device;       /* CUDA device ordinal                                  */
    double R;         /* gas constant, 208 for argon                          */
    double tau;       /* BGK relaxation time                                  */
    double dHS;       /* hard-sphere diameter (tau_variable only)             */
    double vmin;      /* velocity grid lower end (VMin)                       */
    double dv;        /* velocity grid spacing                                */
    double radius;    /* MLS support h (CalcParameters::radius)               */
    int periodic[3];  /* per-axis periodicity (minimum-image stencils)        */
    double L[3];      /* periodic lengths                                     */
    int transport;    /* 0 auto (lattice march when the cloud is a complete
                         lattice and precision is 32, else coefficient
                         gather), 1 always gather, 2 require the march       */
    int particle;     /* 0 auto (streamed rows for a 3-D cloud whose rows fit,
                         in FP32 as three row kernels; else one warp per
                         particle), 1 always the general kernel, 2 require
                         streamed rows (three row kernels in FP32), 3
                         require streamed rows with one warp per particle     */
} alebgk_config;

/* The host cloud in SoA form.  Inputs for alebgk_upload; the download calls
 * fill the non-NULL members of the same struct. */
typedef struct alebgk_cloud
{
    double *xyz;      /* N*3 positions                                        */
    double *meshv;    /* N*3 mesh velocity (meshVx/y/z)                       */
    double *wall;     /* N*7 stored wall state: wnx wny wnz wUx wUy wUz wT    */
    int *boundary;    /* N   wall-particle flag                               */
    int *body_id;     /* N   -1 box wall / fluid, >=0 body surface            */
    int *nnb;         /* N   neighbour count (<= ALEBGK_MAX_NEIGH)            */
    int *nbr;         /* N*ALEBGK_MAX_NEIGH neighbour indices                 */
    double *g;        /* N*gstride distribution (Nv^3, or g1[Nv^2] g2[Nv^2])  */
    double *macro;    /* N*7: rho ux uy uz T p moodFlag                       */
} alebgk_cloud;

/* Counters after the last completed step (cudaLimiterCounts,
 * cudaMlsCounts, cudaMassBudget, cudaTotalMass:
 * Solver/CudaBackend.cu:1986-2030). */
typedef struct alebgk_counters
{
    int64_t steps;            /* steps run since upload                       */
    int transport_flags;      /* particles flagged by the transport MOOD screen */
    int positivity_fixes;     /* particles whose positivity repair fired      */
    int mood_fail;            /* 1 if the post-collision moodCheck failed     */
    int mls_degenerate;       /* particles with a skipped (|pivot|<1e-30) MLS pivot */
    double mass_before;       /* sumMass at the start of the step             */
    double mass_after_transport; /* sumMass after transport (before rescale) */
    double mass_scale;        /* global rescale factor applied               */
    double mass_end;          /* sumMass at the end of the step               */
    int error_word;           /* device-side error bits (0 = none): 2 a lattice
                                 march plane never arrived, 4 a streamed
                                 particle row never arrived, 8 a batch's
                                 persistent grid barrier gave up           */
    int transport_kernel;     /* transport in use: 1 coefficient gather,
                                 2 lattice march                              */
    int particle_kernel;      /* particle stage in use: 1 warp per particle,
                                 2 streamed rows, one warp per particle,
                                 3 streamed rows, three row kernels           */
} alebgk_counters;

/* ---- context --------------------------------------------------------- */

/* Creates a context (no reference counterpart: the reference keeps one
 * static DeviceCloud, Solver/CudaBackend.cu:69-115). */
int alebgk_create(const alebgk_config *cfg, alebgk_ctx **out);

/* Frees every device buffer and the context.
 * Replaces cudaFreeCloud (Solver/CudaBackend.cu:1203-1221). */
int alebgk_destroy(alebgk_ctx *ctx);

/* Message of the last failed call on this context (or the last failed
 * alebgk_create if ctx is NULL).  Copies at most len-1 bytes. */
int alebgk_last_error(const alebgk_ctx *ctx, char *buf, size_t len);

/* ---- state transfer -------------------------------------------------- */

/* Copies the full host cloud to the device and (re)builds the MLS stencil
 * classes and coefficient tables for the given dt.
 * Replaces cudaUploadCloud (Solver/Solver.cpp:68,
 * Solver/CudaBackend.cu:1223-1381); dt is the step the tables are built for
 * (the reference passes it to every cudaStep instead).  With cloud->g and
 * cloud->macro both NULL only the geometry is uploaded; the state follows by
 * alebgk_upload_state or alebgk_upload_rows. */
int alebgk_upload(alebgk_ctx *ctx, const alebgk_cloud *cloud, double dt);

/* Replaces only the distribution and macro fields (same geometry), e.g. a
 * checkpoint restore.  No reference counterpart (cudaUploadCloud's
 * layout-reuse path, Solver/CudaBackend.cu:1262-1263, covers it).
 * g is N x gstride doubles, macro N x 7 (rho, u, v, w, T, p, moodFlag).
 * A precision-32 context whose FP32 rows take at least 32 MB rounds g to
 * FP32 (round to nearest, ties to even) on the host's OpenMP threads, chunk
 * by chunk into pinned staging that the context keeps (four 8 MB chunks),
 * while the copy engine moves the previous chunk.  Smaller clouds and
 * precision-64 contexts copy the FP64 rows and convert on the device; the
 * stored state is the same bits either way.  Returns after the copies. */
int alebgk_upload_state(alebgk_ctx *ctx, const double *g, const double *macro);

/* Moments rho, u, T, p and moodFlag into macro (N*7).
 * Replaces cudaDownloadMoments (Solver/Solver.cpp:71,
 * Solver/CudaBackend.cu:1917-1972); p = rho*R*T as the CPU path computes it
 * (MomentCalculations/Moments.cpp:94). */
int alebgk_download_moments(alebgk_ctx *ctx, double *macro);

/* Moments plus the full distribution g (N*gstride, FP64).
 * Replaces cudaDownloadFull (Solver/Solver.cpp:72,
 * Solver/CudaBackend.cu:2056-2082). */
int alebgk_download_full(alebgk_ctx *ctx, double *g, double *macro);

/* ---- the step ---------------------------------------------------------- */

/* Enqueues nsteps full time steps with the dt given to alebgk_upload:
 * transport, positivity + MOOD screen with linear redo, commit, global mass
 * rescale, diffuse wall, moments, implicit BGK collision, moments, moodCheck
 * (Solver/Solver.cpp:632-705).  No host synchronisation inside.
 * Replaces cudaStep (Solver/Solver.cpp:69-70,
 * Solver/CudaBackend.cu:1505-1870). */
int alebgk_step(alebgk_ctx *ctx, int nsteps);

/* Blocks until all work on the context's stream has finished and returns
 * ALEBGK_EDEVICE if a device-side check set the error word. */
int alebgk_sync(alebgk_ctx *ctx);

/* Runs nsteps steps bracketed by CUDA events recorded on the context's own
 * stream, synchronises, and returns the device time in *ms.  Replaces the
 * reference's event-timed steady window ALEBGK_PROFILE_FROM/LEN
 * (Solver/CudaBackend.cu:1518-1623). */
int alebgk_step_timed(alebgk_ctx *ctx, int nsteps, float *ms);

/* Runs nsteps steps kernel by kernel (no graph) with a CUDA event between
 * every launch, and returns the summed device time of each stage in
 * ms_per_stage[0..ALEBGK_NSTAGES-1] (transport, particle, redo, sigma,
 * fixup, mass_sum, scale_mood, recollide, mass_end, step_begin).
 * Replaces the one-shot [GPU-PROFILE] table of
 * Solver/CudaBackend.cu:1518-1623. */
#define ALEBGK_NSTAGES 10
int alebgk_profile_steps(alebgk_ctx *ctx, int nsteps, float *ms_per_stage);

/* ---- diagnostics ------------------------------------------------------- */

/* Replaces cudaLimiterCounts, cudaMlsCounts, cudaMassBudget
 * (Solver/CudaBackend.cu:1986-2030). */
int alebgk_get_counters(alebgk_ctx *ctx, alebgk_counters *out);

/* Total gas mass sum(g dv^d) on the device.
 * Replaces cudaTotalMass (Solver/CudaBackend.cu:2018-2024). */
int alebgk_total_mass(alebgk_ctx *ctx, double *mass);

/* Per-particle x-momentum change applied by the last wall BC (N values,
 * zero for interior particles).
 * Replaces cudaWallMomentum (Solver/CudaBackend.cu:1977-1983). */
int alebgk_wall_momentum(alebgk_ctx *ctx, double *dpx);

/* Device pointers of the current distribution (row stride ldf elements,
 * FP32 or FP64 per cfg.precision) for callers that keep data on the GPU.
 * No reference counterpart. */
int alebgk_device_state(alebgk_ctx *ctx, void **f, int *ldf, int *elem_bytes);

/* ---- rigid bodies ------------------------------------------------------ */

/* Surface-stress force and torque on each body from the current device g,
 * relative to each surface particle's stored wall velocity:
 * P_ab = sum f c_a c_b dv^3, t = -n.P, F += area t, T += area r x t.
 * Restates computeBodyLoads (RigidBody/BodyDynamics.cpp:17-97).
 * body_centre: nbodies*3; body_area: nbodies; out: nbodies*6 (F, T). */
int alebgk_body_loads(alebgk_ctx *ctx, int nbodies, const double *body_centre,
                      const double *body_area, double *out);

/* The loads of alebgk_body_loads without any device allocation.  No
 * counterpart in the reference.  For callers that must not allocate: one
 * that advances several cavities on separate streams of a device (the
 * cudaFree of the allocating call synchronises the whole device and stalls
 * every other stream), and one that has reserved the device memory for its
 * own pools (an allocation could fail mid-run).  Sums run per block and then
 * over blocks, so results match alebgk_body_loads to rounding, not bitwise.
 * Limits: 1..ALEBGK_NOALLOC_MAX_BODIES bodies; larger counts return
 * ALEBGK_EINVAL.  Scratch: one fixed 114,432-byte device array per device,
 * shared by all contexts on it, so overlapping calls on one device race and
 * must be serialised by the caller.  The first call on a device looks the
 * array up and should come before any stream capture; so should the first
 * call after a device reset, which looks it up again in the new context. */
#define ALEBGK_NOALLOC_MAX_BODIES 16
int alebgk_body_loads_noalloc(alebgk_ctx *ctx, int nbodies, const double *body_centre,
                              const double *body_area, double *out);

/* One rigid body: shape and the 32-double state of alebgk_case_bodies
 * (centre 0-2, velocity 3-5, 2-D spin 6, angular velocity 7-9, force
 * 10-12, 2-D torque 13, torque 14-16, 2-D orientation 17-18, mass 19,
 * moment of inertia 20, temperature 21, body-to-world rotation 22-30,
 * surface area per surface point 31).  RigidBody/Geometry.hpp:19-362. */
typedef struct alebgk_body
{
    int kind;          /* 0 square, 1 circle (2-D); 2 sphere, 3 cube (3-D) */
    int rotates;       /* free to spin under the hydrodynamic torque        */
    double size;       /* side (square, cube) or radius (circle, sphere)    */
    double state[32];
} alebgk_body;

/* One Heun Newton-Euler step of the bodies after a completed alebgk_step
 * (moveRigidBodies, RigidBody/BodyDynamics.cpp:352-638): loads at the
 * stored wall state and at the predicted one (on the device, FP64), rigid
 * motion of the surface particles with the old body state, Newton-Euler
 * with the averaged loads, box-wall contact with a gap of 0.4 dx, and the
 * surface particles' new normal, wall velocity and mesh velocity.  bodies
 * is read and updated in place; box = xleft, xright, ybottom, ytop, zfront,
 * zback (DomainBoundary, Core/Types.hpp:73).  The surface particles move,
 * so the next alebgk_step returns ALEBGK_ESTATE until the cloud is uploaded
 * again (alebgk_download_geometry gives the moved geometry; the reference
 * runs its cloud management in between, Solver.cpp:373-401). */
int alebgk_body_step(alebgk_ctx *ctx, int nbodies, alebgk_body *bodies,
                     const double *box, double dx, double dt);

/* Positions (N*3), mesh velocities (N*3) and wall state (N*7) as stored on
 * the device; any pointer may be NULL.  No reference counterpart (the
 * reference's device state is never read back; cudaSyncBodies,
 * Solver/CudaBackend.cu:1884-1916, writes it). */
int alebgk_download_geometry(alebgk_ctx *ctx, double *xyz, double *meshv, double *wall);

/* Writes the surface wall velocity V + w x r of trial body states onto the
 * surface particles on the device (RigidBody/BodyDynamics.cpp:103-125).
 * state: nbodies*6 (V, w); body_centre: nbodies*3. */
int alebgk_body_set_surface_velocity(alebgk_ctx *ctx, int nbodies,
                                     const double *body_centre,
                                     const double *state);

/* ---- launch shapes, steady residual, batches ------------------------------
 * No reference counterpart: the reference runs one cavity per process. */

/* Launch shapes of the general kernels: threads per block of the
 * coefficient-gather transport (a multiple of 32 in 32..256, or 0: the
 * transport runs inside the particle kernel, each warp building its
 * particle's row in shared memory; same sums, same results) and particles
 * (warps) per block of the warp-per-particle kernel (1..8; 0 = as many as
 * their shared-memory rows allow).  The lattice march and the streamed
 * particle kernel have fixed shapes.  Drops the captured step graphs. */
int alebgk_set_launch(alebgk_ctx *ctx, int transport_threads, int particle_warps);
int alebgk_get_launch(alebgk_ctx *ctx, int *transport_threads, int *particle_warps);

/* Rounding floor of the MOOD NAD screen in FP32 mode: a slack of
 * rel * max(|lo|, |hi|) added to the reference's (MLSTransport.cpp:370),
 * where lo, hi is the neighbours' density range.  The default is 64 * 2^-24
 * in FP32 mode and 0 in FP64 mode: the FP32 transported density carries
 * rounding far above the reference's 1e-9 absolute slack near a uniform
 * state.  Drops the captured step graphs. */
int alebgk_set_nad_floor(alebgk_ctx *ctx, double rel);

/* Velocities per lane of the lattice march: 2 (default; packed
 * fma.rn.f32x2 on two adjacent velocities, 64 velocities per block) or 1
 * (one velocity per lane, 32 per block).  Both widths give the same bits.
 * Drops the captured step graphs. */
int alebgk_set_march_width(alebgk_ctx *ctx, int velocities_per_lane);

/* Times every candidate launch shape over `steps` steps, each on a device
 * snapshot of the state that is restored afterwards, and keeps the fastest;
 * *best_ms (may be NULL) is its time per step. */
int alebgk_autotune(alebgk_ctx *ctx, int steps, float *best_ms);

/* Steady residual of the last step over the interior particles: the largest
 * of ||d rho|| / ||rho||, ||d(rho ux)|| / ||rho c||, ||d(rho uy)|| / ||rho c||
 * and ||d(rho E)|| / ||rho E|| (2-norms over particles, E = |u|^2/2 + 3RT/2).
 * c is the speed set by alebgk_set_residual_speed (a lid speed, or the flow
 * speed |u| so that momentum changes are measured against the flow's own
 * momentum), else sqrt(RT), the thermal speed.  The reference defines no
 * residual. */
int alebgk_residual(alebgk_ctx *ctx, double *res);

/* Speed scale c of the residual's momentum terms: a positive speed (a
 * cavity's lid speed), a negative value for the flow speed |u| itself (the
 * momentum field's own norm), or 0 (the default) for the thermal speed.  A
 * batch copies it when the batch is created. */
int alebgk_set_residual_speed(alebgk_ctx *ctx, double speed);

/* The same measure between the macros of the previous call and now,
 * divided by the steps in between: the mean change per step over the
 * interval, in which the FP32 rounding noise of single steps averages out.
 * The first call only takes the snapshot and returns -1. */
int alebgk_residual_interval(alebgk_ctx *ctx, double *res);

/* Independent cavities on one device advanced in lockstep by one CUDA graph
 * launch per step, with each context's residual.  The contexts stay usable
 * on their own between batch calls, as long as they stay in step. */
typedef struct alebgk_batch alebgk_batch;
int alebgk_batch_create(int n, alebgk_ctx **ctxs, alebgk_batch **out);
int alebgk_batch_step(alebgk_batch *b, int nsteps);
/* mode 0 (default): the contexts split into groups of about equal work,
 * each group stepped by one launch per step stage over its contexts (the
 * groups are parallel branches of the graph), when the contexts share
 * precision and Chu layers and run the plain kernels; else mode 1.
 * mode 1: every context's own step as a branch of one graph.
 * mode 2: under the conditions of mode 0, the whole step of every context
 * in one persistent cooperative launch per step (the stages' blocks spread
 * over the resident grid, a grid-wide barrier between stages); else mode 1.
 * staged reports the form the captured graphs hold (the number of stage
 * groups -- 1 for the persistent launch -- or 0 for per-context branches).
 * set_groups sets the stage groups wanted in mode 0 (default 4).  All
 * forms give every context exactly the state of its own steps. */
int alebgk_batch_set_mode(alebgk_batch *b, int mode);
int alebgk_batch_get_mode(alebgk_batch *b, int *mode, int *staged);
int alebgk_batch_set_groups(alebgk_batch *b, int groups);
/* Polls of the persistent launch's grid barrier before it gives up
 * (default 2^24, polls >= 0).  A barrier that gives up ends the launch and
 * sets bit 8 of the first context's error word (alebgk_sync then returns
 * ALEBGK_EDEVICE); the step's state is then undefined. */
int alebgk_batch_set_spin_limit(alebgk_batch *b, long long polls);
/* Times `steps` steps of each form (stage launches in 1, 2, 4 and 8
 * groups, the persistent launch, per-context branches) and keeps the
 * fastest; *best_ms = its time per step.  The timed steps are real steps:
 * the batch advances by (steps + 2) per form tried (forms = 2 + the group
 * counts in 1, 2, 4, 8 not above the number of contexts). */
int alebgk_batch_autotune(alebgk_batch *b, int steps, float *best_ms);
int alebgk_batch_residuals(alebgk_batch *b, double *out);   /* n residuals */
int alebgk_batch_sync(alebgk_batch *b);
int alebgk_batch_destroy(alebgk_batch *b);

/* ---- learned warm start (2-D cavities) -----------------------------------
 * The reference has no counterpart: it always starts from the Maxwellian at
 * rest (Initialization/InitialConditions.cpp:18-80).
 *
 * 13 moments of the current 2-D state, per particle 9 FP64 values
 * rho, ux, uy, T, sigma_xx, sigma_xy, sigma_yy, q_x, q_y (sigma the traceless
 * stress, q the heat flux) taken with the discrete sums of
 * MomentCalculations/Moments.cpp:66-97.  out_dev is DEVICE memory, N x 9. */
int alebgk_moments13(alebgk_ctx *ctx, double *out_dev);

/* Seeds the 2-D state from 13-moment fields by Grad's 13-moment expansion in
 * the Chu representation (g1, g2).  The moments of particle i are
 * shift[c] + scale[c] * net_dev[i * ldnet + c], c = 0..8, in the order of
 * alebgk_moments13 (net_dev DEVICE FP32, e.g. the network output rows).
 * The macros and mass bookkeeping are reset from the seeded rows, as after
 * alebgk_upload_state. */
int alebgk_seed_grad13(alebgk_ctx *ctx, const float *net_dev, int ldnet,
                       const double *scale, const double *shift);

/* Coordinate network: 64 features (x, y, scaled log density, scaled lid
 * Mach number, and sin/cos(k pi x), sin/cos(k pi y), k = 1..12) -> 4 tanh
 * layers of width 128 -> 16 outputs (9 used).  BF16 weights, FP32
 * accumulation in tensor memory, FP32 master weights and Adam state.
 * Points are DEVICE float4 rows (x/L, y/L, a, b); idx_dev (optional) picks
 * the batch's rows; targets and outputs are DEVICE FP32 rows of 16. */
typedef struct alebgk_net alebgk_net;
int alebgk_net_nparams(void);
int alebgk_net_create(int device, alebgk_net **out);
void alebgk_net_destroy(alebgk_net *net);
const char *alebgk_net_last_error(const alebgk_net *net);
/* FP32 parameters, flat: W0[128][64], W1..W3[128][128], W4[16][128],
 * b0..b3[128], b4[16]; rows 9..15 of W4 and b4 are kept zero. */
int alebgk_net_set_params(alebgk_net *net, const float *host);
int alebgk_net_get_params(alebgk_net *net, float *host);
int alebgk_net_forward(alebgk_net *net, const float *pts_dev, const int *idx_dev, int n,
                       float *out_dev);
/* Gradient of sum_i sum_c w_c (O_ic - T_ic)^2 / n over the batch (no update);
 * grad_host receives alebgk_net_nparams() floats. */
int alebgk_net_grad(alebgk_net *net, const float *pts_dev, const float *tgt_dev,
                    const int *idx_dev, int n, const float *chan_w, float *grad_host,
                    float *loss_host);
/* One Adam step on that loss; loss_host may be NULL (no synchronisation). */
int alebgk_net_train_step(alebgk_net *net, const float *pts_dev, const float *tgt_dev,
                          const int *idx_dev, int n, const float *chan_w, float lr,
                          float beta1, float beta2, float eps, float *loss_host);
int alebgk_net_sync(alebgk_net *net);

/* Where alebgk_upload and alebgk_upload_geometry build the stencil classes
 * and MLS coefficient tables: 0 (default) both on the device, bitwise equal
 * to the host builders, except for clouds the lattice march takes (its plan
 * needs the host tables); 1 always on the host; 2 host classes with device
 * tables (the path a hash collision of two different stencil keys takes).
 * Process-wide; for checks of one against another. */
int alebgk_set_coeff_builder(int which);

/* alebgk_upload for a cloud whose particle set is unchanged: geometry, wall
 * state, mesh velocity, neighbour lists and tables are replaced, the
 * distribution, macros and mass bookkeeping stay on the device (cloud->g and
 * cloud->macro are not read).  For the body steps in which cloud management
 * leaves the particle set alone.  Where the tables are solved on the device
 * the refresh is in place: the stencil classes and slot lists are built on
 * the device from the uploaded geometry and the context's buffers are kept
 * (only tables that must grow are reallocated).  The context's captured
 * step graphs are dropped, and a batch holding it rebuilds its own. */
int alebgk_upload_geometry(alebgk_ctx *ctx, const alebgk_cloud *cloud, double dt);

/* Neighbour lists of the context's current device positions (body surface
 * particles included), as Initialization/NeighbourSearch.cpp:17-99 builds
 * them: grid = x0, y0, z0 (box origin), hBox, vBox, wBox (voxel sizes),
 * radius; boxes = voxel counts per axis.  nnb (N) and nbr (N x
 * ALEBGK_MAX_NEIGH, -1 padded) are host buffers. */
int alebgk_neighbours_device(alebgk_ctx *ctx, const double *grid, const int *boxes, int *nnb,
                             int *nbr);

/* Cloud management after a body motion (RigidBody/CloudManagement.cpp:17-275
 * in the order of Solver.cpp:381-395): remove, neighbour rebuild, merge,
 * refill, with the all-particle tests and the rebuilds on device `device`
 * and the result bitwise equal to the reference's.  Input: the host cloud
 * (N particles, gstride values per row; nnb/nbr unused), the bodies, and
 * prm = dx, minDist, radius, xleft, xright, ybottom, ytop, zfront, zback,
 * vmin, dv, R, hBox, vBox, wBox; iprm = dim, Nv, nbh, nbv, nbw.  The managed
 * cloud (new N, neighbour lists rebuilt) lives in *out until
 * alebgk_managed_free; alebgk_managed_info gives N, removed, merged, added,
 * needState.  With cloud->g and cloud->macro NULL the call only decides: it
 * stops with needState = 1 as soon as the particle set would change (then
 * call again with the state), and otherwise returns the same cloud with
 * rebuilt neighbour lists.  With cloud->macro set and cloud->g NULL (plan
 * mode) it manages the cloud as with the state but keeps no distribution:
 * alebgk_managed_plan gives, per row of the result, its origin in the input
 * (a[j] >= 0: input row a[j], or the mean of input rows a[j] and b[j] when
 * b[j] >= 0, as mergeCloseParticles forms it) or, for a[j] < 0, row
 * -1 - a[j] of `fresh` (the refill Maxwellians, `added` rows of gstride
 * FP64 values).  alebgk_rows_build then builds the distribution on the
 * device. */
typedef struct alebgk_managed alebgk_managed;
int alebgk_manage_cloud(int device, const double *prm, const int *iprm, int nbodies,
                        const alebgk_body *bodies, int N, int gstride,
                        const alebgk_cloud *cloud, alebgk_managed **out);
int alebgk_managed_info(const alebgk_managed *m, int *info);
int alebgk_managed_cloud(alebgk_managed *m, alebgk_cloud *view);
void alebgk_managed_free(alebgk_managed *m);
int alebgk_managed_plan(const alebgk_managed *m, int *a, int *b, double *fresh);

/* The distribution of a managed cloud, built on the device from ctx's
 * current one by a plan of alebgk_managed_plan (n rows, nfresh fresh rows):
 * every value is what alebgk_download_full, the host management and
 * alebgk_upload give it, computed without the host round trip.  The rows
 * (FP64, device memory) live in *out until alebgk_upload_rows or
 * alebgk_rows_free; ctx may be destroyed in between. */
typedef struct alebgk_rows alebgk_rows;
int alebgk_rows_build(alebgk_ctx *ctx, int n, const int *a, const int *b, int nfresh,
                      const double *fresh, alebgk_rows **out);
/* Installs rows as the distribution of ctx, whose cloud was uploaded without
 * a state (alebgk_upload with cloud->g and cloud->macro NULL uploads the
 * geometry only), with the host macros (N*7) as alebgk_upload_state takes
 * them; frees the rows. */
int alebgk_upload_rows(alebgk_ctx *ctx, alebgk_rows *rows, const double *macro);
void alebgk_rows_free(alebgk_rows *rows);

/* ---- slab mode ---------------------------------------------------------------
 * One cavity split into slabs along its outermost lattice axis, one context
 * per slab (the reference's decomposed mode, Solver/MpiExchange.cpp:114-466,
 * driven from one process).  Each context holds its slab's owned particles
 * [own_lo[i], own_hi[i]) and ghost copies of the neighbouring slabs' rows.
 * copies: ncopies rows of 5 ints (dst slab, dst first particle, src slab, src
 * first particle, particle count): after every step, the ghost block is
 * refreshed from its owner (f and macros).  The global mass sums and the
 * moodCheck flag are combined over the slabs in slab order.  Contexts may
 * sit on different devices (peer access is enabled); they must not be
 * stepped on their own while in a group. */
typedef struct alebgk_slab alebgk_slab;
int alebgk_slab_create(int n, alebgk_ctx **ctxs, const int *own_lo, const int *own_hi,
                       int ncopies, const int *copies, alebgk_slab **out);
int alebgk_slab_step(alebgk_slab *g, int nsteps);
int alebgk_slab_sync(alebgk_slab *g);
int alebgk_slab_destroy(alebgk_slab *g);

/* Multi-process slab runs: one slab per process, the reference's decomposed
 * mode with its MPI exchanges (Solver/MpiExchange.cpp:199-466,
 * MomentCalculations/Conservation.cpp:33-36,76-84) left to the host's
 * collectives.  Each rank uploads its slab (owned rows plus ghost rows, as
 * for alebgk_slab_create) and then:
 *   init(nranks, own range, words): the owned mass; all-gather the 4 words
 *     in rank order and pass them to combine(phase 4);
 *   per step, for seg = 0..3: segment(seg, words); all-gather; combine(seg);
 *   then the ghost rows of the state being written: rows(get) of the owned
 *     rows a neighbour needs, exchange, rows(put) into the ghost rows;
 *   finish(): the step's state becomes current.
 * words = the slab's owned-range partial sums (3) and its moodCheck flag;
 * all = nranks x 4 words in rank order.  rows moves `count` rows of f (the
 * storage type, ldf values each) and of the macros (6 doubles each) of the
 * state the step in progress writes.  The arithmetic of the combine is the
 * single-process slab group's, so both runs give the same state. */
int alebgk_rank_slab_init(alebgk_ctx *ctx, int nranks, int own_lo, int own_hi, double *words);
int alebgk_rank_slab_segment(alebgk_ctx *ctx, int seg, double *words);
int alebgk_rank_slab_combine(alebgk_ctx *ctx, int phase, int nranks, const double *all);
int alebgk_rank_slab_rows(alebgk_ctx *ctx, int start, int count, void *f_rows,
                          double *macro_rows, int put);
int alebgk_rank_slab_finish(alebgk_ctx *ctx);

/* ---- restart files ------------------------------------------------------
 * The reference's checkpoint layout (Core/Checkpoint.hpp:37-236, magic
 * "ALEBGK01", version 1): header, one record per particle, N*gStride FP64
 * values of g, one record per body.  Files written here restore with the
 * reference's ckpt::restore, and the reference's files read here. */
typedef struct alebgk_ckpt_header
{
    uint64_t N;
    uint64_t gstride;
    uint64_t step;
    double t;
    uint32_t dim;
    uint32_t nbodies;
} alebgk_ckpt_header;

/* Header of a restart file (host only). */
int alebgk_checkpoint_header(const char *path, alebgk_ckpt_header *out);

/* Reads a restart file into host arrays (host only): the non-NULL members
 * xyz, meshv, wall, boundary, body_id, g, macro of cloud (nnb, nbr
 * untouched: the reference rebuilds neighbour lists after a restore),
 * voxel (N, may be NULL) and the state and rotates flag of nbodies bodies
 * (may be NULL).  Fails, reading nothing past the header, if the file's N,
 * gstride, dim or body count differs from *expect. */
int alebgk_checkpoint_read(const char *path, const alebgk_ckpt_header *expect,
                           alebgk_cloud *cloud, int *voxel, alebgk_body *bodies);

/* Writes the context's state as a restart file: g (FP64, staged through
 * pinned buffers, device copy overlapping the file write), macros,
 * positions, mesh velocity and wall state from the device, boundary flags
 * and body ids from the upload.  vgrid = {vlo, vhi, dv} per particle (NULL:
 * from the configuration), voxel may be NULL (0), bodies may be NULL if
 * nbodies is 0.  The file is written to path.tmp and renamed.  Replaces
 * ckpt::save (Core/Checkpoint.hpp:84-155) after a cudaDownloadFull. */
int alebgk_checkpoint_save(alebgk_ctx *ctx, const char *path, int64_t step, double t,
                           const double *vgrid, const int *voxel, int nbodies,
                           const alebgk_body *bodies);

/* ---- field output -------------------------------------------------------
 * The reference's save-cycle output (Core/Output.hpp:17-115, called from
 * Solver/Solver.cpp:548-560): an ASCII VTK frame, interior diagnostics, a
 * timeseries.csv row and the printStep line; and a binary dump of the same
 * fields at full precision (no reference counterpart: the VTK frame keeps
 * seven significant digits). */
typedef struct
{
    double rho_avg, KE, T_avg, p_avg;  /* interior averages (KE = 0.5 rho |u|^2) */
    int mood_count;                    /* interior particles with moodFlag set   */
    int n;                             /* interior particles                     */
} alebgk_diag;

/* The reference's ASCII VTK frame (writeVTK, Core/Output.hpp:17-51) from host
 * arrays: positions xyz (N*3), per-particle rho ux uy uz T p moodFlag (macro,
 * N*7, the layout of alebgk_download_moments), boundary flags (N), Nv_local =
 * Nv for every particle, and the time in the title line.  Every number is
 * printed as the reference's stream prints it (scientific, six decimals), so
 * the file is the reference's byte for byte for the same data.  Formatted in
 * parallel (OpenMP), written once.  ALEBGK_EIO if the file cannot be
 * written. */
int alebgk_vtk_write_host(const char *path, int N, const double *xyz, const double *macro,
                          const int *boundary, int Nv, double time);

/* The same for the context's current state (positions and moments from the
 * device, boundary flags from the upload) into outdir/output_%06d.vtk, the
 * reference's frame name.  Replaces writeVTK after cudaDownloadMoments
 * (Solver/Solver.cpp:552-556). */
int alebgk_write_vtk(alebgk_ctx *ctx, const char *outdir, int step, double time);

/* Interior averages in particle order (computeDiagnostics,
 * Core/Output.hpp:66-85), from host arrays or from the context. */
int alebgk_diagnostics_host(int N, const double *macro, const int *boundary, alebgk_diag *out);
int alebgk_diagnostics(alebgk_ctx *ctx, alebgk_diag *out);

/* One timeseries.csv row (writeTimeseries, Core/Output.hpp:91-106).  header
 * != 0 truncates the file and writes the column line first, which the
 * reference does on its first call in the process; 0 appends. */
int alebgk_write_timeseries(const char *path, double t, const alebgk_diag *d, int header);

/* The reference's step line (printStep, Core/Output.hpp:111-115) into buf;
 * ALEBGK_EINVAL if it does not fit in len bytes. */
int alebgk_format_step(char *buf, size_t len, int step, double t, double dt,
                       const alebgk_diag *d);

/* Binary field dump: this header, then xyz (N*3 FP64), macro (N*7 FP64, the
 * layout of alebgk_download_moments) and boundary (N int32), little endian
 * as the device writes them.  Written to path.tmp and renamed.  read_fields
 * fills the header and the non-NULL arrays; ALEBGK_EIO on a short file or a
 * wrong magic or version. */
typedef struct
{
    char magic[8];            /* "ALBGKFLD" */
    uint32_t version;         /* 1 */
    uint32_t dim;
    uint64_t N;
    int64_t step;
    double t;
} alebgk_fields_header;
int alebgk_write_fields(alebgk_ctx *ctx, const char *path, int64_t step, double t);
int alebgk_read_fields(const char *path, alebgk_fields_header *h, double *xyz, double *macro,
                       int *boundary);

/* ---- host-side MLS coefficient tables (no device work) -------------------
 * The stencil classes and FP64 transport coefficients that alebgk_upload
 * builds: gt[i][k] = sum_s coef[cls[i]][s][k] * g[slots[i][s]][k], slot 0 =
 * the particle itself (coefficient 1 where the reference keeps the old value:
 * outgoing wall nodes, MLSTransport/MLSTransport.cpp:144-150, and nodes
 * without a weighted neighbour, :182).  No reference counterpart: the
 * reference re-solves the normal equations for every node of every step
 * (MLSTransport/MLSTransport.cpp:129-186). */
typedef struct alebgk_coeffs alebgk_coeffs;
int alebgk_coeff_build(const alebgk_config *cfg, const alebgk_cloud *cloud,
                       double dt, alebgk_coeffs **out);
/* info[0..4] = ncls, S (slot stride), V (nodes per layer),
 *              particles with a skipped pivot, N */
int alebgk_coeff_info(const alebgk_coeffs *t, int *info);
/* cls: N, nslot: N, slots: N*S, coef: ncls*S*V (any may be NULL) */
int alebgk_coeff_get(const alebgk_coeffs *t, int *cls, int *nslot, int *slots,
                     double *coef);
void alebgk_coeff_free(alebgk_coeffs *t);

/* ---- host-side case set-up (no device work) -----------------------------
 * Builds one of the reference's six cases (TestCases/TestCases.cpp:56-294,
 * Initialization/*.cpp, TestCases/main.cpp:193-345) on the host.  Nx, Nv,
 * dt <= 0 keep the case defaults; mls_order 1 or 2; fixed_body = --fixed. */
int alebgk_case_build(const char *name, int Nx, int Nv, double dt,
                      int mls_order, int fixed_body, double body_scale,
                      alebgk_case **out);
void alebgk_case_free(alebgk_case *c);

/* The same with the lid speed (m/s), initial density and relaxation time
 * of the case overridden where > 0 (the batched-cavity workloads vary
 * them; the reference varies them by editing TestCases.cpp). */
int alebgk_case_build_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                         int fixed_body, double body_scale, double lid_speed, double rho0,
                         double tau, alebgk_case **out);

/* info[0..7]  = N, dim, Nv, gstride, nbodies, mls_order, Nx, moving_bodies
 * prm[0..23]  = dt, tau, R, dx, dy, dz, radius, minDist, dv, vmin, vmax,
 *               rho0, Tw, xleft, xright, ybottom, ytop, zfront, zback,
 *               dt_requested, tfinal, dHS, lid_speed, save_every */
int alebgk_case_info(const alebgk_case *c, int *info, double *prm);

/* Fills a cloud view whose members point into the case's own host arrays
 * (valid until alebgk_case_free). */
int alebgk_case_view(alebgk_case *c, alebgk_cloud *view);

/* Body state: per body 32 doubles: cx cy cz velx vely velz angularVel omx omy
 * omz forcex forcey forcez torque tqx tqy tqz ox oy mass I T Rm[9] area. */
int alebgk_case_bodies(const alebgk_case *c, double *out);

/* Shape of every body of the case: kind (alebgk_body), rotates, size. */
int alebgk_case_body_shapes(const alebgk_case *c, int *kind, int *rotates, double *size);

/* ---- lattice set-up on the device -------------------------------------------
 * The reference's cases can be set up on the GPU instead of by
 * alebgk_case_build_ex on the host: the lattice
 * (Initialization/ParticleGeneration.cpp:30-200), the wall state
 * (Core/MLSBasis.hpp:228-287, TestCases/TestCases.cpp:230-249), the rigid
 * bodies embedded (Initialization/BodyEmbedding.cpp:18-104: lattice particles
 * inside a body or within 0.4 dx of its surface dropped, in order, the
 * surface particles appended), the voxel bins and neighbour lists
 * (Initialization/NeighbourSearch.cpp:17-99) and the rest-state Maxwellian
 * (Initialization/InitialConditions.cpp:18-80), each bitwise equal to the
 * host set-up.  The host computes only the bodies' surface points (a few
 * hundred records).  The stencil classes and transport coefficients are
 * built as alebgk_upload builds them.
 *
 * alebgk_lattice_info_ex: info/prm as alebgk_case_info, without a host cloud.
 * For a case with bodies the particle count after the embedding comes from
 * the device set-up, run on `device`.  fixed_body and body_scale as in
 * alebgk_case_build (the --fixed flag and the body size factor). */
int alebgk_lattice_info_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                           int fixed_body, double body_scale, double lid_speed, double rho0,
                           double tau, int device, int *info, double *prm);
/* The bodies of a lattice case (host only): count, state (32 doubles per
 * body, the layout of alebgk_case_bodies), kind, rotates, size (any may be
 * NULL). */
int alebgk_lattice_bodies(const char *name, int Nx, int Nv, double dt, int mls_order,
                          int fixed_body, double body_scale, int *nbodies, double *state,
                          int *kind, int *rotates, double *size);
/* The device-built arrays, copied to host buffers (any may be NULL): xyz N*3,
 * wall N*7, boundary N, body_id N, nnb N, nbr N*ALEBGK_MAX_NEIGH (-1 padded). */
int alebgk_lattice_build_device_ex(const char *name, int Nx, int Nv, double dt, int mls_order,
                                   int fixed_body, double body_scale, double lid_speed,
                                   double rho0, double tau, int device, double *xyz,
                                   double *wall, int *boundary, int *body_id, int *nnb,
                                   int *nbr);
/* alebgk_upload for a lattice case set up on the device: the context (made
 * from the alebgk_lattice_info_ex configuration) gets the same state that
 * alebgk_upload of the host-built case gives it. */
int alebgk_upload_lattice_ex(alebgk_ctx *ctx, const char *name, int Nx, int Nv, double dt,
                             int mls_order, int fixed_body, double body_scale, double lid_speed,
                             double rho0, double tau);
/* The same without bodies' options (fixed_body 0, body_scale 1, device 0). */
int alebgk_lattice_info(const char *name, int Nx, int Nv, double dt, int mls_order,
                        double lid_speed, double rho0, double tau, int *info, double *prm);
int alebgk_lattice_build_device(const char *name, int Nx, int Nv, double dt, int mls_order,
                                double lid_speed, double rho0, double tau, int device,
                                double *xyz, double *wall, int *boundary, int *nnb, int *nbr);
int alebgk_upload_lattice(alebgk_ctx *ctx, const char *name, int Nx, int Nv, double dt,
                          int mls_order, double lid_speed, double rho0, double tau);

/* Fills a solver configuration from a case (precision 32 or 64). */
int alebgk_case_config(const alebgk_case *c, int precision, int device,
                       alebgk_config *cfg);

#ifdef __cplusplus
}
#endif

#endif /* ALEBGK_H */
