/*
 * galaxy_gpu.h -- C ABI of the B200 polar-grid particle-mesh step.
 *
 * The entry points replace the lib15 subroutines of GALAXY v15 that make up
 * the polar-grid (p2d / p3d) particle-mesh step.  Each one names the
 * reference routine it stands in for (paths relative to the GALAXY source
 * tree).  The reference keeps its state in COMMON blocks; here the state is
 * an opaque context created by gx_grdset.
 *
 * Conventions
 *  - Every entry point returns GX_OK (0) or a negative GX_ERR_* code; the
 *    message is available from gx_last_error().  Nothing aborts the process.
 *  - Pointers passed in are host pointers, valid for the duration of the
 *    call only.  Device memory is owned by the context.
 *  - A context is not re-entrant: one host thread at a time; all work is
 *    serialised on the context's own CUDA stream.
 *  - Coordinates are in grid units: positions x, y[, z]; velocities are
 *    displacements per step and accelerations are velocity changes per step
 *    (reference: SRC/lib15/stpgrp.f:26-32).  Particle arrays at the boundary
 *    are AoS float32 records of 2*ndim words, (x, y[, z], vx, vy[, vz]),
 *    the coordinate layout of the reference's .pcs records
 *    (SRC/lib15/loadup.f:36-140).
 *  - Grid arrays (mass, fields) use the reference mesh layout: index
 *    ((ir * ngz + iz) * na + it) for ring ir, plane iz, spoke it
 *    (SRC/lib15/weight.f:236, ncl - 1).
 */
#ifndef GALAXY_GPU_H
#define GALAXY_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GX_OK               0
#define GX_ERR_ARG         -1   /* invalid argument / configuration        */
#define GX_ERR_CUDA        -2   /* CUDA runtime error                      */
#define GX_ERR_STATE       -3   /* call out of order (e.g. no Green table) */
#define GX_ERR_NOMEM       -4   /* device allocation failed                */
#define GX_ERR_TIMEOUT     -5   /* a bounded device wait gave up           */
#define GX_ERR_RANGE       -6   /* size beyond a stated limit              */
#define GX_ERR_DEVICE      -7   /* device-side check raised its error word */

/* radial coordinate maps u(r) (SRC/lib15/uofgr.f:22-36, grofu.f:25-41) */
#define GX_RMAP_STDPOL      0   /* u = ln(1 + r) / a,  r = e^{a u} - 1              */
#define GX_RMAP_LOG         1   /* u = ln(r) / a + uoffs, uoffs = -ln(r0)/a; hole r<r0 */

/* softening rules (SRC/lib15/setgrd.f:178-189) */
#define GX_SOFT_PLUMMER     1
#define GX_SOFT_SPLINE      2

/* arithmetic of the step */
#define GX_PREC_MIXED       0   /* FP32 bulk, FP64 Green table/diagnostics  */
#define GX_PREC_FP64        1   /* plain FP64 path (the comparison baseline) */
#define GX_PREC_MIXED_TC05  2   /* gx_sfp_sum only: the tcgen05 (TMEM) tensor path */

/* flags */
#define GX_FLAG_COMPENSATED 1   /* compensated (two-float) position update  */
#define GX_FLAG_QUADRATIC   2   /* p3d 'inte 3': 27-point quadratic interpolation
                                   (weight.f:251-314, massgn.f:173-202,
                                   grdacc.f:267-299) instead of the 8-point one */
#define GX_FLAG_WHOLE_GRID  4   /* time-step zones: the field over the whole grid
                                   on every step (the 'wholeg' option, findf.f:41)
                                   instead of partial-grid solves */
#define GX_FLAG_PLANE_SPLIT 16  /* 3D mixed path on nranks > 1: each rank runs the
                                   radial contraction only for the vertical
                                   wavenumbers kz with kz mod nranks == rank and the
                                   ranks sum the contracted spectra (the reference's
                                   MPI plane split, SRC/lib15_mpi/p3convp.f:180-190,
                                   276-326); needs nr a multiple of 4, <= 128 */
#define GX_FLAG_SORTED_DEPOSIT 8 /* mixed path: step with the row-sorted deposit
                                   (counting sort of the cell rows, staged
                                   fixed-point items, combine) instead of the
                                   fused pass over the bucketed particle store;
                                   the two give bitwise identical results */
#define GX_FLAG_ROWBLOCK_TRANSFORMS 32 /* 3D mixed path: the field solve's transforms
                                   with the kernels that take any grid (per block of
                                   ring-plane rows or per ring and field type),
                                   instead of the per-ring kernels that hold a ring's
                                   planes, spectra and tables in shared memory; the
                                   results agree to FP32 rounding */
#define GX_MAX_WEIGHTS     27   /* weights per particle of gx_weight          */

/* grid arrays for gx_get_grid / gx_set_mass */
#define GX_GRID_MASS        0   /* mass (after the pmass scaling)            */
#define GX_GRID_FR          1   /* radial force (before polcat)              */
#define GX_GRID_FT          2   /* azimuthal force (before polcat)           */
#define GX_GRID_FZ          3   /* vertical force (3D)                       */
#define GX_GRID_POT         4   /* potential                                 */
#define GX_GRID_FX          5   /* Cartesian x force (after polcat)          */
#define GX_GRID_FY          6   /* Cartesian y force (after polcat)          */

/* Green-function component types, reference itype order
 * (SRC/lib15/p3conv.f:10-12): radial, azimuthal, vertical, potential */
#define GX_GREEN_FR         0
#define GX_GREEN_FT         1
#define GX_GREEN_FZ         2
#define GX_GREEN_POT        3

#define GX_MAX_SKIP        16
#define GX_MAX_ZONES        8   /* time-step zones (gx_set_zones)            */

/* Grid and run parameters: the p2d/p3d cards of the reference
 * (SRC/lib15/p2dset.f:22-80, p3dset.f:22-101, filset.f:101-142) plus the
 * unit scalings that setrun/loadup derive (SRC/lib15/loadup.f:97-99). */
typedef struct GxConfig {
    int32_t ndim;        /* 2 (p2d) or 3 (p3d)                               */
    int32_t nr;          /* grid rings                                        */
    int32_t na;          /* spokes (forced even)                              */
    int32_t ngz;         /* planes (3D; must be 3^i 5^j); ignored for 2D      */
    float   dzg;         /* plane spacing in grid units (3D)                  */
    int32_t ng;          /* sectoral harmonics m = 0 .. ng-1 (HASH + 1)       */
    int32_t nsect;       /* sector symmetry (1 = whole plane)                 */
    int32_t nskip;       /* extra harmonics to skip ('skip' card)             */
    int32_t skip[GX_MAX_SKIP];
    int32_t rmap;        /* GX_RMAP_*                                         */
    float   rmap_a;      /* u scale a; 0 selects the reference alpha = 2pi/na */
    float   rmap_r0;     /* inner edge for GX_RMAP_LOG                        */
    float   softl;       /* softening length, grid units                      */
    int32_t tsoft;       /* GX_SOFT_*                                         */
    float   pmass;       /* particle mass in internal units (M lscale^3 ts^2) */
    int32_t halo;        /* rigid force on every particle on the grid: 0 none;
                            1 cored isothermal halo (ISOT, frhalo.f:55-56);
                            2 softened Kuz'min-Toomre disc, the analytic
                            radial force of a run whose m = 0 harmonic is
                            skipped (filset.f:3-5, axifrc.f, frdisc.f:27-29) */
    float   halo_v2;     /* 1: asymptotic v^2 (M_h / r_c); 2: disc mass
                            M lscale^3 ts^2; internal units                   */
    float   halo_rc;     /* 1: core radius; 2: (1 + epsilon) rscale lscale;
                            grid units                                        */
    int32_t precision;   /* GX_PREC_*                                         */
    int32_t flags;       /* GX_FLAG_*                                         */
    int32_t device;      /* CUDA device ordinal                               */
} GxConfig;

/* Grid geometry derived by setgrd (SRC/lib15/setgrd.f:52-200). */
typedef struct GxGeometry {
    int32_t nr, na, ngz, ng, mmax, nsect, mesh;
    float   alpha;       /* 2 pi / na                                         */
    float   ua;          /* scale of u(r) actually used                       */
    float   uoffs;       /* offset of GX_RMAP_LOG                             */
    float   rinh;        /* inner edge, grofu(0)                              */
    float   rgrid;       /* outer edge, grofu(nr - 1)                         */
    float   zm;          /* half-height of the grid, 0.5 dzg (ngz - 1)        */
    float   thmax;       /* na / nsect                                        */
    int32_t nact;        /* active harmonics (lg false)                       */
    uint8_t lg[260];     /* lg[m] != 0: harmonic m skipped (filset.f:116-141) */
} GxGeometry;

/* Global integrals of icheck (SRC/lib15/icheck.f:61-92), FP64 sums. */
typedef struct GxDiag {
    double ke;           /* sum m v^2 (reference keeps the 1/2 outside)      */
    double pe;           /* 1/2 sum m phi                                     */
    double lz;           /* sum m (x vy - y vx)                               */
    double virial;       /* sum m x . a                                       */
    double a2_re, a2_im; /* sum m e^{2 i phi} / sum m                         */
    int64_t n_on_grid;
} GxDiag;

/* Abel-Jacobi basis of the SFP method (sf2d): set k, the selected
 * functions m = minm..maxm (step nsect) x n = minn..maxn (filset.f:101-114),
 * and the roots and coefficients the reference reads from Basis/ajKK.dat
 * (SRC/lib15/ajsetup.f:23-58).  roots[(m*(maxn+1) + n)*maxn + i] is the
 * (i+1)-th root of U_nm, i < n; xcoeff[(m*(maxn+1) + n)*(k+1) + i] is the
 * coefficient of (1 - r^2)^i (ajfun.f:33-47). */
typedef struct GxSfpBasis {
    int32_t k;
    int32_t minm, maxm, minn, maxn, nsect;
    int32_t nrtab;          /* radii of the reference's look-up table (sfptab)   */
    const double* roots;
    const double* xcoeff;
} GxSfpBasis;

typedef struct GxCtx GxCtx;

/* grdset + setgrd: validate the cards, derive the geometry, allocate the
 * device arrays.  SRC/lib15/grdset.f:23-42, SRC/lib15/setgrd.f:52-200. */
int gx_grdset(const GxConfig* cfg, GxCtx** out);

/* Release every resource of the context. */
void gx_destroy(GxCtx* ctx);

/* Text of the last error on this context (or of the last failed
 * gx_grdset when ctx is NULL). */
const char* gx_last_error(const GxCtx* ctx);

/* Derived geometry (setgrd results). */
int gx_geometry(const GxCtx* ctx, GxGeometry* geo);

/* greenm: build the transformed Green table on the device in FP64 and keep
 * it resident (the reference writes it to a .grt file and re-reads it every
 * step).  SRC/lib15/greenm.f:27-36, p2grnm.f:73-219, p3grnm.f:94-263. */
int gx_greenm(GxCtx* ctx);

/* Copy one Green component out (FP64 build rounded as stored), layout
 * [m][kz][is][ir] for 3D and [m][is][ir] for 2D, for m = 0 .. ng-1 and, in
 * 3D, the ngz + 1 vertical wavenumbers kz = 0 .. ngz of the doubled grid
 * (GX_GREEN_FZ, a sine transform, is zero at kz = 0 and kz = ngz).  type = GX_GREEN_*.  n = ng * nkz * nr * nr. */
int gx_green_get(GxCtx* ctx, int type, double* out, int64_t n);

/* loadup: copy n AoS particle records (2*ndim float32 words each) into the
 * device SoA store.  SRC/lib15/loadup.f:36-140. */
int gx_loadup(GxCtx* ctx, const float* coords, int64_t n);

/* weight: cell numbers (ncl - 1, or -1 off the grid / in the hole) and the
 * 4 (2D) or 8 (3D) interpolation weights, 8 floats per particle, of n AoS
 * particle records; with GX_FLAG_QUADRATIC the central node's number and
 * 27 weights, 27 floats per particle.  old != 0 selects the interpolation
 * form (no sector folding).  SRC/lib15/weight.f:61-101 (p2d), 196-250 (p3d
 * linear), 251-314 (p3d quadratic). */
int gx_weight(GxCtx* ctx, const float* coords, int64_t n, int old, int32_t* ncl, float* wt);

/* dumpp (coordinates only): copy the particle records back out, in the
 * order they were loaded.  SRC/lib15/dumpp.f:246-387. */
int gx_unload(GxCtx* ctx, float* coords);

/* masset: clear, assign every particle's mass (massgn) and scale by pmass.
 * SRC/lib15/masset.f, massgn.f:68-89 (p2d), 140-172 (p3d), scaled.f:89-92. */
int gx_masset(GxCtx* ctx);

/* Test-mass placement of p2ckst/p3ckst: install a mesh-sized mass array
 * (already scaled) directly.  SRC/lib15/p3ckst.f. */
int gx_set_mass(GxCtx* ctx, const float* mass);

/* findf: solve for the fields of the current mass array (p2fndf/p3fndf)
 * and convert to Cartesian components (polcat).  lpot != 0 also returns
 * the potential.  SRC/lib15/findf.f:34-80, p2fndf.f:25-66, p3fndf.f:36-104,
 * polcat.f:22-41. */
int gx_findf(GxCtx* ctx, int lpot);

/* findf without polcat (ptest stubs polcat out, SRC/progs/ptest.f:91-101). */
int gx_findf_polar(GxCtx* ctx, int lpot);

/* Copy a mesh array out.  which = GX_GRID_*.  mesh floats. */
int gx_get_grid(GxCtx* ctx, int which, float* out);

/* getacc/grdacc: accelerations (ndim per particle, AoS) and potentials of
 * every particle at its current position from the current fields, plus the
 * rigid halo.  pot may be NULL.  SRC/lib15/getacc.f:36-162,
 * grdacc.f:40-84 (p2d), 189-266 (p3d). */
int gx_getacc(GxCtx* ctx, float* acc, float* pot);

/* step: nsteps x { findf; getacc; stpgrp; massgn; scaled }.  phys != 0
 * requests potentials on the last step (analysis step).
 * SRC/lib15/step.f:135-290, SRC/progs/galaxy.f:107-148. */
int gx_step(GxCtx* ctx, int nsteps, int phys);

/* Multiple time-step zones (SRC/lib15/setrun.f:208-219, 770-790): zone i
 * (1-based) holds the particles at radius >= zbr[i-1] (cylindrical in 2D,
 * spherical in 3D; zbr[0] is ignored, zone 1 starts at the centre) and
 * steps every nstep[i-1] base steps with that multiple of the base step
 * (nstep[0] = 1, zbr ascending inside the grid, grid units).  Call before
 * gx_loadup, which then gives every particle its zone (loadup.f:177-181,
 * zoneno.f) and scales its velocity to its zone's step (adjvls.f); gx_unload
 * undoes the scaling.  With more than one zone gx_step follows step.f: zone
 * i moves at the steps divisible by nstep[i-1], accelerations scaled by
 * nstep^2 (getacc.f:141-150), particles crossing a boundary change step
 * (rezgrp.f, chstep.f) and particles leaving the grid move to the outer
 * zone's step (addoff.f); each zone keeps its own mass array and the solve
 * uses their linear interpolation in time (masscl.f:64-96, zoncmb.f:46-129).
 * On steps where only zones 1..m < nzones move and no potential is wanted,
 * the field is synthesised only over the rings from jrad(1) to krad(m)
 * (findf.f:41-54, p3fndf.f:66-80): the forces on every moving particle are
 * those of the whole-grid solve, the other rings keep their last field.
 * GX_FLAG_WHOLE_GRID solves the whole grid on every step.  Mixed path; no
 * compensated positions, ensembles, adjoint or guard zones.  nzones = 1
 * restores the single-zone step. */
int gx_set_zones(GxCtx* ctx, int32_t nzones, const int32_t* nstep, const float* zbr);

/* The ring ranges (1-based, inclusive) of the next step's solve: rings[0..1]
 * the source rings jrs..krs holding mass, rings[2..3] the field rings jrf..krf
 * (1..nr on whole-grid steps) -- what findf.f:49-53 reports.  After gx_masset. */
int gx_zone_rings(GxCtx* ctx, int32_t* rings);

/* Zone of every particle in load order (1..nzones, nzones + 1 off the
 * grid) and the step counter; zone may be NULL. */
int gx_zone_info(GxCtx* ctx, int32_t* zone, int32_t* istep);

/* tmcent: move velocities half a step back (start != 0) or forward using
 * the current fields.  SRC/lib15/tmcent.f:83-90, tmcgrp.f. */
int gx_tmcent(GxCtx* ctx, int start);

/* icheck: KE, PE, Lz, virial and the m=2 amplitude, FP64 sums.
 * SRC/lib15/icheck.f:61-92. */
int gx_icheck(GxCtx* ctx, GxDiag* diag);

/* danl: sectoral harmonics of the surface density on the grid rings, as
 * densty.f:82-118, 190-250 writes them to the results file: the current
 * mass projected onto one plane, divided by each ring's area (ring i spans
 * grofu(i - 1/2) .. grofu(i + 1/2)) and scaled by sigmaf = 1 / (lscale ts^2);
 * then per ring the m = 0 term (the sum over spokes) and, for
 * m = 1 .. ng - 1, the cosine and sine sums divided by it.  w holds
 * 2 ng nr floats: real parts [nr][ng] (m = 0: the sum), then imaginary
 * parts [nr][ng] (m = 0: 0). */
int gx_danl(GxCtx* ctx, double sigmaf, float* w);

/* Device time of the last gx_step (ms, CUDA events on the context stream). */
int gx_last_step_ms(const GxCtx* ctx, float* ms);

/* Number of kernels launched by the last gx_step call. */
int gx_last_launch_count(const GxCtx* ctx, int64_t* n);

/* Multi-GPU particle decomposition (the reference's MPI overlay,
 * SRC/lib15_mpi/massum.f:54-65, p2manlp.f:164-233, p3manlp.f:102): every
 * rank holds its own particles and a full grid; once bound to a
 * communicator, every findf reduces the active ring range (min/max) and
 * sums the forward spectrum of the active harmonics over the ranks, so all
 * ranks solve for the fields of all particles.  gx_comm_unique_id fills
 * 128 bytes on one rank, the caller broadcasts them, and every rank calls
 * gx_comm_init with them.  Mixed path only. */
int gx_comm_unique_id(char* id128);
int gx_comm_init(GxCtx* ctx, const char* id128, int nranks, int rank);

/* The same exchanges through the host, for ranks that communicate through a
 * host process group (e.g. torch.distributed over gloo): the library copies
 * each buffer to host memory, calls fn(user, op, dtype, data, count) to
 * reduce the count elements at data in place over all ranks, and copies the
 * result back.  op is GX_OP_SUM, GX_OP_MIN or GX_OP_MAX; dtype GX_DT_INT32
 * or GX_DT_FLOAT32; fn returns 0 on success.  Every rank must make the same
 * calls in the same order (as it must with NCCL).  Replaces a communicator
 * bound by gx_comm_init.  Mixed path only.  (massum.f:54-65, p2manlp.f:208,
 * p3manlp.f:102, p3convp.f:276-326 exchange the same quantities over MPI.) */
#define GX_OP_SUM 0
#define GX_OP_MIN 1
#define GX_OP_MAX 2
#define GX_DT_INT32 0
#define GX_DT_FLOAT32 1
typedef int (*gx_host_reduce_fn)(void* user, int op, int dtype, void* data, int64_t count);
int gx_comm_host(GxCtx* ctx, int nranks, int rank, gx_host_reduce_fn fn, void* user);

/* massgn + scaled without allocating memory.  No counterpart in the
 * reference: it is for callers that may not allocate device memory when they
 * deposit mass, e.g. a host code that owns a fixed device memory pool, or a
 * time loop that must not wait on the allocator.  d_coords (n AoS records of
 * 2*ndim floats) and d_mass (mesh floats) are device pointers owned by the
 * caller; cfg gives the grid as for gx_grdset (mixed path only).  The result
 * equals the gx_masset mass array of the same particles (fixed-point
 * quantum 2^-32 instead of 2^-20).
 *  - Working memory is one file-scope device array of 2^22 cells (32 MiB),
 *    held by every GPU that loads the library until the process exits; a
 *    grid with more than 4194304 cells is rejected with GX_ERR_RANGE before
 *    any work is queued.
 *  - The first call on a device looks the array up (cudaGetSymbolAddress)
 *    with that device current.  Under CUDA's default lazy module loading
 *    that first call is also when the device loads the module and reserves
 *    the 32 MiB, so it can fail for lack of memory: make it at set-up, as a
 *    warm-up call with n = 0, before any stream capture.  The address is
 *    kept for the life of the process; cudaDeviceReset between calls is not
 *    supported.
 *  - The call selects cfg->device while it queues its work and puts the
 *    caller's current device back before it returns.
 *  - All calls share the array and each call clears it first, so calls
 *    whose work overlaps on the GPU (different streams, threads or
 *    processes sharing a context) race and must be serialised by the
 *    caller.
 *  - Work is queued on stream (a cudaStream_t); with stream NULL the call
 *    returns after the work completed.  Returns GX_OK or GX_ERR_ARG /
 *    GX_ERR_RANGE / GX_ERR_CUDA; no message is recorded. */
int gx_massgn_noalloc(const GxConfig* cfg, const float* d_coords, int64_t n, float* d_mass,
                      void* stream);

/* SFP method (sf2d, Abel-Jacobi basis).  A GxSfp holds the basis (as
 * Chebyshev series, built in FP64 from roots and coefficients) and a device
 * copy of particle positions.  SRC/lib15/sfpset.f:31-126,
 * sfptab.f:43-78, ajfun.f:33-47, ajsetup.f:23-58. */
typedef struct GxSfp GxSfp;
int gx_sfp_init(const GxSfpBasis* basis, double maxr, int device, GxSfp** out);
void gx_sfp_destroy(GxSfp* sfp);
const char* gx_sfp_last_error(const GxSfp* sfp);

/* Copy n particle records (stride floats each; x, y first, then vx, vy
 * when stride >= 4, else zero velocities) to the device. */
int gx_sfp_load(GxSfp* sfp, const float* coords, int64_t n, int stride);

/* sfpsum/sfpadd + scaled: coefficients of the loaded particles with
 * r <= maxr, x pmass / maxr^2, into coeff[n * (2 maxm + 1) + m + maxm]
 * (cosine terms at +m, sine terms at -m).  precision GX_PREC_MIXED runs the
 * moment contraction on the tensor cores with warp-level mma.sync m16n8k16
 * FP16 (operands split into FP16 hi and lo parts, 3 products, FP32
 * accumulate per 1024-particle chunk, FP64 across chunks);
 * GX_PREC_MIXED_TC05 on the tcgen05 tensor cores (all four hi/lo products
 * in one MMA of M = 128, N = 48, K = 16 per 16 particles, accumulator in
 * TMEM drained to FP64 every 1024 particles per CTA; at most 32 Chebyshev
 * terms and maxm <= 8); GX_PREC_FP64 on the CUDA cores in FP64.
 * SRC/lib15/sfpsum.f:26-47, sfpadd.f:37-93, scaled.f:53-72. */
int gx_sfp_sum(GxSfp* sfp, int precision, double pmass, double* coeff);

/* sfpacc: Cartesian accelerations [n][2] and potentials [n] (pot may be
 * NULL) of the loaded particles from scaled coefficients (FP64 evaluation).
 * SRC/lib15/sfpacc.f:41-112, 249-259. */
int gx_sfp_acc(GxSfp* sfp, const double* coeff, float* acc, float* pot);

/* Device ms and kernel launches of the last gx_sfp_sum. */
int gx_sfp_last_ms(const GxSfp* sfp, float* ms, int64_t* launches);

/* The SFP-driven time loop of the sf2d code (SRC/lib15/step.f:135-290:
 * getacc -> sfpacc, stpgrp, massgn -> sfpadd, sfpsum at step.f:250): nsteps
 * leapfrog steps of the loaded particles in the field of their own
 * coefficients.  Per step: the coefficients of the current positions
 * (gx_sfp_sum's arithmetic at `precision`, scaled by pmass), then
 * v += a(x) dt, x += v dt (stpgrp.f:26-32 with the time step explicit:
 * positions, velocities and dt in the caller's units, G = 1).  The
 * particles stay on the device; coeff_out (may be NULL) receives the
 * coefficients of the final positions. */
int gx_sfp_step(GxSfp* sfp, int nsteps, double dt, int precision, double pmass, double* coeff_out);

/* The loaded particles as n records of 4 floats (x, y, vx, vy). */
int gx_sfp_unload(GxSfp* sfp, float* coords);

/* Adjoint of nsteps mixed-path steps (2D, one sector) of the loaded
 * particles for the objective J = |A2(t_final)|, A2 = (1/n) sum_p
 * e^{2 i phi_p} over all particles.  The forward sweep (the arithmetic of
 * gx_step: massgn, findf + polcat, getacc with the ISOT halo, stpgrp) keeps
 * a checkpoint every ckpt_every steps; the reverse sweep recomputes the
 * trajectory backwards by time reversal (reset at each checkpoint) and
 * applies the transposed step: interpolation slopes, halo Jacobian, and the
 * transposed field solve (forward DFT, radial contraction with the same
 * Green table, synthesis, polcat, all transposed).  Outputs: J, grad[n][4] =
 * dJ/d(x, y, vx, vy) of the initial records in load order, dtheta[2] =
 * dJ/d(halo_rc, halo_v2) in config units, drift (may be NULL) = largest
 * |position difference| between the time-reversed trajectory and the
 * checkpoints.  Afterwards the context holds the initial particles and
 * their mass again.  No reference counterpart (the reference has no
 * gradients); its forward arithmetic is step.f:135-290 / stpgrp.f:26-32. */
int gx_adjoint(GxCtx* ctx, int nsteps, int ckpt_every, double* J, float* grad, double* dtheta,
               float* drift);

/* Ensemble of independent 2D discs sharing one grid geometry (one Green
 * table), advanced together: every step is one persistent cooperative
 * launch for all discs (field solve per disc, then push + deposit of every
 * particle), and batches of 16 step launches are replayed from a CUDA graph.
 * Each disc follows the single-disc run of SRC/progs/galaxy.f:107-148
 * (findf, getacc + stpgrp, massgn: the same cell keys, weights and integer
 * deposit; FP32 transforms summed in a different order, so fields agree to
 * FP32 rounding, not bitwise).  No single reference routine: it batches the
 * reference's per-run loop over runs.
 *  - cfg: the shared 2D grid (ndim 2, mixed precision; cfg->pmass ignored);
 *    at most 12800 cells (16 B per cell of shared memory).
 *  - counts[ndisc], pmass[ndisc]: particles and particle mass of each disc;
 *    coords: sum(counts) records (x, y, vx, vy) in grid units, disc after
 *    disc.  max_steps bounds the recorded A2 series.
 *  - create builds the Green table, deposits the initial mass (masset) and
 *    records A2 at step 0. */
typedef struct GxEnsemble GxEnsemble;
int gx_ensemble_create(const GxConfig* cfg, int ndisc, const int64_t* counts, const float* pmass,
                       const float* coords, int max_steps, GxEnsemble** out);
void gx_ensemble_destroy(GxEnsemble* ens);
const char* gx_ensemble_last_error(const GxEnsemble* ens);

/* Autotuner: times each (threads per CTA, particles per chunk) candidate
 * over a few steps from a snapshot of the state, restores the state and
 * keeps the fastest; returns the choice. */
int gx_ensemble_tune(GxEnsemble* ens, int* threads, int* chunk);

/* Current launch shape: threads per CTA, particles per chunk, CTAs, and
 * whether the steps are replayed from a CUDA graph (1) or launched one by
 * one (0). */
int gx_ensemble_config(const GxEnsemble* ens, int* threads, int* chunk, int* grid, int* graph);

/* Advance every disc nsteps leapfrog steps. */
int gx_ensemble_step(GxEnsemble* ens, int nsteps);
int gx_ensemble_steps_done(const GxEnsemble* ens, int64_t* n);

/* m = 2 amplitude of every disc after every step:
 * out[(s * ndisc + d) * 2 + {0, 1}] = mean over the disc's particles on the
 * grid of (cos 2 phi, sin 2 phi), s = 0 .. steps_done (FP64 sums). */
int gx_ensemble_a2(GxEnsemble* ens, double* out, int64_t cap);

/* Particle records (x, y, vx, vy) of all discs, in the order of create. */
int gx_ensemble_unload(GxEnsemble* ens, float* coords);

/* Device ms and kernel launches of the last gx_ensemble_step. */
int gx_ensemble_last_ms(const GxEnsemble* ens, float* ms, int64_t* launches);

/* Page-locked host buffers for gx_loadup/gx_unload (cudaMallocHost in the
 * library's own runtime).  No reference counterpart. */
int gx_host_alloc(int64_t bytes, void** ptr);
int gx_host_free(void* ptr);

/* Phase timing of gx_step: on != 0 records CUDA events between the phases
 * of every step (forward transform, radial contraction, synthesis,
 * particle pass, sort, deposit, mass combine, other) on the context
 * stream.  No reference counterpart (instrumentation). */
int gx_set_profile(GxCtx* ctx, int on);

/* Accumulated device ms and step counts per phase since the last
 * gx_set_profile(ctx, 1); arrays of 8. */
int gx_phase_ms(const GxCtx* ctx, float* ms, int64_t* count);

#ifdef __cplusplus
}
#endif
#endif /* GALAXY_GPU_H */
