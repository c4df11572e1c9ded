/*
 * gx_oracle.h -- CPU restatement of the GALAXY v15 polar-grid PM step.
 *
 * TEST INFRASTRUCTURE ONLY.  The CUDA path's results are checked against it:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it.  The product path (galaxy_b200/libgalaxy_gpu.so) never links or
 * calls it.
 *
 * The reference (Fortran 77, SRC/lib15) cannot be compiled here (no
 * Fortran compiler), so each routine below restates the reference routine it
 * names, in the reference's loop order, in two flavours built from one
 * template (gx_oracle_tmpl.h):
 *   *_f64  FP64 throughout (the accuracy oracle),
 *   *_f32  FP32 "mirror": the reference's single-precision expressions and
 *          operation order (keys, weights, kernels, sums).  Transforms are
 *          direct sums with the FFTPACK conventions, not FFTPACK itself.
 * Parity pin: tests/test_oracle_ftest.py checks the p3d point-mass field
 * values printed in EXAMPLES/p3d/ftest/run999.lis:26-30.
 *
 * Layouts (shared with the CUDA library):
 *   particle records   AoS, 2*ndim words: x, y[, z], vx, vy[, vz]
 *   mesh arrays        [ir][iz][it]  (ncl - 1 of SRC/lib15/weight.f:236)
 *   Green table        [type 0..3][m 0..ng-1][kz 0..nkz-1][is][ir]
 *                      type: 0 radial, 1 azimuthal, 2 vertical, 3 potential;
 *                      nkz = ngz + 1 (3D) or 1 (2D)
 *   direct table       [type][is][ir][jz 0..nkz-1][k 0..na/2]
 */
#ifndef GX_ORACLE_H
#define GX_ORACLE_H
#include <stdint.h>
#include "../include/galaxy_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

int ox_geometry(const GxConfig* cfg, GxGeometry* geo, char* err, int errlen);
/* host threads of the restated loops; 1 (the default) runs them in the
 * reference's sequential order */
int ox_set_threads(int n);
int64_t ox_green_size(const GxConfig* cfg);
int64_t ox_direct_size(const GxConfig* cfg);

#define OX_DECL(R, S)                                                          \
int ox_green_##S(const GxConfig* cfg, R* G, R* D);                             \
int ox_weight_##S(const GxConfig* cfg, int old, int64_t n, const R* pos,       \
                  int32_t* key, R* wt, uint8_t* on);                           \
int ox_massgn_##S(const GxConfig* cfg, int64_t n, const int32_t* key,          \
                  const R* wt, const uint8_t* on, R* mass, int32_t* jrk);      \
int ox_findf_##S(const GxConfig* cfg, const R* G, const R* mass, int lpot,     \
                 int jrs, int krs, R* fields);                                 \
int ox_polcat_##S(const GxConfig* cfg, R* fields);                             \
int ox_grdacc_##S(const GxConfig* cfg, int64_t n, const R* pos,                \
                  const R* fields, int phys, R* acc, R* pot);                  \
int ox_masset_##S(const GxConfig* cfg, int64_t n, const R* pos, R* mass,       \
                  int32_t* jrk);                                               \
int ox_particle_pass_##S(const GxConfig* cfg, int64_t n, R* pos, const R* fields,   \
                         R* mass, int32_t* jrk);                               \
int ox_step_##S(const GxConfig* cfg, const R* G, int64_t n, R* pos, R* mass,   \
                int32_t* jrk, int nsteps, int phys, R* fields);                \
int ox_direct_field_##S(const GxConfig* cfg, const R* D, int nmass,            \
                        const int32_t* mr, const int32_t* mt,                  \
                        const int32_t* mz, const R* mm, int lpot, R* fields);

OX_DECL(double, f64)
OX_DECL(float, f32)

/* SFP Abel-Jacobi method (gx_oracle_sfp.c), FP64 */
double ox_ajfun(const GxSfpBasis* b, int m, int n, double r);
double ox_ajder(const GxSfpBasis* b, int m, int n, double r);
int ox_sfp_coeffs(const GxSfpBasis* b, int64_t n, const double* pos, int stride, double maxr,
                  double pmass, double* coeff);
int ox_sfp_acc(const GxSfpBasis* b, const double* coeff, int64_t n, const double* pos, int stride,
               double maxr, double* acc, double* pot);

/* adjoint of the 2D step in FP64 (gx_oracle_adj.h): J = |A2(x_T)| over
 * all particles; pos records (x, y, vx, vy); grad [n][4]; dtheta = dJ/d
 * (halo_rc, halo_v2) */
int ox_adj_forward(const GxConfig* cfg, const double* G, int64_t n, double* pos, int nsteps,
                   double* a2, double* J);
int ox_adj_gradient(const GxConfig* cfg, const double* G, int64_t n, const double* pos0,
                    int nsteps, double* grad, double* dtheta, double* J);

/* multiple time-step zones of the p2d/p3d step in FP64 (gx_oracle_zone.h).
 * Zone codes 1..nzones, nzones + 1 off the grid; zm, zo [nzones][mesh]. */
typedef struct OxZones {
    int32_t nzones;
    int32_t nstep[GX_MAX_ZONES];
    double zbr[GX_MAX_ZONES];      /* zbr[0] unused: zone 1 starts at the centre */
    int32_t istep;
    int32_t lstep[GX_MAX_ZONES][2];  /* step numbers of the older and newer arrays */
    int32_t jrk[GX_MAX_ZONES][2];    /* 1-based ring range of each zone's mass */
} OxZones;
int ox_zone_setup(const GxConfig* cfg, OxZones* z, int64_t n, double* pos, int32_t* zone);
int ox_zone_unscale(const GxConfig* cfg, const OxZones* z, int64_t n, double* pos,
                    const int32_t* zone);
int ox_zone_masset(const GxConfig* cfg, OxZones* z, int64_t n, const double* pos,
                   const int32_t* zone, double* zm, double* zo, int32_t* jrk);
int ox_zone_step(const GxConfig* cfg, OxZones* z, const double* G, int64_t n, double* pos,
                 int32_t* zone, double* zm, double* zo, int32_t* jrk, int nsteps);

/* danl density harmonics of the grid rings in FP64 (densty.f); w is
 * 2 ng nr: real parts [nr][ng] then imaginary parts */
int ox_danl(const GxConfig* cfg, const double* mass, double sigmaf, double* w);

/* icheck-style integrals in FP64 from FP64 particle records and potentials */
int ox_icheck(const GxConfig* cfg, int64_t n, const double* pos,
              const double* acc, const double* pot, double pmass_phys,
              GxDiag* d);

#ifdef __cplusplus
}
#endif
#endif
