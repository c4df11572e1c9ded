/* gx_shim_driver.c -- a C program in the place of GALAXY's Fortran main
 * program and its iso_c_binding shim, on the library's C ABI alone
 * (include/galaxy_gpu.h, libgalaxy_gpu.so).  Test infrastructure: it shows
 * that a compiled caller drives the path with nothing but the C ABI.
 *
 * It reads the grid cards of a run file in the reference's .dat syntax
 * (the values grdset / setgrd take from the COMMON blocks:
 * SRC/lib15/grdset.f:23-42, setgrd.f:52-200, p3dset.f:22-101,
 * filset.f:116-142) into a GxConfig field by field, then calls the entry
 * points in the order of SRC/progs/galaxy.f: greenm (galaxy.f:76), the
 * particle load and masset (galaxy.f:98), tmcent, and per step findf(phys)
 * + step (galaxy.f:114-118, both done by gx_step), the integral check on
 * analysis steps, and the particles out as at dumpp.
 *
 *   gx_shim_driver <run.dat> <records.f32> <n> <nsteps> <iphys> <out.f32> <checks.txt>
 *
 * Cards read: "grid type p2d|p3d", "grid size nr na [ngz]", "z spacing",
 * "hash", "softl <length> <rule>", "sect", "skip <m...>", "lscale",
 * "zones <n>" followed by n - 1 lines "<step ratio> <radius>" (radii in
 * model units, times lscale for the grid), and two lines the shim fills
 * from elsewhere: "gx pmass <mass in internal units>" (loadup.f:97-99) and
 * "gx isot <v^2> <rc>" (the rigid halo in grid units, frhalo.f:55-56).
 * Exit status 0 on success; on a library error the message of
 * gx_last_error and status 2, as crash.f stops the run. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "galaxy_gpu.h"

static GxCtx* ctx = NULL;

static void check(int rc, const char* where) {
    if (rc == GX_OK) return;
    fprintf(stderr, "crash in %s: %s (%d)\n", where, gx_last_error(ctx), rc);
    if (ctx) gx_destroy(ctx);
    exit(2);
}

int main(int argc, char** argv) {
    if (argc != 8) {
        fprintf(stderr, "usage: %s run.dat records.f32 n nsteps iphys out.f32 checks.txt\n", argv[0]);
        return 1;
    }
    GxConfig cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.nsect = 1;
    cfg.tsoft = GX_SOFT_PLUMMER;
    cfg.rmap = GX_RMAP_STDPOL;  /* the reference's u = ln(1 + r) / alpha */
    cfg.precision = GX_PREC_MIXED;
    int nzones = 1, nstep[GX_MAX_ZONES] = {1};
    float zrad[GX_MAX_ZONES] = {0.f}, lscale = 1.f;
    FILE* f = fopen(argv[1], "r");
    if (!f) {
        perror(argv[1]);
        return 1;
    }
    char line[512];
    int zone_lines = 0;
    while (fgets(line, sizeof line, f)) {
        char* hash = strchr(line, '#');
        if (hash) *hash = 0;
        if (zone_lines > 0) {  /* "<step ratio> <radius>" of the next zone */
            int k = nzones - zone_lines;
            if (sscanf(line, "%d %f", &nstep[k], &zrad[k]) == 2) zone_lines--;
            continue;
        }
        char t[64];
        if (sscanf(line, "grid type %63s", t) == 1) cfg.ndim = strcmp(t, "p3d") == 0 ? 3 : 2;
        else if (strncmp(line, "grid size", 9) == 0) {
            int n3 = sscanf(line + 9, "%d %d %d", &cfg.nr, &cfg.na, &cfg.ngz);
            if (n3 < 3) cfg.ngz = 1;
        } else if (sscanf(line, "z spacing %f", &cfg.dzg) == 1) {
        } else if (sscanf(line, "hash %d", &cfg.ng) == 1) {
            cfg.ng += 1;  /* harmonics m = 0 .. hash */
        } else if (strncmp(line, "softl", 5) == 0) {
            sscanf(line + 5, "%f %d", &cfg.softl, &cfg.tsoft);
        } else if (sscanf(line, "sect %d", &cfg.nsect) == 1) {
        } else if (strncmp(line, "skip", 4) == 0) {
            char* p = line + 4;
            int m, used;
            while (cfg.nskip < GX_MAX_SKIP && sscanf(p, "%d%n", &m, &used) == 1) {
                cfg.skip[cfg.nskip++] = m;
                p += used;
            }
        } else if (sscanf(line, "lscale %f", &lscale) == 1) {
        } else if (sscanf(line, "zones %d", &nzones) == 1) {
            if (nzones < 1 || nzones > GX_MAX_ZONES) return 1;
            zone_lines = nzones - 1;
        } else if (sscanf(line, "gx pmass %f", &cfg.pmass) == 1) {
        } else if (sscanf(line, "gx isot %f %f", &cfg.halo_v2, &cfg.halo_rc) == 2) {
            cfg.halo = 1;
        }
    }
    fclose(f);
    const int nw = 2 * cfg.ndim;
    const long long n = atoll(argv[3]);
    const int nsteps = atoi(argv[4]), iphys = atoi(argv[5]);
    float* rec = (float*)malloc(sizeof(float) * nw * (n > 0 ? n : 1));
    f = fopen(argv[2], "rb");
    if (!f || fread(rec, sizeof(float) * nw, (size_t)n, f) != (size_t)n) {
        fprintf(stderr, "cannot read %lld records from %s\n", n, argv[2]);
        return 1;
    }
    fclose(f);

    check(gx_grdset(&cfg, &ctx), "GRDSET");
    check(gx_greenm(ctx), "GREENM");
    if (nzones > 1) {
        float zbr[GX_MAX_ZONES];
        for (int k = 0; k < nzones; k++) zbr[k] = zrad[k] * lscale;
        check(gx_set_zones(ctx, nzones, nstep, zbr), "SETRUN");
    }
    check(gx_loadup(ctx, rec, n), "LOADUP");
    check(gx_masset(ctx), "MASSET");
    check(gx_findf(ctx, 0), "FINDF");
    check(gx_tmcent(ctx, 1), "TMCENT");
    FILE* out = fopen(argv[7], "w");
    for (int istep = 1; istep <= nsteps; istep++) {
        const int phys = (iphys > 0) && (istep % iphys == 0);
        check(gx_step(ctx, 1, phys), "STEP");
        if (phys) {
            GxDiag d;
            check(gx_findf(ctx, 1), "FINDF");
            check(gx_icheck(ctx, &d), "ICHECK");
            fprintf(out, "%d %.9e %.9e %.9e\n", istep, d.ke, d.pe, d.lz);
        }
    }
    fclose(out);
    check(gx_unload(ctx, rec), "DUMPP");
    f = fopen(argv[6], "wb");
    fwrite(rec, sizeof(float) * nw, (size_t)n, f);
    fclose(f);
    gx_destroy(ctx);
    free(rec);
    return 0;
}
