/*
 * Drop-in drivers chanfast2 / chanfast4 / channel2 / channel4 in C over the
 * chanfast_cuda C ABI.
 *
 * Same arguments and file protocol as the reference drivers (chanfast.h:1-21,
 * chanfast.c:71-992 / 995-1916; channel.h:1-21, channel.c:71-1018 /
 * 1021-1968, the same loop with the fully implicit substep).  One GPU holds
 * the whole grid, so the pencil decomposition p_row x p_col has nothing to
 * split:
 *   - a single process (no MPI launcher, or one rank) runs whatever p_row x
 *     p_col it is given, with a one-line note on stderr when that is not
 *     1 x 1 -- the reference's main.c passes 2 x 2 (main.c:9-10);
 *   - under an MPI launcher with N > 1 ranks, p_row x p_col must equal N as
 *     in the reference (chanfast.c:87; CF_EINVAL otherwise); rank 0 then
 *     runs the whole grid on its GPU and writes every file, and the other
 *     ranks return at once without touching a GPU or a file.  The rank and
 *     size come from the launcher's environment (Open MPI, MPICH / Hydra,
 *     PMIx, Slurm), so the library needs no MPI itself.
 * The run itself:
 *   - read outputdir/{u,v,w,c}_it<it>.dat (raw FP64, C order [nx][ny][nz],
 *     io.c:259-297)
 *   - for it in [it, nt): CFL of the current field (get.c:390-416), adapt dt
 *     if cflmode == 1, append "it dt cfl" to outputdir/cfl.dat; three RK3
 *     substeps on the GPU; append the mass-flux and scalar-mean statistics of
 *     the last substep to outputdir/pstat.dat and outputdir/cstat.dat
 *     (chanfast.c:525-528, 612-615)
 *   - every istat steps: the statistics of chanfast.c:658-857 (channel.c:
 *     692-891) as ASCII files (io.c:22-35, one %+e per line): xy averages,
 *     correlations, moments and x / y spectra, zp.dat and zw.dat, then the
 *     restart files outputdir/{u,v,w,c}_it<it+1>.dat (io.c:211-257)
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "chanfast_cuda.h"

static int read_field(cf_instance *inst, int field, const char *name, int it, size_t n)
{
    char fname[256];
    snprintf(fname, sizeof fname, "outputdir/%s_it%d.dat", name, it);
    FILE *fp = fopen(fname, "rb");
    if (!fp) return CF_EIO;
    double *buf = (double *) malloc(n * sizeof(double));
    if (!buf) { fclose(fp); return CF_ENOMEM; }
    size_t got = fread(buf, sizeof(double), n, fp);
    fclose(fp);
    int rc = got == n ? cf_set_field(inst, field, buf, CF_LAYOUT_INTERIOR) : CF_EIO;
    free(buf);
    return rc;
}

static int write_field(cf_instance *inst, int field, const char *name, int it, size_t n)
{
    char fname[256];
    snprintf(fname, sizeof fname, "outputdir/%s_it%d.dat", name, it);
    double *buf = (double *) malloc(n * sizeof(double));
    if (!buf) return CF_ENOMEM;
    int rc = cf_get_field(inst, field, buf, CF_LAYOUT_INTERIOR);
    if (rc == CF_OK) {
        FILE *fp = fopen(fname, "wb");
        if (!fp) rc = CF_EIO;
        else {
            if (fwrite(buf, sizeof(double), n, fp) != n) rc = CF_EIO;
            if (fclose(fp) != 0) rc = CF_EIO;
        }
    }
    free(buf);
    return rc;
}

/* io_write_ascii (io.c:22-35) */
static int write_ascii(const double *u, size_t n, const char *name, int it)
{
    char fname[256];
    if (it >= 0) snprintf(fname, sizeof fname, "outputdir/%s_it%d.dat", name, it);
    else snprintf(fname, sizeof fname, "outputdir/%s.dat", name);
    FILE *fp = fopen(fname, "w");
    if (!fp) return CF_EIO;
    for (size_t i = 0; i < n; i++) fprintf(fp, "%+e\n", u[i]);
    return fclose(fp) == 0 ? CF_OK : CF_EIO;
}

/* The istat block of chanfast.c:658-843 in its order. */
static int write_stats(cf_instance *inst, const cf_config *cfg, int it)
{
    const size_t n2 = (size_t) cfg->nz + 2 * cfg->ngz;
    const size_t nsx = (size_t) (cfg->nx / 2 + 1) * n2 * 2, nsy = (size_t) (cfg->ny / 2 + 1) * n2 * 2;
    double *prof = (double *) malloc(n2 * sizeof(double));
    double *sx = (double *) malloc(nsx * sizeof(double)), *sy = (double *) malloc(nsy * sizeof(double));
    double *zw = (double *) malloc(n2 * sizeof(double));
    int rc = prof && sx && sy && zw ? CF_OK : CF_ENOMEM;
    static const struct { const char *name; int f; } avg[] = {
        {"u_avg", CF_U}, {"v_avg", CF_V}, {"w_avg", CF_W}, {"c_avg", CF_C}, {"p_avg", CF_P}};
    static const struct { const char *name; int a, b; } pairs[] = {
        {"uu", CF_U, CF_U}, {"vv", CF_V, CF_V}, {"ww", CF_W, CF_W}, {"cc", CF_C, CF_C},
        {"pp", CF_P, CF_P}, {"wu", CF_W, CF_U}, {"uc", CF_U, CF_C}, {"wc", CF_W, CF_C}};
    char name[64];
    for (int q = 0; q < 5 && rc == CF_OK; q++) {
        rc = cf_xy_avg(inst, avg[q].f, prof);
        if (rc == CF_OK) rc = write_ascii(prof, n2, avg[q].name, it);
    }
    for (int q = 0; q < 8 && rc == CF_OK; q++) {
        rc = cf_xy_corr(inst, pairs[q].a, pairs[q].b, prof);
        snprintf(name, sizeof name, "%s_corr", pairs[q].name);
        if (rc == CF_OK) rc = write_ascii(prof, n2, name, it);
    }
    for (int q = 3; q <= 4 && rc == CF_OK; q++) {
        rc = cf_xy_moment(inst, CF_U, (double) q, prof);
        snprintf(name, sizeof name, "u_mom%d", q);
        if (rc == CF_OK) rc = write_ascii(prof, n2, name, it);
    }
    for (int q = 0; q < 8 && rc == CF_OK; q++) {
        rc = cf_xy_spec(inst, pairs[q].a, pairs[q].b, sx, sy);
        snprintf(name, sizeof name, "%s_specx", pairs[q].name);
        if (rc == CF_OK) rc = write_ascii(sx, nsx, name, it);
        snprintf(name, sizeof name, "%s_specy", pairs[q].name);
        if (rc == CF_OK) rc = write_ascii(sy, nsy, name, it);
    }
    if (rc == CF_OK) rc = cf_z_coords(inst, prof, zw);
    if (rc == CF_OK) rc = write_ascii(prof, n2, "zp", -1);
    if (rc == CF_OK) rc = write_ascii(zw, n2, "zw", -1);
    free(prof);
    free(sx);
    free(sy);
    free(zw);
    return rc;
}

/* io_append_ascii (io.c:5-19) */
static int append_ascii(const double *u, int n, const char *filename)
{
    FILE *fp = fopen(filename, "a");
    if (!fp) return CF_EIO;
    fprintf(fp, "%+e", u[0]);
    for (int i = 1; i < n; i++) fprintf(fp, " %+e", u[i]);
    fprintf(fp, "\n");
    return fclose(fp) == 0 ? CF_OK : CF_EIO;
}

/* World size and rank of this process as its MPI launcher exported them;
 * 1 and 0 when no launcher did. */
static void launcher_rank(int *size, int *rank)
{
    static const char *const sizes[] = {"OMPI_COMM_WORLD_SIZE", "PMI_SIZE", "PMIX_SIZE", "SLURM_NTASKS"};
    static const char *const ranks[] = {"OMPI_COMM_WORLD_RANK", "PMI_RANK", "PMIX_RANK", "SLURM_PROCID"};
    *size = 1;
    *rank = 0;
    for (int q = 0; q < 4; q++) {
        const char *s = getenv(sizes[q]), *r = getenv(ranks[q]);
        if (s && r && atoi(s) > 0) {
            *size = atoi(s);
            *rank = atoi(r);
            return;
        }
    }
}

static int run(int order, int scheme, int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
               int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
               double dt, double want_cfl, int cflmode, double nu, double prandtl,
               double dpdx, double want_uvolavg, int uvolavgmode,
               double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
               double betg_x, double betg_y, double betg_z)
{
    if (p_row < 1 || p_col < 1 || istat <= 0) return CF_EINVAL;
    int nproc, rank;
    launcher_rank(&nproc, &rank);
    if (nproc > 1) {
        if (p_row * p_col != nproc) return CF_EINVAL;
        if (rank != 0) return CF_OK;
    } else if (p_row * p_col != 1) {
        fprintf(stderr, "%s%d: p_row x p_col = %d x %d: one GPU holds the whole %d x %d x %d grid\n",
                scheme == CF_SCHEME_CHANNEL ? "channel" : "chanfast", order, p_row, p_col, nx, ny, nz);
    }
    cf_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.order = order;
    cfg.nx = nx; cfg.ny = ny; cfg.nz = nz;
    cfg.ngx = nghost_x; cfg.ngy = nghost_y; cfg.ngz = nghost_z;
    cfg.uvolavgmode = uvolavgmode; cfg.cvolavgmode = cvolavgmode;
    cfg.lx = lx; cfg.ly = ly; cfg.lz = lz;
    cfg.dt = dt; cfg.nu = nu; cfg.prandtl = prandtl; cfg.dpdx = dpdx;
    cfg.want_uvolavg = want_uvolavg; cfg.want_cvolavg = want_cvolavg;
    cfg.setuframe = setuframe; cfg.setvframe = setvframe;
    cfg.betg_x = betg_x; cfg.betg_y = betg_y; cfg.betg_z = betg_z;
    cfg.scheme = scheme;

    cf_instance *inst = NULL;
    int rc = cf_create(&cfg, NULL, &inst);
    if (rc) return rc;
    const size_t n = (size_t) nx * ny * nz;
    const char *names[4] = {"u", "v", "w", "c"};
    const int fields[4] = {CF_U, CF_V, CF_W, CF_C};
    for (int f = 0; f < 4 && rc == CF_OK; f++) rc = read_field(inst, fields[f], names[f], it, n);

    double log[10];
    for (; rc == CF_OK && it < nt; it++) {
        double cfl = 0.0;
        rc = cf_cfl(inst, dt, &cfl);
        if (rc) break;
        if (cflmode == 1) {  /* chanfast.c:388-391 */
            double ndt = dt * (cfl > 0.0 ? want_cfl / cfl : 1.0);
            cfl = cfl > 0.0 ? want_cfl : cfl;
            if (ndt != dt) {
                dt = ndt;
                rc = cf_set_dt(inst, dt);
                if (rc) break;
            }
        }
        double row[3] = {(double) it, dt, cfl};
        rc = append_ascii(row, 3, "outputdir/cfl.dat");
        if (rc) break;
        rc = cf_step(inst, 3);
        if (rc) break;
        long got = cf_get_log(inst, log, 1);
        if (got != 1) { rc = got < 0 ? (int) got : CF_ECUDA; break; }
        double ps[6] = {(double) (it + 1), log[0], log[1], log[2], log[3], log[4]};
        double cs[6] = {(double) (it + 1), log[5], log[6], log[7], log[8], log[9]};
        rc = append_ascii(ps, 6, "outputdir/pstat.dat");
        if (rc == CF_OK) rc = append_ascii(cs, 6, "outputdir/cstat.dat");
        if (rc == CF_OK && (it + 1) % istat == 0) {
            rc = write_stats(inst, &cfg, it + 1);
            for (int f = 0; f < 4 && rc == CF_OK; f++) rc = write_field(inst, fields[f], names[f], it + 1, n);
        }
    }
    int rc2 = cf_destroy(inst);
    return rc ? rc : rc2;
}

int chanfast2_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                     int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                     double dt, double want_cfl, int cflmode, double nu, double prandtl,
                     double dpdx, double want_uvolavg, int uvolavgmode,
                     double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                     double betg_x, double betg_y, double betg_z)
{
    return run(2, CF_SCHEME_CHANFAST, p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z, lx, ly, lz,
               dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg, uvolavgmode, want_cvolavg,
               cvolavgmode, setuframe, setvframe, betg_x, betg_y, betg_z);
}

int chanfast4_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                     int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                     double dt, double want_cfl, int cflmode, double nu, double prandtl,
                     double dpdx, double want_uvolavg, int uvolavgmode,
                     double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                     double betg_x, double betg_y, double betg_z)
{
    return run(4, CF_SCHEME_CHANFAST, p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z, lx, ly, lz,
               dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg, uvolavgmode, want_cvolavg,
               cvolavgmode, setuframe, setvframe, betg_x, betg_y, betg_z);
}

void chanfast2(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
               int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
               double dt, double want_cfl, int cflmode, double nu, double prandtl,
               double dpdx, double want_uvolavg, int uvolavgmode,
               double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
               double betg_x, double betg_y, double betg_z)
{
    int rc = chanfast2_status(p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
                              lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg,
                              uvolavgmode, want_cvolavg, cvolavgmode, setuframe, setvframe,
                              betg_x, betg_y, betg_z);
    if (rc) fprintf(stderr, "chanfast2: %s\n", cf_strerror(rc));
}

void chanfast4(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
               int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
               double dt, double want_cfl, int cflmode, double nu, double prandtl,
               double dpdx, double want_uvolavg, int uvolavgmode,
               double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
               double betg_x, double betg_y, double betg_z)
{
    int rc = chanfast4_status(p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
                              lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg,
                              uvolavgmode, want_cvolavg, cvolavgmode, setuframe, setvframe,
                              betg_x, betg_y, betg_z);
    if (rc) fprintf(stderr, "chanfast4: %s\n", cf_strerror(rc));
}

int channel2_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                    int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                    double dt, double want_cfl, int cflmode, double nu, double prandtl,
                    double dpdx, double want_uvolavg, int uvolavgmode,
                    double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                    double betg_x, double betg_y, double betg_z)
{
    return run(2, CF_SCHEME_CHANNEL, p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
               lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg, uvolavgmode,
               want_cvolavg, cvolavgmode, setuframe, setvframe, betg_x, betg_y, betg_z);
}

int channel4_status(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
                    int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
                    double dt, double want_cfl, int cflmode, double nu, double prandtl,
                    double dpdx, double want_uvolavg, int uvolavgmode,
                    double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
                    double betg_x, double betg_y, double betg_z)
{
    return run(4, CF_SCHEME_CHANNEL, p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
               lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg, uvolavgmode,
               want_cvolavg, cvolavgmode, setuframe, setvframe, betg_x, betg_y, betg_z);
}

void channel2(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
              int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
              double dt, double want_cfl, int cflmode, double nu, double prandtl,
              double dpdx, double want_uvolavg, int uvolavgmode,
              double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
              double betg_x, double betg_y, double betg_z)
{
    int rc = channel2_status(p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
                             lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg,
                             uvolavgmode, want_cvolavg, cvolavgmode, setuframe, setvframe,
                             betg_x, betg_y, betg_z);
    if (rc) fprintf(stderr, "channel2: %s\n", cf_strerror(rc));
}

void channel4(int p_row, int p_col, int nx, int ny, int nz, int it, int nt, int istat,
              int nghost_x, int nghost_y, int nghost_z, double lx, double ly, double lz,
              double dt, double want_cfl, int cflmode, double nu, double prandtl,
              double dpdx, double want_uvolavg, int uvolavgmode,
              double want_cvolavg, int cvolavgmode, double setuframe, double setvframe,
              double betg_x, double betg_y, double betg_z)
{
    int rc = channel4_status(p_row, p_col, nx, ny, nz, it, nt, istat, nghost_x, nghost_y, nghost_z,
                             lx, ly, lz, dt, want_cfl, cflmode, nu, prandtl, dpdx, want_uvolavg,
                             uvolavgmode, want_cvolavg, cvolavgmode, setuframe, setvframe,
                             betg_x, betg_y, betg_z);
    if (rc) fprintf(stderr, "channel4: %s\n", cf_strerror(rc));
}
