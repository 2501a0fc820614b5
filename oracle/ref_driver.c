/*
 * Oracle driver around the UNMODIFIED reference sources -- TEST
 * INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file.
 *
 * The reference keeps its state inside chanfast2/chanfast4 (chanfast.c:71-992,
 * 995-1916) and only exchanges fields through restart files.  To compare the
 * pressure and per-substep intermediates, this driver performs the same setup
 * as chanfast.c:85-192 and then replays the RK3 substep body of
 * chanfast.c:395-656 (order 2) / :1319-1580 (order 4), calling the reference's
 * own step functions in the same order with the same arguments.  The only
 * differences from chanfast are: fields come from and go back to caller
 * memory instead of restart files, the ASCII logs are kept in memory, and
 * dt is fixed (cflmode = 0).  tests/ checks this replay against the real
 * chanfast2/chanfast4 entry points (bit-identical u, v, w, c).
 *
 * ref_channel_substeps replays the fully implicit substep of channel2 /
 * channel4 (channel.c:392-690 / :1342-1640) the same way: explicit terms
 * without the x-y Laplacian, then per field the 3-D Helmholtz operator,
 * FFT3D_FWD, solve_helmholtz_{u,w}, FFT3D_BWD; tests/ checks it against the
 * real channel2/channel4 entry points (ref_channel).
 *
 * Also exported: the case-1 style projection (cases.c:426-470) used to make
 * initial states divergence-free, and the reference divergence operator.
 */
#include <setjmp.h>
#include <stdint.h>
#include <string.h>
#include <unistd.h>

#include "check.h"
#include "d3tensor.h"
#include "c3tensor.h"
#include "decomp.h"
#include "transpose.h"
#include "fft.h"
#include "ghostz.h"
#include "ghost.h"
#include "get.h"
#include "rk3.h"
#include "fourth.h"
#include "pressure.h"
#include "diffuseu.h"
#include "diffusew.h"
#include "advect.h"
#include "scalar.h"
#include "chanfast.h"
#include "channel.h"
#include "cases.h"

extern jmp_buf *shim_abort_target;

typedef struct ref_params {
    int order, nx, ny, nz, ngx, ngy, ngz;
    int uvolavgmode, cvolavgmode;
    double lx, ly, lz, dt, nu, prandtl, dpdx;
    double want_uvolavg, want_cvolavg, setuframe, setvframe;
    double betg_x, betg_y, betg_z;
} ref_params;

#define REF_LOG_COLS 10

typedef struct ref_ctx {
    ref_params prm;
    MPI_Comm comm_cart;
    MPI_Datatype cplx_t;
    decomp_plan *decomp_d, *decomp_c;
    transpose_plan *transp_d, *transp_c;
    fftx_plan *fftx_p;
    ffty_plan *ffty_p;
    ghostz_plan *ghostz_p;
    int local_nx, local_ny, n0, n1, n2, local_size;
    double dx, dy;
    double *xp, *xu, *yp, *yv, *dz, *zp, *zw, *avg;
    double ***zwork_d1;
    fftw_complex ***zwork_c1;
    double ***bc_3d, ***hbc_3d, ***u_3d, ***v_3d, ***w_3d, ***c_3d, ***p_3d, ***h_3d;
    double ***m1_3d, ***m2_3d, ***m3_3d;
    double ***f_3d[4], ***g_3d[4];
    double *fcur[4], *gcur[4];   /* current f/g pointers (swapped each substep) */
    long substep;                /* substeps done so far */
    double *log;                 /* REF_LOG_COLS values per substep */
    long log_cap;
} ref_ctx;

static double uframe_s, vframe_s;
static double bc_u_bot(double x, double y) { (void) x; (void) y; return 0.0 - uframe_s; }
static double bc_u_top(double x, double y) { (void) x; (void) y; return 0.0 - uframe_s; }
static double bc_v_bot(double x, double y) { (void) x; (void) y; return 0.0 - vframe_s; }
static double bc_v_top(double x, double y) { (void) x; (void) y; return 0.0 - vframe_s; }
static double bc_w_bot(double x, double y) { (void) x; (void) y; return 0.0; }
static double bc_w_top(double x, double y) { (void) x; (void) y; return 0.0; }
static double bc_c_bot(double x, double y) { (void) x; (void) y; return -0.5; }
static double bc_c_top(double x, double y) { (void) x; (void) y; return +0.5; }

#define GUARD(errval) \
    jmp_buf jb_; \
    shim_abort_target = &jb_; \
    if (setjmp(jb_)) { shim_abort_target = NULL; return errval; }
#define UNGUARD() (shim_abort_target = NULL)

#define PAD3(c) (c)->ghostz_p->zst_pad[0], (c)->ghostz_p->zen_pad[0], \
                (c)->ghostz_p->zst_pad[1], (c)->ghostz_p->zen_pad[1], \
                (c)->ghostz_p->zst_pad[2], (c)->ghostz_p->zen_pad[2]
#define FLAT(c, t) (&((t)[(c)->ghostz_p->zst_pad[0]][(c)->ghostz_p->zst_pad[1]][(c)->ghostz_p->zst_pad[2]]))

static void module_init(int order, int nz, int ngz)
{
    if (order == 2) {
        diffuseu_initialize2(nz, ngz);
        diffusew_initialize2(nz, ngz);
        pressure_initialize2(nz, ngz);
    } else {
        diffuseu_initialize4(nz, ngz);
        diffusew_initialize4(nz, ngz);
        pressure_initialize4(nz, ngz);
    }
}

static void module_fini(int order)
{
    if (order == 2) {
        diffuseu_finalize2();
        diffusew_finalize2();
        pressure_finalize2();
    } else {
        diffuseu_finalize4();
        diffusew_finalize4();
        pressure_finalize4();
    }
}

/* Setup as chanfast.c:85-192 (decomposition, transposes, FFT plans, halo
 * plan, grid metrics with the cosine-stretched dz, and the padded fields). */
void *ref_create(const ref_params *prm)
{
    ref_ctx *c = (ref_ctx *) calloc(1, sizeof(ref_ctx));
    GUARD(NULL);
    c->prm = *prm;
    int dims[2] = {1, 1}, periodic[2] = {1, 1}, coord[2];
    MPI_Cart_create(MPI_COMM_WORLD, 2, dims, periodic, 0, &c->comm_cart);
    MPI_Cart_coords(c->comm_cart, 0, 2, coord);
    MPI_Type_contiguous(2, MPI_DOUBLE, &c->cplx_t);
    MPI_Type_commit(&c->cplx_t);
    int nx = prm->nx, ny = prm->ny, nz = prm->nz;
    int ngx = prm->ngx, ngy = prm->ngy, ngz = prm->ngz;

    c->decomp_d = create_decomp_plan(dims, coord, nx, ny, nz + 2 * ngz);
    decomp_plan *d = c->decomp_d;
    c->transp_d = create_transpose_plan(dims, &c->comm_cart, MPI_DOUBLE,
        d->xst, d->xen, d->xsz, d->yst, d->yen, d->ysz, d->zst, d->zen, d->zsz,
        d->x1st, d->x1en, d->x1dist, d->y1st, d->y1en, d->y1dist,
        d->y2st, d->y2en, d->y2dist, d->z2st, d->z2en, d->z2dist);
    c->decomp_c = create_decomp_plan(dims, coord, nx / 2 + 1, ny, nz + 2 * ngz);
    decomp_plan *dc = c->decomp_c;
    c->transp_c = create_transpose_plan(dims, &c->comm_cart, c->cplx_t,
        dc->xst, dc->xen, dc->xsz, dc->yst, dc->yen, dc->ysz, dc->zst, dc->zen, dc->zsz,
        dc->x1st, dc->x1en, dc->x1dist, dc->y1st, dc->y1en, dc->y1dist,
        dc->y2st, dc->y2en, dc->y2dist, dc->z2st, dc->z2en, dc->z2dist);
    c->fftx_p = create_fftx_plan(nx, d->xst, d->xen, d->xsz, dc->xst, dc->xen, dc->xsz);
    c->ffty_p = create_ffty_plan(ny, dc->yst, dc->yen, dc->ysz);
    c->ghostz_p = create_ghostz_plan(&c->comm_cart, MPI_DOUBLE, d->zst, d->zen, d->zsz, ngx, ngy);

    c->local_nx = d->zsz[0];
    c->local_ny = d->zsz[1];
    c->n0 = c->local_nx + 2 * ngx;
    c->n1 = c->local_ny + 2 * ngy;
    c->n2 = nz + 2 * ngz;
    c->local_size = c->n0 * c->n1 * c->n2;
    c->dx = prm->lx / (double) nx;
    c->dy = prm->ly / (double) ny;

    int n0 = c->n0, n1 = c->n1, n2 = c->n2;
    c->xp = (double *) malloc(sizeof(double) * n0);
    c->xu = (double *) malloc(sizeof(double) * n0);
    c->yp = (double *) malloc(sizeof(double) * n1);
    c->yv = (double *) malloc(sizeof(double) * n1);
    c->dz = (double *) malloc(sizeof(double) * n2);
    c->zp = (double *) malloc(sizeof(double) * n2);
    c->zw = (double *) malloc(sizeof(double) * n2);
    c->avg = (double *) malloc(sizeof(double) * n2);
    for (int i = 0; i < n0; i++) {
        int ix = ((d->zst[0] - 1 + i - ngx) + nx) % nx;
        c->xu[i] = (double) (ix + 1) * c->dx;
        c->xp[i] = ((double) (ix + 1) - 0.5) * c->dx;
    }
    for (int j = 0; j < n1; j++) {
        int iy = ((d->zst[1] - 1 + j - ngy) + ny) % ny;
        c->yv[j] = (double) (iy + 1) * c->dy;
        c->yp[j] = ((double) (iy + 1) - 0.5) * c->dy;
    }
    for (int iz = 0; iz < nz; iz++)
        c->dz[iz + ngz] = prm->lz * 0.5 * (cos(M_PI * (double) iz / (double) nz)
                                         - cos(M_PI * (double) (iz + 1) / (double) nz));
    ghost_even_z(c->dz, 1, 1, nz, 0, 0, ngz);
    get_z_at_p(c->dz, c->zp, nz, ngz);
    get_z_at_w(c->dz, c->zw, nz, ngz);

    c->zwork_d1 = d3tensor(d->zst[0], d->zen[0], d->zst[1], d->zen[1], d->zst[2], d->zen[2]);
    c->zwork_c1 = c3tensor(dc->zst[0], dc->zen[0], dc->zst[1], dc->zen[1], dc->zst[2], dc->zen[2]);
    c->bc_3d = d3tensor(PAD3(c));
    c->hbc_3d = d3tensor(PAD3(c));
    c->u_3d = d3tensor(PAD3(c));
    c->v_3d = d3tensor(PAD3(c));
    c->w_3d = d3tensor(PAD3(c));
    c->c_3d = d3tensor(PAD3(c));
    c->p_3d = d3tensor(PAD3(c));
    c->h_3d = d3tensor(PAD3(c));
    c->m1_3d = d3tensor(PAD3(c));
    c->m2_3d = d3tensor(PAD3(c));
    c->m3_3d = d3tensor(PAD3(c));
    for (int q = 0; q < 4; q++) {
        c->f_3d[q] = d3tensor(PAD3(c));
        c->g_3d[q] = d3tensor(PAD3(c));
        c->fcur[q] = FLAT(c, c->f_3d[q]);
        c->gcur[q] = FLAT(c, c->g_3d[q]);
    }
    double *all[] = {FLAT(c, c->u_3d), FLAT(c, c->v_3d), FLAT(c, c->w_3d), FLAT(c, c->c_3d),
                     FLAT(c, c->p_3d), FLAT(c, c->h_3d), FLAT(c, c->bc_3d), FLAT(c, c->hbc_3d),
                     FLAT(c, c->m1_3d), FLAT(c, c->m2_3d), FLAT(c, c->m3_3d),
                     c->fcur[0], c->fcur[1], c->fcur[2], c->fcur[3],
                     c->gcur[0], c->gcur[1], c->gcur[2], c->gcur[3]};
    for (size_t a = 0; a < sizeof(all) / sizeof(all[0]); a++)
        for (int i = 0; i < c->local_size; i++) all[a][i] = FILL_VALUE;
    c->log_cap = 0;
    c->log = NULL;
    UNGUARD();
    return c;
}

void ref_destroy(void *vc)
{
    ref_ctx *c = (ref_ctx *) vc;
    if (!c) return;
    decomp_plan *d = c->decomp_d, *dc = c->decomp_c;
    free(c->xp); free(c->xu); free(c->yp); free(c->yv);
    free(c->dz); free(c->zp); free(c->zw); free(c->avg);
    free_d3tensor(c->zwork_d1, d->zst[0], d->zen[0], d->zst[1], d->zen[1], d->zst[2], d->zen[2]);
    free_c3tensor(c->zwork_c1, dc->zst[0], dc->zen[0], dc->zst[1], dc->zen[1], dc->zst[2], dc->zen[2]);
    double ***t[] = {c->bc_3d, c->hbc_3d, c->u_3d, c->v_3d, c->w_3d, c->c_3d, c->p_3d, c->h_3d,
                     c->m1_3d, c->m2_3d, c->m3_3d,
                     c->f_3d[0], c->f_3d[1], c->f_3d[2], c->f_3d[3],
                     c->g_3d[0], c->g_3d[1], c->g_3d[2], c->g_3d[3]};
    for (size_t a = 0; a < sizeof(t) / sizeof(t[0]); a++) free_d3tensor(t[a], PAD3(c));
    destroy_ghostz_plan(c->ghostz_p);
    destroy_fftx_plan(c->fftx_p);
    destroy_ffty_plan(c->ffty_p);
    destroy_transpose_plan(c->transp_d);
    destroy_decomp_plan(c->decomp_d);
    destroy_transpose_plan(c->transp_c);
    destroy_decomp_plan(c->decomp_c);
    MPI_Type_free(&c->cplx_t);
    free(c->log);
    free(c);
}

void ref_dims(void *vc, int out[3])
{
    ref_ctx *c = (ref_ctx *) vc;
    out[0] = c->n0; out[1] = c->n1; out[2] = c->n2;
}

void ref_metrics(void *vc, double *dz, double *zp, double *zw)
{
    ref_ctx *c = (ref_ctx *) vc;
    memcpy(dz, c->dz, sizeof(double) * c->n2);
    memcpy(zp, c->zp, sizeof(double) * c->n2);
    memcpy(zw, c->zw, sizeof(double) * c->n2);
}

/* Field slots: 0 u, 1 v, 2 w, 3 c, 4 p, 5 h (scratch), 6..9 f (current), 10..13 g. */
static double *slot(ref_ctx *c, int s)
{
    switch (s) {
    case 0: return FLAT(c, c->u_3d);
    case 1: return FLAT(c, c->v_3d);
    case 2: return FLAT(c, c->w_3d);
    case 3: return FLAT(c, c->c_3d);
    case 4: return FLAT(c, c->p_3d);
    case 5: return FLAT(c, c->h_3d);
    default:
        if (s >= 6 && s < 10) return c->fcur[s - 6];
        if (s >= 10 && s < 14) return c->gcur[s - 10];
        return NULL;
    }
}

int ref_set_field(void *vc, int s, const double *src)
{
    ref_ctx *c = (ref_ctx *) vc;
    double *dst = slot(c, s);
    if (!dst) return -1;
    memcpy(dst, src, sizeof(double) * (size_t) c->local_size);
    return 0;
}

int ref_get_field(void *vc, int s, double *dst)
{
    ref_ctx *c = (ref_ctx *) vc;
    double *src = slot(c, s);
    if (!src) return -1;
    memcpy(dst, src, sizeof(double) * (size_t) c->local_size);
    return 0;
}

long ref_log(void *vc, double *out, long max_rows)
{
    ref_ctx *c = (ref_ctx *) vc;
    long n = c->substep < max_rows ? c->substep : max_rows;
    if (out && n > 0) memcpy(out, c->log, sizeof(double) * REF_LOG_COLS * (size_t) n);
    return c->substep;
}

/* FFT3D_FWD / FFT3D_BWD of chanfast.c:21-55 on the context's plans. */
static void fft3d_fwd(ref_ctx *c, double ***a)
{
    decomp_plan *d = c->decomp_d, *dc = c->decomp_c;
    ghostz_truncate_double(a, c->zwork_d1, c->ghostz_p);
    transpose_z_to_x(&(c->zwork_d1[d->zst[0]][d->zst[1]][d->zst[2]]),
                     &(c->fftx_p->work_d[d->xst[0]][d->xst[1]][d->xst[2]]), c->transp_d);
    fftx_d2c(c->fftx_p);
    transpose_x_to_y(&(c->fftx_p->work_c[dc->xst[0]][dc->xst[1]][dc->xst[2]]),
                     &(c->ffty_p->work_i[dc->yst[0]][dc->yst[1]][dc->yst[2]]), c->transp_c);
    ffty_i2o(c->ffty_p);
    transpose_y_to_z(&(c->ffty_p->work_o[dc->yst[0]][dc->yst[1]][dc->yst[2]]),
                     &(c->zwork_c1[dc->zst[0]][dc->zst[1]][dc->zst[2]]), c->transp_c);
}

static void fft3d_bwd(ref_ctx *c, double ***a)
{
    decomp_plan *d = c->decomp_d, *dc = c->decomp_c;
    transpose_z_to_y(&(c->zwork_c1[dc->zst[0]][dc->zst[1]][dc->zst[2]]),
                     &(c->ffty_p->work_o[dc->yst[0]][dc->yst[1]][dc->yst[2]]), c->transp_c);
    ffty_o2i(c->ffty_p);
    transpose_y_to_x(&(c->ffty_p->work_i[dc->yst[0]][dc->yst[1]][dc->yst[2]]),
                     &(c->fftx_p->work_c[dc->xst[0]][dc->xst[1]][dc->xst[2]]), c->transp_c);
    fftx_c2d(c->fftx_p);
    transpose_x_to_z(&(c->fftx_p->work_d[d->xst[0]][d->xst[1]][d->xst[2]]),
                     &(c->zwork_d1[d->zst[0]][d->zst[1]][d->zst[2]]), c->transp_d);
    ghostz_pad_double(a, c->zwork_d1, c->ghostz_p);
}

/* Pressure solve + projection exactly as chanfast.c:569-585 (order 2) /
 * 1493-1509 (order 4): divergence -> FFT -> Poisson -> inverse FFT ->
 * periodic p halo -> project with coefficient `abdt`. */
static void pressure_step(ref_ctx *c, double abdt)
{
    const ref_params *q = &c->prm;
    int lnx = c->local_nx, lny = c->local_ny, nz = q->nz;
    double *u = FLAT(c, c->u_3d), *v = FLAT(c, c->v_3d), *w = FLAT(c, c->w_3d);
    double *p = FLAT(c, c->p_3d), *h = FLAT(c, c->h_3d);
    decomp_plan *dc = c->decomp_c;
    if (q->order == 2)
        divergence2(u, v, w, h, lnx, lny, nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz);
    else
        divergence4(u, v, w, h, lnx, lny, nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz);
    fft3d_fwd(c, c->h_3d);
    fftw_complex *zc = &(c->zwork_c1[dc->zst[0]][dc->zst[1]][dc->zst[2]]);
    if (q->order == 2)
        pressure_poisson2(zc, q->nx, dc->zsz[0], dc->zst[0] - 1, q->ny, dc->zsz[1], dc->zst[1] - 1,
                          nz, q->ngz, c->dx, c->dy, c->dz, abdt);
    else
        pressure_poisson4(zc, q->nx, dc->zsz[0], dc->zst[0] - 1, q->ny, dc->zsz[1], dc->zst[1] - 1,
                          nz, q->ngz, c->dx, c->dy, c->dz, abdt);
    fft3d_bwd(c, c->p_3d);
    ghostz_periodic(p, c->ghostz_p);
    if (q->order == 2)
        project2(u, v, w, p, lnx, lny, nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz, abdt);
    else
        project4(u, v, w, p, lnx, lny, nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz, abdt);
}

/* Case-1 style projection of the current (u, v, w) with time step `dt`
 * (cases.c:426-470): periodic halos, then the pressure step. */
int ref_project(void *vc, double dt)
{
    ref_ctx *c = (ref_ctx *) vc;
    GUARD(-1);
    module_init(c->prm.order, c->prm.nz, c->prm.ngz);
    ghostz_periodic(FLAT(c, c->u_3d), c->ghostz_p);
    ghostz_periodic(FLAT(c, c->v_3d), c->ghostz_p);
    ghostz_periodic(FLAT(c, c->w_3d), c->ghostz_p);
    pressure_step(c, dt);
    module_fini(c->prm.order);
    UNGUARD();
    return 0;
}

/* The reference divergence of the current (u, v, w) after periodic halos,
 * into `out` (padded layout).  Works on copies: divergence4 rewrites w ghosts
 * in place (pressure.c:80-97). */
int ref_divergence(void *vc, double *out)
{
    ref_ctx *c = (ref_ctx *) vc;
    const ref_params *q = &c->prm;
    GUARD(-1);
    module_init(q->order, q->nz, q->ngz);
    size_t nb = sizeof(double) * (size_t) c->local_size;
    double *u = (double *) malloc(nb), *v = (double *) malloc(nb), *w = (double *) malloc(nb);
    memcpy(u, FLAT(c, c->u_3d), nb);
    memcpy(v, FLAT(c, c->v_3d), nb);
    memcpy(w, FLAT(c, c->w_3d), nb);
    ghostz_periodic(u, c->ghostz_p);
    ghostz_periodic(v, c->ghostz_p);
    ghostz_periodic(w, c->ghostz_p);
    for (int i = 0; i < c->local_size; i++) out[i] = 0.0;
    if (q->order == 2)
        divergence2(u, v, w, out, c->local_nx, c->local_ny, q->nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz);
    else
        divergence4(u, v, w, out, c->local_nx, c->local_ny, q->nz, q->ngx, q->ngy, q->ngz, c->dx, c->dy, c->dz);
    free(u); free(v); free(w);
    module_fini(q->order);
    UNGUARD();
    return 0;
}

typedef void (*bcfn_t)(double *, int, int, int, int, int, int, double *, double *, double *,
                       double (*)(double, double), double (*)(double, double), int, int);
typedef void (*opfn_t)(double *, double *, int, int, int, int, int, int, double *, double);
typedef void (*solvefn_t)(double *, double *, int, int, int, int, int, int, double *, double,
                          double, double, int, int);
typedef void (*lapfn_t)(double *, double *, int, int, int, int, int, int, double, double, double);
typedef void (*mflux_t)(double *, double *, double *, double *, double *, double *,
                        int, int, int, int, int, int, double, double, double *);
typedef void (*adv_t)(double *, double *, double *, double *, double *,
                      int, int, int, int, int, int, double, double, double *);
typedef void (*op3fn_t)(double *, double *, int, int, int, int, int, int, double, double, double *, double);
typedef void (*spfn_t)(fftw_complex *, int, int, int, int, int, int, int, int, double, double, double *,
                       double, double, double, int, int);

/* Run `nsub` RK3 substeps, continuing the substep counter and the f/g
 * history kept in the context.  scheme 0: chanfast (chanfast.c:395-656 /
 * 1319-1580); scheme 1: channel (channel.c:392-690 / 1342-1640). */
static int substeps_impl(ref_ctx *c, long nsub, int scheme)
{
    const ref_params *q = &c->prm;
    GUARD(-1);
    int o4 = q->order == 4;
    bcfn_t apply_bc_u = o4 ? apply_bc_u4 : apply_bc_u2;
    bcfn_t apply_bc_w = o4 ? apply_bc_w4 : apply_bc_w2;
    opfn_t hop_u = o4 ? helmholtz1d_operator_u4 : helmholtz1d_operator_u2;
    opfn_t hop_w = o4 ? helmholtz1d_operator_w4 : helmholtz1d_operator_w2;
    solvefn_t solve_u = o4 ? solve_helmholtz1d_u4 : solve_helmholtz1d_u2;
    solvefn_t solve_w = o4 ? solve_helmholtz1d_w4 : solve_helmholtz1d_w2;
    lapfn_t lap_u = o4 ? add_laplacexy_operator_u4 : add_laplacexy_operator_u2;
    lapfn_t lap_w = o4 ? add_laplacexy_operator_w4 : add_laplacexy_operator_w2;
    mflux_t mfx = o4 ? massfluxx4 : massfluxx2, mfy = o4 ? massfluxy4 : massfluxy2,
            mfz = o4 ? massfluxz4 : massfluxz2;
    adv_t adu = o4 ? advectu4 : advectu2, adv = o4 ? advectv4 : advectv2,
          adw = o4 ? advectw4 : advectw2;
    op3fn_t hop3_u = o4 ? helmholtz_operator_u4 : helmholtz_operator_u2;
    op3fn_t hop3_w = o4 ? helmholtz_operator_w4 : helmholtz_operator_w2;
    spfn_t spec_u = o4 ? solve_helmholtz_u4 : solve_helmholtz_u2;
    spfn_t spec_w = o4 ? solve_helmholtz_w4 : solve_helmholtz_w2;
    const int implicit3d = scheme == 1;
    decomp_plan *dc = c->decomp_c;

    module_init(q->order, q->nz, q->ngz);
    uframe_s = q->setuframe;
    vframe_s = q->setvframe;

    int lnx = c->local_nx, lny = c->local_ny, nz = q->nz;
    int ngx = q->ngx, ngy = q->ngy, ngz = q->ngz, n2 = c->n2, ls = c->local_size;
    double dx = c->dx, dy = c->dy, *dz = c->dz, nu = q->nu, pr = q->prandtl, dt = q->dt;
    double *xu = c->xu, *xp = c->xp, *yv = c->yv, *yp = c->yp, *avg = c->avg;
    double *u = FLAT(c, c->u_3d), *v = FLAT(c, c->v_3d), *w = FLAT(c, c->w_3d), *cc = FLAT(c, c->c_3d);
    double *h = FLAT(c, c->h_3d), *bc = FLAT(c, c->bc_3d), *hbc = FLAT(c, c->hbc_3d);
    double *m1 = FLAT(c, c->m1_3d), *m2 = FLAT(c, c->m2_3d), *m3 = FLAT(c, c->m3_3d);
    const int DU = DIRICHU, DW = DIRICHW;

    if (c->log_cap < c->substep + nsub) {
        c->log_cap = c->substep + nsub;
        c->log = (double *) realloc(c->log, sizeof(double) * REF_LOG_COLS * (size_t) c->log_cap);
    }

    for (long s = 0; s < nsub; s++) {
        int step = (int) (c->substep % 3);
        for (int f = 0; f < 4; f++) { double *t = c->fcur[f]; c->fcur[f] = c->gcur[f]; c->gcur[f] = t; }
        double *fu = c->fcur[0], *fv = c->fcur[1], *fw = c->fcur[2], *fc = c->fcur[3];
        double *gu = c->gcur[0], *gv = c->gcur[1], *gw = c->gcur[2], *gc = c->gcur[3];

        ghostz_periodic(u, c->ghostz_p);
        apply_bc_u(u, lnx, lny, nz, ngx, ngy, ngz, xu, yp, dz, bc_u_bot, bc_u_top, DU, DU);
        ghostz_periodic(v, c->ghostz_p);
        apply_bc_u(v, lnx, lny, nz, ngx, ngy, ngz, xp, yv, dz, bc_v_bot, bc_v_top, DU, DU);
        ghostz_periodic(cc, c->ghostz_p);
        apply_bc_u(cc, lnx, lny, nz, ngx, ngy, ngz, xp, yp, dz, bc_c_bot, bc_c_top, DU, DU);
        ghostz_periodic(w, c->ghostz_p);
        apply_bc_w(w, lnx, lny, nz, ngx, ngy, ngz, xp, yp, dz, bc_w_bot, bc_w_top, DW, DW);

        mfx(u, v, w, m1, m2, m3, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        adu(u, m1, m2, m3, fu, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        mfy(u, v, w, m1, m2, m3, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        adv(v, m1, m2, m3, fv, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        mfz(u, v, w, m1, m2, m3, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        adw(w, m1, m2, m3, fw, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        if (!implicit3d) {   /* channel.c:419-438 has no explicit x-y diffusion */
            lap_u(u, fu, lnx, lny, nz, ngx, ngy, ngz, dx, dy, nu);
            lap_u(v, fv, lnx, lny, nz, ngx, ngy, ngz, dx, dy, nu);
            lap_w(w, fw, lnx, lny, nz, ngx, ngy, ngz, dx, dy, nu);
        }
        flux_quick(u, v, w, cc, m1, m2, m3, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        advect_scalar(m1, m2, m3, fc, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz);
        if (!implicit3d)
            lap_u(cc, fc, lnx, lny, nz, ngx, ngy, ngz, dx, dy, nu / pr);
        if (o4)
            add_buoyancy4(cc, fu, fv, fw, q->betg_x, q->betg_y, q->betg_z, lnx, lny, nz, ngx, ngy, ngz);
        else
            add_buoyancy2(cc, fu, fv, fw, q->betg_x, q->betg_y, q->betg_z, lnx, lny, nz, ngx, ngy, ngz);
        ghostz_periodic(fu, c->ghostz_p);
        ghostz_periodic(fv, c->ghostz_p);
        ghostz_periodic(fw, c->ghostz_p);
        ghostz_periodic(fc, c->ghostz_p);

        double nuadt = nu * rk3_alp[step] * dt;
        double nubdt = nu * rk3_bet[step] * dt;
        double abdt = (rk3_alp[step] + rk3_bet[step]) * dt;
        double gamdt = rk3_gam[step] * dt;
        double zetdt = rk3_zet[step] * dt;
        double *row = c->log + REF_LOG_COLS * (size_t) c->substep;

        /* u (chanfast.c:465-536), v (:538-556), c (:558-623), w (:625-642) */
        for (int fld = 0; fld < 4; fld++) {
            double *x = fld == 0 ? u : fld == 1 ? v : fld == 2 ? cc : w;
            double *fx = fld == 0 ? fu : fld == 1 ? fv : fld == 2 ? fc : fw;
            double *gx = fld == 0 ? gu : fld == 1 ? gv : fld == 2 ? gc : gw;
            double *xb = fld == 0 ? xu : xp, *yb = fld == 1 ? yv : yp;
            double (*bb)(double, double) = fld == 0 ? bc_u_bot : fld == 1 ? bc_v_bot : fld == 2 ? bc_c_bot : bc_w_bot;
            double (*bt)(double, double) = fld == 0 ? bc_u_top : fld == 1 ? bc_v_top : fld == 2 ? bc_c_top : bc_w_top;
            int isw = fld == 3;
            double kap = fld == 2 ? 1.0 / pr : 1.0;
            bcfn_t abc = isw ? apply_bc_w : apply_bc_u;
            opfn_t hop = isw ? hop_w : hop_u;
            solvefn_t slv = isw ? solve_w : solve_u;
            int bt_ = isw ? DW : DU;
            double na = fld == 2 ? nuadt / pr : nuadt;
            double nb = fld == 2 ? nubdt / pr : nubdt;
            (void) kap;

            abc(x, lnx, lny, nz, ngx, ngy, ngz, xb, yb, dz, bb, bt, bt_, bt_);
            if (implicit3d) {   /* channel.c:455-485 (u); same for v, c, w */
                op3fn_t hop3 = isw ? hop3_w : hop3_u;
                hop3(x, h, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz, na);
                for (int i = 0; i < ls; i++) h[i] += gamdt * fx[i] + zetdt * gx[i];
                for (int i = 0; i < ls; i++) bc[i] = 0.0;
                abc(bc, lnx, lny, nz, ngx, ngy, ngz, xb, yb, dz, bb, bt, bt_, bt_);
                hop3(bc, hbc, lnx, lny, nz, ngx, ngy, ngz, dx, dy, dz, -nb);
                for (int i = 0; i < ls; i++) h[i] -= hbc[i];
                fft3d_fwd(c, c->h_3d);
                (isw ? spec_w : spec_u)(&(c->zwork_c1[dc->zst[0]][dc->zst[1]][dc->zst[2]]),
                                        q->nx, dc->zsz[0], dc->zst[0] - 1, q->ny, dc->zsz[1], dc->zst[1] - 1,
                                        nz, ngz, dx, dy, dz, -nb, 0.0, 0.0, bt_, bt_);
                double ***x3 = fld == 0 ? c->u_3d : fld == 1 ? c->v_3d : fld == 2 ? c->c_3d : c->w_3d;
                fft3d_bwd(c, x3);
                ghostz_periodic(x, c->ghostz_p);
            } else {
                hop(x, h, lnx, lny, nz, ngx, ngy, ngz, dz, na);
                for (int i = 0; i < ls; i++) h[i] += gamdt * fx[i] + zetdt * gx[i];
                for (int i = 0; i < ls; i++) bc[i] = 0.0;
                abc(bc, lnx, lny, nz, ngx, ngy, ngz, xb, yb, dz, bb, bt, bt_, bt_);
                hop(bc, hbc, lnx, lny, nz, ngx, ngy, ngz, dz, -nb);
                for (int i = 0; i < ls; i++) h[i] -= hbc[i];
                slv(x, h, lnx, lny, nz, ngx, ngy, ngz, dz, -nb, 0.0, 0.0, bt_, bt_);
            }
            abc(x, lnx, lny, nz, ngx, ngy, ngz, xb, yb, dz, bb, bt, bt_, bt_);

            if (fld == 0 || fld == 2) {
                /* mass-flux / scalar-mean control (chanfast.c:485-536, 572-623) */
                double kk = fld == 0 ? nu : nu / pr;
                double s0[4], s1[4];
                for (int pass = 0; pass < 2; pass++) {
                    double *src = pass == 0 ? x : h;
                    if (pass == 1) {
                        for (int i = 0; i < ls; i++) h[i] = gamdt;
                        slv(h, h, lnx, lny, nz, ngx, ngy, ngz, dz, -nb, 0.0, 0.0, bt_, bt_);
                    }
                    get_xy_avg(src, avg, lnx, lny, nz, ngx, ngy, ngz, q->nx, q->ny);
                    double *o = pass == 0 ? s0 : s1;
                    o[0] = get_z_avg(avg, nz, ngz, dz);
                    if (o4) {
                        o[1] = kk * (a1 * (avg[ngz] - avg[ngz - 1]) + a2 * (avg[ngz + 1] - avg[ngz - 2]))
                               / (0.5 * (dz[ngz] + dz[ngz - 1]));
                        o[2] = kk * (a1 * (avg[n2 - ngz] - avg[n2 - ngz - 1]) + a2 * (avg[n2 - ngz + 1] - avg[n2 - ngz - 2]))
                               / (0.5 * (dz[n2 - ngz] + dz[n2 - ngz - 1]));
                    } else {
                        o[1] = kk * (avg[ngz] - avg[ngz - 1]) / (0.5 * (dz[ngz] + dz[ngz - 1]));
                        o[2] = kk * (avg[n2 - ngz] - avg[n2 - ngz - 1]) / (0.5 * (dz[n2 - ngz] + dz[n2 - ngz - 1]));
                    }
                    o[3] = nz % 2 == 0 ? 0.5 * (avg[ngz + nz / 2 - 1] + avg[ngz + nz / 2]) : avg[ngz + nz / 2];
                }
                double m;
                if (fld == 0)
                    m = q->uvolavgmode == 1 ? (q->want_uvolavg - uframe_s - s0[0]) / s1[0] : -q->dpdx;
                else
                    m = q->cvolavgmode == 1 ? (q->want_cvolavg - s0[0]) / s1[0] : 0.0;
                for (int t = 0; t < 4; t++) s0[t] += s1[t] * m;
                for (int i = 0; i < ls; i++) {
                    x[i] += h[i] * m;
                    fx[i] += m;
                }
                double *r = row + (fld == 0 ? 0 : 5);
                r[0] = m;
                r[1] = s0[1];
                r[2] = s0[2];
                r[3] = s0[0];
                r[4] = s0[3];
            }
        }

        pressure_step(c, abdt);
        c->substep++;
    }
    module_fini(q->order);
    UNGUARD();
    return 0;
}

int ref_substeps(void *vc, long nsub) { return substeps_impl((ref_ctx *) vc, nsub, 0); }
int ref_channel_substeps(void *vc, long nsub) { return substeps_impl((ref_ctx *) vc, nsub, 1); }

/* The real drivers, unmodified, run inside directory `workdir` (they read and
 * write outputdir/ relative to the current directory). */
typedef void (*driver_t)(int, int, int, int, int, int, int, int, int, int, int, double, double, double,
                         double, double, int, double, double, double, double, int, double, int, double,
                         double, double, double, double);

#define DRIVER_PARAMS const char *workdir, int order, int nx, int ny, int nz, int it, int nt, int istat, \
                      int ngx, int ngy, int ngz, double lx, double ly, double lz, double dt, \
                      double want_cfl, int cflmode, double nu, double prandtl, double dpdx, \
                      double want_uvolavg, int uvolavgmode, double want_cvolavg, int cvolavgmode, \
                      double setuframe, double setvframe, double betg_x, double betg_y, double betg_z
#define DRIVER_ARGS nx, ny, nz, it, nt, istat, ngx, ngy, ngz, lx, ly, lz, dt, want_cfl, cflmode, \
                    nu, prandtl, dpdx, want_uvolavg, uvolavgmode, want_cvolavg, cvolavgmode, \
                    setuframe, setvframe, betg_x, betg_y, betg_z

static int run_driver(driver_t drv, const char *workdir, int nx, int ny, int nz, int it, int nt, int istat,
                      int ngx, int ngy, int ngz, double lx, double ly, double lz, double dt,
                      double want_cfl, int cflmode, double nu, double prandtl, double dpdx,
                      double want_uvolavg, int uvolavgmode, double want_cvolavg, int cvolavgmode,
                      double setuframe, double setvframe, double betg_x, double betg_y, double betg_z)
{
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) return -2;
    if (chdir(workdir) != 0) return -3;
    jmp_buf jb;
    shim_abort_target = &jb;
    if (setjmp(jb)) {
        shim_abort_target = NULL;
        if (chdir(cwd) != 0) return -4;
        return -1;
    }
    drv(1, 1, DRIVER_ARGS);
    shim_abort_target = NULL;
    if (chdir(cwd) != 0) return -4;
    return 0;
}

int ref_chanfast(DRIVER_PARAMS)
{
    return run_driver(order == 2 ? chanfast2 : chanfast4, workdir, DRIVER_ARGS);
}

int ref_channel(DRIVER_PARAMS)
{
    return run_driver(order == 2 ? channel2 : channel4, workdir, DRIVER_ARGS);
}

/* Known-answer cases of cases.c (case0..case16) at one rank. */
int ref_case(int which, int nx, int ny, int nz, int ng)
{
    GUARD(-1);
    switch (which) {
    case 0: case0(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 1: case1(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 2: case2(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 3: case3(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 4: case4(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 5: case5(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 6: case6(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 7: case7(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 8: case8(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 9: case9(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 10: case10(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 11: case11(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 12: case12(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 13: case13(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 14: case14(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 15: case15(1, 1, nx, ny, nz, ng, ng, ng); break;
    case 16: case16(1, 1, nx, ny, nz, ng, ng, ng); break;
    default: UNGUARD(); return -2;
    }
    fflush(stdout);
    UNGUARD();
    return 0;
}
