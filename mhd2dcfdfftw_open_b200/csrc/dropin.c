/*
 * The reference's hot-path entry points on the GPU (include/mhd_gpu_dropin.h).
 *
 * The reference keeps its state in globals defined by its initialize.c
 * (declared in its initialize.h:11-69, `real` = double); this file declares
 * the ones it uses with the same names and types.  By default each entry
 * point uploads the global arrays it reads, runs the operator of
 * libmhdgpu.so on them, and downloads the arrays it writes, so the host
 * globals stay exactly what the reference's own routines would leave there.
 * In resident mode (mhdgpu_dropin_resident, or MHDGPU_DROPIN_RESIDENT=1) the
 * device copies are authoritative: each array crosses PCIe on its first use
 * only, and results come back in mhdgpu_dropin_sync_host, which a driver
 * calls before it reads the globals itself (mhd.c's checkDivB and writeArray).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mhd_gpu.h"
#include "mhd_gpu_dropin.h"

/* --- the reference's globals (initialize.c:15-79, divBcleaning.c:4) ------ */
extern int NVAR;
extern int boundaryTypeX;
extern double cfl, Tmax, dtOut;
extern size_t nx, ny, iSize, jSize;
extern double Lx, Ly;
extern double adiabaticIdx, resistivity, viscosity;
extern int Hall, divBcleaning, outDivB;
extern double di;
extern double Ch_divBcleaning, Cp_divBcleaning;
extern double Cr_divBCleaning;
extern double *uu, *dudx, *dudy, *d2udx2, *d2udy2, *d2Bdx2, *d2Bdy2;
extern double *divB, *ddivBdx, *ddivBdy, *Efield, *dEdx, *dEdy, *dudt, *dudtRK;
extern double *uuHaloX0, *uuHaloX1, *divBHaloX0, *divBHaloX1, *EfieldHaloX0, *EfieldHaloX1;

static mhdgpu_ctx *g_ctx = NULL;
static mhdgpu_params g_p;  /* the parameters g_ctx was created with */
static int g_reported = 0;

/* Resident mode (mhdgpu_dropin_resident): the device arrays are the
 * authoritative copy.  An array is uploaded on its first use only
 * (g_uploaded), results stay on the device (g_dev_newer marks arrays whose
 * host copy is stale) and reach the host in mhdgpu_dropin_sync_host. */
static int g_resident = -1;  /* -1: not decided yet (MHDGPU_DROPIN_RESIDENT) */
static unsigned char g_uploaded[MHDGPU_NARRAYS], g_dev_newer[MHDGPU_NARRAYS];

static int resident(void)
{
    if (g_resident < 0) {
        const char *e = getenv("MHDGPU_DROPIN_RESIDENT");
        g_resident = e && atoi(e) != 0;
    }
    return g_resident;
}

static void report(const char *where, int rc)
{
    if (rc != MHDGPU_OK && !g_reported) {
        fprintf(stderr, "mhdgpu drop-in: %s failed: %s\n", where, mhdgpu_error_string(rc));
        g_reported = 1;
    }
}

static int same_params(const mhdgpu_params *a, const mhdgpu_params *b)
{
    return a->boundaryTypeX == b->boundaryTypeX && a->cfl == b->cfl && a->Tmax == b->Tmax &&
           a->dtOut == b->dtOut && a->nx == b->nx && a->ny == b->ny && a->Lx == b->Lx &&
           a->Ly == b->Ly && a->adiabaticIdx == b->adiabaticIdx && a->Hall == b->Hall &&
           a->di == b->di && a->resistivity == b->resistivity && a->viscosity == b->viscosity &&
           a->divBcleaning == b->divBcleaning && a->outDivB == b->outDivB;
}

/* the context, created from the globals initialize() has set; a caller that
 * changes any of them between calls gets a context made for the new values */
static mhdgpu_ctx *ctx(void)
{
    mhdgpu_params p;
    memset(&p, 0, sizeof p);
    p.boundaryTypeX = boundaryTypeX;
    p.cfl = cfl;
    p.Tmax = Tmax;
    p.dtOut = dtOut;
    p.nx = (long)nx;
    p.ny = (long)ny;
    p.Lx = Lx;
    p.Ly = Ly;
    p.adiabaticIdx = adiabaticIdx;
    p.Hall = Hall;
    p.di = di;
    p.resistivity = resistivity;
    p.viscosity = viscosity;
    p.divBcleaning = divBcleaning;
    p.outDivB = outDivB;
    if (g_ctx && same_params(&p, &g_p)) return g_ctx;
    if (g_ctx) mhdgpu_destroy(g_ctx);
    g_ctx = NULL;
    /* a new context starts from the host globals */
    memset(g_uploaded, 0, sizeof g_uploaded);
    memset(g_dev_newer, 0, sizeof g_dev_newer);
    const char *dev = getenv("MHDGPU_DEVICE");
    int rc = mhdgpu_create(&p, dev ? atoi(dev) : 0, &g_ctx);
    if (rc != MHDGPU_OK) {
        report("context creation", rc);
        g_ctx = NULL;
        return NULL;
    }
    g_p = p;
    return g_ctx;
}

/* the context array mirroring a reference global, or -1 */
static int which(const double *a)
{
    const double *g[MHDGPU_NARRAYS] = {uu, dudx, dudy, d2udx2, d2udy2, d2Bdx2, d2Bdy2, divB,
                                       ddivBdx, ddivBdy, Efield, dEdx, dEdy, dudt, dudtRK};
    if (!a) return -1;
    for (int k = 0; k < MHDGPU_NARRAYS; k++)
        if (g[k] == a) return k;
    return -1;
}

static double *host_of(int k)
{
    double *g[MHDGPU_NARRAYS] = {uu, dudx, dudy, d2udx2, d2udy2, d2Bdx2, d2Bdy2, divB,
                                 ddivBdx, ddivBdy, Efield, dEdx, dEdy, dudt, dudtRK};
    return g[k];
}

static int up(mhdgpu_ctx *c, int k)
{
    double *h = host_of(k);
    if (!h || !mhdgpu_device_array(c, k)) return MHDGPU_OK;  /* not allocated: not used */
    if (resident() && (g_uploaded[k] || g_dev_newer[k])) return MHDGPU_OK;
    int rc = mhdgpu_set_array(c, k, h);
    if (!rc) g_uploaded[k] = 1;
    return rc;
}

static int down(mhdgpu_ctx *c, int k)
{
    double *h = host_of(k);
    if (!h || !mhdgpu_device_array(c, k)) return MHDGPU_OK;
    if (resident()) {
        g_dev_newer[k] = 1;
        return MHDGPU_OK;
    }
    return mhdgpu_get_array(c, k, h);
}

void mhdgpu_dropin_resident(int on)
{
    if (resident() && !on) mhdgpu_dropin_sync_host();
    g_resident = on != 0;
}

void mhdgpu_dropin_sync_host(void)
{
    if (!g_ctx) return;
    for (int k = 0; k < MHDGPU_NARRAYS; k++) {
        if (!g_dev_newer[k]) continue;
        double *h = host_of(k);
        int rc = h && mhdgpu_device_array(g_ctx, k) ? mhdgpu_get_array(g_ctx, k, h) : MHDGPU_OK;
        report("mhdgpu_dropin_sync_host", rc);
        if (!rc) g_dev_newer[k] = 0;
    }
}

void mhdgpu_dropin_sync_device(void)
{
    memset(g_uploaded, 0, sizeof g_uploaded);
    memset(g_dev_newer, 0, sizeof g_dev_newer);
}

static void deriv(const char *name, int dir, int order, int nv, double *in, int start,
                  double *out)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int ki = which(in), ko = which(out);
    if (ki < 0 || ko < 0) {
        report(name, MHDGPU_ERR_INVALID);
        return;
    }
    int rc = up(c, ki);
    if (!rc) rc = dir == 0 ? mhdgpu_deriv_x(c, nv, ki, start, ko, order)
                           : mhdgpu_deriv_y(c, nv, ki, start, ko, order);
    if (!rc) rc = down(c, ko);
    report(name, rc);
}

void derivX(int nv, double *arrMain, double *arrHalo0, double *arrHalo1, double *arrDeriv,
            int iVarStartMain, int iVarStartHalo)
{
    (void)arrHalo0; (void)arrHalo1; (void)iVarStartHalo;  /* periodic wrap is in the kernel */
    deriv("derivX", 0, 1, nv, arrMain, iVarStartMain, arrDeriv);
}

void derivXX(int nv, double *arrMain, double *arrHalo0, double *arrHalo1, double *arrDeriv,
             int iVarStartMain, int iVarStartHalo)
{
    (void)arrHalo0; (void)arrHalo1; (void)iVarStartHalo;
    deriv("derivXX", 0, 2, nv, arrMain, iVarStartMain, arrDeriv);
}

void derivY(int nv, double *arrMain, double *arrDeriv, int iVarStartMain)
{
    deriv("derivY", 1, 1, nv, arrMain, iVarStartMain, arrDeriv);
}

void derivYY(int nv, double *arrMain, double *arrDeriv, int iVarStartMain)
{
    deriv("derivYY", 1, 2, nv, arrMain, iVarStartMain, arrDeriv);
}

void calcEfield(void)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int rc = up(c, MHDGPU_UU);
    if (!rc) rc = mhdgpu_calc_efield(c);
    if (!rc) rc = down(c, MHDGPU_EFIELD);
    report("calcEfield", rc);
}

void calcDivB(void)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int rc = up(c, MHDGPU_DUDX);
    if (!rc) rc = up(c, MHDGPU_DUDY);
    if (!rc) rc = mhdgpu_calc_divb(c);
    if (!rc) rc = down(c, MHDGPU_DIVB);
    report("calcDivB", rc);
}

void calcRHS(void)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    static const int reads[] = {MHDGPU_UU, MHDGPU_DUDX, MHDGPU_DUDY, MHDGPU_D2UDX2,
                                MHDGPU_D2UDY2, MHDGPU_D2BDX2, MHDGPU_D2BDY2, MHDGPU_DDIVBDX,
                                MHDGPU_DDIVBDY, MHDGPU_DEDX, MHDGPU_DEDY};
    int rc = MHDGPU_OK;
    for (size_t k = 0; k < sizeof reads / sizeof reads[0] && !rc; k++) rc = up(c, reads[k]);
    if (!rc) rc = mhdgpu_calc_rhs(c);
    if (!rc) rc = down(c, MHDGPU_DUDT);
    report("calcRHS", rc);
}

void filtering(void)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int rc = up(c, MHDGPU_UU);
    if (!rc) rc = mhdgpu_filtering(c);
    if (!rc) rc = down(c, MHDGPU_UU);
    report("filtering", rc);
}

/* rkInit (timeAdvance.c:20-27): stage coefficients and dudtRK = 0, here and
 * on the device */
void rkInit(double dt)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int rc = mhdgpu_rk_init(c, dt);
    if (resident()) {  /* zeroed on the device, which is authoritative */
        g_uploaded[MHDGPU_DUDTRK] = 1;
        g_dev_newer[MHDGPU_DUDTRK] = 1;
    } else {
        memset(dudtRK, 0, sizeof(double) * (size_t)NVAR * iSize * jSize);
    }
    report("rkInit", rc);
}

void rkExecute(int iRK)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return;
    int rc = up(c, MHDGPU_UU);
    if (!rc) rc = up(c, MHDGPU_DUDT);
    if (!rc) rc = up(c, MHDGPU_DUDTRK);
    if (!rc) rc = mhdgpu_rk_execute(c, iRK);
    if (!rc) rc = down(c, MHDGPU_UU);
    if (!rc) rc = down(c, MHDGPU_DUDTRK);
    report("rkExecute", rc);
}

/* calcDt (timeAdvance.c:38-153); with hyperbolic cleaning it also sets the
 * reference's Ch_divBcleaning / Cp_divBcleaning (divBcleaning.c:7-10) */
double calcDt(double dt0)
{
    mhdgpu_ctx *c = ctx();
    if (!c) return dt0;
    double dt = dt0;
    int rc = up(c, MHDGPU_UU);
    if (!rc) rc = mhdgpu_calc_dt(c, dt0, &dt);
    if (!rc && divBcleaning == 2) {
        double ch = 0.0, cp = 0.0;
        rc = mhdgpu_get_cleaning_speeds(c, &ch, &cp);
        Ch_divBcleaning = ch;
        Cp_divBcleaning = sqrt(Cr_divBCleaning * ch);
    }
    report("calcDt", rc);
    return dt;
}

/* The single-rank periodic halo exchange of parallel.c:13-24: the left halo
 * holds rows nx-2, nx-1 and the right halo rows 0, 1 of every field. */
static void halo(const double *a, int nf, double *h0, double *h1)
{
    if (!a || !h0 || !h1) return;
    const size_t n = iSize, m = jSize;
    for (int v = 0; v < nf; v++)
        for (int r = 0; r < 2; r++) {
            memcpy(h0 + ((size_t)v * 2 + r) * m, a + ((size_t)v * n + (n - 2 + r)) * m,
                   sizeof(double) * m);
            memcpy(h1 + ((size_t)v * 2 + r) * m, a + ((size_t)v * n + r) * m, sizeof(double) * m);
        }
}

/* In resident mode the host arrays are stale between syncs; the kernels wrap
 * periodically and never read these halos, so they are left alone. */
void sendrecvHaloPointsX(void)
{
    if (!resident()) halo(uu, NVAR, uuHaloX0, uuHaloX1);
}
void sendrecvHaloPointsdivBX(void)
{
    if (!resident()) halo(divB, 1, divBHaloX0, divBHaloX1);
}
void sendrecvHaloPointsEfieldX(void)
{
    if (!resident()) halo(Efield, 3, EfieldHaloX0, EfieldHaloX1);
}
