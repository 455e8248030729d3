/*
 * TEST INFRASTRUCTURE -- the oracle.  A single-threaded CPU restatement of the reference's
 * explicit-dynamics step (GMollon/MELODY2D, Code/*.h) on the flattened model of
 * include/melgpu.h.  It exists to check the GPU solver; the product library never links it.
 *
 * Pinning: tests/test_oracle_vs_reference.py runs this oracle and the reference solver itself
 * (oracle/_ref/ref_harness, compiled from the reference sources) on the same generated inputs and
 * requires identical state.  Every function below names the reference lines it restates; the
 * arithmetic keeps the reference's operation order so results agree bit for bit (compile with
 * -ffp-contract=off, as oracle/Makefile does).
 */
#include "mel_oracle.h"
#include "../melody2d_b200/csrc/mel_rsqrt.h"
#include "../melody2d_b200/csrc/mel_sincos.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* x^(-1/2), and the cosine and sine that turn rigid bodies, as the reference computes them (glibc
 * pow, cos, sin) or correctly rounded (the GPU's values); see orc_set_rsqrt_mode. */
static int g_cr_rsqrt = 0;
static inline double orc_rsqrt(double x) { return g_cr_rsqrt ? mel_rsqrt(x) : pow(x, -0.5); }
static inline double orc_cos(double x) { return g_cr_rsqrt ? mel_cos(x) : cos(x); }
static inline double orc_sin(double x) { return g_cr_rsqrt ? mel_sin(x) : sin(x); }
void orc_set_rsqrt_mode(int correctly_rounded) { g_cr_rsqrt = correctly_rounded; }

typedef struct { int n, cap; mel_contact* a; } cvec;
typedef struct { int body2, border2, shift; } nbr_t;
typedef struct { int body, node; double f[3]; } send_t;
typedef struct { int n, cap; send_t* a; } svec;

struct orc_model {
    double xmin, xmax, gx, gy, time, dt, tend, cup, next_cup;
    int solver; double sp[8]; int flags[MEL_NFLAGS];
    int nmat; int* mat_type; double* mat_p;
    int nlaw; int* law_type; int* law_len; double* law_p; int* table;
    /* bodies */
    int nb; int *btype, *bmat, *bper, *bstatus; double* bdist;
    int *nptr, *bptr, *gptr, *cptr, *nreg, *reg_off;
    double* rg;           /* [nb*MEL_RIGID_NF] */
    double* rg_tmp;       /* [nb*6] x,y,r displacement_temporary, velocity_temporary */
    double* rf;           /* [nb*15] contact, body, dirichlet, neumann, damping (x,y,r) */
    double* rtot;         /* [nb*3] */
    double* drv;          /* [nb*8] drivendof (Body.h:164) */
    double* works;        /* [nb*7] */
    double* terr;         /* [nb] total_error */
    double* merr;         /* [nb] max_error */
    int*    nmerr;        /* [nb] node_for_max_error */
    double* bfms;         /* [nb] factor_mass_scaling (rigid) */
    double* bdfms;        /* [nb] delta_factor_mass_scaling */
    double* bmms;         /* [nb] mass_mass_scaling */
    double* bmaxfms;      /* [nb] max_factor_mass_scaling */
    /* nodes */
    int nn; double *X0, *mass, *invm, *dom; int *sptr, *sidx; double* sN;
    double *x, *u, *v, *a, *up, *vp, *ap, *upt, *ut;
    double *freg, *fint, *fcon, *fself, *fbody, *fdir, *fneu, *fdamp, *falid, *ftot;
    double *ide, *err, *errn, *fms, *dfms, *mms;
    /* borders */
    int nbd; int *bd_body, *bd_per, *bd_int, *bd_bef, *bd_aft, *bd_ptr, *bd_nodes;
    int* bc_type; double* bc_param; int* hptr; double *ht, *hv;
    double *bc_value, *bc_vel;   /* [2*nbd] */
    int *s_node[4], *s_shift[4];
    double *blen, *blen0, *cpx, *cpy, *bcpx, *bcpy;
    double *prox;                /* [nbd*4] xmin,xmax,ymin,ymax */
    int *shmin, *shmax;
    /* Gauss points */
    int ng; int *gsp, *gsi; double *gN, *gdx, *gdy, *gw, *gJ;
    double* eenergy;             /* [nb] Elastic_energy summed (always 0, Model.h:28,72) */
    int ndeact; double* deact;   /* DEACTIVATION entries, MEL_DEACT_NF doubles each */
    int* cells;
    int nmx; int* mx_ptr; int* mx_dofs; double *mx_k, *mx_c;
    int* alid_ptr; double *alid_t, *alid_v, *alid_ab;   /* ALID histories and nodal alpha, beta (or NULL) */
    double* damage;       /* [nb] Body::damage, the running value of Update_damage */
    int dmg_bodies[16], dmg_n, dmg_count, dmg_cap; double* dmg_log;   /* Monitoring's Damage entries (tests) */
    /* dynamic lists */
    cvec* cont; nbr_t** nbl; int* nbn; int* nbc; svec* send;
    /* Solver_step storage (Body::Store/Restore, Body.h:2601-2659) */
    cvec* s_cont; double *s_node_blob, *s_body_blob, *s_border_blob;
    long stale;
    double stats[5];
};

/* ------------------------------------------------------------------------------------------ */
/* small helpers                                                                               */
/* ------------------------------------------------------------------------------------------ */
static void* xcalloc(size_t n, size_t s) { void* p = calloc(n ? n : 1, s); return p; }
#define NEWD(n) ((double*)xcalloc((size_t)(n), sizeof(double)))
#define NEWI(n) ((int*)xcalloc((size_t)(n), sizeof(int)))
static double* dupd(const double* s, size_t n) { double* p = NEWD(n); if (s && n) memcpy(p, s, n * sizeof(double)); return p; }
static int* dupi(const int* s, size_t n) { int* p = NEWI(n); if (s && n) memcpy(p, s, n * sizeof(int)); return p; }

static void cpush(cvec* v, const mel_contact* c) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 16; v->a = (mel_contact*)realloc(v->a, (size_t)v->cap * sizeof(mel_contact)); }
    v->a[v->n++] = *c;
}
static void spush(svec* v, int body, int node, double f0, double f1, double f2) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 64; v->a = (send_t*)realloc(v->a, (size_t)v->cap * sizeof(send_t)); }
    send_t* s = &v->a[v->n++]; s->body = body; s->node = node; s->f[0] = f0; s->f[1] = f1; s->f[2] = f2;
}

static inline int nb_nodes(const orc_model* m, int b) { return m->nptr[b + 1] - m->nptr[b]; }
static inline int nb_borders(const orc_model* m, int b) { return m->bptr[b + 1] - m->bptr[b]; }
static inline int bd_count(const orc_model* m, int gb) { return m->bd_ptr[gb + 1] - m->bd_ptr[gb]; }
/* global border index of body-local border j of body b */
static inline int gbd(const orc_model* m, int b, int j) { return m->bptr[b] + j; }
static inline int is_active(const orc_model* m, int b) { return m->bstatus[b] != MEL_STATUS_INACTIVE; }

/* ------------------------------------------------------------------------------------------ */
/* Tools.h                                                                                     */
/* ------------------------------------------------------------------------------------------ */
/* Closest_2_segment, "Linear" interpolant (Code/Tools.h:106-219).  Outputs that the reference
 * leaves unassigned on some paths are left untouched here as well. */
static void closest_2_segment_linear(double Xs, double Ys, double X0, double Y0, double X1, double Y1,
                                     double X2, double Y2, double X3, double Y3,
                                     double* Gap, double* Xsi, double* Xnorm, double* Ynorm, double* Xtan,
                                     double* Ytan, double* N0, double* N1, double* N2, double* N3, int* flag)
{
    double Xclosest, Yclosest;
    double ilength = orc_rsqrt((X2 - X1) * (X2 - X1) + (Y2 - Y1) * (Y2 - Y1));
    double ilengthm = orc_rsqrt((X1 - X0) * (X1 - X0) + (Y1 - Y0) * (Y1 - Y0));
    double ilengthp = orc_rsqrt((X3 - X2) * (X3 - X2) + (Y3 - Y2) * (Y3 - Y2));
    *Xtan = (X2 - X1) * ilength;
    *Ytan = (Y2 - Y1) * ilength;
    *Xnorm = *Ytan;
    *Ynorm = -*Xtan;
    double Xtanm = (X1 - X0) * ilengthm, Ytanm = (Y1 - Y0) * ilengthm;
    double Xtanp = (X3 - X2) * ilengthp, Ytanp = (Y3 - Y2) * ilengthp;
    double xt = *Xtan, yt = *Ytan;
    if (((Xs - X1) * (Xtanm + xt) + (Ys - Y1) * (Ytanm + yt)) * (xt * (Xtanm + xt) + yt * (Ytanm + yt)) >= 0.) {
        if (((Xs - X2) * (xt + Xtanp) + (Ys - Y2) * (yt + Ytanp)) * (xt * (xt + Xtanp) + yt * (yt + Ytanp)) <= 0.) {
            double xsi = -1. + 2. * ((X2 - X1) * (Xs - X1) + (Y2 - Y1) * (Ys - Y1)) * ilength * ilength;
            *Xsi = xsi;
            if ((xsi < 1.) && (xsi > -1.)) {
                *Xnorm = yt; *Ynorm = -xt;
                Xclosest = 0.5 * (X1 + X2) + xsi * 0.5 * (X2 - X1);
                Yclosest = 0.5 * (Y1 + Y2) + xsi * 0.5 * (Y2 - Y1);
                *Gap = *Xnorm * (Xs - Xclosest) + *Ynorm * (Ys - Yclosest);
                *N0 = 0.; *N1 = 0.5 * (1. - xsi); *N2 = 0.5 * (1. + xsi); *N3 = 0.;
                *flag = 0;
            } else if (xsi == -1.) {
                *Xnorm = yt; *Ynorm = -xt;
                *Gap = *Xnorm * (Xs - X1) + *Ynorm * (Ys - Y1);
                *N0 = 0.; *N1 = 1.; *N2 = 0.; *N3 = 0.;
                *flag = -1;
            } else if (xsi < -1.) {
                double invdistm = orc_rsqrt((Xs - X1) * (Xs - X1) + (Ys - Y1) * (Ys - Y1));
                double xn = (Xs - X1) * invdistm, yn = (Ys - Y1) * invdistm;
                if (-yn * (xt + Xtanm) + xn * (yt + Ytanm) < 0.) { xn = -xn; yn = -yn; }
                *Xnorm = xn; *Ynorm = yn; *Xtan = -yn; *Ytan = xn;
                *Gap = xn * (Xs - X1) + yn * (Ys - Y1);
                *N0 = 0.; *N1 = 1.; *N2 = 0.; *N3 = 0.;
                *Xsi = -1.;
                *flag = -2;
            } else if (xsi == 1.) {
                *Xnorm = yt; *Ynorm = -xt;
                *Gap = *Xnorm * (Xs - X2) + *Ynorm * (Ys - Y2);
                *N0 = 0.; *N1 = 0.; *N2 = 1.; *N3 = 0.;
                *flag = 1;
            } else if (xsi > 1.) {
                double invdistp = orc_rsqrt((Xs - X2) * (Xs - X2) + (Ys - Y2) * (Ys - Y2));
                double xn = (Xs - X2) * invdistp, yn = (Ys - Y2) * invdistp;
                if (-yn * (xt + Xtanp) + xn * (yt + Ytanp) < 0.) { xn = -xn; yn = -yn; }
                *Xnorm = xn; *Ynorm = yn; *Xtan = -yn; *Ytan = xn;
                *Gap = xn * (Xs - X2) + yn * (Ys - Y2);
                *N0 = 0.; *N1 = 0.; *N2 = 1.; *N3 = 0.;
                *Xsi = 1.;
                *flag = 2;
            }
        } else {
            *flag = 3;
            *Xsi = 1.;
        }
    } else {
        *flag = -3;
        *Xsi = -1.;
    }
}

/* Closest_2_segment_self (Code/Tools.h:319-369).  Its trailing statements run unconditionally,
 * so the flag is always -3; the other outputs follow the reference's branches. */
static void closest_2_segment_self(double Xs, double Ys, double X1, double Y1, double X2, double Y2,
                                   double* Gap, double* Xsi, double* Xnorm, double* Ynorm, double* Xtan,
                                   double* Ytan, double* N0, double* N1, double* N2, double* N3, int* flag)
{
    double ilength = orc_rsqrt((X2 - X1) * (X2 - X1) + (Y2 - Y1) * (Y2 - Y1));
    double xt = (X2 - X1) * ilength, yt = (Y2 - Y1) * ilength;
    *Xtan = xt; *Ytan = yt;
    if (((Xs - X1) * xt + (Ys - Y1) * yt) * (xt * xt + yt * yt) >= 0.) {
        if (((Xs - X2) * xt + (Ys - Y2) * yt) * (xt * xt + yt * yt) <= 0.) {
            double xsi = -1. + 2. * ((X2 - X1) * (Xs - X1) + (Y2 - Y1) * (Ys - Y1)) * ilength * ilength;
            *Xsi = xsi;
            if ((xsi < 1.) && (xsi > -1.)) {
                *Xnorm = yt; *Ynorm = -xt;
                double Xc = 0.5 * (X1 + X2) + xsi * 0.5 * (X2 - X1);
                double Yc = 0.5 * (Y1 + Y2) + xsi * 0.5 * (Y2 - Y1);
                *Gap = *Xnorm * (Xs - Xc) + *Ynorm * (Ys - Yc);
                *N0 = 0.; *N1 = 0.5 * (1. - xsi); *N2 = 0.5 * (1. + xsi); *N3 = 0.;
            }
        } else {
            *Xsi = 1.;
        }
    } else {
        *Xsi = -1.;
    }
    *flag = -3;
}

/* Detect_Segment_Proximity (Code/Proximity.h:8-27) */
static int detect_segment_proximity(double Xs, double Ys, double X1, double Y1, double X2, double Y2, double dd)
{
    dd = dd * dd;
    if ((Xs - X1) * (Xs - X1) + (Ys - Y1) * (Ys - Y1) < dd) return 1;
    if ((Xs - X2) * (Xs - X2) + (Ys - Y2) * (Ys - Y2) < dd) return 1;
    double dx = X2 - X1, dy = Y2 - Y1;
    double a = dx * dx + dy * dy;
    double Xsi = -1. + 2. * (dx * (Xs - X1) + dy * (Ys - Y1)) / a;
    if ((Xsi < 1.) && (Xsi > -1.)) {
        double b = dy * (Xs - 0.5 * (X1 + X2) - Xsi * 0.5 * dx) - dx * (Ys - 0.5 * (Y1 + Y2) - Xsi * 0.5 * dy);
        if (b * b < a * dd) return 1;
    }
    return 0;
}

static double triangle_surface(double x0, double y0, double x1, double y1, double x2, double y2)
{   /* Code/Tools.h:377-380 */
    return 0.5 * fabs((x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0));
}

static double triangle_inertia(double x0, double y0, double x1, double y1, double x2, double y2, double xc, double yc)
{   /* Code/Tools.h:388-412 */
    double area, PP, PQ, QQ, inertia = 0;
    area = triangle_surface(xc, yc, x0, y0, x1, y1);
    PP = (x0 - xc) * (x0 - xc) + (y0 - yc) * (y0 - yc);
    PQ = (x0 - xc) * (x1 - xc) + (y0 - yc) * (y1 - yc);
    QQ = (x1 - xc) * (x1 - xc) + (y1 - yc) * (y1 - yc);
    inertia += area * (PP + PQ + QQ);
    area = triangle_surface(xc, yc, x1, y1, x2, y2);
    PP = (x1 - xc) * (x1 - xc) + (y1 - yc) * (y1 - yc);
    PQ = (x1 - xc) * (x2 - xc) + (y1 - yc) * (y2 - yc);
    QQ = (x2 - xc) * (x2 - xc) + (y2 - yc) * (y2 - yc);
    inertia += area * (PP + PQ + QQ);
    area = triangle_surface(xc, yc, x2, y2, x0, y0);
    PP = (x2 - xc) * (x2 - xc) + (y2 - yc) * (y2 - yc);
    PQ = (x2 - xc) * (x0 - xc) + (y2 - yc) * (y0 - yc);
    QQ = (x0 - xc) * (x0 - xc) + (y0 - yc) * (y0 - yc);
    inertia += area * (PP + PQ + QQ);
    return fabs(inertia / 6.);
}

/* ------------------------------------------------------------------------------------------ */
/* Model.h contact laws                                                                        */
/* ------------------------------------------------------------------------------------------ */
static void law_frictionless(double kn, double gapn, double* gapt, double* Pn, double* Pt)
{   /* Code/Model.h:81-90 */
    if (gapn > 0.) *Pn = 0.; else *Pn = -kn * gapn;
    *Pt = 0.; *gapt = 0.;
}
static void law_cohesion(double kn, double kt, double gtang, double gtens, double gapn, double* gapt, double* Pn, double* Pt)
{   /* Code/Model.h:97-116 */
    *Pn = -kn * gapn; *Pt = -kt * *gapt;
    if (*Pn < -gtens) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
    else if (fabs(*Pt) > gtang) { if (*gapt > 0.) *Pt = -gtang; else *Pt = gtang; *gapt = -*Pt / kt; }
}
static void law_mohr_coulomb(double kn, double kt, double fric, double coh, double tens, double gapn, double* gapt, double* Pn, double* Pt)
{   /* Code/Model.h:123-142 */
    *Pn = -kn * gapn; *Pt = -kt * *gapt;
    if (*Pn < -tens) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
    else if (fabs(*Pt) > coh + fric * *Pn) {
        if (*gapt > 0.) *Pt = -coh - fric * *Pn; else *Pt = coh + fric * *Pn;
        *gapt = -*Pt / kt;
    }
}
static void law_damped_mc(double kn, double kt, double fric, double coh, double tens, double damp, double mass, double length,
                          double gapn, double vgapn, double* gapt, double vgapt, double* Pn, double* Pt, double* W)
{   /* Code/Model.h:149-180 */
    *Pn = 0.;
    if (gapn < 0.) { *Pn = -damp * vgapn * 2. * sqrt(mass * kn / length); *W += *Pn * vgapn; }
    *Pn -= kn * gapn;
    if (*Pn < -tens) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
    else {
        double Pt_damp = -damp * vgapt * 2. * sqrt(mass * kt / length);
        *Pt = -kt * *gapt + Pt_damp;
        if (fabs(*Pt) > coh + fric * *Pn) {
            if (*gapt > 0.) *Pt = -coh - fric * *Pn; else *Pt = coh + fric * *Pn;
            *gapt = -*Pt / kt;
            *W += *Pt * vgapt;
        } else *W += Pt_damp * vgapt;
    }
}
static void law_two_slopes_mc(double kn, double kt, double fric, double coh, double tens, double rati, double gapn, double vgapn,
                              double* gapt, double vgapt, double* Pn, double* Pt)
{   /* Code/Model.h:212-243 */
    (void)vgapt;
    if (vgapn <= 0.) *Pn = -kn * gapn; else *Pn = -kn * gapn * rati;
    if (*Pn < -tens) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
    else {
        *Pt = -kt * *gapt;
        if (fabs(*Pt) > coh + fric * *Pn) {
            if (*gapt > 0.) *Pt = -coh - fric * *Pn; else *Pt = coh + fric * *Pn;
            *gapt = -*Pt / kt;
        }
    }
}
static void czm_kmax_branch(double kini, double Pnlim, double gapnres, double Pnres, double NTratio, double gapn, double* gapt,
                            double* Damage, double* Pn, double* Pt, double gapnmax, double gaptmax, int which)
{
    double kmax;
    if (which == 1) { gapnmax = gapn; gaptmax = gapnmax * NTratio; }
    else if (which == 2) { gaptmax = fabs(*gapt); gapnmax = gaptmax / NTratio; }
    else if (which == 3) {
        if (gapn / gapnmax > fabs(*gapt) / gaptmax) { gapnmax = gapn; gaptmax = gapnmax * NTratio; }
        else { gaptmax = fabs(*gapt); gapnmax = gaptmax / NTratio; }
    }
    (void)gaptmax;
    *Damage = (gapnmax - Pnlim / kini) / (gapnres - Pnlim / kini);
    kmax = (Pnlim * (1. - *Damage) + Pnres * *Damage) / gapnmax;
    if (gapn < 0.) *Pn = -kini * gapn; else *Pn = -kmax * gapn;
    *Pt = -kmax * *gapt;
}
static void law_czm_linear(double kini, double Pnlim, double gapnlim, double Pnres, double NTratio, double gapn, double* gapt,
                           double* Damage, double* Pn, double* Pt)
{   /* Code/Model.h:250-336 */
    if (*Damage >= 1.) {
        *Pn = -kini * gapn; *Pt = -kini * *gapt;
        if (*Pn < -Pnres) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
        else if (fabs(*Pt) > Pnres * NTratio) {
            if (*gapt > 0.) *Pt = -Pnres * NTratio; else *Pt = Pnres * NTratio;
            *gapt = -*Pt / kini;
        }
    } else {
        double gapnmax = Pnlim / kini * (1. - *Damage) + gapnlim * *Damage;
        double gaptmax = gapnmax * NTratio;
        if (gapn < gapnmax && fabs(*gapt) < gaptmax) {
            double kmax = (Pnlim * (1. - *Damage) + Pnres * *Damage) / gapnmax;
            if (gapn < 0.) *Pn = -kini * gapn; else *Pn = -kmax * gapn;
            *Pt = -kmax * *gapt;
        } else if (gapn > gapnmax && fabs(*gapt) < gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 1);
        } else if (gapn < gapnmax && fabs(*gapt) > gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 2);
        } else if (gapn > gapnmax && fabs(*gapt) > gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 3);
        }
    }
}
static void law_czm_fatigue(double kini, double Pnlim, double gapnres, double Pnres, double NTratio, double Pnfat, double Raten,
                            double Ratet, double gapn, double* gapt, double* Damage, double* Pn, double* Pt)
{   /* Code/Model.h:343-446 */
    if (*Damage < 1.) {
        double gapnmax = Pnlim / kini * (1. - *Damage) + gapnres * *Damage;
        double gaptmax = gapnmax * NTratio;
        if (gapn < gapnmax && fabs(*gapt) < gaptmax) {
            double Pnm = *Pn, Ptm = *Pt;
            double kmax = (Pnlim * (1. - *Damage) + Pnres * *Damage) / gapnmax;
            if (gapn < 0.) *Pn = -kini * gapn; else *Pn = -kmax * gapn;
            *Pt = -kmax * *gapt;
            double Pnmax = Pnlim * (1. - *Damage) + Pnres * *Damage;
            if ((fabs(*Pn) > Pnfat) && (fabs(*Pn) > fabs(Pnm))) {
                double Ratiopn = (fabs(*Pn) - Pnfat) / (Pnmax - Pnfat);
                double Deltapn = fabs(*Pn) - fabs(Pnm);
                *Damage = *Damage + Ratiopn * Raten * Deltapn;
            }
            if ((fabs(*Pt) > NTratio * Pnfat) && (fabs(*Pt) > fabs(Ptm))) {
                double Ratiopt = (fabs(*Pt) - Pnfat * NTratio) / (NTratio * (Pnmax - Pnfat));
                double Deltapt = fabs(*Pt) - fabs(Ptm);
                *Damage = *Damage + Ratiopt * Ratet * Deltapt;
            }
        } else if (gapn > gapnmax && fabs(*gapt) < gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 1);
        } else if (gapn < gapnmax && fabs(*gapt) > gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 2);
        } else if (gapn > gapnmax && fabs(*gapt) > gaptmax) {
            czm_kmax_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, Damage, Pn, Pt, gapnmax, gaptmax, 3);
        }
    }
    if (*Damage >= 1.) {
        *Damage = 1.;
        *Pn = -kini * gapn; *Pt = -kini * *gapt;
        if (*Pn < -Pnres) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
        else if (fabs(*Pt) > Pnres * NTratio) {
            if (*gapt > 0.) *Pt = -Pnres * NTratio; else *Pt = Pnres * NTratio;
            *gapt = -*Pt / kini;
        }
    }
}
static void law_bonded_mc(double kn, double kt, double kbond, double fricbond, double cohbond, double tensbond, double fricfree,
                          double cohfree, double tensfree, double damp, double mass, double length, double gapn, double vgapn,
                          double* gapt, double vgapt, double* Damage, double* Pn, double* Pt)
{   /* Code/Model.h:453-505 */
    if (*Damage >= 1.) {
        *Pn = -kn * gapn - damp * vgapn * 2. * sqrt(mass * kn / length);
        if (*Pn < -tensfree) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
        else *Pt = -kt * *gapt - damp * vgapt * 2. * sqrt(mass * kt / length);
        if (fabs(*Pt) > cohfree + fricfree * *Pn) {
            if (*gapt > 0.) *Pt = -cohfree - fricfree * *Pn; else *Pt = cohfree + fricfree * *Pn;
            *gapt = -*Pt / kt;
        }
    } else {
        if (gapn < 0.) *Pn = -kn * gapn - damp * vgapn * 2. * sqrt(mass * kn / length);
        else *Pn = -kbond * gapn - damp * vgapn * 2. * sqrt(mass * kbond / length);
        *Pt = -kt * *gapt - damp * vgapt * 2. * sqrt(mass * kt / length);
        if (*Pn < -tensbond) {
            *Damage = 1.;
            if (*Pn < -tensfree) { *Pn = 0.; *Pt = 0.; *gapt = 0.; }
        }
        if (fabs(*Pt) > cohbond + fricbond * *Pn) {
            *Damage = 1.;
            if (*gapt > 0.) *Pt = -cohfree - fricfree * *Pn; else *Pt = cohfree + fricfree * *Pn;
            *gapt = -*Pt / kt;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Body.h: set-up                                                                              */
/* ------------------------------------------------------------------------------------------ */
/* Body::Initialize_segments (Code/Body.h:403-606) */
static void initialize_segments(orc_model* m, int b)
{
    double period = m->xmax - m->xmin;
    int nbrd = nb_borders(m, b);
    int n0 = m->nptr[b];
    for (int i = 0; i < nbrd; i++) {
        int g = gbd(m, b, i);
        int nbn = bd_count(m, g);
        int off = m->bd_ptr[g];
        const int* bn = m->bd_nodes + off;
        int gb = gbd(m, b, m->bd_bef[g]);
        int ga = gbd(m, b, m->bd_aft[g]);
        const int* bnb = m->bd_nodes + m->bd_ptr[gb];
        const int* bna = m->bd_nodes + m->bd_ptr[ga];
        int per = m->bd_per[g];
        for (int j = 0; j < nbn; j++)
            for (int k = 0; k < 4; k++) { m->s_node[k][off + j] = 0; m->s_shift[k][off + j] = 0; }
        m->s_node[0][off] = bnb[bd_count(m, gb) - 2];
        m->s_node[1][off] = bn[0];
        m->s_node[2][off] = bn[1];
        m->s_node[3][off] = bn[2];
        if (per == MEL_PER_PERIODIC && i == 0) m->s_shift[0][off] = -1;
        else if (per == MEL_PER_PERIODIC) m->s_shift[0][off] = 1;
        for (int j = 1; j < nbn - 2; j++) {
            m->s_node[0][off + j] = bn[j - 1];
            m->s_node[1][off + j] = bn[j];
            m->s_node[2][off + j] = bn[j + 1];
            m->s_node[3][off + j] = bn[j + 2];
        }
        m->s_node[0][off + nbn - 2] = bn[nbn - 3];
        m->s_node[1][off + nbn - 2] = bn[nbn - 2];
        m->s_node[2][off + nbn - 2] = bn[nbn - 1];
        m->s_node[3][off + nbn - 2] = bna[1];
        if (per == MEL_PER_PERIODIC && i == 0) { m->s_shift[2][off + nbn - 2] = 1; m->s_shift[3][off + nbn - 2] = 1; }
        else if (per == MEL_PER_PERIODIC) { m->s_shift[2][off + nbn - 2] = -1; m->s_shift[3][off + nbn - 2] = -1; }
        m->s_node[0][off + nbn - 1] = bn[nbn - 2];
        m->s_node[1][off + nbn - 1] = bn[nbn - 1];
        m->s_node[2][off + nbn - 1] = bna[1];
        m->s_node[3][off + nbn - 1] = bna[2];
        if (per == MEL_PER_PERIODIC) {
            int s = (i == 0) ? 1 : -1;
            m->s_shift[1][off + nbn - 1] = s; m->s_shift[2][off + nbn - 1] = s; m->s_shift[3][off + nbn - 1] = s;
        }
        for (int j = 0; j < nbn; j++) {
            double x0 = m->X0[2 * (n0 + m->s_node[0][off + j])] + m->s_shift[0][off + j] * period;
            double y0 = m->X0[2 * (n0 + m->s_node[0][off + j]) + 1];
            double x1 = m->X0[2 * (n0 + m->s_node[1][off + j])] + m->s_shift[1][off + j] * period;
            double y1 = m->X0[2 * (n0 + m->s_node[1][off + j]) + 1];
            double x2 = m->X0[2 * (n0 + m->s_node[2][off + j])] + m->s_shift[2][off + j] * period;
            double y2 = m->X0[2 * (n0 + m->s_node[2][off + j]) + 1];
            double L = 0.5 * sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0)) + 0.5 * sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1));
            m->blen[off + j] = L;
            m->blen0[off + j] = L;
        }
    }
}

/* The stiffness re-assembly of Body::Update_material (Code/Body.h:2784-2859): E and Nu from the
 * material (Body.h:2727-2746), the plane-strain elasticity matrix scaled by E/((1+Nu)(1-2Nu)), and per
 * Gauss point the local matrix of the support's dofs, each entry summed from 0 in the reference's
 * four-term order; every upper-triangle pair (dof0 <= dof1) adds L*weight*jacobian into the first
 * MATRICES entry with those dofs (pairs without an entry are dropped).  The first-entry lookup is a
 * dense table over the body's dof pairs instead of the reference's linear search; the sums are
 * the same. */
static void assemble_stiffness(orc_model* m, int b)
{
    const double* P = m->mat_p + MEL_MAT_NPARAM * m->bmat[b];
    double E = 0., Nu = 0.;
    if (m->mat_type[m->bmat[b]] == MEL_MAT_ELASTIC_LINEAR) {
        double Mu = P[3], Lambda = P[4];
        E = Mu * (3. * Lambda + 2. * Mu) / (Lambda + Mu);
        Nu = Mu / (2. * Lambda + 2. * Mu);
    } else if (m->mat_type[m->bmat[b]] == MEL_MAT_NEOHOOKEAN) {
        double Mu = P[3], Kappa = P[4];
        E = 9. * Kappa * Mu / (3. * Kappa + Mu);
        Nu = (3. * Kappa - 2. * Mu) / (6. * Kappa + 2. * Mu);
    }
    double C[3][3] = { { 1. - Nu, Nu, 0 }, { Nu, 1. - Nu, 0 }, { 0, 0, 1. - 2. * Nu } };
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C[i][j] *= E / ((1. + Nu) * (1. - 2. * Nu));
    const int nd = 2 * nb_nodes(m, b);
    int* first = (int*)malloc(sizeof(int) * (size_t)nd * nd);
    for (size_t k = 0; k < (size_t)nd * nd; k++) first[k] = -1;
    for (int i = m->mx_ptr[b + 1] - 1; i >= m->mx_ptr[b]; i--) {
        m->mx_k[i] = 0.;
        first[(size_t)m->mx_dofs[2 * i] * nd + m->mx_dofs[2 * i + 1]] = i;
    }
    for (int g = m->gptr[b]; g < m->gptr[b + 1]; g++) {
        const int s0 = m->gsp[g], nin = m->gsp[g + 1] - s0;
        const double* xd = m->gdx + s0; const double* yd = m->gdy + s0;
        double* L = (double*)calloc((size_t)4 * nin * nin, sizeof(double));
        const int w = 2 * nin;
        for (int ii = 0; ii < nin; ii++)
            for (int jj = 0; jj < nin; jj++) {
                double* e = L + (size_t)(2 * ii) * w + 2 * jj;       /* x row, x column */
                *e += xd[ii] * C[0][0] * xd[jj]; *e += xd[ii] * C[0][2] * yd[jj];
                *e += yd[ii] * C[2][0] * xd[jj]; *e += yd[ii] * C[2][2] * yd[jj];
                e = L + (size_t)(2 * ii) * w + 2 * jj + 1;           /* x row, y column */
                *e += xd[ii] * C[0][1] * yd[jj]; *e += xd[ii] * C[0][2] * xd[jj];
                *e += yd[ii] * C[2][1] * yd[jj]; *e += yd[ii] * C[2][2] * xd[jj];
                e = L + (size_t)(2 * ii + 1) * w + 2 * jj;           /* y row, x column */
                *e += yd[ii] * C[1][0] * xd[jj]; *e += yd[ii] * C[1][2] * yd[jj];
                *e += xd[ii] * C[2][0] * xd[jj]; *e += xd[ii] * C[2][2] * yd[jj];
                e = L + (size_t)(2 * ii + 1) * w + 2 * jj + 1;       /* y row, y column */
                *e += yd[ii] * C[1][1] * yd[jj]; *e += yd[ii] * C[1][2] * xd[jj];
                *e += xd[ii] * C[2][1] * yd[jj]; *e += xd[ii] * C[2][2] * xd[jj];
            }
        for (int i = 0; i < w; i++) {
            const int dof0 = 2 * m->gsi[s0 + i / 2] + (i - 2 * (i / 2));
            for (int j = 0; j < w; j++) {
                const int dof1 = 2 * m->gsi[s0 + j / 2] + (j - 2 * (j / 2));
                if (dof1 < dof0) continue;
                const int n = first[(size_t)dof0 * nd + dof1];
                if (n >= 0) m->mx_k[n] += L[(size_t)i * w + j] * m->gw[g] * m->gJ[g];
            }
        }
        free(L);
    }
    free(first);
}

/* Body::Update_material (Code/Body.h:2708-2906): masses (flags[4]), stiffness (flags[5]) and
 * damping (flags[6]) entries rebuilt from the material, in that order; the matrix updates act on
 * the MATRICES triplets and are skipped when there are none. */
static void update_material(orc_model* m, int b)
{
    const double* P = m->mat_p + MEL_MAT_NPARAM * m->bmat[b];
    double Rho = P[0], Alpha = P[1], Beta = P[2];
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        if (m->flags[4] == 1) {
            double* rg = m->rg + MEL_RIGID_NF * b;
            rg[MEL_RG_MASS] = 0.;
            for (int i = 0; i < nb_nodes(m, b); i++) { m->mass[2 * (n0 + i)] = 0.; m->mass[2 * (n0 + i) + 1] = 0.; }
            for (int g = m->gptr[b]; g < m->gptr[b + 1]; g++)
                for (int j = m->gsp[g]; j < m->gsp[g + 1]; j++)
                    for (int k = m->gsp[g]; k < m->gsp[g + 1]; k++) {
                        double dm = m->gw[g] * m->gJ[g] * m->gN[j] * m->gN[k];
                        m->mass[2 * (n0 + m->gsi[j])] += dm;
                        m->mass[2 * (n0 + m->gsi[j]) + 1] += dm;
                    }
            for (int i = 0; i < nb_nodes(m, b); i++) {
                double* mm = m->mass + 2 * (n0 + i);
                mm[0] *= Rho; mm[1] *= Rho;
                m->invm[2 * (n0 + i)] = 1. / mm[0];
                m->invm[2 * (n0 + i) + 1] = 1. / mm[1];
                rg[MEL_RG_MASS] += sqrt(mm[0] * mm[0] + mm[1] * mm[1]);
                rg[MEL_RG_INV_MASS] = 1 / rg[MEL_RG_MASS];
            }
        }
        if (m->flags[5] == 1 && m->mx_ptr) assemble_stiffness(m, b);
        if (m->flags[6] == 1 && m->mx_ptr) {
            for (int i = m->mx_ptr[b]; i < m->mx_ptr[b + 1]; i++) {
                int d0 = m->mx_dofs[2 * i], d1 = m->mx_dofs[2 * i + 1];
                if (d0 == d1) m->mx_c[i] = Alpha * m->mx_k[i] + Beta * m->mass[2 * (n0 + d0 / 2)];
                else m->mx_c[i] = Alpha * m->mx_k[i];
            }
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        double mass = 0., inertia = 0.;
        for (int c = m->cptr[b]; c < m->cptr[b + 1]; c++) {
            int a0 = m->cells[3 * c], a1 = m->cells[3 * c + 1], a2 = m->cells[3 * c + 2];
            double x0 = m->X0[2 * (n0 + a0)], y0 = m->X0[2 * (n0 + a0) + 1];
            double x1 = m->X0[2 * (n0 + a1)], y1 = m->X0[2 * (n0 + a1) + 1];
            double x2 = m->X0[2 * (n0 + a2)], y2 = m->X0[2 * (n0 + a2) + 1];
            double xc = (x0 + x1 + x2) / 3., yc = (y0 + y1 + y2) / 3.;
            double surf = triangle_surface(x0, y0, x1, y1, x2, y2);
            mass += surf;
            inertia += surf * ((xc - rg[MEL_RG_X0]) * (xc - rg[MEL_RG_X0]) + (yc - rg[MEL_RG_Y0]) * (yc - rg[MEL_RG_Y0]));
            inertia += triangle_inertia(x0, y0, x1, y1, x2, y2, xc, yc);
        }
        mass *= Rho; inertia *= Rho;
        rg[MEL_RG_MASS] = mass; rg[MEL_RG_INERTIA] = inertia;
        rg[MEL_RG_INV_MASS] = 1. / mass; rg[MEL_RG_INV_INERTIA] = 1. / inertia;
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Border.h / Body.h: boundary conditions                                                       */
/* ------------------------------------------------------------------------------------------ */
/* Border::Update_bc (Code/Border.h:120-215) for direction d of global border g */
static void border_update_bc(orc_model* m, int g, int d, double Time)
{
    int t = m->bc_type[2 * g + d];
    if (t == MEL_BC_DRIVEN) return;
    const double* ti = m->ht + m->hptr[2 * g + d];
    const double* va = m->hv + m->hptr[2 * g + d];
    int nh = m->hptr[2 * g + d + 1] - m->hptr[2 * g + d];
    double* val = &m->bc_value[2 * g + d];
    double* vel = &m->bc_vel[2 * g + d];
    if (t == MEL_BC_SOFT) {
        int n = 0, ex = 0;
        *val = 0.;
        while (ex == 0 && n + 1 < nh) {
            double t0 = ti[n], p0 = va[n], t1 = ti[n + 1], p1 = va[n + 1];
            if (Time >= t1) *val = *val + (t1 - t0) * (p1 + p0) * 0.5;
            else {
                *val = *val + (Time - t0) * (p0 + (p1 - p0) / (t1 - t0) * ((Time - t0) * 0.5));
                *vel = p0 + (p1 - p0) / (t1 - t0) * (Time - t0);
                ex = 1;
            }
            n++;
        }
    } else if (t == MEL_BC_ORIENTED || t == MEL_BC_FOLLOWING) {
        for (int n = 0; n + 1 < nh; n++) {
            double t0 = ti[n], p0 = va[n], t1 = ti[n + 1], p1 = va[n + 1];
            if ((t0 <= Time) & (Time <= t1)) { *val = p0 + (p1 - p0) / (t1 - t0) * (Time - t0); break; }
        }
    } else if (t == MEL_BC_NONE) {
        *val = 0.;
    }
}

/* Body::Update_bc (Code/Body.h:335-395) */
static void body_update_bc(orc_model* m, int b, double Time)
{
    double* drv = m->drv + 8 * b;
    for (int n = 0; n < nb_borders(m, b); n++) {
        int g = gbd(m, b, n);
        border_update_bc(m, g, 0, Time);
        border_update_bc(m, g, 1, Time);
        for (int d = 0; d < 2; d++) {
            if (m->bc_type[2 * g + d] != MEL_BC_DRIVEN) continue;
            const double* ti = m->ht + m->hptr[2 * g + d];
            const double* va = m->hv + m->hptr[2 * g + d];
            int nh = m->hptr[2 * g + d + 1] - m->hptr[2 * g + d];
            int base = 4 * d;
            drv[base] = 1.;
            drv[base + 1] = 0.;
            int ex = 0, nbh = 0;
            while (ex == 0 && nbh + 1 < nh) {
                double t0 = ti[nbh], p0 = va[nbh], t1 = ti[nbh + 1], p1 = va[nbh + 1];
                if (Time >= t1) drv[base + 1] += (t1 - t0) * (p1 + p0) * 0.5;
                else {
                    drv[base + 1] += (Time - t0) * (p0 + (p1 - p0) / (t1 - t0) * ((Time - t0) * 0.5));
                    drv[base + 2] = (Time - t0) * (p1 - p0) / (t1 - t0);
                    drv[base + 3] = (p1 - p0) / (t1 - t0);
                    ex = 1;
                }
                nbh++;
            }
        }
    }
}

/* Body::Update_borders (Code/Body.h:614-661) */
static void update_borders(orc_model* m, int b)
{
    if (m->btype[b] != MEL_BODY_DEFORMABLE) return;
    double period = m->xmax - m->xmin;
    int n0 = m->nptr[b];
    for (int i = 0; i < nb_borders(m, b); i++) {
        int g = gbd(m, b, i);
        int nbn = bd_count(m, g), off = m->bd_ptr[g];
        int simple = m->bd_per[g] == MEL_PER_SIMPLE;
        for (int j = 0; j < nbn; j++) {
            int e = off + j;
            double x0 = m->x[2 * (n0 + m->s_node[0][e])] + period * m->s_shift[0][e];
            double y0 = m->x[2 * (n0 + m->s_node[0][e]) + 1];
            double x1 = m->x[2 * (n0 + m->s_node[1][e])] + period * m->s_shift[1][e];
            double y1 = m->x[2 * (n0 + m->s_node[1][e]) + 1];
            double x2 = m->x[2 * (n0 + m->s_node[2][e])] + period * m->s_shift[2][e];
            double y2 = m->x[2 * (n0 + m->s_node[2][e]) + 1];
            double L;
            if (j == 0) {
                if (simple) L = sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) * 0.5;
                else L = (sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) + sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0))) * 0.5;
            } else if (j == nbn - 1) {
                if (simple) L = sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0)) * 0.5;
                else L = (sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) + sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0))) * 0.5;
            } else
                L = (sqrt((x2 - x1) * (x2 - x1) + (y2 - y1) * (y2 - y1)) + sqrt((x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0))) * 0.5;
            m->blen[e] = L;
        }
    }
}

/* Body::Update_bc_forces (Code/Body.h:669-901) */
static void update_bc_forces(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int n = 0; n < nb_nodes(m, b); n++) {
            int k = 2 * (n0 + n);
            m->fneu[k] = 0.; m->fneu[k + 1] = 0.; m->fdir[k] = 0.; m->fdir[k + 1] = 0.;
        }
        for (int i = 0; i < nb_borders(m, b); i++) {
            int g = gbd(m, b, i);
            int nbn = bd_count(m, g), off = m->bd_ptr[g];
            int tx = m->bc_type[2 * g], ty = m->bc_type[2 * g + 1];
            for (int j = 0; j < nbn; j++) { m->bcpx[off + j] = 0.; m->bcpy[off + j] = 0.; }
            if (tx == MEL_BC_NONE && ty == MEL_BC_NONE) continue;
            double xv = m->bc_value[2 * g], yv = m->bc_value[2 * g + 1];
            double xvel = m->bc_vel[2 * g], yvel = m->bc_vel[2 * g + 1];
            for (int n = 0; n < nbn - 1; n++) {
                int e = off + n;
                int bnode = m->bd_nodes[e];
                double length = m->blen[e];
                double* px = &m->bcpx[e]; double* py = &m->bcpy[e];
                int gn = n0 + bnode;
                double ftx = 0., fty = 0., ftpx = 0., ftpy = 0.;
                if (tx == MEL_BC_FOLLOWING || ty == MEL_BC_FOLLOWING) {
                    int a = n0 + m->s_node[0][e], c = n0 + m->s_node[2][e];
                    double x0 = m->X0[2 * a], y0 = m->X0[2 * a + 1], x2 = m->X0[2 * c], y2 = m->X0[2 * c + 1];
                    double xp0 = m->x[2 * a], yp0 = m->x[2 * a + 1], xp2 = m->x[2 * c], yp2 = m->x[2 * c + 1];
                    double invl = orc_rsqrt((x2 - x0) * (x2 - x0) + (y2 - y0) * (y2 - y0));
                    double invlp = orc_rsqrt((xp2 - xp0) * (xp2 - xp0) + (yp2 - yp0) * (yp2 - yp0));
                    ftx = (x2 - x0) * invl; fty = (y2 - y0) * invl;
                    ftpx = (xp2 - xp0) * invlp; ftpy = (yp2 - yp0) * invlp;
                }
                if (tx == MEL_BC_ORIENTED) *px = xv;
                else if (tx == MEL_BC_FOLLOWING) {
                    *px += xv * (ftx * ftpx + fty * ftpy);
                    *py += xv * (ftx * ftpy - fty * ftpx);
                } else if (tx == MEL_BC_SOFT) {
                    double pen = m->bc_param[4 * g], dmp = m->bc_param[4 * g + 1];
                    *px = pen * (xv - m->u[2 * gn]) - dmp * (xvel - m->v[2 * gn]);
                }
                if (ty == MEL_BC_ORIENTED) *py = yv;
                else if (ty == MEL_BC_FOLLOWING) {
                    *px += yv * (fty * ftpx - ftx * ftpy);
                    *py += yv * (fty * ftpy + ftx * ftpx);
                } else if (ty == MEL_BC_SOFT) {
                    double pen = m->bc_param[4 * g + 2], dmp = m->bc_param[4 * g + 3];
                    *py = pen * (yv - m->u[2 * gn + 1]) - dmp * (yvel - m->v[2 * gn + 1]);
                }
                for (int j = m->sptr[gn]; j < m->sptr[gn + 1]; j++) {
                    double sf = m->sN[j];
                    double fxn = 0., fyn = 0., fxd = 0., fyd = 0.;
                    if (tx == MEL_BC_ORIENTED) fxn = *px * length * sf;
                    else if (tx == MEL_BC_FOLLOWING) { fxn = *px * length * sf; fyn = *py * length * sf; }
                    else if (tx == MEL_BC_SOFT) fxd = *px * length * sf;
                    if (ty == MEL_BC_ORIENTED) fyn = *py * length * sf;
                    else if (ty == MEL_BC_FOLLOWING) { fxn = *px * length * sf; fyn = *py * length * sf; }
                    else if (ty == MEL_BC_SOFT) fyd = *py * length * sf;
                    int t = n0 + m->sidx[j];
                    m->fneu[2 * t] += fxn; m->fneu[2 * t + 1] += fyn;
                    m->fdir[2 * t] += fxd; m->fdir[2 * t + 1] += fyd;
                }
            }
        }
    } else {
        double* rf = m->rf + 15 * b;
        const double* rg = m->rg + MEL_RIGID_NF * b;
        rf[9] = rf[10] = rf[11] = 0.;   /* neumann */
        rf[6] = rf[7] = rf[8] = 0.;     /* dirichlet */
        for (int i = 0; i < nb_borders(m, b); i++) {
            int g = gbd(m, b, i);
            int nbn = bd_count(m, g), off = m->bd_ptr[g];
            int tx = m->bc_type[2 * g], ty = m->bc_type[2 * g + 1];
            for (int j = 0; j < nbn; j++) { m->bcpx[off + j] = 0.; m->bcpy[off + j] = 0.; }
            if (tx == MEL_BC_NONE && ty == MEL_BC_NONE) continue;
            double xv = m->bc_value[2 * g], yv = m->bc_value[2 * g + 1];
            double xvel = m->bc_vel[2 * g], yvel = m->bc_vel[2 * g + 1];
            for (int n = 0; n < nbn; n++) {
                int e = off + n;
                int gn = n0 + m->bd_nodes[e];
                double length = m->blen[e];
                double fxn = 0., fyn = 0., fxd = 0., fyd = 0.;
                if (tx == MEL_BC_ORIENTED || tx == MEL_BC_FOLLOWING) { m->bcpx[e] = xv; fxn = m->bcpx[e] * length; }
                else if (tx == MEL_BC_SOFT) {
                    double pen = m->bc_param[4 * g], dmp = m->bc_param[4 * g + 1];
                    m->bcpx[e] = pen * (xv - m->u[2 * gn]) + dmp * (xvel - m->v[2 * gn]);
                    fxd = m->bcpx[e] * length;
                } else if (tx == MEL_BC_DRIVEN) { m->bcpx[e] = 0.; fxd = 0.; }
                if (ty == MEL_BC_ORIENTED || ty == MEL_BC_FOLLOWING) { m->bcpy[e] = yv; fyn = m->bcpy[e] * length; }
                else if (ty == MEL_BC_SOFT) {
                    double pen = m->bc_param[4 * g + 2], dmp = m->bc_param[4 * g + 3];
                    m->bcpy[e] = pen * (yv - m->u[2 * gn + 1]) + dmp * (yvel - m->v[2 * gn + 1]);
                    fyd = m->bcpy[e] * length;
                } else if (ty == MEL_BC_DRIVEN) { m->bcpy[e] = 0.; fyd = 0.; }
                double dx = m->x[2 * gn] - rg[MEL_RG_XC];
                double dy = m->x[2 * gn + 1] - rg[MEL_RG_YC];
                rf[9] += fxn; rf[10] += fyn; rf[11] += -fxn * dy + fyn * dx;
                rf[6] += fxd; rf[7] += fyd; rf[8] += -fxd * dy + fyd * dx;
            }
        }
    }
}

/* Body::Update_body_forces (Code/Body.h:909-929) */
static void update_body_forces(orc_model* m, int b)
{
    double gx = m->gx, gy = m->gy;
    if (m->bstatus[b] == MEL_STATUS_NOGRAVITY) { gx = 0.; gy = 0.; }
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            m->fbody[2 * i] = m->mass[2 * i] * gx;
            m->fbody[2 * i + 1] = m->mass[2 * i + 1] * gy;
        }
    } else {
        double* rf = m->rf + 15 * b;
        rf[3] = m->rg[MEL_RIGID_NF * b + MEL_RG_MASS] * gx;
        rf[4] = m->rg[MEL_RIGID_NF * b + MEL_RG_MASS] * gy;
    }
}

/* Body::Update_damping_forces (Code/Body.h:1057-1154) */
static void update_damping_forces(orc_model* m, int b)
{
    if (m->btype[b] != MEL_BODY_DEFORMABLE) return;
    int n0 = m->nptr[b];
    for (int i = n0; i < m->nptr[b + 1]; i++) { m->fdamp[2 * i] = 0.; m->fdamp[2 * i + 1] = 0.; }
    if (!m->mx_ptr) return;
    for (int i = m->mx_ptr[b]; i < m->mx_ptr[b + 1]; i++) {
        int dof0 = m->mx_dofs[2 * i], dof1 = m->mx_dofs[2 * i + 1];
        double d = m->mx_c[i];
        int node0 = dof0 / 2, dir0 = dof0 - node0 * 2, node1 = dof1 / 2, dir1 = dof1 - node1 * 2;
        int a = n0 + node0, c = n0 + node1;
        if (dir0 == 0 && dir1 == 0) {
            m->fdamp[2 * a] -= m->vp[2 * c] * d;
            if (dof0 != dof1) m->fdamp[2 * c] -= m->vp[2 * a] * d;
        } else if (dir0 == 0 && dir1 == 1) {
            m->fdamp[2 * a] -= m->vp[2 * c + 1] * d;
            m->fdamp[2 * c + 1] -= m->vp[2 * a] * d;
        } else if (dir0 == 1 && dir1 == 0) {
            m->fdamp[2 * a + 1] -= m->vp[2 * c] * d;
            m->fdamp[2 * c] -= m->vp[2 * a + 1] * d;
        } else {
            m->fdamp[2 * a + 1] -= m->vp[2 * c + 1] * d;
            if (dof0 != dof1) m->fdamp[2 * c + 1] -= m->vp[2 * a + 1] * d;
        }
    }
}

/* Body::Update_alid_forces (Code/Body.h:1163-1296): the layer's reference velocity of each
 * direction interpolated in its history at Time (the first interval holding Time; the reference
 * scans past the end of its vector when none does, here the value stays 0), the nodal term
 * -beta m (v - pv), then the stiffness entries' terms -(v_param - pv) d with
 * d = k / (1/alpha0 + 1/alpha1), in entry order; a direction without history gets no force */
static void update_alid_forces(orc_model* m, int b, double T)
{
    if (m->btype[b] != MEL_BODY_DEFORMABLE || !m->alid_ptr) return;
    int flag[2];
    double pv[2] = { 0., 0. };
    for (int dir = 0; dir < 2; dir++) {
        int h0 = m->alid_ptr[2 * b + dir], h1 = m->alid_ptr[2 * b + dir + 1];
        flag[dir] = h1 > h0;
        for (int k = h0; k + 1 < h1; k++) {
            double t0 = m->alid_t[k], p0 = m->alid_v[k], t1 = m->alid_t[k + 1], p1 = m->alid_v[k + 1];
            if ((t0 <= T) & (T <= t1)) { pv[dir] = p0 + (p1 - p0) / (t1 - t0) * (T - t0); break; }
        }
    }
    if (!flag[0] && !flag[1]) return;          /* flag_alid == 0 */
    int n0 = m->nptr[b];
    for (int i = n0; i < m->nptr[b + 1]; i++) {
        double beta = m->alid_ab[2 * i + 1];
        m->falid[2 * i] = flag[0] ? -beta * m->mass[2 * i] * (m->v[2 * i] - pv[0]) : 0.;
        m->falid[2 * i + 1] = flag[1] ? -beta * m->mass[2 * i + 1] * (m->v[2 * i + 1] - pv[1]) : 0.;
    }
    if (!m->mx_ptr) return;
    for (int i = m->mx_ptr[b]; i < m->mx_ptr[b + 1]; i++) {
        int dof0 = m->mx_dofs[2 * i], dof1 = m->mx_dofs[2 * i + 1];
        int node0 = dof0 / 2, dir0 = dof0 - node0 * 2, node1 = dof1 / 2, dir1 = dof1 - node1 * 2;
        int a = n0 + node0, c = n0 + node1;
        double d = m->mx_k[i] / (1. / m->alid_ab[2 * a] + 1. / m->alid_ab[2 * c]);
        if (dir0 == 0 && dir1 == 0) {
            if (flag[0]) m->falid[2 * a] += -(m->vp[2 * c] - pv[0]) * d;
            if ((dof0 != dof1) && flag[0]) m->falid[2 * c] += -(m->vp[2 * a] - pv[0]) * d;
        } else if (dir0 == 0 && dir1 == 1) {
            if (flag[0]) m->falid[2 * a] += -(m->vp[2 * c + 1] - pv[1]) * d;
            if (flag[1]) m->falid[2 * c + 1] += -(m->vp[2 * a] - pv[0]) * d;
        } else if (dir0 == 1 && dir1 == 0) {
            if (flag[1]) m->falid[2 * a + 1] += -(m->vp[2 * c] - pv[0]) * d;
            if (flag[0]) m->falid[2 * c] += -(m->vp[2 * a + 1] - pv[1]) * d;
        } else {
            if (flag[1]) m->falid[2 * a + 1] += -(m->vp[2 * c + 1] - pv[1]) * d;
            if ((dof0 != dof1) && flag[1]) m->falid[2 * c + 1] += -(m->vp[2 * a + 1] - pv[1]) * d;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Contacts                                                                                     */
/* ------------------------------------------------------------------------------------------ */
/* Body::Initialize_contact_forces (Code/Body.h:1305-1333) */
static void initialize_contact_forces(orc_model* m, int b)
{
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) { m->fcon[2 * i] = 0.; m->fcon[2 * i + 1] = 0.; }
    } else {
        double* rf = m->rf + 15 * b; rf[0] = rf[1] = rf[2] = 0.;
    }
    m->send[b].n = 0;
}

static inline void seg_nodes(const orc_model* m, int bodyM, int borderM, int seg, int* nd, int* sh)
{
    int e = m->bd_ptr[gbd(m, bodyM, borderM)] + seg;
    for (int k = 0; k < 4; k++) { nd[k] = m->s_node[k][e]; sh[k] = m->s_shift[k][e]; }
}

/* Body::Update_contacts (Code/Body.h:1341-1634).  shape[] persists across contacts of the body
 * exactly like the reference's function-scope shapeM0..3. */
static void update_contacts(orc_model* m, int b)
{
    double period = m->xmax - m->xmin;
    double shape[4] = { 0., 0., 0., 0. };
    int flag = 0;
    cvec* cv = &m->cont[b];
    for (int ic = 0; ic < cv->n; ic++) {
        mel_contact* c = &cv->a[ic];
        int nodeS = c->nodeS, bodyM = c->bodyM, borderM = c->borderM, shiftM = c->shiftM, segmentM = c->segmentM;
        int gM = gbd(m, bodyM, borderM);
        int per = m->bd_per[gM];
        double gapn = c->gapn, gapt = c->gapt, xsi = c->xsi, xnorm = c->xnorm, ynorm = c->ynorm, xtan = c->xtan, ytan = c->ytan;
        int nd[4], sh[4];
        seg_nodes(m, bodyM, borderM, segmentM, nd, sh);
        double xsi_previous = xsi;
        int s0 = m->nptr[b] + nodeS, mb = m->nptr[bodyM];
        double xs = m->x[2 * s0], ys = m->x[2 * s0 + 1];
        double X[4], Y[4];
        for (int k = 0; k < 4; k++) { X[k] = m->x[2 * (mb + nd[k])] + period * (shiftM + sh[k]); Y[k] = m->x[2 * (mb + nd[k]) + 1]; }
        int flag_in = flag;
        double sh_in[4] = { shape[0], shape[1], shape[2], shape[3] };
        if (b == bodyM && (nd[0] == nodeS || nd[3] == nodeS))
            closest_2_segment_self(xs, ys, X[1], Y[1], X[2], Y[2], &gapn, &xsi, &xnorm, &ynorm, &xtan, &ytan,
                                   &shape[0], &shape[1], &shape[2], &shape[3], &flag);
        else
            closest_2_segment_linear(xs, ys, X[0], Y[0], X[1], Y[1], X[2], Y[2], X[3], Y[3], &gapn, &xsi, &xnorm, &ynorm,
                                     &xtan, &ytan, &shape[0], &shape[1], &shape[2], &shape[3], &flag);
        (void)flag_in; (void)sh_in;
        int set1 = (flag == -2 || flag == -1 || flag == 0 || flag == 1 || flag == 2) && !(b == bodyM && (nd[0] == nodeS || nd[3] == nodeS));
        if (flag == -2 || flag == -3) {
            gapt = gapt + 0.5 * (-1. - xsi_previous) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
            if (per == MEL_PER_SIMPLE) {
                if (segmentM == 0) { borderM = m->bd_bef[gM]; segmentM = bd_count(m, gbd(m, bodyM, borderM)) - 2; }
                else segmentM--;
            } else if (per == MEL_PER_PERIODIC) {
                if (segmentM == 0) {
                    if (borderM == 0) shiftM--; else if (borderM == 1) shiftM++;
                    segmentM = bd_count(m, gbd(m, bodyM, borderM)) - 2;
                } else segmentM--;
            } else {
                if (segmentM == 0) segmentM = bd_count(m, gbd(m, bodyM, borderM)) - 2; else segmentM--;
            }
            seg_nodes(m, bodyM, borderM, segmentM, nd, sh);
            for (int k = 0; k < 4; k++) { X[k] = m->x[2 * (mb + nd[k])] + period * (shiftM + sh[k]); Y[k] = m->x[2 * (mb + nd[k]) + 1]; }
            xsi = 1.;
            int wset = 0;
            double before[4] = { shape[0], shape[1], shape[2], shape[3] };
            if (b == bodyM && (nd[0] == nodeS || nd[3] == nodeS))
                closest_2_segment_self(xs, ys, X[1], Y[1], X[2], Y[2], &gapn, &xsi, &xnorm, &ynorm, &xtan, &ytan,
                                       &shape[0], &shape[1], &shape[2], &shape[3], &flag);
            else
                closest_2_segment_linear(xs, ys, X[0], Y[0], X[1], Y[1], X[2], Y[2], X[3], Y[3], &gapn, &xsi, &xnorm, &ynorm,
                                         &xtan, &ytan, &shape[0], &shape[1], &shape[2], &shape[3], &flag);
            wset = (flag == -2 || flag == -1 || flag == 0 || flag == 1 || flag == 2);
            (void)before;
            if (!wset && !set1) m->stale++;
            gapt = gapt + 0.5 * (-1. + xsi) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
            c->bodyM = bodyM; c->borderM = borderM; c->shiftM = shiftM; c->segmentM = segmentM;
        } else if (flag == 2 || flag == 3) {
            gapt = gapt + 0.5 * (-1. + xsi_previous) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
            int last = bd_count(m, gM) - 2;
            if (per == MEL_PER_SIMPLE) {
                if (segmentM == last) { borderM = m->bd_aft[gM]; segmentM = 0; } else segmentM++;
            } else if (per == MEL_PER_PERIODIC) {
                if (segmentM == last) { if (borderM == 0) shiftM++; else if (borderM == 1) shiftM--; segmentM = 0; }
                else segmentM++;
            } else {
                if (segmentM == last) segmentM = 0; else segmentM++;
            }
            seg_nodes(m, bodyM, borderM, segmentM, nd, sh);
            for (int k = 0; k < 4; k++) { X[k] = m->x[2 * (mb + nd[k])] + period * (shiftM + sh[k]); Y[k] = m->x[2 * (mb + nd[k]) + 1]; }
            xsi = -1.;
            double before[4] = { shape[0], shape[1], shape[2], shape[3] };
            if (b == bodyM && (nd[0] == nodeS || nd[3] == nodeS))
                closest_2_segment_self(xs, ys, X[1], Y[1], X[2], Y[2], &gapn, &xsi, &xnorm, &ynorm, &xtan, &ytan,
                                       &shape[0], &shape[1], &shape[2], &shape[3], &flag);
            else
                closest_2_segment_linear(xs, ys, X[0], Y[0], X[1], Y[1], X[2], Y[2], X[3], Y[3], &gapn, &xsi, &xnorm, &ynorm,
                                         &xtan, &ytan, &shape[0], &shape[1], &shape[2], &shape[3], &flag);
            int wset = (flag == -2 || flag == -1 || flag == 0 || flag == 1 || flag == 2);
            (void)before;
            if (!wset && !set1) m->stale++;
            gapt = gapt + 0.5 * (1. + xsi) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
            c->bodyM = bodyM; c->borderM = borderM; c->shiftM = shiftM; c->segmentM = segmentM;
        } else {
            gapt = gapt + 0.5 * (xsi - xsi_previous) * sqrt((X[2] - X[1]) * (X[2] - X[1]) + (Y[2] - Y[1]) * (Y[2] - Y[1]));
        }
        double vsx = m->v[2 * s0], vsy = m->v[2 * s0 + 1];
        double vgapx = vsx - (shape[0] * m->v[2 * (mb + nd[0])] + shape[1] * m->v[2 * (mb + nd[1])] +
                              shape[2] * m->v[2 * (mb + nd[2])] + shape[3] * m->v[2 * (mb + nd[3])]);
        double vgapy = vsy - (shape[0] * m->v[2 * (mb + nd[0]) + 1] + shape[1] * m->v[2 * (mb + nd[1]) + 1] +
                              shape[2] * m->v[2 * (mb + nd[2]) + 1] + shape[3] * m->v[2 * (mb + nd[3]) + 1]);
        c->gapn = gapn; c->vgapn = vgapx * xnorm + vgapy * ynorm;
        c->gapt = gapt; c->vgapt = vgapx * xtan + vgapy * ytan;
        c->xsi = xsi; c->xnorm = xnorm; c->ynorm = ynorm; c->xtan = xtan; c->ytan = ytan;
        for (int k = 0; k < 4; k++) { c->nodeM[k] = nd[k]; c->shapeM[k] = shape[k]; c->shiftMk[k] = sh[k]; }
    }
}

/* Body::Update_contact_forces (Code/Body.h:1642-1941) */
static void update_contact_forces(orc_model* m, int b, double Deltat)
{
    double period = m->xmax - m->xmin;
    cvec* cv = &m->cont[b];
    double* rg = m->rg + MEL_RIGID_NF * b;
    for (int ic = 0; ic < cv->n; ic++) {
        mel_contact* c = &cv->a[ic];
        double W = 0.;
        int e = m->bd_ptr[gbd(m, b, c->borderS)] + c->border_nodeS;
        double length = m->blen[e], initial_length = m->blen0[e];
        double gapn = c->gapn, vgapn = c->vgapn, gapt = c->gapt, vgapt = c->vgapt;
        int nodeS = c->nodeS, bodyM = c->bodyM, shiftM = c->shiftM;
        double xnorm = c->xnorm, ynorm = c->ynorm, xtan = c->xtan, ytan = c->ytan, effm = c->effective_mass;
        int li = m->table[m->bmat[b] * m->nmat + m->bmat[bodyM]];
        if (li <= -1) continue;
        int type = m->law_type[li];
        const double* P = m->law_p + MEL_LAW_NPARAM * li;
        double Pn = 0., Pt = 0.;
        if (type == MEL_LAW_FRICTIONLESS) law_frictionless(P[0], gapn, &gapt, &Pn, &Pt);
        else if (type == MEL_LAW_COHESION) law_cohesion(P[0], P[1], P[2] * 0.5, P[3] * 0.5, gapn, &gapt, &Pn, &Pt);
        else if (type == MEL_LAW_MOHR_COULOMB) law_mohr_coulomb(P[0], P[1], P[2], P[3] * 0.5, P[4] * 0.5, gapn, &gapt, &Pn, &Pt);
        else if (type == MEL_LAW_DAMPED_MOHR_COULOMB)
            law_damped_mc(P[0], P[1], P[2], P[3] * 0.5, P[4] * 0.5, P[5], effm, initial_length, gapn, vgapn, &gapt, vgapt, &Pn, &Pt, &W);
        else if (type == MEL_LAW_TWO_SLOPES_MOHR_COULOMB)
            law_two_slopes_mc(P[0], P[1], P[2], P[3] * 0.5, P[4] * 0.5, P[5], gapn, vgapn, &gapt, vgapt, &Pn, &Pt);
        else if (type == MEL_LAW_BONDED_MOHR_COULOMB) {
            double Damage = c->internal[0];
            Pn = c->internal[1]; Pt = c->internal[2];
            if (c->nb_internal == 0) {
                Damage = 1.; c->nb_internal = 3; c->internal[0] = 1.; c->internal[1] = 0.; c->internal[2] = 0.;
            }
            law_bonded_mc(P[0], P[1], P[2], P[3], P[4] * 0.5, P[5] * 0.5, P[6], P[7] * 0.5, P[8] * 0.5, P[9], effm, initial_length,
                          gapn, vgapn, &gapt, vgapt, &Damage, &Pn, &Pt);
            c->internal[0] = Damage; c->internal[1] = Pn; c->internal[2] = Pt;
        } else if (type == MEL_LAW_CZM_LINEAR) {
            double Damage = c->internal[0];
            if (c->nb_internal == 0) { Damage = 1.; c->nb_internal = 1; c->internal[0] = 1.; }
            law_czm_linear(P[0], P[1] * 0.5, P[2], P[3] * 0.5, P[4], gapn, &gapt, &Damage, &Pn, &Pt);
            c->internal[0] = Damage;
        } else if (type == MEL_LAW_CZM_FATIGUE) {
            double Damage = c->internal[0];
            Pn = c->internal[1]; Pt = c->internal[2];
            if (c->nb_internal == 0) {
                Damage = 1.; c->nb_internal = 3; c->internal[0] = 1.; c->internal[1] = 0.; c->internal[2] = 0.;
            }
            law_czm_fatigue(P[0], P[1] * 0.5, P[2], P[3] * 0.5, P[4], P[5], P[6], P[7], gapn, &gapt, &Damage, &Pn, &Pt);
            c->internal[0] = Damage; c->internal[1] = Pn; c->internal[2] = Pt;
        }
        double Px = xnorm * Pn + xtan * Pt, Py = ynorm * Pn + ytan * Pt;
        double Fsx, Fsy;
        if (m->law_len[li] == MEL_LENGTH_FIXED) { Fsx = Px * initial_length; Fsy = Py * initial_length; W *= initial_length * Deltat; }
        else { Fsx = Px * length; Fsy = Py * length; W *= length * Deltat; }
        c->gapn = gapn; c->gapt = gapt; c->length = length; c->fx = Fsx; c->fy = Fsy;
        m->works[7 * b + 1] += 0.5 * W;
        m->works[7 * bodyM + 1] += 0.5 * W;
        int s0 = m->nptr[b] + nodeS;
        if (m->btype[b] == MEL_BODY_DEFORMABLE) {
            for (int j = m->sptr[s0]; j < m->sptr[s0 + 1]; j++) {
                int t = m->nptr[b] + m->sidx[j];
                m->fcon[2 * t] += Fsx * m->sN[j];
                m->fcon[2 * t + 1] += Fsy * m->sN[j];
            }
        } else {
            double dx = m->x[2 * s0] - rg[MEL_RG_XC], dy = m->x[2 * s0 + 1] - rg[MEL_RG_YC];
            double* rf = m->rf + 15 * b;
            rf[0] += Fsx; rf[1] += Fsy; rf[2] += -Fsx * dy + Fsy * dx;
        }
        if (m->btype[bodyM] == MEL_BODY_DEFORMABLE) {
            for (int k = 0; k < 4; k++) {
                int mn = m->nptr[bodyM] + c->nodeM[k];
                double sk = c->shapeM[k];
                for (int j = m->sptr[mn]; j < m->sptr[mn + 1]; j++)
                    spush(&m->send[b], bodyM, m->sidx[j], -Fsx * sk * m->sN[j], -Fsy * sk * m->sN[j], 0.);
            }
        } else {
            const double* rgm = m->rg + MEL_RIGID_NF * bodyM;
            double dx = m->x[2 * s0] - rgm[MEL_RG_XC] - shiftM * period;
            double dy = m->x[2 * s0 + 1] - rgm[MEL_RG_YC];
            spush(&m->send[b], bodyM, -1, -Fsx, -Fsy, Fsx * dy - Fsy * dx);
        }
    }
}

/* Body::Send_contact_forces (Code/Body.h:1948-1967) */
static void send_contact_forces(orc_model* m, int b)
{
    svec* s = &m->send[b];
    for (int j = 0; j < s->n; j++) {
        int tb = s->a[j].body, n = s->a[j].node;
        if (n == -1) {
            double* rf = m->rf + 15 * tb;
            rf[0] += s->a[j].f[0]; rf[1] += s->a[j].f[1]; rf[2] += s->a[j].f[2];
        } else {
            int t = m->nptr[tb] + n;
            m->fcon[2 * t] += s->a[j].f[0];
            m->fcon[2 * t + 1] += s->a[j].f[1];
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Internal forces and node update                                                             */
/* ------------------------------------------------------------------------------------------ */
/* Body::Update_internal_forces (Code/Body.h:937-1049) + Apply_Elastic_Linear / Apply_NeoHookean
 * (Code/Model.h:19-73), one region. */
static void update_internal_forces(orc_model* m, int b, int region)
{
    const double* P = m->mat_p + MEL_MAT_NPARAM * m->bmat[b];
    int mtype = m->mat_type[m->bmat[b]];
    int n0 = m->nptr[b], R = m->nreg[b];
    int G = m->gptr[b + 1] - m->gptr[b];
    int npr = (int)ceil((double)G / (double)R);
    int ga = m->gptr[b] + region * npr, gb = m->gptr[b] + (region + 1) * npr;
    if (gb > m->gptr[b + 1]) gb = m->gptr[b + 1];
    double* freg = m->freg + m->reg_off[b];
    for (int i = ga; i < gb; i++) {
        double c0;
        if (mtype == MEL_MAT_ELASTIC_LINEAR) {
            double E11 = 0., E12 = 0., E22 = 0.;
            for (int j = m->gsp[i]; j < m->gsp[i + 1]; j++) {
                int t = n0 + m->gsi[j];
                E11 += m->gdx[j] * m->up[2 * t];
                E12 += m->gdx[j] * m->up[2 * t + 1] + m->gdy[j] * m->up[2 * t];
                E22 += m->gdy[j] * m->up[2 * t + 1];
            }
            E12 = 0.5 * E12;
            double Mu = P[3], Lambda = P[4];
            double J = 1. + E11 + E22;
            double S33 = Lambda * (J - 1.);
            Mu = 2 * Mu;
            double S11 = S33 + Mu * E11, S22 = S33 + Mu * E22, S12 = Mu * E12;
            c0 = m->gw[i] * m->gJ[i];
            for (int j = m->gsp[i]; j < m->gsp[i + 1]; j++) {
                int l = m->gsi[j];
                freg[(l * R + region) * 2] -= c0 * (m->gdx[j] * S11 + m->gdy[j] * S12);
                freg[(l * R + region) * 2 + 1] -= c0 * (m->gdy[j] * S22 + m->gdx[j] * S12);
            }
        } else {
            double F11 = 1., F12 = 0., F21 = 0., F22 = 1.;
            for (int j = m->gsp[i]; j < m->gsp[i + 1]; j++) {
                int t = n0 + m->gsi[j];
                F11 += m->gdx[j] * m->up[2 * t];
                F12 += m->gdy[j] * m->up[2 * t];
                F21 += m->gdx[j] * m->up[2 * t + 1];
                F22 += m->gdy[j] * m->up[2 * t + 1];
            }
            double Mu = P[3], Kappa = P[4];
            double F11F12 = F11 * F11 + F12 * F12, F21F22 = F21 * F21 + F22 * F22;
            double J = F11 * F22 - F12 * F21;
            double invJ = 1. / J;
            double K = Kappa * (J - 1.);
            double MuJ53 = Mu * pow(J, -1.666666666667);
            double trBover3 = 0.333333333333 * (F11F12 + F21F22 + 1.);
            double sig11 = K + MuJ53 * (F11F12 - trBover3);
            double sig22 = K + MuJ53 * (F21F22 - trBover3);
            double sig12 = MuJ53 * (F11 * F21 + F12 * F22);
            double S11 = (F12 * (F12 * sig22 - F22 * sig12) - F22 * (F12 * sig12 - F22 * sig11)) * invJ;
            double S22 = (F11 * (F11 * sig22 - F21 * sig12) - F21 * (F11 * sig12 - F21 * sig11)) * invJ;
            double S12 = (F21 * (F12 * sig12 - F22 * sig11) - F11 * (F12 * sig22 - F22 * sig12)) * invJ;
            c0 = m->gw[i] * m->gJ[i];
            for (int j = m->gsp[i]; j < m->gsp[i + 1]; j++) {
                int l = m->gsi[j];
                freg[(l * R + region) * 2] -= c0 * (m->gdx[j] * (F11 * S11 + F12 * S12) + m->gdy[j] * (F12 * S22 + F11 * S12));
                freg[(l * R + region) * 2 + 1] -= c0 * (m->gdx[j] * (F21 * S11 + F22 * S12) + m->gdy[j] * (F22 * S22 + F21 * S12));
            }
        }
    }
}

/* Body::Sum_up_forces (Code/Body.h:1975-2015) and Node::Sum_up_forces (Code/Node.h:212-225) */
static void sum_up_forces(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        int R = m->nreg[b];
        double* freg = m->freg + m->reg_off[b];
        for (int l = 0; l < nb_nodes(m, b); l++) {
            int i = n0 + l;
            double fx = 0., fy = 0.;
            for (int r = 0; r < R; r++) {
                fx += freg[(l * R + r) * 2]; fy += freg[(l * R + r) * 2 + 1];
                freg[(l * R + r) * 2] = 0.; freg[(l * R + r) * 2 + 1] = 0.;
            }
            m->fint[2 * i] = fx; m->fint[2 * i + 1] = fy;
            m->ftot[2 * i] = m->fint[2 * i] + m->fcon[2 * i] + m->fself[2 * i] + m->fbody[2 * i] + m->fdir[2 * i] + m->fneu[2 * i] + m->fdamp[2 * i] + m->falid[2 * i];
            m->ftot[2 * i + 1] = m->fint[2 * i + 1] + m->fcon[2 * i + 1] + m->fself[2 * i + 1] + m->fbody[2 * i + 1] + m->fdir[2 * i + 1] + m->fneu[2 * i + 1] + m->fdamp[2 * i + 1] + m->falid[2 * i + 1];
        }
    } else {
        double* rf = m->rf + 15 * b;
        double* t = m->rtot + 3 * b;
        for (int d = 0; d < 3; d++) t[d] = rf[d] + rf[3 + d] + rf[6 + d] + rf[9 + d] + rf[12 + d];
        for (int l = 0; l < nb_nodes(m, b); l++) {
            int i = n0 + l;
            m->fcon[2 * i] = rf[0]; m->fcon[2 * i + 1] = rf[1];
            m->fbody[2 * i] = rf[3]; m->fbody[2 * i + 1] = rf[4];
            m->fdir[2 * i] = rf[6]; m->fdir[2 * i + 1] = rf[7];
            m->fneu[2 * i] = rf[9]; m->fneu[2 * i + 1] = rf[10];
            m->fdamp[2 * i] = rf[12]; m->fdamp[2 * i + 1] = rf[13];
            m->ftot[2 * i] = t[0]; m->ftot[2 * i + 1] = t[1];
        }
    }
}

/* Body::Apply_Newton (Code/Body.h:2023-2043), Node::Apply_Newton (Code/Node.h:227-231) */
static void apply_newton(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    double* rg = m->rg + MEL_RIGID_NF * b;
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            m->ap[2 * i] = m->ftot[2 * i] * m->invm[2 * i] / m->fms[2 * i];
            m->ap[2 * i + 1] = m->ftot[2 * i + 1] * m->invm[2 * i + 1] / m->fms[2 * i + 1];
        }
    } else {
        double* t = m->rtot + 3 * b;
        rg[MEL_RG_XA] = t[0] * rg[MEL_RG_INV_MASS] / m->bfms[b];
        rg[MEL_RG_YA] = t[1] * rg[MEL_RG_INV_MASS] / m->bfms[b];
        rg[MEL_RG_RA] = t[2] * rg[MEL_RG_INV_INERTIA] / m->bfms[b];
    }
    for (int i = n0; i < m->nptr[b + 1]; i++) { m->a[2 * i] = rg[MEL_RG_XA]; m->a[2 * i + 1] = rg[MEL_RG_YA]; }
}

/* Body::Apply_Euler (Code/Body.h:2051-2118), Node::Apply_Euler (Code/Node.h:239-245) */
static void apply_euler(orc_model* m, int b, double Deltat)
{
    double* W = m->works + 7 * b;
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            double vx = m->vp[2 * i] + 0.5 * Deltat * m->ap[2 * i];
            double vy = m->vp[2 * i + 1] + 0.5 * Deltat * m->ap[2 * i + 1];
            W[0] += Deltat * (vx * m->fint[2 * i] + vy * m->fint[2 * i + 1]);
            W[2] += Deltat * (vx * m->fbody[2 * i] + vy * m->fbody[2 * i + 1]);
            W[3] += Deltat * (vx * m->fdir[2 * i] + vy * m->fdir[2 * i + 1]);
            W[4] += Deltat * (vx * m->fneu[2 * i] + vy * m->fneu[2 * i + 1]);
            W[5] += Deltat * (vx * m->fdamp[2 * i] + vy * m->fdamp[2 * i + 1]);
            W[6] += Deltat * (vx * m->falid[2 * i] + vy * m->falid[2 * i + 1]);
            m->vp[2 * i] = m->vp[2 * i] + Deltat * m->ap[2 * i];
            m->vp[2 * i + 1] = m->vp[2 * i + 1] + Deltat * m->ap[2 * i + 1];
            m->up[2 * i] = m->up[2 * i] + Deltat * m->vp[2 * i];
            m->up[2 * i + 1] = m->up[2 * i + 1] + Deltat * m->vp[2 * i + 1];
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        double* rf = m->rf + 15 * b;
        double* t = m->rtot + 3 * b;
        double* drv = m->drv + 8 * b;
        double vx = rg[MEL_RG_XV] + 0.5 * Deltat * rg[MEL_RG_XA];
        double vy = rg[MEL_RG_YV] + 0.5 * Deltat * rg[MEL_RG_YA];
        double vr = rg[MEL_RG_RV] + 0.5 * Deltat * rg[MEL_RG_RA];
        W[2] += Deltat * (vx * rf[3] + vy * rf[4] + vr * rf[5]);
        W[3] += Deltat * (vx * rf[6] + vy * rf[7] + vr * rf[8]);
        W[4] += Deltat * (vx * rf[9] + vy * rf[10] + vr * rf[11]);
        W[5] += Deltat * (vx * rf[12] + vy * rf[13] + vr * rf[14]);
        if (drv[0] == 0.) {
            rg[MEL_RG_XV] += Deltat * rg[MEL_RG_XA];
            rg[MEL_RG_XD] = rg[MEL_RG_XD] + Deltat * rg[MEL_RG_XV];
        } else if (drv[0] == 1.) {
            rg[MEL_RG_XA] = drv[3]; rg[MEL_RG_XV] = drv[2]; rg[MEL_RG_XD] = drv[1];
            rf[6] = rg[MEL_RG_MASS] * rg[MEL_RG_XA] - t[0];
        }
        if (drv[4] == 0.) {
            rg[MEL_RG_YV] += Deltat * rg[MEL_RG_YA];
            rg[MEL_RG_YD] = rg[MEL_RG_YD] + Deltat * rg[MEL_RG_YV];
        } else if (drv[4] == 1.) {
            rg[MEL_RG_YA] = drv[7]; rg[MEL_RG_YV] = drv[6]; rg[MEL_RG_YD] = drv[5];
            rf[7] = rg[MEL_RG_MASS] * rg[MEL_RG_YA] - t[1];
        }
        if (drv[0] == 0. && drv[4] == 0. && !m->bper[b]) {
            rg[MEL_RG_RV] += Deltat * rg[MEL_RG_RA];
            rg[MEL_RG_RD] = rg[MEL_RG_RD] + Deltat * rg[MEL_RG_RV];
        } else { rg[MEL_RG_RV] = 0.; rg[MEL_RG_RD] = 0.; }
    }
}

/* Body::Apply_Euler_temporary (Code/Body.h:2126-2168), Node::Apply_Euler_temporary (Node.h:247-251) */
static void apply_euler_temporary(orc_model* m, int b, double Deltat)
{
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            m->upt[2 * i] = m->up[2 * i] + Deltat * (m->vp[2 * i] + Deltat * m->ap[2 * i]);
            m->upt[2 * i + 1] = m->up[2 * i + 1] + Deltat * (m->vp[2 * i + 1] + Deltat * m->ap[2 * i + 1]);
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        double* tm = m->rg_tmp + 6 * b;
        double* drv = m->drv + 8 * b;
        if (drv[0] == 0.) { tm[3] = rg[MEL_RG_XV] + Deltat * rg[MEL_RG_XA]; tm[0] = rg[MEL_RG_XD] + Deltat * tm[3]; }
        else if (drv[0] == 1.) { tm[3] = drv[2]; tm[0] = drv[1]; }
        if (drv[4] == 0.) { tm[4] = rg[MEL_RG_YV] + Deltat * rg[MEL_RG_YA]; tm[1] = rg[MEL_RG_YD] + Deltat * tm[4]; }
        else if (drv[4] == 1.) { tm[4] = drv[6]; tm[1] = drv[5]; }
        if (drv[0] == 0. && drv[4] == 0. && !m->bper[b]) { tm[5] = rg[MEL_RG_RV] + Deltat * rg[MEL_RG_RA]; tm[2] = rg[MEL_RG_RD] + Deltat * tm[5]; }
        else { tm[5] = 0.; tm[2] = 0.; }
    }
}

/* Body::Update_kinematics (Code/Body.h:2176-2227) */
static void update_kinematics(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            double dx = 0., dy = 0., vx = 0., vy = 0., ax = 0., ay = 0.;
            for (int j = m->sptr[i]; j < m->sptr[i + 1]; j++) {
                int t = n0 + m->sidx[j];
                double s = m->sN[j];
                dx += s * m->up[2 * t]; dy += s * m->up[2 * t + 1];
                vx += s * m->vp[2 * t]; vy += s * m->vp[2 * t + 1];
                ax += s * m->ap[2 * t]; ay += s * m->ap[2 * t + 1];
            }
            m->u[2 * i] = dx; m->u[2 * i + 1] = dy;
            m->v[2 * i] = vx; m->v[2 * i + 1] = vy;
            m->a[2 * i] = ax; m->a[2 * i + 1] = ay;
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            double dx = m->X0[2 * i] - rg[MEL_RG_X0], dy = m->X0[2 * i + 1] - rg[MEL_RG_Y0];
            double dr = rg[MEL_RG_RD] - rg[MEL_RG_R0];
            m->u[2 * i] = rg[MEL_RG_XD] + dx * orc_cos(dr) - dy * orc_sin(dr) - dx;
            m->u[2 * i + 1] = rg[MEL_RG_YD] + dx * orc_sin(dr) + dy * orc_cos(dr) - dy;
            m->v[2 * i] = rg[MEL_RG_XV]; m->v[2 * i + 1] = rg[MEL_RG_YV];
        }
    }
}

/* Body::Update_kinematics_temporary (Code/Body.h:2235-2264) */
static void update_kinematics_temporary(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            double dx = 0., dy = 0.;
            for (int j = m->sptr[i]; j < m->sptr[i + 1]; j++) {
                int t = n0 + m->sidx[j];
                dx += m->sN[j] * m->upt[2 * t]; dy += m->sN[j] * m->upt[2 * t + 1];
            }
            m->ut[2 * i] = dx; m->ut[2 * i + 1] = dy;
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        double* tm = m->rg_tmp + 6 * b;
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            double dx = m->X0[2 * i] - rg[MEL_RG_X0], dy = m->X0[2 * i + 1] - rg[MEL_RG_Y0];
            double dr = tm[2] - rg[MEL_RG_R0];
            m->ut[2 * i] = tm[0] + dx * orc_cos(dr) - dy * orc_sin(dr) - dx;
            m->ut[2 * i + 1] = tm[1] + dx * orc_sin(dr) + dy * orc_cos(dr) - dy;
        }
    }
}

/* Body::Update_current_positions (Code/Body.h:2272-2302), Node.h:233-237 */
static void update_current_positions(orc_model* m, int b)
{
    int n0 = m->nptr[b];
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            m->x[2 * i] = m->X0[2 * i] + m->u[2 * i];
            m->x[2 * i + 1] = m->X0[2 * i + 1] + m->u[2 * i + 1];
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        rg[MEL_RG_XC] = rg[MEL_RG_X0] + rg[MEL_RG_XD];
        rg[MEL_RG_YC] = rg[MEL_RG_Y0] + rg[MEL_RG_YD];
        rg[MEL_RG_RC] = rg[MEL_RG_R0] + rg[MEL_RG_RD];
        for (int i = n0; i < m->nptr[b + 1]; i++) {
            double dx = m->X0[2 * i] - rg[MEL_RG_X0], dy = m->X0[2 * i + 1] - rg[MEL_RG_Y0];
            double dr = rg[MEL_RG_RD] - rg[MEL_RG_R0];
            m->x[2 * i] = rg[MEL_RG_XC] + dx * orc_cos(dr) - dy * orc_sin(dr);
            m->x[2 * i + 1] = rg[MEL_RG_YC] + dx * orc_sin(dr) + dy * orc_cos(dr);
            dx = m->x[2 * i] - rg[MEL_RG_XC];
            dy = m->x[2 * i + 1] - rg[MEL_RG_YC];
            m->v[2 * i] = -dy * rg[MEL_RG_RV] + rg[MEL_RG_XV];
            m->v[2 * i + 1] = dx * rg[MEL_RG_RV] + rg[MEL_RG_YV];
        }
    }
}

/* Node::Compute_error / Body::Compute_error (Code/Node.h:253-272, Code/Body.h:2528-2553) */
static void compute_error(orc_model* m, int b)
{
    double* drv = m->drv + 8 * b;
    m->terr[b] = 0.;
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        m->merr[b] = 0.; m->nmerr[b] = 0;
        for (int l = 0; l < nb_nodes(m, b); l++) {
            int i = m->nptr[b] + l;
            if (drv[0] == 1.) m->err[2 * i] = 0.; else m->err[2 * i] = m->u[2 * i] - m->ut[2 * i];
            if (drv[4] == 1.) m->err[2 * i + 1] = 0.; else m->err[2 * i + 1] = m->u[2 * i + 1] - m->ut[2 * i + 1];
            double en = sqrt(m->err[2 * i] * m->err[2 * i] + m->err[2 * i + 1] * m->err[2 * i + 1]) * m->ide[i];
            m->terr[b] += en;
            if (en == 0.) en = 1.e-16;
            m->errn[i] = en;
            if (en > m->merr[b]) { m->merr[b] = en; m->nmerr[b] = l; }
        }
    } else {
        double* rg = m->rg + MEL_RIGID_NF * b;
        double* tm = m->rg_tmp + 6 * b;
        if (drv[0] != 1.) m->terr[b] += (rg[MEL_RG_XD] - tm[0]) * (rg[MEL_RG_XD] - tm[0]);
        if (drv[4] != 1.) m->terr[b] += (rg[MEL_RG_YD] - tm[1]) * (rg[MEL_RG_YD] - tm[1]);
        m->terr[b] = 0.1 * sqrt(m->terr[b]) / m->bdist[3 * b];
        if (m->terr[b] == 0.) m->terr[b] = 1.e-16;
        m->merr[b] = m->terr[b]; m->nmerr[b] = -1;
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) m->errn[i] = m->terr[b];
    }
}

/* Node::Compute_mass_scaling / Body::Compute_mass_scaling (Code/Node.h:274-320, Body.h:2559-2594) */
static void compute_mass_scaling(orc_model* m, int b)
{
    double Target_error = m->sp[0], MaxMS = m->sp[3], CtrlMS = m->sp[4], ErrFac = m->sp[5], Decr = m->sp[6];
    m->bmms[b] = 0.;
    if (m->btype[b] == MEL_BODY_DEFORMABLE) {
        m->bmaxfms[b] = 0.;
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            for (int d = 0; d < 2; d++) {
                double e = fabs(m->err[2 * i + d] * m->ide[i]);
                if (e >= Target_error * ErrFac) {
                    m->dfms[2 * i + d] = pow((e - Target_error * ErrFac), CtrlMS);
                    m->fms[2 * i + d] += m->dfms[2 * i + d];
                    if (m->fms[2 * i + d] > MaxMS) m->fms[2 * i + d] = MaxMS;
                } else {
                    if (m->fms[2 * i + d] != 1) m->fms[2 * i + d] *= Decr;
                    if (m->fms[2 * i + d] < 1) m->fms[2 * i + d] = 1;
                }
            }
            double f = (m->fms[2 * i] + m->fms[2 * i + 1]) * 0.5;
            if (f > m->bmaxfms[b]) m->bmaxfms[b] = f;
            double mx = m->mass[2 * i], my = m->mass[2 * i + 1];
            m->mms[i] = sqrt(mx * mx * m->fms[2 * i] * m->fms[2 * i] + my * my * m->fms[2 * i + 1] * m->fms[2 * i + 1]);
            m->bmms[b] += m->mms[i];
        }
    } else {
        if (m->terr[b] >= Target_error * ErrFac) {
            m->bdfms[b] = pow((m->terr[b] - Target_error * ErrFac), CtrlMS);
            m->bfms[b] += m->bdfms[b];
            if (m->bfms[b] >= MaxMS) m->bfms[b] = MaxMS;
        } else {
            if (m->bfms[b] != 1) m->bfms[b] *= Decr;
            if (m->bfms[b] < 1) m->bfms[b] = 1;
        }
        m->bmms[b] = m->rg[MEL_RIGID_NF * b + MEL_RG_MASS] * m->bfms[b];
    }
}

/* Update_contact_pressures (Code/Proximity.h:1014-1069) */
static void update_contact_pressures(orc_model* m)
{
    for (int i = 0; i < m->nbd; i++)
        for (int k = m->bd_ptr[i]; k < m->bd_ptr[i + 1]; k++) { m->cpx[k] = 0.; m->cpy[k] = 0.; }
    for (int b = 0; b < m->nb; b++) {
        for (int j = 0; j < m->cont[b].n; j++) {
            mel_contact* c = &m->cont[b].a[j];
            int eM = m->bd_ptr[gbd(m, c->bodyM, c->borderM)];
            int eS = m->bd_ptr[gbd(m, b, c->borderS)] + c->border_nodeS;
            double fx = c->fx, fy = c->fy, il = 1. / c->length;
            m->cpx[eS] += fx * il; m->cpy[eS] += fy * il;
            m->cpx[eM + c->segmentM] -= fx * il * c->shapeM[1];
            m->cpy[eM + c->segmentM] -= fy * il * c->shapeM[1];
            m->cpx[eM + c->segmentM + 1] -= fx * il * c->shapeM[2];
            m->cpy[eM + c->segmentM + 1] -= fy * il * c->shapeM[2];
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Proximity (Code/Proximity.h:48-473)                                                          */
/* ------------------------------------------------------------------------------------------ */
static void nbr_push(orc_model* m, int b, int body2, int border2, int shift)
{
    if (m->nbn[b] == m->nbc[b]) {
        m->nbc[b] = m->nbc[b] ? 2 * m->nbc[b] : 8;
        m->nbl[b] = (nbr_t*)realloc(m->nbl[b], (size_t)m->nbc[b] * sizeof(nbr_t));
    }
    nbr_t* n = &m->nbl[b][m->nbn[b]++];
    n->body2 = body2; n->border2 = border2; n->shift = shift;
}

int orc_update_proximity(orc_model* m)
{
    double period = m->xmax - m->xmin;
    double invperiod = 1. / period;
    for (int i = 0; i < m->nb; i++) {
        m->nbn[i] = 0;
        if (!is_active(m, i)) continue;
        for (int j = 0; j < nb_borders(m, i); j++) {
            int g = gbd(m, i, j);
            double xmin = 1.e100, xmax = -1.e100, ymin = 1.e100, ymax = -1.e100;
            for (int k = m->bd_ptr[g]; k < m->bd_ptr[g + 1]; k++) {
                int n = m->nptr[i] + m->bd_nodes[k];
                double x = m->x[2 * n], y = m->x[2 * n + 1], d = m->bdist[3 * i + 1];
                if (x - d < xmin) xmin = x - d;
                if (x + d > xmax) xmax = x + d;
                if (y - d < ymin) ymin = y - d;
                if (y + d > ymax) ymax = y + d;
            }
            m->prox[4 * g] = xmin; m->prox[4 * g + 1] = xmax; m->prox[4 * g + 2] = ymin; m->prox[4 * g + 3] = ymax;
            m->shmin[g] = (int)floor((xmin - m->xmin) * invperiod);
            m->shmax[g] = (int)floor((xmax - m->xmin) * invperiod);
        }
    }
    for (int b1 = 0; b1 < m->nb; b1++) {
        if (!is_active(m, b1)) continue;
        for (int r1 = 0; r1 < nb_borders(m, b1); r1++) {
            int g1 = gbd(m, b1, r1);
            double xmin1 = m->prox[4 * g1], xmax1 = m->prox[4 * g1 + 1], ymin1 = m->prox[4 * g1 + 2], ymax1 = m->prox[4 * g1 + 3];
            for (int b2 = 0; b2 < m->nb; b2++) {
                if (!is_active(m, b2) || b1 == b2) continue;
                for (int r2 = 0; r2 < nb_borders(m, b2); r2++) {
                    int g2 = gbd(m, b2, r2);
                    double xmin2 = m->prox[4 * g2], xmax2 = m->prox[4 * g2 + 1], ymin2 = m->prox[4 * g2 + 2], ymax2 = m->prox[4 * g2 + 3];
                    if ((ymax2 < ymin1) || (ymax1 < ymin2)) continue;
                    for (int s = m->shmin[g1] - m->shmax[g2]; s <= m->shmax[g1] - m->shmin[g2]; s++) {
                        if ((xmax2 + s * period > xmin1) && (xmin2 + s * period < xmax1)) {
                            int ok = 1;
                            for (int q = 0; q < m->nbn[b1]; q++) {
                                nbr_t* n = &m->nbl[b1][q];
                                if (n->body2 == b2 && n->border2 == r2 && n->shift == s) { ok = 0; break; }
                            }
                            if (ok) nbr_push(m, b1, b2, r2, s);
                        }
                    }
                }
            }
        }
    }
    /* local proximities */
    cvec* fresh = (cvec*)xcalloc((size_t)m->nb, sizeof(cvec));
    for (int bS = 0; bS < m->nb; bS++) {
        mel_contact nc; memset(&nc, 0, sizeof nc);
        int flag = 0;
        for (int rS = 0; rS < nb_borders(m, bS); rS++) {
            int gS = gbd(m, bS, rS);
            int nS = bd_count(m, gS);
            for (int q = 0; q < m->nbn[bS]; q++) {
                int bM = m->nbl[bS][q].body2, rM = m->nbl[bS][q].border2, shM = m->nbl[bS][q].shift;
                int gM = gbd(m, bM, rM);
                int nM = bd_count(m, gM);
                double effm;
                const double* rgM = m->rg + MEL_RIGID_NF * bM;
                const double* rgS = m->rg + MEL_RIGID_NF * bS;
                if (rgM[MEL_RG_MASS] == 0.) effm = 0.;
                else if (rgS[MEL_RG_MASS] == 0.) effm = 0.;
                else effm = 1. / (rgM[MEL_RG_INV_MASS] + rgS[MEL_RG_INV_MASS]);
                for (int kS = 0; kS < nS; kS++) {
                    int eS = m->bd_ptr[gS] + kS;
                    int NodeS = m->bd_nodes[eS];
                    double length = m->blen[eS];
                    int s0 = m->nptr[bS] + NodeS;
                    double Xs = m->x[2 * s0], Ys = m->x[2 * s0 + 1];
                    for (int seg = 0; seg < nM - 1; seg++) {
                        int eM = m->bd_ptr[gM] + seg;
                        int mb = m->nptr[bM];
                        double X1 = m->x[2 * (mb + m->s_node[1][eM])] + period * (shM + m->s_shift[1][eM]);
                        double Y1 = m->x[2 * (mb + m->s_node[1][eM]) + 1];
                        double X2 = m->x[2 * (mb + m->s_node[2][eM])] + period * (shM + m->s_shift[2][eM]);
                        double Y2 = m->x[2 * (mb + m->s_node[2][eM]) + 1];
                        if (detect_segment_proximity(Xs, Ys, X1, Y1, X2, Y2, m->bdist[3 * bS + 1]) == 0) continue;
                        double X0 = m->x[2 * (mb + m->s_node[0][eM])] + period * (shM + m->s_shift[0][eM]);
                        double Y0 = m->x[2 * (mb + m->s_node[0][eM]) + 1];
                        double X3 = m->x[2 * (mb + m->s_node[3][eM])] + period * (shM + m->s_shift[3][eM]);
                        double Y3 = m->x[2 * (mb + m->s_node[3][eM]) + 1];
                        double Gapn = 0, Xsi = 0., Xn = 0, Yn = 0, Xt = 0, Yt = 0, N0 = 0, N1 = 0, N2 = 0, N3 = 0;
                        closest_2_segment_linear(Xs, Ys, X0, Y0, X1, Y1, X2, Y2, X3, Y3, &Gapn, &Xsi, &Xn, &Yn, &Xt, &Yt,
                                                 &N0, &N1, &N2, &N3, &flag);
                        if ((flag == -2 || flag == -1 || flag == 0) && (Gapn > -m->bdist[3 * bS + 2])) {
                            int exists = 0;
                            cvec* old = &m->cont[bS];
                            for (int k = 0; k < old->n; k++) {
                                mel_contact* o = &old->a[k];
                                if (o->borderS == rS && o->border_nodeS == kS && o->bodyM == bM && o->borderM == rM &&
                                    abs(o->segmentM - seg) <= 1) { nc = *o; exists = 1; break; }
                            }
                            if (!exists) {
                                nc.bodyS = bS; nc.borderS = rS; nc.border_nodeS = kS; nc.nodeS = NodeS;
                                nc.bodyM = bM; nc.borderM = rM; nc.shiftM = shM; nc.segmentM = seg;
                                for (int k = 0; k < 4; k++) { nc.nodeM[k] = m->s_node[k][eM]; nc.shiftMk[k] = m->s_shift[k][eM]; }
                                nc.shapeM[0] = N0; nc.shapeM[1] = N1; nc.shapeM[2] = N2; nc.shapeM[3] = N3;
                                nc.gapn = Gapn; nc.gapt = 0.; nc.xsi = Xsi; nc.xnorm = Xn; nc.ynorm = Yn; nc.xtan = Xt; nc.ytan = Yt;
                                nc.effective_mass = effm; nc.length = length; nc.fx = 0.; nc.fy = 0.;
                                nc.nb_internal = 0; nc.internal[0] = 0.; nc.internal[1] = 0.; nc.internal[2] = 0.;
                            }
                            cpush(&fresh[bS], &nc);
                        }
                    }
                }
            }
        }
    }
    for (int b = 0; b < m->nb; b++) { free(m->cont[b].a); m->cont[b] = fresh[b]; }
    free(fresh);
    /* self proximities (Code/Proximity.h:332-470); they search the list just built */
    if (m->flags[8] == 0) {
        for (int bS = 0; bS < m->nb; bS++) {
            if (m->btype[bS] == MEL_BODY_RIGID || m->bper[bS]) continue;
            mel_contact nc; memset(&nc, 0, sizeof nc);
            int flag = 0;
            int nreg_before = m->cont[bS].n;
            double effm = m->rg[MEL_RIGID_NF * bS + MEL_RG_MASS];
            for (int rS = 0; rS < nb_borders(m, bS); rS++) {
                int gS = gbd(m, bS, rS);
                int nS = bd_count(m, gS);
                for (int kS = 0; kS < nS; kS++) {
                    int eS = m->bd_ptr[gS] + kS;
                    int NodeS = m->bd_nodes[eS];
                    double length = m->blen[eS];
                    int s0 = m->nptr[bS] + NodeS;
                    double Xs = m->x[2 * s0], Ys = m->x[2 * s0 + 1];
                    for (int rM = 0; rM < nb_borders(m, bS); rM++) {
                        int gM = gbd(m, bS, rM);
                        int nM = bd_count(m, gM);
                        for (int seg = 0; seg < nM - 1; seg++) {
                            int eM = m->bd_ptr[gM] + seg;
                            int mb = m->nptr[bS];
                            int NM1 = m->s_node[1][eM], NM2 = m->s_node[2][eM];
                            if (NM1 == NodeS) continue;
                            double X1 = m->x[2 * (mb + NM1)], Y1 = m->x[2 * (mb + NM1) + 1];
                            if (NM2 == NodeS) continue;
                            double X2 = m->x[2 * (mb + NM2)], Y2 = m->x[2 * (mb + NM2) + 1];
                            if (detect_segment_proximity(Xs, Ys, X1, Y1, X2, Y2, m->bdist[3 * bS + 1]) == 0) continue;
                            int NM0 = m->s_node[0][eM], NM3 = m->s_node[3][eM];
                            double X0 = m->x[2 * (mb + NM0)], Y0 = m->x[2 * (mb + NM0) + 1];
                            double X3 = m->x[2 * (mb + NM3)], Y3 = m->x[2 * (mb + NM3) + 1];
                            double Gapn = 0, Xsi = 0., Xn = 0, Yn = 0, Xt = 0, Yt = 0, N0 = 0, N1 = 0, N2 = 0, N3 = 0;
                            if (NM0 == NodeS || NM3 == NodeS)
                                closest_2_segment_self(Xs, Ys, X1, Y1, X2, Y2, &Gapn, &Xsi, &Xn, &Yn, &Xt, &Yt, &N0, &N1, &N2, &N3, &flag);
                            else
                                closest_2_segment_linear(Xs, Ys, X0, Y0, X1, Y1, X2, Y2, X3, Y3, &Gapn, &Xsi, &Xn, &Yn, &Xt, &Yt,
                                                         &N0, &N1, &N2, &N3, &flag);
                            if (flag == 0 && (Gapn > -m->bdist[3 * bS + 2])) {
                                int exists = 0;
                                for (int k = 0; k < nreg_before; k++) {
                                    mel_contact* o = &m->cont[bS].a[k];
                                    if (o->borderS == rS && o->border_nodeS == kS && o->bodyM == bS && o->borderM == rM &&
                                        abs(o->segmentM - seg) <= 1) { nc = *o; exists = 1; break; }
                                }
                                if (!exists) {
                                    nc.bodyS = bS; nc.borderS = rS; nc.border_nodeS = kS; nc.nodeS = NodeS;
                                    nc.bodyM = bS; nc.borderM = rM; nc.shiftM = 0; nc.segmentM = seg;
                                    nc.nodeM[0] = NM0; nc.nodeM[1] = NM1; nc.nodeM[2] = NM2; nc.nodeM[3] = NM3;
                                    for (int k = 0; k < 4; k++) nc.shiftMk[k] = 0;
                                    nc.shapeM[0] = N0; nc.shapeM[1] = N1; nc.shapeM[2] = N2; nc.shapeM[3] = N3;
                                    nc.gapn = Gapn; nc.gapt = 0.; nc.xsi = Xsi; nc.xnorm = Xn; nc.ynorm = Yn; nc.xtan = Xt; nc.ytan = Yt;
                                    nc.effective_mass = effm; nc.length = length; nc.fx = 0.; nc.fy = 0.;
                                    nc.nb_internal = 0; nc.internal[0] = nc.internal[1] = nc.internal[2] = 0.;
                                }
                                cpush(&m->cont[bS], &nc);
                            }
                        }
                    }
                }
            }
        }
    }
    return 0;
}

/* Initialize_CZM (Code/Proximity.h:481-541) */
static void initialize_czm(orc_model* m)
{
    for (int b = 0; b < m->nb; b++) update_contacts(m, b);
    m->flags[3] = 0;
    for (int bS = 0; bS < m->nb; bS++) {
        for (int ic = 0; ic < m->cont[bS].n; ic++) {
            mel_contact* c = &m->cont[bS].a[ic];
            int li = m->table[m->bmat[bS] * m->nmat + m->bmat[c->bodyM]];
            if (li < 0) continue;
            const double* P = m->law_p + MEL_LAW_NPARAM * li;
            int t = m->law_type[li];
            double gi;
            if (t == MEL_LAW_CZM_LINEAR) { gi = P[5]; c->nb_internal = 1; c->internal[0] = (c->gapn < gi) ? 0. : 1.; }
            else if (t == MEL_LAW_CZM_FATIGUE || t == MEL_LAW_BONDED_MOHR_COULOMB) {
                gi = (t == MEL_LAW_CZM_FATIGUE) ? P[8] : P[10];
                c->nb_internal = 3; c->internal[0] = (c->gapn < gi) ? 0. : 1.; c->internal[1] = 0.; c->internal[2] = 0.;
            }
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Step drivers (Code/Solver.h)                                                                 */
/* ------------------------------------------------------------------------------------------ */
static void force_evaluation(orc_model* m, double law_dt, double bc_time, int update_bc_first, double alid_time)
{
    for (int i = 0; i < m->nb; i++) {
        if (!is_active(m, i)) continue;
        initialize_contact_forces(m, i);
        if (update_bc_first) body_update_bc(m, i, bc_time);
        update_borders(m, i);
        update_contacts(m, i);
    }
    for (int i = 0; i < m->nb; i++) {
        if (!is_active(m, i)) continue;
        update_bc_forces(m, i);
        update_body_forces(m, i);
        update_damping_forces(m, i);
        update_alid_forces(m, i, alid_time);
        update_contact_forces(m, i, law_dt);
    }
    for (int i = 0; i < m->nb; i++) send_contact_forces(m, i);
    for (int i = 0; i < m->nb; i++) {
        if (!is_active(m, i) || m->btype[i] != MEL_BODY_DEFORMABLE) continue;
        for (int r = 0; r < m->nreg[i]; r++) update_internal_forces(m, i, r);
    }
}

/* Euler_step (Code/Solver.h:10-88) */
static void euler_step(orc_model* m)
{
    force_evaluation(m, m->dt, 0., 0, m->time);
    for (int i = 0; i < m->nb; i++) {
        if (!is_active(m, i)) continue;
        sum_up_forces(m, i);
        apply_newton(m, i);
        body_update_bc(m, i, m->time + m->dt);
        apply_euler(m, i, m->dt);
        update_kinematics(m, i);
        update_current_positions(m, i);
    }
    m->time += m->dt;
    update_contact_pressures(m);
}

/* Body::Store / Body::Restore (Code/Body.h:2601-2659): the full node, border and contact state
 * plus works and rigid kinematics. */
#define NODE_BLOB 40
static void store_all(orc_model* m)
{
    double* const arrs[] = { m->x, m->u, m->v, m->a, m->up, m->vp, m->ap, m->upt, m->ut, m->fint, m->fcon, m->fself,
                             m->fbody, m->fdir, m->fneu, m->fdamp, m->falid, m->ftot, m->fms, m->err };
    for (int k = 0; k < 20; k++) memcpy(m->s_node_blob + (size_t)k * 2 * m->nn, arrs[k], sizeof(double) * 2 * m->nn);
    for (int b = 0; b < m->nb; b++) {
        double* sb = m->s_body_blob + 16 * b;
        memcpy(sb, m->works + 7 * b, 7 * sizeof(double));
        sb[7] = m->bdfms[b];
        const double* rg = m->rg + MEL_RIGID_NF * b;
        for (int k = 0; k < 3; k++) { sb[8 + k] = rg[MEL_RG_XC + k]; sb[11 + k] = rg[MEL_RG_XD + k]; }
        sb[14] = rg[MEL_RG_XV]; sb[15] = rg[MEL_RG_YV];
        m->s_body_blob[16 * m->nb + b] = rg[MEL_RG_RV];
        m->s_cont[b].n = 0;
        for (int j = 0; j < m->cont[b].n; j++) cpush(&m->s_cont[b], &m->cont[b].a[j]);
    }
    int ne = m->bd_ptr[m->nbd];
    double* const barr[] = { m->blen, m->cpx, m->cpy, m->bcpx, m->bcpy };
    for (int k = 0; k < 5; k++) memcpy(m->s_border_blob + (size_t)k * ne, barr[k], sizeof(double) * ne);
    memcpy(m->s_border_blob + (size_t)5 * ne, m->bc_value, sizeof(double) * 2 * m->nbd);
    memcpy(m->s_border_blob + (size_t)5 * ne + 2 * m->nbd, m->bc_vel, sizeof(double) * 2 * m->nbd);
}
static void restore_all(orc_model* m)
{
    double* const arrs[] = { m->x, m->u, m->v, m->a, m->up, m->vp, m->ap, m->upt, m->ut, m->fint, m->fcon, m->fself,
                             m->fbody, m->fdir, m->fneu, m->fdamp, m->falid, m->ftot, m->fms, m->err };
    for (int k = 0; k < 20; k++) memcpy(arrs[k], m->s_node_blob + (size_t)k * 2 * m->nn, sizeof(double) * 2 * m->nn);
    for (int b = 0; b < m->nb; b++) {
        double* sb = m->s_body_blob + 16 * b;
        memcpy(m->works + 7 * b, sb, 7 * sizeof(double));
        m->bdfms[b] = sb[7];
        if (m->btype[b] == MEL_BODY_RIGID) {
            double* rg = m->rg + MEL_RIGID_NF * b;
            for (int k = 0; k < 3; k++) { rg[MEL_RG_XC + k] = sb[8 + k]; rg[MEL_RG_XD + k] = sb[11 + k]; }
            rg[MEL_RG_XV] = sb[14]; rg[MEL_RG_YV] = sb[15]; rg[MEL_RG_RV] = m->s_body_blob[16 * m->nb + b];
        }
        m->cont[b].n = 0;
        for (int j = 0; j < m->s_cont[b].n; j++) cpush(&m->cont[b], &m->s_cont[b].a[j]);
    }
    int ne = m->bd_ptr[m->nbd];
    double* const barr[] = { m->blen, m->cpx, m->cpy, m->bcpx, m->bcpy };
    for (int k = 0; k < 5; k++) memcpy(barr[k], m->s_border_blob + (size_t)k * ne, sizeof(double) * ne);
    memcpy(m->bc_value, m->s_border_blob + (size_t)5 * ne, sizeof(double) * 2 * m->nbd);
    memcpy(m->bc_vel, m->s_border_blob + (size_t)5 * ne + 2 * m->nbd, sizeof(double) * 2 * m->nbd);
}

static void dt_update(orc_model* m, double c1, double c2)
{   /* the correction law shared by the adaptive schemes (Code/Solver.h:349-357) */
    if (c1 > c2) m->dt = m->dt / pow(c1, m->sp[1]);
    else m->dt = m->dt / pow(c2, m->sp[1]);
    if (m->dt > m->cup) m->dt = m->cup;
}

/* Solver_step (Code/Solver.h:98-486) */
static void solver_step(orc_model* m)
{
    double Target_error = m->sp[0], Accepted_ratio = m->sp[2], Inv_Target_error = m->sp[7];
    store_all(m);
    int ok = 0, neval = 0;
    double max_error = 0., mean_error = 0., total_mass = 0., max_mass = 0.;
    while (!ok) {
        neval++;
        force_evaluation(m, m->dt * 0.5, 0., 0, m->time);
        for (int i = 0; i < m->nb; i++) {
            if (!is_active(m, i)) continue;
            sum_up_forces(m, i);
            apply_newton(m, i);
            apply_euler_temporary(m, i, m->dt);
            update_kinematics_temporary(m, i);
            apply_euler(m, i, m->dt * 0.5);
            update_kinematics(m, i);
            update_current_positions(m, i);
        }
        force_evaluation(m, m->dt * 0.5, m->time + m->dt * 0.5, 1, m->time + m->dt * 0.5);
        for (int i = 0; i < m->nb; i++) {
            if (!is_active(m, i)) continue;
            sum_up_forces(m, i);
            apply_newton(m, i);
            body_update_bc(m, i, m->time + m->dt);
            apply_euler(m, i, m->dt * 0.5);
            update_kinematics(m, i);
            update_current_positions(m, i);
            compute_error(m, i);
            if (m->solver == MEL_SOLVER_MASS_SCALING || m->solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING) compute_mass_scaling(m, i);
        }
        mean_error = 0.; max_error = 0.;
        int nnodes = 0;
        for (int i = 0; i < m->nb; i++) {
            if (!is_active(m, i)) continue;
            mean_error += m->terr[i];
            nnodes += nb_nodes(m, i);
            if (m->merr[i] > max_error) max_error = m->merr[i];
        }
        mean_error /= nnodes;
        if (m->solver == MEL_SOLVER_MASS_SCALING || m->solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING) {
            total_mass = 0.; max_mass = 0.;
            for (int i = 0; i < m->nb; i++) {
                if (!is_active(m, i)) continue;
                total_mass += m->bmms[i];
                double inv = m->rg[MEL_RIGID_NF * i + MEL_RG_INV_MASS];
                if (m->bmms[i] * inv > max_mass) max_mass = m->bmms[i] * inv;
            }
        }
        double error = max_error;
        if (m->solver == MEL_SOLVER_ADAPTIVE_EULER) {
            if (error > Target_error * Accepted_ratio) { ok = 0; restore_all(m); dt_update(m, error / Target_error, 1. / Accepted_ratio); }
            else { ok = 1; m->time += m->dt; dt_update(m, error / Target_error, 1. / Accepted_ratio); update_contact_pressures(m); }
        }
        if (m->solver == MEL_SOLVER_EULER_2) {
            ok = 1; m->time += m->dt; dt_update(m, error / Target_error, 1. / Accepted_ratio); update_contact_pressures(m);
        }
        if (m->solver == MEL_SOLVER_MASS_SCALING) {
            if (max_error > Target_error * Accepted_ratio) { ok = 0; restore_all(m); dt_update(m, max_error * Inv_Target_error, 1. / Accepted_ratio); }
            else { ok = 1; m->time += m->dt; dt_update(m, max_error * Inv_Target_error, 1. / Accepted_ratio); update_contact_pressures(m); }
        }
        if (m->solver == MEL_SOLVER_ADAPTIVE_MASS_SCALING) {
            if (max_mass > Accepted_ratio + 0.05) { ok = 0; restore_all(m); dt_update(m, max_mass, 1. / Accepted_ratio); }
            else {
                ok = 1; m->time += m->dt;
                double c2 = 1. / Accepted_ratio;
                m->dt = m->dt / pow(c2, m->sp[1]);
                if (m->dt > m->cup) m->dt = m->cup;
                update_contact_pressures(m);
            }
        }
        if (neval > 1000) break;   /* the reference loops until success; a cap keeps tests bounded */
    }
    m->stats[0] = neval; m->stats[1] = max_error; m->stats[2] = mean_error; m->stats[3] = total_mass; m->stats[4] = max_mass;
}

/* nodal force of kind k (total, internal, contact, body, dirichlet, neumann, damping, alid) of
 * global node i, as Node holds it after Sum_up_forces */
static void node_force(const orc_model* m, int i, int k, double* fx, double* fy)
{
    const double* a[8] = { m->ftot, m->fint, m->fcon, m->fbody, m->fdir, m->fneu, m->fdamp, m->falid };
    *fx = a[k][2 * i]; *fy = a[k][2 * i + 1];
}

/* Body::Update_damage (Code/Body.h:2667-2700): per border node the smallest internal[0] of the
 * body's contact elements on that node that carry internal variables (1 when none does), averaged
 * over the border nodes, and never below the previous value */
static double update_damage(orc_model* m, int b)
{
    double total_nodes = 0., dmg = 0.;
    const double previous = m->damage[b];
    const cvec* cv = &m->cont[b];
    for (int i = 0; i < m->bptr[b + 1] - m->bptr[b]; i++) {
        const int g = m->bptr[b] + i;
        const int nbn = m->bd_ptr[g + 1] - m->bd_ptr[g];
        total_nodes += nbn;
        for (int j = 0; j < nbn; j++) {
            double d = 1.;
            for (int k = 0; k < cv->n; k++) {
                const mel_contact* c = &cv->a[k];
                if (c->borderS == i && c->border_nodeS == j && c->nb_internal > 0 && c->internal[0] < d) d = c->internal[0];
            }
            dmg += d;
        }
    }
    dmg = dmg / total_nodes;
    if (dmg < previous) dmg = previous;
    m->damage[b] = dmg;
    return dmg;
}
void orc_get_damage(orc_model* m, double* out) { memcpy(out, m->damage, sizeof(double) * m->nb); }
int orc_get_matrices(orc_model* m, double* k, double* c)
{
    if (!m->mx_ptr) return 0;
    memcpy(k, m->mx_k, sizeof(double) * m->nmx);
    memcpy(c, m->mx_c, sizeof(double) * m->nmx);
    return m->nmx;
}
double orc_update_damage(orc_model* m, int b) { return update_damage(m, b); }

/* Update_status (Code/Proximity.h:550-1007): entries of type position, displacement, velocity,
 * acceleration (e = {type, kind, body, node, mode, threshold}) and force (e = {4, kind, force kind,
 * body, node, mode, threshold}); x, y, r start at 0 and carry over between entries */
static void update_status(orc_model* m)
{
    double x = 0., y = 0., r = 0., mm;
    for (int k = 0; k < m->ndeact; k++) {
        const double* e = m->deact + MEL_DEACT_NF * k;
        const int type = (int)e[0], kind = (int)e[1];
        int body, mode;
        double thr;
        if (type >= 0 && type <= 3) {
            body = (int)e[2];
            const int node = (int)e[3];
            mode = (int)e[4]; thr = e[5];
            const double* arr = type == 0 ? m->x : type == 1 ? m->u : type == 2 ? m->v : m->a;
            const int rx = type == 0 ? MEL_RG_XC : type == 1 ? MEL_RG_XD : type == 2 ? MEL_RG_XV : MEL_RG_XA;
            const int n0 = m->nptr[body];
            if (node >= 0) { x = arr[2 * (n0 + node)]; y = arr[2 * (n0 + node) + 1]; }
            else if (m->btype[body] == MEL_BODY_DEFORMABLE) {
                x = 0.; y = 0.; mm = 0.;
                for (int j = n0; j < m->nptr[body + 1]; j++) {
                    x += arr[2 * j] * m->mass[2 * j];
                    y += arr[2 * j + 1] * m->mass[2 * j + 1];
                    mm += m->mass[2 * j];
                }
                x /= mm; y /= mm;
            } else {
                const double* rg = m->rg + MEL_RIGID_NF * body;
                x = rg[rx]; y = rg[rx + 1]; r = rg[rx + 2];
            }
        } else if (type == 4) {
            const int fk = (int)e[2];
            body = (int)e[3];
            const int node = (int)e[4];
            mode = (int)e[5]; thr = e[6];
            if (node >= 0) {
                if (fk <= 6) node_force(m, m->nptr[body] + node, fk, &x, &y);
            } else if (m->btype[fk] == MEL_BODY_DEFORMABLE) {
                /* Code/Proximity.h:866-882: the type and node count of body number <force kind> */
                x = 0.; y = 0.;
                const int n0 = m->nptr[body], cnt = m->nptr[fk + 1] - m->nptr[fk];
                for (int j = 0; j < cnt; j++) {
                    double fx, fy;
                    if (fk == 0) { node_force(m, n0 + j, 0, &fx, &fy); x += fx; y += fy; }
                    else if (fk == 1) { node_force(m, n0 + j, 6, &fx, &fy); x += fx; y += fy; }
                }
            } else {
                const double* rf = m->rf + 15 * body;
                if (fk == 0) { x = m->rtot[3 * body]; y = m->rtot[3 * body + 1]; r = m->rtot[3 * body + 2]; }
                else if (fk >= 2 && fk <= 6) { const int q = 3 * (fk - 2); x = rf[q]; y = rf[q + 1]; r = rf[q + 2]; }
            }
        } else if (type == 8) {
            /* Damage (e = {8, body, mode, threshold}), Code/Proximity.h:988-998 */
            body = (int)e[1];
            mode = (int)e[2]; thr = e[3];
            const double dm = update_damage(m, body);
            if ((mode == 0 && dm <= thr) || (mode == 1 && dm == thr) || (mode == 2 && dm >= thr))
                m->bstatus[body] = MEL_STATUS_INACTIVE;
            continue;
        } else continue;
        double v;
        if (kind == 0) v = x;
        else if (kind == 1) v = y;
        else if (kind == 2) v = type == 0 ? r : pow(x * x + y * y, 0.5);
        else if (kind == 3 && type != 0) v = r;
        else continue;
        if ((mode == 0 && v <= thr) || (mode == 1 && v == thr) || (mode == 2 && v >= thr))
            m->bstatus[body] = MEL_STATUS_INACTIVE;
    }
}

/* Damage entries of Monitoring (Code/Monitoring.h:385-390): after every step, before its proximity
 * update (Code/main.cpp:173-196), Update_damage of the listed bodies, logged in order */
void orc_monitor_damage(orc_model* m, const int* bodies, int n, int cap)
{
    m->dmg_n = n < 16 ? (n > 0 ? n : 0) : 16;
    for (int i = 0; i < m->dmg_n; i++) m->dmg_bodies[i] = (bodies[i] >= 0 && bodies[i] < m->nb) ? bodies[i] : 0;
    free(m->dmg_log);
    m->dmg_log = NEWD((size_t)(cap > 0 ? cap : 1) * (m->dmg_n > 0 ? m->dmg_n : 1));
    m->dmg_cap = cap;
    m->dmg_count = 0;
}
int orc_damage_log(orc_model* m, double* out)
{
    if (out && m->dmg_log) memcpy(out, m->dmg_log, sizeof(double) * (size_t)m->dmg_count * m->dmg_n);
    return m->dmg_count;
}

int orc_step(orc_model* m, int nsteps, int run_proximity)
{
    for (int s = 0; s < nsteps; s++) {
        if (m->solver == MEL_SOLVER_EULER) euler_step(m);
        else solver_step(m);
        if (m->dmg_n > 0 && m->dmg_count < m->dmg_cap) {
            for (int i = 0; i < m->dmg_n; i++) m->dmg_log[(size_t)m->dmg_count * m->dmg_n + i] = update_damage(m, m->dmg_bodies[i]);
            m->dmg_count++;
        }
        if (run_proximity && m->time > m->next_cup - 1.e-6 * m->dt) {
            m->next_cup = m->next_cup + m->cup;
            orc_update_proximity(m);
            update_status(m);                 /* Code/main.cpp:195 */
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* construction                                                                                 */
/* ------------------------------------------------------------------------------------------ */
int orc_create(const mel_model_desc* d, const int* n_regions, orc_model** out)
{
    orc_model* m = (orc_model*)xcalloc(1, sizeof(orc_model));
    m->xmin = d->period[0]; m->xmax = d->period[1]; m->gx = d->gravity[0]; m->gy = d->gravity[1];
    m->time = d->time; m->dt = d->dt; m->tend = d->tend; m->cup = d->contact_update_period; m->next_cup = d->next_contact_update;
    m->solver = d->solver; memcpy(m->sp, d->solver_params, sizeof m->sp); memcpy(m->flags, d->flags, sizeof m->flags);
    m->nmat = d->n_materials; m->mat_type = dupi(d->material_type, m->nmat); m->mat_p = dupd(d->material_params, (size_t)m->nmat * MEL_MAT_NPARAM);
    m->nlaw = d->n_laws; m->law_type = dupi(d->law_type, m->nlaw); m->law_len = dupi(d->law_length, m->nlaw);
    m->law_p = dupd(d->law_params, (size_t)m->nlaw * MEL_LAW_NPARAM); m->table = dupi(d->contacts_table, (size_t)m->nmat * m->nmat);
    int nb = m->nb = d->n_bodies;
    m->ndeact = d->n_deactivated;
    m->deact = d->n_deactivated > 0 ? dupd(d->deactivated, (size_t)d->n_deactivated * MEL_DEACT_NF) : NULL;
    m->btype = dupi(d->body_type, nb); m->bmat = dupi(d->body_material, nb); m->bper = dupi(d->body_periodic, nb);
    m->bstatus = dupi(d->body_status, nb); m->bdist = dupd(d->body_dist, 3 * (size_t)nb);
    m->nptr = dupi(d->body_node_ptr, nb + 1); m->bptr = dupi(d->body_border_ptr, nb + 1); m->gptr = dupi(d->body_gp_ptr, nb + 1);
    m->cptr = dupi(d->body_cell_ptr, nb + 1);
    m->nreg = NEWI(nb); m->reg_off = NEWI(nb + 1);
    for (int b = 0; b < nb; b++) {
        m->nreg[b] = (n_regions && n_regions[b] > 0) ? n_regions[b] : 1;
        m->reg_off[b + 1] = m->reg_off[b] + 2 * (m->nptr[b + 1] - m->nptr[b]) * m->nreg[b];
    }
    m->rg = dupd(d->rigid, (size_t)nb * MEL_RIGID_NF);
    m->rg_tmp = NEWD(6 * nb); m->rf = NEWD(15 * nb); m->rtot = NEWD(3 * nb); m->drv = NEWD(8 * nb); m->works = NEWD(7 * nb);
    m->terr = NEWD(nb); m->merr = NEWD(nb); m->nmerr = NEWI(nb); m->bfms = NEWD(nb); m->bdfms = NEWD(nb); m->bmms = NEWD(nb);
    m->bmaxfms = NEWD(nb); m->eenergy = NEWD(nb); m->damage = NEWD(nb);
    for (int b = 0; b < nb; b++) m->bfms[b] = 1.;
    int nn = m->nn = d->n_nodes;
    m->X0 = dupd(d->node_x0, 2 * (size_t)nn); m->mass = dupd(d->node_mass, 2 * (size_t)nn); m->invm = dupd(d->node_inv_mass, 2 * (size_t)nn);
    m->dom = dupd(d->node_domain, nn);
    m->sptr = dupi(d->node_sup_ptr, nn + 1);
    m->sidx = dupi(d->node_sup_idx, m->sptr[nn]); m->sN = dupd(d->node_sup_N, m->sptr[nn]);
    m->x = NEWD(2 * nn); m->u = NEWD(2 * nn); m->v = NEWD(2 * nn); m->a = NEWD(2 * nn); m->up = NEWD(2 * nn); m->vp = NEWD(2 * nn);
    m->ap = NEWD(2 * nn); m->upt = NEWD(2 * nn); m->ut = NEWD(2 * nn);
    m->freg = NEWD(m->reg_off[nb]); m->fint = NEWD(2 * nn); m->fcon = NEWD(2 * nn); m->fself = NEWD(2 * nn); m->fbody = NEWD(2 * nn);
    m->fdir = NEWD(2 * nn); m->fneu = NEWD(2 * nn); m->fdamp = NEWD(2 * nn); m->falid = NEWD(2 * nn); m->ftot = NEWD(2 * nn);
    m->ide = NEWD(nn); m->err = NEWD(2 * nn); m->errn = NEWD(nn); m->fms = NEWD(2 * nn); m->dfms = NEWD(2 * nn); m->mms = NEWD(nn);
    for (int i = 0; i < 2 * nn; i++) { m->fms[i] = 1.; m->dfms[i] = 1.; }
    orc_set_node_state(m, d->node_state);
    for (int b = 0; b < nb; b++)
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            if (m->btype[b] == MEL_BODY_DEFORMABLE) {
                int ns = m->sptr[i + 1] - m->sptr[i];
                m->ide[i] = ns ? 1. / (m->dom[i] * sqrt(3.1415927 / 4. / ns)) : 0.;   /* Code/IO.h:1814 */
            } else m->ide[i] = 1. / m->bdist[3 * b];                                  /* Code/IO.h:1619 */
        }
    int nbd = m->nbd = d->n_borders;
    m->bd_body = dupi(d->border_body, nbd); m->bd_per = dupi(d->border_periodicity, nbd); m->bd_int = dupi(d->border_interpolant, nbd);
    m->bd_bef = dupi(d->border_before, nbd); m->bd_aft = dupi(d->border_after, nbd); m->bd_ptr = dupi(d->border_node_ptr, nbd + 1);
    int ne = m->bd_ptr[nbd];
    m->bd_nodes = dupi(d->border_nodes, ne);
    m->bc_type = dupi(d->border_bc_type, 2 * nbd); m->bc_param = dupd(d->border_bc_param, 4 * (size_t)nbd);
    m->hptr = dupi(d->border_hist_ptr, 2 * nbd + 1);
    m->ht = dupd(d->hist_time, m->hptr[2 * nbd]); m->hv = dupd(d->hist_value, m->hptr[2 * nbd]);
    m->bc_value = NEWD(2 * nbd); m->bc_vel = NEWD(2 * nbd);
    for (int k = 0; k < 4; k++) { m->s_node[k] = NEWI(ne); m->s_shift[k] = NEWI(ne); }
    m->blen = NEWD(ne); m->blen0 = NEWD(ne); m->cpx = NEWD(ne); m->cpy = NEWD(ne); m->bcpx = NEWD(ne); m->bcpy = NEWD(ne);
    m->prox = NEWD(4 * nbd); m->shmin = NEWI(nbd); m->shmax = NEWI(nbd);
    int ng = m->ng = d->n_gauss;
    m->gsp = dupi(d->gp_sup_ptr, ng + 1);
    int nge = m->gsp[ng];
    m->gsi = dupi(d->gp_sup_idx, nge); m->gN = dupd(d->gp_N, nge); m->gdx = dupd(d->gp_dNdx, nge); m->gdy = dupd(d->gp_dNdy, nge);
    m->gw = dupd(d->gp_weight, ng); m->gJ = dupd(d->gp_jacobian, ng);
    m->cells = dupi(d->cells, 3 * (size_t)d->n_cells);
    m->nmx = d->n_matrix;
    if (d->n_matrix > 0 && d->body_matrix_ptr) {
        m->mx_ptr = dupi(d->body_matrix_ptr, nb + 1); m->mx_dofs = dupi(d->matrix_dofs, 2 * (size_t)d->n_matrix);
        m->mx_k = dupd(d->matrix_stiffness, d->n_matrix); m->mx_c = dupd(d->matrix_damping, d->n_matrix);
    }
    if (d->body_alid_ptr && d->alid_time && d->alid_value && d->node_alid) {
        m->alid_ptr = dupi(d->body_alid_ptr, 2 * (size_t)nb + 1);
        int nh = m->alid_ptr[2 * nb];
        m->alid_t = dupd(d->alid_time, nh); m->alid_v = dupd(d->alid_value, nh);
        m->alid_ab = dupd(d->node_alid, 2 * (size_t)nn);
    }
    m->cont = (cvec*)xcalloc((size_t)nb, sizeof(cvec)); m->s_cont = (cvec*)xcalloc((size_t)nb, sizeof(cvec));
    m->nbl = (nbr_t**)xcalloc((size_t)nb, sizeof(nbr_t*)); m->nbn = NEWI(nb); m->nbc = NEWI(nb);
    m->send = (svec*)xcalloc((size_t)nb, sizeof(svec));
    m->s_node_blob = NEWD((size_t)20 * 2 * nn); m->s_body_blob = NEWD(17 * (size_t)nb);
    m->s_border_blob = NEWD((size_t)5 * ne + 4 * (size_t)nbd);
    for (int b = 0; b < nb; b++) initialize_segments(m, b);
    /* rigid nodes take their positions from the body (Load_dynamic KINEMATICS -> Update_current_positions) */
    for (int b = 0; b < nb; b++) if (m->btype[b] == MEL_BODY_RIGID) update_current_positions(m, b);
    /* set-up of Code/main.cpp:104-127 */
    for (int b = 0; b < nb; b++) update_borders(m, b);
    for (int b = 0; b < nb; b++) body_update_bc(m, b, m->time);
    orc_update_proximity(m);
    if (m->flags[3] == 1) initialize_czm(m);
    for (int b = 0; b < nb; b++) update_material(m, b);
    orc_update_proximity(m);
    if (m->flags[3] == 1) initialize_czm(m);
    *out = m;
    return 0;
}

void orc_get_body_status(const orc_model* m, int* status) { memcpy(status, m->bstatus, sizeof(int) * (size_t)m->nb); }

void orc_destroy(orc_model* m)
{
    if (!m) return;
    /* process-lifetime test object: release the large arrays */
    for (int b = 0; b < m->nb; b++) { free(m->cont[b].a); free(m->s_cont[b].a); free(m->nbl[b]); free(m->send[b].a); }
    free(m->cont); free(m->s_cont); free(m->nbl); free(m->send);
    free(m->freg); free(m->gsi); free(m->gN); free(m->gdx); free(m->gdy); free(m->s_node_blob);
    free(m);
}

/* ------------------------------------------------------------------------------------------ */
/* accessors                                                                                    */
/* ------------------------------------------------------------------------------------------ */
double orc_time(orc_model* m) { return m->time; }
double orc_dt(orc_model* m) { return m->dt; }
long orc_stale_shape_events(orc_model* m) { return m->stale; }
void orc_solver_stats(orc_model* m, double* o) { memcpy(o, m->stats, sizeof m->stats); }
void orc_get_contact_pressures(orc_model* m, double* px, double* py)
{
    int ne = m->bd_ptr[m->nbd];
    memcpy(px, m->cpx, sizeof(double) * ne);
    memcpy(py, m->cpy, sizeof(double) * ne);
}

int orc_n_contacts(orc_model* m) { int n = 0; for (int b = 0; b < m->nb; b++) n += m->cont[b].n; return n; }
int orc_get_contacts(orc_model* m, mel_contact* out, int cap)
{
    int n = 0;
    for (int b = 0; b < m->nb; b++)
        for (int j = 0; j < m->cont[b].n; j++) {
            if (n < cap) { out[n] = m->cont[b].a[j]; out[n].bodyS = b; }
            n++;
        }
    return n;
}
int orc_set_contacts(orc_model* m, const mel_contact* c, int n)
{
    for (int b = 0; b < m->nb; b++) m->cont[b].n = 0;
    for (int k = 0; k < n; k++) {
        if (c[k].bodyS < 0 || c[k].bodyS >= m->nb) return 1;
        cpush(&m->cont[c[k].bodyS], &c[k]);
    }
    return 0;
}
void orc_get_node_state(orc_model* m, double* st)
{
    for (int i = 0; i < m->nn; i++) {
        double* s = st + 12 * i;
        s[0] = m->u[2 * i]; s[1] = m->u[2 * i + 1]; s[2] = m->v[2 * i]; s[3] = m->v[2 * i + 1]; s[4] = m->a[2 * i]; s[5] = m->a[2 * i + 1];
        s[6] = m->up[2 * i]; s[7] = m->up[2 * i + 1]; s[8] = m->vp[2 * i]; s[9] = m->vp[2 * i + 1]; s[10] = m->ap[2 * i]; s[11] = m->ap[2 * i + 1];
    }
}
void orc_set_node_state(orc_model* m, const double* st)
{
    if (!st) return;
    for (int i = 0; i < m->nn; i++) {
        const double* s = st + 12 * i;
        m->u[2 * i] = s[0]; m->u[2 * i + 1] = s[1]; m->v[2 * i] = s[2]; m->v[2 * i + 1] = s[3]; m->a[2 * i] = s[4]; m->a[2 * i + 1] = s[5];
        m->up[2 * i] = s[6]; m->up[2 * i + 1] = s[7]; m->vp[2 * i] = s[8]; m->vp[2 * i + 1] = s[9]; m->ap[2 * i] = s[10]; m->ap[2 * i + 1] = s[11];
        m->x[2 * i] = m->X0[2 * i] + m->u[2 * i];
        m->x[2 * i + 1] = m->X0[2 * i + 1] + m->u[2 * i + 1];
    }
    for (int b = 0; m->btype && b < m->nb; b++) if (m->btype[b] == MEL_BODY_RIGID) update_current_positions(m, b);
}
void orc_get_positions(orc_model* m, double* xy) { memcpy(xy, m->x, sizeof(double) * 2 * m->nn); }
void orc_get_forces(orc_model* m, double* fint, double* fcon, double* fneu, double* fdir, double* ftot)
{
    size_t s = sizeof(double) * 2 * m->nn;
    if (fint) memcpy(fint, m->fint, s);
    if (fcon) memcpy(fcon, m->fcon, s);
    if (fneu) memcpy(fneu, m->fneu, s);
    if (fdir) memcpy(fdir, m->fdir, s);
    if (ftot) memcpy(ftot, m->ftot, s);
}
void orc_get_rigid(orc_model* m, double* rigid, double* rf)
{
    if (rigid) memcpy(rigid, m->rg, sizeof(double) * MEL_RIGID_NF * m->nb);
    if (rf) for (int b = 0; b < m->nb; b++) memcpy(rf + 12 * b, m->rf + 15 * b, 12 * sizeof(double));
}
void orc_set_time(orc_model* m, double time, double dt, double next_contact_update)
{
    m->time = time; m->dt = dt; m->next_cup = next_contact_update;
}

void orc_set_rigid(orc_model* m, const double* rigid)
{
    memcpy(m->rg, rigid, sizeof(double) * MEL_RIGID_NF * m->nb);
    for (int b = 0; b < m->nb; b++) if (m->btype[b] == MEL_BODY_RIGID) update_current_positions(m, b);
}
void orc_get_works(orc_model* m, double* w) { memcpy(w, m->works, sizeof(double) * 7 * m->nb); }
int orc_get_neighbours(orc_model* m, int* rows, int cap)
{
    int n = 0;
    for (int b = 0; b < m->nb; b++)
        for (int q = 0; q < m->nbn[b]; q++) {
            if (n < cap) { rows[4 * n] = b; rows[4 * n + 1] = m->nbl[b][q].body2; rows[4 * n + 2] = m->nbl[b][q].border2; rows[4 * n + 3] = m->nbl[b][q].shift; }
            n++;
        }
    return n;
}
void orc_monitor(orc_model* m, mel_monitor* o)
{   /* Code/Monitoring.h:88-101 (mean displacement), 528-531 (kinetic energy) */
    memset(o, 0, sizeof *o);
    o->time = m->time;
    double ke = 0., ux = 0., uy = 0., mt = 0.;
    for (int b = 0; b < m->nb; b++) {
        for (int i = m->nptr[b]; i < m->nptr[b + 1]; i++) {
            ke += 0.5 * m->v[2 * i] * m->v[2 * i] * m->mass[2 * i];
            ke += 0.5 * m->v[2 * i + 1] * m->v[2 * i + 1] * m->mass[2 * i + 1];
            if (m->btype[b] == MEL_BODY_DEFORMABLE) { ux += m->u[2 * i] * m->mass[2 * i]; uy += m->u[2 * i + 1] * m->mass[2 * i + 1]; mt += m->mass[2 * i]; }
        }
    }
    o->kinetic_energy = ke;
    o->mean_displacement[0] = mt > 0 ? ux / mt : 0.;
    o->mean_displacement[1] = mt > 0 ? uy / mt : 0.;
    int r = 0;
    for (int b = 0; b < m->nb && r < 4; b++) {
        if (m->btype[b] != MEL_BODY_RIGID) continue;
        o->rigid_force[2 * r] = m->rf[15 * b]; o->rigid_force[2 * r + 1] = m->rf[15 * b + 1];
        o->rigid_dirichlet[2 * r] = m->rf[15 * b + 6]; o->rigid_dirichlet[2 * r + 1] = m->rf[15 * b + 7];
        r++;
    }
    int act = 0, nc = 0;
    for (int b = 0; b < m->nb; b++)
        for (int j = 0; j < m->cont[b].n; j++) { nc++; if (m->cont[b].a[j].fx != 0. || m->cont[b].a[j].fy != 0.) act++; }
    o->active_contacts = act; o->n_contacts = nc;
}
