// Device restatement of the reference's projection geometry and contact laws.
// Operation order follows the reference exactly; this translation unit is compiled with
// -fmad=false so no multiply-add is contracted, and pow(x,-0.5) is the correctly rounded
// mel_rsqrt (mel_rsqrt.h).
#pragma once
#include "mel_rsqrt.h"

namespace mel {

struct Proj {       // outputs of Closest_2_segment (unassigned outputs keep their inputs)
    double gap, xsi, xn, yn, xt, yt, N[4];
    int flag;
};

// Closest_2_segment, "Linear" interpolant (Code/Tools.h:106-219)
__device__ __forceinline__ void closest_linear(double Xs, double Ys, double X0, double Y0, double X1, double Y1,
                                               double X2, double Y2, double X3, double Y3, Proj& p)
{
    double ilength = mel_rsqrt((X2 - X1) * (X2 - X1) + (Y2 - Y1) * (Y2 - Y1));
    double ilengthm = mel_rsqrt((X1 - X0) * (X1 - X0) + (Y1 - Y0) * (Y1 - Y0));
    double ilengthp = mel_rsqrt((X3 - X2) * (X3 - X2) + (Y3 - Y2) * (Y3 - Y2));
    double xt = (X2 - X1) * ilength, yt = (Y2 - Y1) * ilength;
    p.xt = xt; p.yt = yt; p.xn = yt; p.yn = -xt;
    double Xtanm = (X1 - X0) * ilengthm, Ytanm = (Y1 - Y0) * ilengthm;
    double Xtanp = (X3 - X2) * ilengthp, Ytanp = (Y3 - Y2) * ilengthp;
    if (((Xs - X1) * (Xtanm + xt) + (Ys - Y1) * (Ytanm + yt)) * (xt * (Xtanm + xt) + yt * (Ytanm + yt)) >= 0.) {
        if (((Xs - X2) * (xt + Xtanp) + (Ys - Y2) * (yt + Ytanp)) * (xt * (xt + Xtanp) + yt * (yt + Ytanp)) <= 0.) {
            double xsi = -1. + 2. * ((X2 - X1) * (Xs - X1) + (Y2 - Y1) * (Ys - Y1)) * ilength * ilength;
            p.xsi = xsi;
            if ((xsi < 1.) && (xsi > -1.)) {
                p.xn = yt; p.yn = -xt;
                double Xc = 0.5 * (X1 + X2) + xsi * 0.5 * (X2 - X1);
                double Yc = 0.5 * (Y1 + Y2) + xsi * 0.5 * (Y2 - Y1);
                p.gap = p.xn * (Xs - Xc) + p.yn * (Ys - Yc);
                p.N[0] = 0.; p.N[1] = 0.5 * (1. - xsi); p.N[2] = 0.5 * (1. + xsi); p.N[3] = 0.;
                p.flag = 0;
            } else if (xsi == -1.) {
                p.xn = yt; p.yn = -xt;
                p.gap = p.xn * (Xs - X1) + p.yn * (Ys - Y1);
                p.N[0] = 0.; p.N[1] = 1.; p.N[2] = 0.; p.N[3] = 0.;
                p.flag = -1;
            } else if (xsi < -1.) {
                double invd = mel_rsqrt((Xs - X1) * (Xs - X1) + (Ys - Y1) * (Ys - Y1));
                double xn = (Xs - X1) * invd, yn = (Ys - Y1) * invd;
                if (-yn * (xt + Xtanm) + xn * (yt + Ytanm) < 0.) { xn = -xn; yn = -yn; }
                p.xn = xn; p.yn = yn; p.xt = -yn; p.yt = xn;
                p.gap = xn * (Xs - X1) + yn * (Ys - Y1);
                p.N[0] = 0.; p.N[1] = 1.; p.N[2] = 0.; p.N[3] = 0.;
                p.xsi = -1.; p.flag = -2;
            } else if (xsi == 1.) {
                p.xn = yt; p.yn = -xt;
                p.gap = p.xn * (Xs - X2) + p.yn * (Ys - Y2);
                p.N[0] = 0.; p.N[1] = 0.; p.N[2] = 1.; p.N[3] = 0.;
                p.flag = 1;
            } else if (xsi > 1.) {
                double invd = mel_rsqrt((Xs - X2) * (Xs - X2) + (Ys - Y2) * (Ys - Y2));
                double xn = (Xs - X2) * invd, yn = (Ys - Y2) * invd;
                if (-yn * (xt + Xtanp) + xn * (yt + Ytanp) < 0.) { xn = -xn; yn = -yn; }
                p.xn = xn; p.yn = yn; p.xt = -yn; p.yt = xn;
                p.gap = xn * (Xs - X2) + yn * (Ys - Y2);
                p.N[0] = 0.; p.N[1] = 0.; p.N[2] = 1.; p.N[3] = 0.;
                p.xsi = 1.; p.flag = 2;
            }
        } else { p.flag = 3; p.xsi = 1.; }
    } else { p.flag = -3; p.xsi = -1.; }
}

// Closest_2_segment_self (Code/Tools.h:319-369): the flag always ends at -3
__device__ __forceinline__ void closest_self(double Xs, double Ys, double X1, double Y1, double X2, double Y2, Proj& p)
{
    double ilength = mel_rsqrt((X2 - X1) * (X2 - X1) + (Y2 - Y1) * (Y2 - Y1));
    double xt = (X2 - X1) * ilength, yt = (Y2 - Y1) * ilength;
    p.xt = xt; p.yt = yt;
    if (((Xs - X1) * xt + (Ys - Y1) * yt) * (xt * xt + yt * yt) >= 0.) {
        if (((Xs - X2) * xt + (Ys - Y2) * yt) * (xt * xt + yt * yt) <= 0.) {
            double xsi = -1. + 2. * ((X2 - X1) * (Xs - X1) + (Y2 - Y1) * (Ys - Y1)) * ilength * ilength;
            p.xsi = xsi;
            if ((xsi < 1.) && (xsi > -1.)) {
                p.xn = yt; p.yn = -xt;
                double Xc = 0.5 * (X1 + X2) + xsi * 0.5 * (X2 - X1);
                double Yc = 0.5 * (Y1 + Y2) + xsi * 0.5 * (Y2 - Y1);
                p.gap = p.xn * (Xs - Xc) + p.yn * (Ys - Yc);
                p.N[0] = 0.; p.N[1] = 0.5 * (1. - xsi); p.N[2] = 0.5 * (1. + xsi); p.N[3] = 0.;
            }
        } else p.xsi = 1.;
    } else p.xsi = -1.;
    p.flag = -3;
}

// Detect_Segment_Proximity (Code/Proximity.h:8-27)
__device__ __forceinline__ int detect_proximity(double Xs, double Ys, double X1, double Y1, double X2, double Y2, double dd)
{
    dd = dd * dd;
    if ((Xs - X1) * (Xs - X1) + (Ys - Y1) * (Ys - Y1) < dd) return 1;
    if ((Xs - X2) * (Xs - X2) + (Ys - Y2) * (Ys - Y2) < dd) return 1;
    double dx = X2 - X1, dy = Y2 - Y1;
    double a = dx * dx + dy * dy;
    double xsi = -1. + 2. * (dx * (Xs - X1) + dy * (Ys - Y1)) / a;
    if ((xsi < 1.) && (xsi > -1.)) {
        double b = dy * (Xs - 0.5 * (X1 + X2) - xsi * 0.5 * dx) - dx * (Ys - 0.5 * (Y1 + Y2) - xsi * 0.5 * dy);
        if (b * b < a * dd) return 1;
    }
    return 0;
}

// ---- contact laws (Code/Model.h:81-506) --------------------------------------------------
__device__ __forceinline__ void czm_branch(double kini, double Pnlim, double gapnres, double Pnres, double NTratio,
                                           double gapn, double& gapt, double& D, double& Pn, double& Pt,
                                           double gapnmax, double gaptmax, int which)
{
    if (which == 1) { gapnmax = gapn; gaptmax = gapnmax * NTratio; }
    else if (which == 2) { gaptmax = fabs(gapt); gapnmax = gaptmax / NTratio; }
    else {
        if (gapn / gapnmax > fabs(gapt) / gaptmax) { gapnmax = gapn; gaptmax = gapnmax * NTratio; }
        else { gaptmax = fabs(gapt); gapnmax = gaptmax / NTratio; }
    }
    D = (gapnmax - Pnlim / kini) / (gapnres - Pnlim / kini);
    double kmax = (Pnlim * (1. - D) + Pnres * D) / gapnmax;
    if (gapn < 0.) Pn = -kini * gapn; else Pn = -kmax * gapn;
    Pt = -kmax * gapt;
}

__device__ __forceinline__ void apply_law(int type, const double* P, double effm, double initial_length, double gapn,
                                          double vgapn, double& gapt, double vgapt, double& Pn, double& Pt,
                                          double& W, int& nb_internal, double* internal)
{
    switch (type) {
    case MEL_LAW_FRICTIONLESS: {
        double kn = P[0];
        if (gapn > 0.) Pn = 0.; else Pn = -kn * gapn;
        Pt = 0.; gapt = 0.;
    } break;
    case MEL_LAW_COHESION: {
        double kn = P[0], kt = P[1], gtang = P[2] * 0.5, gtens = P[3] * 0.5;
        Pn = -kn * gapn; Pt = -kt * gapt;
        if (Pn < -gtens) { Pn = 0.; Pt = 0.; gapt = 0.; }
        else if (fabs(Pt) > gtang) { if (gapt > 0.) Pt = -gtang; else Pt = gtang; gapt = -Pt / kt; }
    } break;
    case MEL_LAW_MOHR_COULOMB: {
        double kn = P[0], kt = P[1], fric = P[2], coh = P[3] * 0.5, tens = P[4] * 0.5;
        Pn = -kn * gapn; Pt = -kt * gapt;
        if (Pn < -tens) { Pn = 0.; Pt = 0.; gapt = 0.; }
        else if (fabs(Pt) > coh + fric * Pn) {
            if (gapt > 0.) Pt = -coh - fric * Pn; else Pt = coh + fric * Pn;
            gapt = -Pt / kt;
        }
    } break;
    case MEL_LAW_DAMPED_MOHR_COULOMB: {
        double kn = P[0], kt = P[1], fric = P[2], coh = P[3] * 0.5, tens = P[4] * 0.5, damp = P[5];
        double mass = effm, length = initial_length;
        Pn = 0.;
        if (gapn < 0.) { Pn = -damp * vgapn * 2. * sqrt(mass * kn / length); W += Pn * vgapn; }
        Pn -= kn * gapn;
        if (Pn < -tens) { Pn = 0.; Pt = 0.; gapt = 0.; }
        else {
            double Pt_damp = -damp * vgapt * 2. * sqrt(mass * kt / length);
            Pt = -kt * gapt + Pt_damp;
            if (fabs(Pt) > coh + fric * Pn) {
                if (gapt > 0.) Pt = -coh - fric * Pn; else Pt = coh + fric * Pn;
                gapt = -Pt / kt;
                W += Pt * vgapt;
            } else W += Pt_damp * vgapt;
        }
    } break;
    case MEL_LAW_TWO_SLOPES_MOHR_COULOMB: {
        double kn = P[0], kt = P[1], fric = P[2], coh = P[3] * 0.5, tens = P[4] * 0.5, rati = P[5];
        if (vgapn <= 0.) Pn = -kn * gapn; else Pn = -kn * gapn * rati;
        if (Pn < -tens) { Pn = 0.; Pt = 0.; gapt = 0.; }
        else {
            Pt = -kt * gapt;
            if (fabs(Pt) > coh + fric * Pn) {
                if (gapt > 0.) Pt = -coh - fric * Pn; else Pt = coh + fric * Pn;
                gapt = -Pt / kt;
            }
        }
    } break;
    case MEL_LAW_BONDED_MOHR_COULOMB: {
        double kn = P[0], kt = P[1], kbond = P[2], fricbond = P[3], cohbond = P[4] * 0.5, tensbond = P[5] * 0.5;
        double fricfree = P[6], cohfree = P[7] * 0.5, tensfree = P[8] * 0.5, damp = P[9];
        double mass = effm, length = initial_length;
        double D = internal[0];
        Pn = internal[1]; Pt = internal[2];
        if (nb_internal == 0) { D = 1.; nb_internal = 3; internal[0] = 1.; internal[1] = 0.; internal[2] = 0.; }
        if (D >= 1.) {
            Pn = -kn * gapn - damp * vgapn * 2. * sqrt(mass * kn / length);
            if (Pn < -tensfree) { Pn = 0.; Pt = 0.; gapt = 0.; }
            else Pt = -kt * gapt - damp * vgapt * 2. * sqrt(mass * kt / length);
            if (fabs(Pt) > cohfree + fricfree * Pn) {
                if (gapt > 0.) Pt = -cohfree - fricfree * Pn; else Pt = cohfree + fricfree * Pn;
                gapt = -Pt / kt;
            }
        } else {
            if (gapn < 0.) Pn = -kn * gapn - damp * vgapn * 2. * sqrt(mass * kn / length);
            else Pn = -kbond * gapn - damp * vgapn * 2. * sqrt(mass * kbond / length);
            Pt = -kt * gapt - damp * vgapt * 2. * sqrt(mass * kt / length);
            if (Pn < -tensbond) {
                D = 1.;
                if (Pn < -tensfree) { Pn = 0.; Pt = 0.; gapt = 0.; }
            }
            if (fabs(Pt) > cohbond + fricbond * Pn) {
                D = 1.;
                if (gapt > 0.) Pt = -cohfree - fricfree * Pn; else Pt = cohfree + fricfree * Pn;
                gapt = -Pt / kt;
            }
        }
        internal[0] = D; internal[1] = Pn; internal[2] = Pt;
    } break;
    case MEL_LAW_CZM_LINEAR: {
        double kini = P[0], Pnlim = P[1] * 0.5, gapnlim = P[2], Pnres = P[3] * 0.5, NTratio = P[4];
        double D = internal[0];
        if (nb_internal == 0) { D = 1.; nb_internal = 1; internal[0] = 1.; }
        if (D >= 1.) {
            Pn = -kini * gapn; Pt = -kini * gapt;
            if (Pn < -Pnres) { Pn = 0.; Pt = 0.; gapt = 0.; }
            else if (fabs(Pt) > Pnres * NTratio) {
                if (gapt > 0.) Pt = -Pnres * NTratio; else Pt = Pnres * NTratio;
                gapt = -Pt / kini;
            }
        } else {
            double gapnmax = Pnlim / kini * (1. - D) + gapnlim * D;
            double gaptmax = gapnmax * NTratio;
            if (gapn < gapnmax && fabs(gapt) < gaptmax) {
                double kmax = (Pnlim * (1. - D) + Pnres * D) / gapnmax;
                if (gapn < 0.) Pn = -kini * gapn; else Pn = -kmax * gapn;
                Pt = -kmax * gapt;
            } else if (gapn > gapnmax && fabs(gapt) < gaptmax) czm_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 1);
            else if (gapn < gapnmax && fabs(gapt) > gaptmax) czm_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 2);
            else if (gapn > gapnmax && fabs(gapt) > gaptmax) czm_branch(kini, Pnlim, gapnlim, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 3);
        }
        internal[0] = D;
    } break;
    case MEL_LAW_CZM_FATIGUE: {
        double kini = P[0], Pnlim = P[1] * 0.5, gapnres = P[2], Pnres = P[3] * 0.5, NTratio = P[4];
        double Pnfat = P[5], Raten = P[6], Ratet = P[7];
        double D = internal[0];
        Pn = internal[1]; Pt = internal[2];
        if (nb_internal == 0) { D = 1.; nb_internal = 3; internal[0] = 1.; internal[1] = 0.; internal[2] = 0.; }
        if (D < 1.) {
            double gapnmax = Pnlim / kini * (1. - D) + gapnres * D;
            double gaptmax = gapnmax * NTratio;
            if (gapn < gapnmax && fabs(gapt) < gaptmax) {
                double Pnm = Pn, Ptm = Pt;
                double kmax = (Pnlim * (1. - D) + Pnres * D) / gapnmax;
                if (gapn < 0.) Pn = -kini * gapn; else Pn = -kmax * gapn;
                Pt = -kmax * gapt;
                double Pnmax = Pnlim * (1. - D) + Pnres * D;
                if ((fabs(Pn) > Pnfat) && (fabs(Pn) > fabs(Pnm))) {
                    double Ratiopn = (fabs(Pn) - Pnfat) / (Pnmax - Pnfat);
                    double Deltapn = fabs(Pn) - fabs(Pnm);
                    D = D + Ratiopn * Raten * Deltapn;
                }
                if ((fabs(Pt) > NTratio * Pnfat) && (fabs(Pt) > fabs(Ptm))) {
                    double Ratiopt = (fabs(Pt) - Pnfat * NTratio) / (NTratio * (Pnmax - Pnfat));
                    double Deltapt = fabs(Pt) - fabs(Ptm);
                    D = D + Ratiopt * Ratet * Deltapt;
                }
            } else if (gapn > gapnmax && fabs(gapt) < gaptmax) czm_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 1);
            else if (gapn < gapnmax && fabs(gapt) > gaptmax) czm_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 2);
            else if (gapn > gapnmax && fabs(gapt) > gaptmax) czm_branch(kini, Pnlim, gapnres, Pnres, NTratio, gapn, gapt, D, Pn, Pt, gapnmax, gaptmax, 3);
        }
        if (D >= 1.) {
            D = 1.;
            Pn = -kini * gapn; Pt = -kini * gapt;
            if (Pn < -Pnres) { Pn = 0.; Pt = 0.; gapt = 0.; }
            else if (fabs(Pt) > Pnres * NTratio) {
                if (gapt > 0.) Pt = -Pnres * NTratio; else Pt = Pnres * NTratio;
                gapt = -Pt / kini;
            }
        }
        internal[0] = D; internal[1] = Pn; internal[2] = Pt;
    } break;
    default: Pn = 0.; Pt = 0.; break;
    }
}

} // namespace mel
