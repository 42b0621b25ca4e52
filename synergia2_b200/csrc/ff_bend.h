// Sector-bend units shared by the host runtime (design-particle propagation,
// host.cc) and the particle kernels (track_impl.cuh).  The reference runs
// the same FF_algorithm templates for its design particle on the host and for
// the bunch on the device (libFF/ff_sbend.h:221-339 and :568-660), so one
// definition here serves both sides.
//
// This header is included INSIDE a namespace (sb2::hostff, sb2::exact,
// sb2::fast); each includer defines SB2_FF (the function qualifiers) and
// SB2_FF_SINCOS (1: evaluate sin and cos of one angle together).
//
//   bend_unit       ff_algorithm.h:255-343  exact sector-bend body
//   bend_edge       ff_algorithm.h:366-450  thin face-angle edge
//   cf_kick5        ff_algorithm.h:596-800  combined-function kick up to the
//                   decapole, from the sector-magnet field potentials of
//                   Zolkin, Phys. Rev. Accel. Beams 20, 043501 (2017),
//                   table XII
//   bend_yoshida6   ff_algorithm.h:2194-2440 sixth-order Yoshida splitting
//                   of a combined-function bend (10 bend units, 9 kicks per
//                   step)
#ifndef SB2_FF
#error "define SB2_FF before including ff_bend.h"
#endif
#ifndef SB2_FF_SINCOS
#define SB2_FF_SINCOS 0
#endif

constexpr double kBendC = 299792458.0;

// Constants of the bend units that depend only on the reference momentum,
// the mass and the bend strength.  The reference evaluates them for every
// particle and unit (ff_algorithm.h:276-285); computed once with the same
// operations they are the same doubles: igib2 = (m/E0)^2 / (1 - (m/E0)^2)
// as ((1/gamma)(1/gamma))(1/beta)(1/beta), cs = (c c 1e-9) strength.
struct BendConst {
    double igib2, cs;
};
SB2_FF BendConst bend_const(double p_ref, double m, double strength)
{
    const double uni = 1.0;
    double p0 = p_ref;
    double E0 = sqrt(p0 * p0 + m * m);
    double igamma = m / E0;
    double ibeta = uni / sqrt(uni - igamma * igamma);
    double csq = kBendC * kBendC * 1e-9;
    BendConst k;
    k.igib2 = igamma * igamma * ibeta * ibeta;
    k.cs = csq * strength;
    return k;
}

// ff_algorithm.h:255-343: the particle moves on its circle through the
// rotation `phase` / translation `term` of one bend piece of angle -theta.
SB2_FF void bend_unit(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double theta,
                      const BendConst& bk, double p_ref, double m, double cdt_ref, double phase_r, double phase_i,
                      double term_r, double term_i)
{
    const double uni = 1.0;
    const double tc = kBendC;
    double p = p_ref * (dpop + uni);
    double E = sqrt(p * p + m * m);
    double psq = (dpop + uni) * (dpop + uni);
    double Ef = uni / sqrt(psq + bk.igib2);
    double beta1 = Ef * xp;
    double beta2 = Ef * yp;
    double beta3 = Ef * sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    double ui_r = 0.0, ui_i = x;
    double vui_r = tc * beta3, vui_i = tc * beta1;
    double iomega = E / bk.cs;
    double bi_r = -vui_i * iomega - ui_r;
    double bi_i = vui_r * iomega - ui_i;
    double bf_r = bi_r * phase_r - bi_i * phase_i + term_r;
    double bf_i = bi_r * phase_i + bi_i * phase_r + term_i;
    double rho = tc * sqrt(beta1 * beta1 + beta3 * beta3) * iomega;
    double dthmphi = asin(bi_r / rho) - asin(bf_r / rho);
#if SB2_FF_SINCOS
    double expf_r, expf_i;
    sincos(dthmphi, &expf_i, &expf_r);
#else
    double expf_r = cos(dthmphi);
    double expf_i = sin(dthmphi);
#endif
    double vuf_i = vui_r * expf_i + vui_i * expf_r;
    double uf_i = (ui_r + bi_r) * expf_i + (ui_i + bi_i) * expf_r - bf_i;
    double dtheta = dthmphi + theta;
    double ncdt = -tc * dtheta * iomega;
    x = uf_i;
    xp = vuf_i / (Ef * tc);
    y = y + beta2 * ncdt;
    cdt = cdt + ncdt - cdt_ref;
}

// ff_algorithm.h:366-450: the same circle through the pure rotation of a
// pole face of angle e (no translation, no reference-time subtraction).
SB2_FF void bend_edge(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double e,
                      double phase_r, double phase_i, const BendConst& bk, double p_ref, double m)
{
    const double uni = 1.0;
    const double tc = kBendC;
    double p = p_ref * (dpop + uni);
    double E = sqrt(p * p + m * m);
    double psq = (dpop + uni) * (dpop + uni);
    double Ef = uni / sqrt(psq + bk.igib2);
    double beta1 = Ef * xp;
    double beta2 = Ef * yp;
    double beta3 = Ef * sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    double ui_r = 0.0, ui_i = x;
    double vui_r = tc * beta3, vui_i = tc * beta1;
    double iomega = E / bk.cs;
    double bi_r = -vui_i * iomega - ui_r;
    double bi_i = vui_r * iomega - ui_i;
    double bf_r = bi_r * phase_r - bi_i * phase_i;
    double bf_i = bi_r * phase_i + bi_i * phase_r;
    double rho = tc * sqrt(beta1 * beta1 + beta3 * beta3) * iomega;
    double dthmphi = asin(bi_r / rho) - asin(bf_r / rho);
#if SB2_FF_SINCOS
    double expf_r, expf_i;
    sincos(dthmphi, &expf_i, &expf_r);
#else
    double expf_r = cos(dthmphi);
    double expf_i = sin(dthmphi);
#endif
    double vuf_i = vui_r * expf_i + vui_i * expf_r;
    double uf_i = (ui_r + bi_r) * expf_i + (ui_i + bi_i) * expf_r - bf_i;
    double dtheta = dthmphi + e;
    double ncdt = -tc * dtheta * iomega;
    x = uf_i;
    xp = vuf_i / (Ef * tc);
    y = y + beta2 * ncdt;
    cdt = cdt + ncdt;
}

// ((k rho) r0) r0 ... with n factors of r0: the multipole prefactor of
// order n+1 in ff_algorithm.h:736-800, in the reference's left-to-right
// product order.
SB2_FF double cf_prefactor(double k, double rho, double r0, int n)
{
    double t = k * rho;
    for (int i = 0; i < n; ++i) t = t * r0;
    return t;
}

// ff_algorithm.h:736-800 (thin_cf_kick_5): normal (kL[2j]) and skew
// (kL[2j+1]) components of orders 2..5 (quadrupole to decapole) in a
// sector magnet of radius r0.  rho = 1 + x/r0 and yb = y/r0 are the
// cylindrical coordinates; for each order the x kick is the ybar
// derivative and the y kick the rho derivative of the field potential
// (Zolkin's F functions).
SB2_FF void cf_kick5(double x, double& xp, double y, double& yp, double r0, const double* kL)
{
    const double rho = 1.0 + x / r0;
    const double yb = y / r0;
    const double r2m1 = rho * rho - 1.0;
    if (kL[0] || kL[1]) { // quadrupole
        const double fyn = log(rho), frn = -1.0 * (yb / rho);
        const double fys = yb, frs = 0.5 / rho * r2m1;
        xp = xp - cf_prefactor(kL[0], rho, r0, 1) * fyn + cf_prefactor(kL[1], rho, r0, 1) * fys;
        yp = yp - cf_prefactor(kL[0], rho, r0, 1) * frn + cf_prefactor(kL[1], rho, r0, 1) * frs;
    }
    if (kL[2] || kL[3]) { // sextupole
        const double lr = log(rho);
        const double fyn = 0.5 * (0.5 * r2m1 - yb * yb - lr);
        const double frn = -0.5 * (yb / rho) * r2m1;
        const double fys = yb * lr;
        const double frs = 0.5 / rho * (-0.5 * r2m1 - yb * yb + rho * rho * lr);
        xp = xp - cf_prefactor(kL[2], rho, r0, 2) * fyn + cf_prefactor(kL[3], rho, r0, 2) * fys;
        yp = yp - cf_prefactor(kL[2], rho, r0, 2) * frn + cf_prefactor(kL[3], rho, r0, 2) * frs;
    }
    if (kL[4] || kL[5]) { // octupole
        const double lr = log(rho);
        const double fyn = -0.25 * r2m1 + 0.5 * (0.5 * (rho * rho + 1.0) - yb * yb) * lr;
        const double frn = (-1.0 / 6.0) * (yb / rho) * (-1.5 * r2m1 - yb * yb + 3.0 * rho * rho * lr);
        const double fys = 0.5 * yb * (0.5 * r2m1 - yb * yb / 3.0 - lr);
        const double frs = 0.25 / rho * (0.25 * (rho * rho * rho * rho - 1.0) - r2m1 * yb * yb - rho * rho * lr);
        xp = xp - cf_prefactor(kL[4], rho, r0, 3) * fyn + cf_prefactor(kL[5], rho, r0, 3) * fys;
        yp = yp - cf_prefactor(kL[4], rho, r0, 3) * frn + cf_prefactor(kL[5], rho, r0, 3) * frs;
    }
    if (kL[6] || kL[7]) { // decapole
        const double lr = log(rho);
        const double r4 = rho * rho * rho * rho, y2 = yb * yb, y4 = yb * yb * yb * yb;
        const double fyn = 0.125 * (0.125 * (r4 + 4.0 * rho * rho - 5.0) - r2m1 * yb * yb + y4 -
                                    (0.5 + rho * rho - 2.0 * yb * yb) * lr);
        const double frn = (-1.0 / 12.0) * (yb / rho) * (r2m1 * (0.75 * (rho * rho + 1.0) - y2) - 3.0 * rho * rho * lr);
        const double fys = -0.25 * yb * r2m1 + (1.0 / 6.0) * yb * (1.5 * (rho * rho + 1.0) - y2) * lr;
        const double frs = 0.125 / rho *
                           (-0.625 * rho * rho * rho * rho + 0.5 * rho * rho + 0.125 + r2m1 * yb * yb + y4 / 3.0 +
                            (1.0 + 0.5 * rho * rho - 2.0 * yb * yb) * rho * rho * lr);
        xp = xp - cf_prefactor(kL[6], rho, r0, 4) * fyn + cf_prefactor(kL[7], rho, r0, 4) * fys;
        yp = yp - cf_prefactor(kL[6], rho, r0, 4) * frn + cf_prefactor(kL[7], rho, r0, 4) * frs;
    }
}

// Yoshida coefficients of the bend splitting (ff_algorithm.h:2013-2023):
// bend pieces c1..c4 of the step angle, kicks d1..d4 of the step strength.
constexpr double kBY6_C[4] = {0.79361246386112147294625603763, -0.206276584816439780698721319354,
                              -0.118008867881292655922412133144, 0.236949573653050744373598734219};
constexpr double kBY6_D[4] = {1.58722492772224294589251207526, -1.99977809735512250728995471397,
                              -1.82324266348482825773733634154, 2.29714181079092974648453380998};

// ff_algorithm.h:2194-2440: `steps` steps of
//   B1 K1 B2 K2 B2 K1 B3 K3 B4 K4 B4 K3 B3 K1 B2 K2 B2 K1 B1
// where Bj is a bend piece of angle c_j * step angle (dphi[j], phase[2j..],
// term[2j..]) with the reference time sub_ref_cdt, and Kj = cf_kick5 with
// the strengths kj (8 values each, the d_j-scaled step strengths).
SB2_FF void bend_yoshida6(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double pref,
                          double m, double sub_ref_cdt, const double* k1, const double* k2, const double* k3,
                          const double* k4, const double* dphi, const double* phase, const double* term, double r0,
                          const BendConst& bk, int steps)
{
    for (int s = 0; s < steps; ++s) {
#define SB2_BY6_B(j)                                                                                                  \
    bend_unit(x, xp, y, yp, cdt, dpop, dphi[j], bk, pref, m, sub_ref_cdt, phase[2 * (j)], phase[2 * (j) + 1],         \
              term[2 * (j)], term[2 * (j) + 1])
        SB2_BY6_B(0); cf_kick5(x, xp, y, yp, r0, k1);
        SB2_BY6_B(1); cf_kick5(x, xp, y, yp, r0, k2);
        SB2_BY6_B(1); cf_kick5(x, xp, y, yp, r0, k1);
        SB2_BY6_B(2); cf_kick5(x, xp, y, yp, r0, k3);
        SB2_BY6_B(3); cf_kick5(x, xp, y, yp, r0, k4);
        SB2_BY6_B(3); cf_kick5(x, xp, y, yp, r0, k3);
        SB2_BY6_B(2); cf_kick5(x, xp, y, yp, r0, k1);
        SB2_BY6_B(1); cf_kick5(x, xp, y, yp, r0, k2);
        SB2_BY6_B(1); cf_kick5(x, xp, y, yp, r0, k1);
        SB2_BY6_B(0);
#undef SB2_BY6_B
    }
}
