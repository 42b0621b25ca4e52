// Particle-pass kernels for sm_100a, compiled twice from this file:
//
//   track.cu       SB2_FAST_MAPS 0, namespace sb2::exact, --fmad=false: every
//                  a*b+c keeps two IEEE roundings and sqrt/div are
//                  IEEE-correct, so the maps reproduce the reference's FP64
//                  arithmetic (libFF/ff_algorithm.h) operation for operation
//                  (the plain FP64 drop-in);
//   track_fast.cu  SB2_FAST_MAPS 1, namespace sb2::fast, --fmad=true: the
//                  same FP64 maps with fused multiply-adds, the exact drift's
//                  two square roots and two divisions folded into one
//                  reciprocal square root (cdt advances by L (1+dpop) / p_z
//                  / beta, algebraically the same quantity) and the particle's
//                  1/beta hoisted out of the Yoshida sub-steps; used by the
//                  mixed-precision path, whose tolerances are set against the
//                  FP64 path and are far above these last-bit differences.
//
// One launch runs a whole sequence of particle-local operations (element
// slice maps, apertures, the space-charge kick, the spatial-moment sums) on
// each particle while its six coordinates stay in registers: the column-major
// N x 7 FP64 array is read once and written once per pass, coalesced (one
// particle per thread, 32 consecutive particles per warp per column).
#pragma once
#include <cuda_runtime.h>
#include <climits>
#include <cstdint>
#include <cstdlib>

#include "sb2_kernels.h"

#ifndef SB2_FAST_MAPS
#error "define SB2_FAST_MAPS (0 or 1) and SB2_TRACK_NS before including track_impl.cuh"
#endif

namespace sb2 {
namespace SB2_TRACK_NS {

constexpr double kC = 299792458.0;

// ---------------------------------------------------------------------------
// ff_algorithm.h units, same operation order as the reference
// ---------------------------------------------------------------------------
__device__ __forceinline__ void drift_unit(double& x, double xp, double& y, double yp, double& cdt,
                                           double dpop, double length, double reference_momentum,
                                           double m, double reference_cdt)
{ // ff_algorithm.h:47-79
    const double uni = 1.0;
    const double sig = (double)((0.0 < length) - (length < 0.0));
    double dp = dpop + uni;
    double inv_npz = uni / sqrt(dp * dp - xp * xp - yp * yp);
    double lxpr = xp * length * inv_npz;
    double lypr = yp * length * inv_npz;
    double D2 = lxpr * lxpr + length * length + lypr * lypr;
    double p = dp * reference_momentum;
    double E2 = p * p + m * m;
    double ibeta2 = E2 / (p * p);
    x = x + lxpr;
    y = y + lypr;
    cdt = cdt + sig * sqrt(D2 * ibeta2) - reference_cdt;
}

#if SB2_FAST_MAPS
// 1/beta of a particle of relative momentum dp = 1 + dpop: sqrt(1 + m^2 /
// (dp pref)^2); constant while dpop is (through every map of a pass but the
// space-charge kick).
__device__ __forceinline__ double inv_beta(double dp, double pref, double m)
{
    const double r = m / (dp * pref);
    return sqrt(1.0 + r * r);
}

// drift_unit with the path length folded: with p_z = sqrt(dp^2 - xp^2 -
// yp^2), the exact drift's sqrt(D2 / beta^2) is |L| dp / p_z / beta, so the
// whole drift costs one reciprocal square root.
__device__ __forceinline__ void drift_unit_ib(double& x, double xp, double& y, double yp, double& cdt, double dp,
                                              double length, double ib, double reference_cdt)
{
    const double inv_npz = rsqrt(dp * dp - xp * xp - yp * yp);
    const double lz = length * inv_npz;
    x = x + xp * lz;
    y = y + yp * lz;
    cdt = cdt + lz * dp * ib - reference_cdt;
}
#endif

__device__ __forceinline__ void thin_quadrupole_unit(double x, double& xp, double y, double& yp,
                                                     double k0, double k1)
{ // ff_algorithm.h:929-936
    xp = xp - k0 * x + k1 * y;
    yp = yp + k0 * y + k1 * x;
}

__device__ __forceinline__ void thin_sextupole_unit(double x, double& xp, double y, double& yp,
                                                    double k0, double k1)
{ // ff_algorithm.h:940-947
    xp = xp - 0.5 * k0 * (x * x - y * y) + k1 * x * y;
    yp = yp + k0 * x * y + 0.5 * k1 * (x * x - y * y);
}

__device__ __forceinline__ void thin_octupole_unit(double x, double& xp, double y, double& yp,
                                                   double k0, double k1)
{ // ff_algorithm.h:951-963
    const double n1 = 0.5, n2 = 1.0 / 3.0;
    xp = xp - n1 * k0 * (x * x * x * n2 - x * y * y) + n1 * k1 * (x * x * y - y * y * y * n2);
    yp = yp - n1 * k0 * (y * y * y * n2 - x * x * y) + n1 * k1 * (x * x * x * n2 - x * y * y);
}

__device__ __forceinline__ double factorial_d(int n)
{ // ff_algorithm.h:1108-1117
    if (n == 0) return 1.0;
    double r = 1;
    for (int i = 1; i <= n; ++i) r *= i;
    return r;
}

__device__ __forceinline__ double qpow_d(double x, int i)
{ // utils/kokkos_types.h:89-95
    double r = 1;
    while (i--) r = r * x;
    return r;
}

__device__ __noinline__ void thin_magnet_unit(double x, double& xp, double y, double& yp, double kl0, double kl1,
                                              int n)
{ // ff_algorithm.h:1122-1168
    for (int k = 0; k < n; k += 4)
        xp = xp - (kl0 * (n - k)) * qpow_d(x, n - k - 1) * qpow_d(y, k) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 2; k < n; k += 4)
        xp = xp + (kl0 * (n - k)) * qpow_d(x, n - k - 1) * qpow_d(y, k) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 1; k < n; k += 4)
        xp = xp + (kl1 * (n - k)) * qpow_d(x, n - k - 1) * qpow_d(y, k) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 3; k < n; k += 4)
        xp = xp - (kl1 * (n - k)) * qpow_d(x, n - k - 1) * qpow_d(y, k) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 4; k <= n; k += 4)
        yp = yp - (kl0 * k) * qpow_d(x, n - k) * qpow_d(y, k - 1) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 2; k <= n; k += 4)
        yp = yp + (kl0 * k) * qpow_d(x, n - k) * qpow_d(y, k - 1) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 1; k <= n; k += 4)
        yp = yp + (kl1 * k) * qpow_d(x, n - k) * qpow_d(y, k - 1) / (factorial_d(n - k) * factorial_d(k));
    for (int k = 3; k <= n; k += 4)
        yp = yp - (kl1 * k) * qpow_d(x, n - k) * qpow_d(y, k - 1) / (factorial_d(n - k) * factorial_d(k));
}

// cf_kick ff_quadrupole.h:22-35
__device__ __noinline__ void quad_cf_kick(double x, double& xp, double y, double& yp, const double* kL)
{
    thin_quadrupole_unit(x, xp, y, yp, kL[0], kL[1]);
    if (kL[2] || kL[3]) thin_quadrupole_unit(x, xp, y, yp, kL[2], kL[3]);
    if (kL[4] || kL[5]) thin_sextupole_unit(x, xp, y, yp, kL[4], kL[5]);
    if (kL[6] || kL[7]) thin_octupole_unit(x, xp, y, yp, kL[6], kL[7]);
    if (kL[8] || kL[9]) thin_magnet_unit(x, xp, y, yp, kL[8], kL[9], 5);
    if (kL[10] || kL[11]) thin_magnet_unit(x, xp, y, yp, kL[10], kL[11], 6);
    if (kL[12] || kL[13]) thin_magnet_unit(x, xp, y, yp, kL[12], kL[13], 7);
    if (kL[14] || kL[15]) thin_magnet_unit(x, xp, y, yp, kL[14], kL[15], 8);
}

// drift_unit with dp = dpop + 1 and ibeta2 = E^2 / p^2 of the particle given
// (same operations, same results; for loops in which dpop is constant)
__device__ __forceinline__ void drift_unit_ibeta2(double& x, double xp, double& y, double yp, double& cdt,
                                                  double dp, double length, double ibeta2, double reference_cdt)
{
    const double uni = 1.0;
    const double sig = (double)((0.0 < length) - (length < 0.0));
    double inv_npz = uni / sqrt(dp * dp - xp * xp - yp * yp);
    double lxpr = xp * length * inv_npz;
    double lypr = yp * length * inv_npz;
    double D2 = lxpr * lxpr + length * length + lypr * lypr;
    x = x + lxpr;
    y = y + lypr;
    cdt = cdt + sig * sqrt(D2 * ibeta2) - reference_cdt;
}

// slot_unit ff_algorithm.h:83-129
__device__ __forceinline__ void slot_unit(double& x, double& xp, double& y, double& yp, double& cdt,
                                          double& dpop, double ct, double st, double pref, double m)
{
    const double uni = 1.0;
    double zp = sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    double p = (dpop + uni) * pref;
    double e = sqrt(p * p + m * m);
    double b0 = xp * pref / e;
    double b1 = yp * pref / e;
    double b2 = zp * pref / e;
    double bp = st * b0 + ct * b2;
    double tau = -x * st / bp;
    double r0 = x + tau * b0;
    double r1 = y + tau * b1;
    double r2 = tau * b2;
    x = r0 * ct - r2 * st;
    y = r1;
    cdt = cdt + tau;
    xp = xp * ct - zp * st;
}

// solenoid_unit ff_algorithm.h:1317-1356 in the reference's argument order
// (its caller passes ks*L as `ks` and ks as `ksl`), with the edge kicks
// :1358-1372 (flags: 1 entry edge, 2 exit edge); out of line: rare op
__device__ __noinline__ void solenoid_op(double& x, double& xp, double& y, double& yp, double& cdt, double dpop,
                                         const double* d, int flags)
{
    const double ks = d[0], ksl = d[1], length = d[2], ref_p = d[3], mass = d[4], ref_cdt = d[5], kse = d[6];
    if (flags & 1) {
        xp = xp + kse * y;
        yp = yp - kse * x;
    }
    const double uni = 1.0;
    double p2 = (uni + dpop) * (uni + dpop);
    double zp = sqrt(p2 - xp * xp - yp * yp);
    double dtheta = ksl / zp;
#if SB2_FAST_MAPS
    double sn, cs;
    sincos(dtheta, &sn, &cs);
#else
    double sn = sin(dtheta);
    double cs = cos(dtheta);
#endif
    double xpi = xp, ypi = yp;
    xp = cs * xpi + sn * ypi;
    yp = (-sn) * xpi + cs * ypi;
    cs = cs - uni;
    x = x + (cs * (-ypi) + sn * xpi) / ks;
    y = y + ((-sn) * (-ypi) + cs * xpi) / ks;
    double en = sqrt(p2 * ref_p * ref_p + mass * mass);
    double duration = length / (zp * ref_p / en);
    cdt = cdt + duration - ref_cdt;
    if (flags & 2) {
        xp = xp - kse * y;
        yp = yp + kse * x;
    }
}

// PropThinRFCavity / PropRFCavity ff_rfcavity.h:23-132 with
// thin_rfcavity_unit ff_algorithm.h:1025-1082 (d: half length, pref,
// mass, ref_cdt_1, ref_cdt_2, w_rf, volt, phi_s, new pref, mhp[12]; steps =
// number of harmonics; flags 1: thin)
__device__ __noinline__ void rfcavity_op(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop,
                                         const double* d, int nh, int flags)
{
    const double half = d[0], pref = d[1], m = d[2], w_rf = d[5], volt = d[6], phi_s = d[7], new_p = d[8];
    const double* mhp = d + 9;
    const bool thin = flags & 1;
    if (!thin) drift_unit(x, xp, y, yp, cdt, dpop, half, pref, m, d[3]);
    if (volt != 0.0) {
        const double anh_phase = 0.0;
        double phase_slip_argument = (cdt * (w_rf / kC)) + anh_phase;
        double strength_factor = 0.0;
        for (int i = 0; i < nh; ++i)
            strength_factor = strength_factor + mhp[i * 3 + 1] * sin(mhp[i * 3] * (phi_s + phase_slip_argument) +
                                                                     mhp[i * 3 + 2]);
        double p = pref * (dpop + 1.0);
        double E = sqrt(p * p + m * m);
        E = E + volt * strength_factor;
        xp = xp * (pref / new_p);
        yp = yp * (pref / new_p);
        dpop = sqrt((E - m) * (E + m)) / new_p - 1.0;
    }
    if (!thin) drift_unit(x, xp, y, yp, cdt, dpop, half, pref, m, d[4]);
}

// bend_unit, bend_edge, cf_kick5, bend_yoshida6 (ff_algorithm.h), shared
// with the host's design-particle propagation
#define SB2_FF __device__ __forceinline__
#define SB2_FF_SINCOS SB2_FAST_MAPS
#include "ff_bend.h"
#undef SB2_FF
#undef SB2_FF_SINCOS

// PropSbendSimd ff_sbend.h:127-215 for one particle (out of line: rare op)
__device__ __noinline__ void sbend_op(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop,
                                      const double* d, int flags)
{
    if (flags & 1) {
        slot_unit(x, xp, y, yp, cdt, dpop, d[0], d[1], d[14], d[15]);
        yp = yp - d[4] * y; // edge_unit ff_algorithm.h:139-148
        xp = xp + d[5] * y;
    }
    const BendConst bk{d[17], d[18]};
    bend_unit(x, xp, y, yp, cdt, dpop, d[8], bk, d[14], d[15], d[16], d[9], d[10], d[11], d[12]);
    if (flags & 2) {
        yp = yp - d[6] * y;
        xp = xp + d[7] * y;
        slot_unit(x, xp, y, yp, cdt, dpop, d[2], d[3], d[14], d[15]);
    }
}

#define SB2_FF __device__ __forceinline__
#include "ff_nllens.h"
#undef SB2_FF
// dipedge_unit ff_algorithm.h:1284-1316 (MAD-X tmfrng): edge focusing
// d[0] = re_2_1, d[1] = re_4_3 and second-order terms d[2..11]
__device__ __noinline__ void dipedge_op(double& x, double& xp, double& y, double& yp, const double* d)
{
    const double* te = d + 2;
    double nx, nxp, ny, nyp;
    nxp = xp + d[0] * x;
    nyp = yp + d[1] * y;
    nx = x + te[0] * x * x + te[1] * y * y;
    nxp = nxp + te[2] * x * x + te[4] * y * y + te[3] * x * xp * 2.0 + te[5] * y * yp * 2.0;
    ny = y + te[6] * x * y * 2.0;
    nyp = nyp + te[7] * x * y * 2.0 + te[8] * x * yp * 2.0 + te[9] * y * xp * 2.0;
    x = nx;
    xp = nxp;
    y = ny;
    yp = nyp;
}

// matrix_unit ff_algorithm.h:2439-2700: kick + linear map + optional
// second-order tensor, summed in the reference's order
__device__ __noinline__ void matrix_op(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop,
                                       const double* d, int flags)
{
    const double v[6] = {x, xp, y, yp, cdt, dpop};
    double nv[6];
    for (int i = 0; i < 6; ++i) {
        double a = d[i];
        for (int j = 0; j < 6; ++j) a = a + d[6 + i * 6 + j] * v[j];
        nv[i] = a;
    }
    if (flags & 1) {
        uint64_t bits;
        memcpy(&bits, &d[42], sizeof(bits));
        const double* tm = reinterpret_cast<const double*>((uintptr_t)bits);
        for (int i = 0; i < 6; ++i) {
            double a = nv[i];
            for (int j = 0; j < 6; ++j)
                for (int l = 0; l < 6; ++l) a = a + __ldg(&tm[(i * 6 + j) * 6 + l]) * v[j] * v[l];
            nv[i] = a;
        }
    }
    x = nv[0];
    xp = nv[1];
    y = nv[2];
    yp = nv[3];
    cdt = nv[4];
    dpop = nv[5];
}

// FF_nllens thin kick (out of line: rare op with atan and log)
__device__ __noinline__ void nllens_op(double x, double& xp, double y, double& yp, const double* d)
{
    nllens_unit(x, xp, y, yp, d + 2);
}

// PropSbendCF ff_sbend.h:221-339 for one particle (combined-function or
// a_n/b_n multipole bend; out of line: rare op).  d: 0 ce1 1 se1 2 ce2
// 3 se2 4 us_kx 5 us_ky 6 ds_kx 7 ds_ky 8 e1 9 e2 10-11 entry-face phase
// 12-13 exit-face phase 14 strength 15 pref_b 16 m_b 17 substep ref_cdt
// 18 r0 19-22 dphi[4] 23-30 phase[4] 31-38 term[4] 39-70 k1..k4 (8 each);
// steps in `steps`, flags bit0 entry edge, bit1 exit edge
__device__ __noinline__ void sbend_cf_op(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop,
                                         const double* d, int steps, int flags)
{
    const BendConst bk{d[71], d[72]};
    if (flags & 1) {
        slot_unit(x, xp, y, yp, cdt, dpop, d[0], d[1], d[15], d[16]);
        yp = yp - d[4] * y; // edge_unit ff_algorithm.h:139-148
        xp = xp + d[5] * y;
        bend_edge(x, xp, y, yp, cdt, dpop, d[8], d[10], d[11], bk, d[15], d[16]);
    }
    bend_yoshida6(x, xp, y, yp, cdt, dpop, d[15], d[16], d[17], d + 39, d + 47, d + 55, d + 63, d + 19, d + 23,
                  d + 31, d[18], bk, steps);
    if (flags & 2) {
        bend_edge(x, xp, y, yp, cdt, dpop, d[9], d[12], d[13], bk, d[15], d[16]);
        yp = yp - d[6] * y;
        xp = xp + d[7] * y;
        slot_unit(x, xp, y, yp, cdt, dpop, d[2], d[3], d[15], d[16]);
    }
}

// yoshida6 ff_algorithm.h:1834-2008 with the drift lengths c_i*step_length,
// the 0.1*step_ref_cdt substep and the d_i-scaled strengths precomputed on
// the host (identical doubles).  kind selects the kick function.
template <int KIND>
__device__ __forceinline__ void yoshida6_op(double& x, double& xp, double& y, double& yp, double& cdt,
                                            double dpop, const MapOp& op)
{
    const double pref = op.d[2], m = op.d[3], sub = op.d[4];
    const double l1 = op.d[5], l2 = op.d[6], l3 = op.d[7], l4 = op.d[8];
    const double* k = op.d + 9;
    constexpr int KS = (KIND == OP_QUAD_CF) ? 16 : 2; // stride between k1..k4
    auto kick = [&](const double* kk) {
        if (KIND == OP_QUAD)
            thin_quadrupole_unit(x, xp, y, yp, kk[0], kk[1]);
        else if (KIND == OP_SEXT_YOSHIDA)
            thin_sextupole_unit(x, xp, y, yp, kk[0], kk[1]);
        else if (KIND == OP_OCT_YOSHIDA)
            thin_octupole_unit(x, xp, y, yp, kk[0], kk[1]);
        else if (KIND == OP_KICK_YOSHIDA) {
            xp = xp + kk[0]; // thin_kicker_unit ff_algorithm.h:994-1000
            yp = yp + kk[1];
        } else {
            double cxp = xp, cyp = yp; // copies: see on_copies
            quad_cf_kick(x, cxp, y, cyp, kk);
            xp = cxp;
            yp = cyp;
        }
    };
    const double* k1 = k;
    const double* k2 = k + KS;
    const double* k3 = k + 2 * KS;
    const double* k4 = k + 3 * KS;
#if SB2_FAST_MAPS
    const double dp = dpop + 1.0;
    const double ib = inv_beta(dp, pref, m);
    auto drift_unit = [&](double& x_, double xp_, double& y_, double yp_, double& cdt_, double, double len, double,
                          double, double sub_) { drift_unit_ib(x_, xp_, y_, yp_, cdt_, dp, len, ib, sub_); };
#else
    // The kicks leave dpop alone, so the drift's 1/beta^2 (E^2 / p^2, one
    // IEEE division) is the same double in all 10 * steps drifts: computed
    // once, with the operations of drift_unit, the results are unchanged.
    const double dp = dpop + 1.0;
    const double pp = dp * pref;
    const double ibeta2 = (pp * pp + m * m) / (pp * pp);
    auto drift_unit = [&](double& x_, double xp_, double& y_, double yp_, double& cdt_, double, double len, double,
                          double, double sub_) { drift_unit_ibeta2(x_, xp_, y_, yp_, cdt_, dp, len, ibeta2, sub_); };
#endif
    for (int i = 0; i < op.steps; ++i) {
        drift_unit(x, xp, y, yp, cdt, dpop, l1, pref, m, sub); kick(k1);
        drift_unit(x, xp, y, yp, cdt, dpop, l2, pref, m, sub); kick(k2);
        drift_unit(x, xp, y, yp, cdt, dpop, l2, pref, m, sub); kick(k1);
        drift_unit(x, xp, y, yp, cdt, dpop, l3, pref, m, sub); kick(k3);
        drift_unit(x, xp, y, yp, cdt, dpop, l4, pref, m, sub); kick(k4);
        drift_unit(x, xp, y, yp, cdt, dpop, l4, pref, m, sub); kick(k3);
        drift_unit(x, xp, y, yp, cdt, dpop, l3, pref, m, sub); kick(k1);
        drift_unit(x, xp, y, yp, cdt, dpop, l2, pref, m, sub); kick(k2);
        drift_unit(x, xp, y, yp, cdt, dpop, l2, pref, m, sub); kick(k1);
        drift_unit(x, xp, y, yp, cdt, dpop, l1, pref, m, sub);
    }
}

// collective/utils.h:9-18
__device__ __forceinline__ void leftmost(double pos, double left, double inv, int& idx, double& off)
{
    double s = (pos - left) * inv - 0.5;
    idx = (int)floor(s);
    off = s - idx;
}


constexpr int kTrackThreads = 256;

// Two compiled variants: FULL runs every op kind; LIGHT omits the Yoshida
// integrators and the sector bend so that passes made only of drifts, thin
// kicks, apertures, the space-charge kick and the moment sums fit in fewer
// registers and run at higher occupancy.
// TRACK_QUAD: the light ops plus the pure-quadrupole Yoshida integrator and
// the (out-of-line) pure-dipole sector bend (the FODO and ring passes), a
// smaller body than the variant that inlines every integrator: 3 CTAs/SM (80 registers, a 20-byte spill) measured 8%
// faster on the FODO quadrupole passes than TRACK_FULL_WIDE at 2 CTAs/SM.
enum TrackVariant { TRACK_LIGHT = 0, TRACK_FULL = 1, TRACK_FULL_WIDE = 2, TRACK_QUAD = 3 };

// CTAs per SM of the prefetching light variants: on the C1 passes 4 (64
// registers) measured 8% faster than 3 (80 registers); 5 was 35% slower.
#ifndef SB2_LIGHT_OCC
#define SB2_LIGHT_OCC 4
#endif
#ifndef SB2_QUAD_OCC
#define SB2_QUAD_OCC 3
#endif
// Minimum resident CTAs per SM for each variant (register budget).
template <int V, int PPT = 1>
struct TrackOcc {
    static constexpr int value =
        V == TRACK_LIGHT ? 3 : (V == TRACK_FULL ? 3 : (V == TRACK_QUAD ? (PPT == 1 ? SB2_QUAD_OCC : 2) : 2));
};

// Runs an out-of-line op on copies of the six coordinates.  A coordinate
// whose address reaches a call that is not inlined is given a stack slot for
// the whole pass, and every op then reloads it from local memory (through
// L1); on copies only the copies live in the stack frame, and only while
// the op runs.
template <class F>
__device__ __forceinline__ void on_copies(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop,
                                          F&& f)
{
    double c0 = x, c1 = xp, c2 = y, c3 = yp, c4 = cdt, c5 = dpop;
    f(c0, c1, c2, c3, c4, c5);
    x = c0;
    xp = c1;
    y = c2;
    yp = c3;
    cdt = c4;
    dpop = c5;
}

// One particle in registers during a pass.
struct Part {
    double x, xp, y, yp, cdt, dpop;
    bool alive;
    int disc;
    int64_t idx; // position in the bunch arrays (loss records read the id there)
};

// Field corners for the kick.  Corner c of a cell is read as (ex, ey, ez);
// FP64: two double2 per cell {ex, ey | ez, 0}; mixed: one float4.
struct Corner {
    double x, y, z;
};
// The field of the cell (ix, iy, iz): one base address and the x, y, z
// strides of the {ex, ey, ez, pad} cells, so the 8 corner loads share one
// 64-bit index.  FP64 cells are 32 bytes (one 256-bit load each; the
// cudaMalloc'd field is 32-byte aligned), FP32 cells 16 bytes.
template <typename T>
struct CellField;
template <>
struct CellField<double> {
    const double* b;
    int64_t sy, sz;
    __device__ __forceinline__ CellField(const TrackParams& p, int ix, int iy, int iz)
        : b(reinterpret_cast<const double*>(p.efield) + 4 * (((int64_t)iz * p.gy + iy) * p.gx + ix)), sy(4 * (int64_t)p.gx),
          sz(4 * (int64_t)p.gx * p.gy)
    {
    }
    // corner c (x fastest, then y, then z)
    __device__ __forceinline__ void corner(int c, Corner& v) const
    {
        const double* a = b + ((c & 1) ? 4 : 0) + (((c >> 1) & 1) ? sy : 0) + ((c >> 2) ? sz : 0);
        double pad;
        asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v.x), "=d"(v.y), "=d"(v.z), "=d"(pad) : "l"(a));
    }
};
template <>
struct CellField<float> {
    const float4* b;
    int64_t sy, sz;
    __device__ __forceinline__ CellField(const TrackParams& p, int ix, int iy, int iz)
        : b(p.efield32 + (((int64_t)iz * p.gy + iy) * p.gx + ix)), sy(p.gx), sz((int64_t)p.gx * p.gy)
    {
    }
    __device__ __forceinline__ void corner(int c, Corner& v) const
    {
        const float4 f = __ldg(b + ((c & 1) ? 1 : 0) + (((c >> 1) & 1) ? sy : 0) + ((c >> 2) ? sz : 0));
        v.x = f.x;
        v.y = f.y;
        v.z = f.z;
    }
};

// zyx::alg_kicker space_charge_3d_kernels.h:91-215: trilinear interpolation
// of E (FP64 or FP32 cells, T) at the particle and the kick of xp, yp, dpop.
template <typename T>
__device__ __forceinline__ void sc_kick(const TrackParams& p, Part& P, double pref, double m)
{
    const ScState& sc = *p.sc;
    if (!sc.valid) return;
    int ix, iy, iz;
    double ox, oy, oz;
    leftmost(P.x, sc.left[0], sc.ih[0], ix, ox);
    leftmost(P.y, sc.left[1], sc.ih[1], iy, oy);
    leftmost(P.cdt, sc.left[2], sc.ih[2], iz, oz);
    const int gx = p.gx, gy = p.gy, gz = p.gz;
    if (!((ix >= 0 && ix < gx - 1) && (iy >= 0 && iy < gy - 1) && (iz >= 0 && iz < gz - 1))) return;
    const double aox = 1.0 - ox, aoy = 1.0 - oy, aoz = 1.0 - oz;
    // each component sums the corners in the reference's order (x fastest,
    // then y, then z), one corner at a time
    const double wz[2] = {aoz, oz}, wy[2] = {aoy, oy}, wx[2] = {aox, ox};
    double vx = 0.0, vy = 0.0, vz = 0.0;
    const CellField<T> field(p, ix, iy, iz);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        Corner f;
        field.corner(c, f);
        const double w = wz[c >> 2] * wy[(c >> 1) & 1] * wx[c & 1];
        if (c == 0) {
            vz = w * f.z;
            vy = w * f.y;
            vx = w * f.x;
        } else {
            vz += w * f.z;
            vy += w * f.y;
            vx += w * f.x;
        }
    }
    const double factor = sc.factor;
    double pp = pref + P.dpop * pref;
    double Eoc_i = sqrt(pp * pp + m * m);
    double Eoc_f = Eoc_i + factor * (-pref) * vz;
    double ddp = (sqrt(Eoc_f * Eoc_f - m * m) - sqrt(Eoc_i * Eoc_i - m * m)) / pref;
    P.dpop += ddp;
    P.yp += factor * vy;
    P.xp += factor * vx;
}

// Applies one op to one particle (apertures, moments and maps).
template <int VARIANT>
__device__ __forceinline__ void apply_op(const TrackParams& p, const MapOp& op, Part& P, int* s_counts,
                                         double* s_mom_col)
{
    constexpr bool kQuad = VARIANT != TRACK_LIGHT;                       // pure-quad Yoshida
    constexpr bool kFull = VARIANT == TRACK_FULL || VARIANT == TRACK_FULL_WIDE; // every integrator
    const int kind = op.kind;
    double& x = P.x;
    double& xp = P.xp;
    double& y = P.y;
    double& yp = P.yp;
    double& cdt = P.cdt;
    double& dpop = P.dpop;
    if (kind >= OP_AP_FINITE && kind <= OP_AP_RECTANGULAR) {
        // discard_applier bunch_particles.h:484-503: discards(i) is reset by
        // every aperture, then set if this one discards.
        P.disc = 0;
        if (P.alive) {
            bool d;
            if (kind == OP_AP_FINITE) {
                if (!isfinite(x) || !isfinite(xp) || !isfinite(y) || !isfinite(yp) || !isfinite(cdt) ||
                    !isfinite(dpop))
                    d = true;
                else {
                    double pt = 1.0 + dpop;
                    d = pt * pt - xp * xp - yp * yp < 0.0;
                }
            } else if (kind == OP_AP_CIRCULAR) {
                double xr = x - op.d[1], yr = y - op.d[2];
                d = (xr * xr + yr * yr) > op.d[0];
            } else if (kind == OP_AP_ELLIPTICAL) {
                double xr = x - op.d[2], yr = y - op.d[3];
                d = (xr * xr / op.d[0] + yr * yr / op.d[1]) > 1.0;
            } else {
                double xr = x - op.d[2], yr = y - op.d[3];
                d = (fabs(xr) > 0.5 * op.d[0]) || (fabs(yr) > 0.5 * op.d[1]);
            }
            if (d) {
                P.disc = 1;
                P.alive = false;
                atomicAdd(&s_counts[op.slot - p.slot_base], 1);
                if (p.loss_buf) { // Diagnostics_loss: coordinates at the aperture
                    const int r = atomicAdd(p.loss_count, 1);
                    if (r < p.loss_cap) {
                        double* rec = p.loss_buf + (int64_t)r * 8;
                        rec[0] = x;
                        rec[1] = xp;
                        rec[2] = y;
                        rec[3] = yp;
                        rec[4] = cdt;
                        rec[5] = dpop;
                        rec[6] = p.parts[P.idx + 6 * p.stride];
                        rec[7] = op.d[10]; // aperture tag (host table: repetition, s, s_n)
                    }
                }
            }
        }
        return;
    }
    if (kind == OP_MOMENTS) {
        if (P.alive) {
            s_mom_col[0 * kTrackThreads] += x;
            s_mom_col[1 * kTrackThreads] += y;
            s_mom_col[2 * kTrackThreads] += cdt;
            s_mom_col[3 * kTrackThreads] += x * x;
            s_mom_col[4 * kTrackThreads] += y * y;
            s_mom_col[5 * kTrackThreads] += cdt * cdt;
        }
        return;
    }
    if (!P.alive) return;
        switch (kind) {
        case OP_DRIFT:
#if SB2_FAST_MAPS
            {
                const double dp = dpop + 1.0;
                drift_unit_ib(x, xp, y, yp, cdt, dp, op.d[0], inv_beta(dp, op.d[1], op.d[2]), op.d[3]);
            }
#else
            drift_unit(x, xp, y, yp, cdt, dpop, op.d[0], op.d[1], op.d[2], op.d[3]);
#endif
            break;
        case OP_QUAD: {
            if constexpr (kQuad) {
                double xx = x - op.d[0], yy = y - op.d[1];
                yoshida6_op<OP_QUAD>(xx, xp, yy, yp, cdt, dpop, op);
                x = xx + op.d[0];
                y = yy + op.d[1];
            }
            break;
        }
        case OP_QUAD_CF: {
            if constexpr (kFull) {
                double xx = x - op.d[0], yy = y - op.d[1];
                yoshida6_op<OP_QUAD_CF>(xx, xp, yy, yp, cdt, dpop, op);
                x = xx + op.d[0];
                y = yy + op.d[1];
            }
            break;
        }
        case OP_SEXT_YOSHIDA:
            if constexpr (kFull) yoshida6_op<OP_SEXT_YOSHIDA>(x, xp, y, yp, cdt, dpop, op);
            break;
        case OP_THIN_QUAD: {
            double xx = x - op.d[0], yy = y - op.d[1];
            thin_quadrupole_unit(xx, xp, yy, yp, op.d[2], op.d[3]);
            break;
        }
        case OP_THIN_SEXT:
            thin_sextupole_unit(x, xp, y, yp, op.d[2], op.d[3]);
            break;
        case OP_OCT_YOSHIDA:
            if constexpr (kFull) yoshida6_op<OP_OCT_YOSHIDA>(x, xp, y, yp, cdt, dpop, op);
            break;
        case OP_THIN_OCT:
            thin_octupole_unit(x, xp, y, yp, op.d[2], op.d[3]);
            break;
        case OP_KICK_YOSHIDA:
            if constexpr (kFull) yoshida6_op<OP_KICK_YOSHIDA>(x, xp, y, yp, cdt, dpop, op);
            break;
        case OP_MATRIX:
            on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double& e, double& f) {
                matrix_op(a, b, c, d, e, f, op.d, op.flags);
            });
            break;
        case OP_DIPEDGE:
            on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double&, double&) {
                dipedge_op(a, b, c, d, op.d);
            });
            break;
        case OP_THIN_NLLENS:
            on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double&, double&) {
                nllens_op(a, b, c, d, op.d);
            });
            break;
        case OP_THIN_KICK:
            xp = xp + op.d[2];
            yp = yp + op.d[3];
            break;
        case OP_KICK_SIMPLE: {
            // simple_kicker ff_patterned_propagator.h:57-100: half drift, kick,
            // half drift (d: half length, pref, mass, half reference cdt, k)
#if SB2_FAST_MAPS
            const double dp = dpop + 1.0;
            const double ib = inv_beta(dp, op.d[1], op.d[2]);
            drift_unit_ib(x, xp, y, yp, cdt, dp, op.d[0], ib, op.d[3]);
            xp = xp + op.d[4];
            yp = yp + op.d[5];
            drift_unit_ib(x, xp, y, yp, cdt, dp, op.d[0], ib, op.d[3]);
#else
            drift_unit(x, xp, y, yp, cdt, dpop, op.d[0], op.d[1], op.d[2], op.d[3]);
            xp = xp + op.d[4];
            yp = yp + op.d[5];
            drift_unit(x, xp, y, yp, cdt, dpop, op.d[0], op.d[1], op.d[2], op.d[3]);
#endif
            break;
        }
        case OP_MPOLE: {
            const double* kl = op.d;
            const int on = op.flags;
            if (on & 1) { xp = xp - kl[0]; yp = yp + kl[1]; }
            if (on & 2) thin_quadrupole_unit(x, xp, y, yp, kl[2], kl[3]);
            if (on & 4) thin_sextupole_unit(x, xp, y, yp, kl[4], kl[5]);
            if (on & 8) thin_octupole_unit(x, xp, y, yp, kl[6], kl[7]);
            for (int nn = 4; nn < 8; ++nn)
                if (on & (1 << nn))
                    on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double&, double&) {
                        thin_magnet_unit(a, b, c, d, kl[nn * 2], kl[nn * 2 + 1], nn + 1);
                    });
            break;
        }
        case OP_SBEND: {
            if constexpr (kQuad)
                on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double& e, double& f) {
                    sbend_op(a, b, c, d, e, f, op.d, op.flags);
                });
            break;
        }
        case OP_SBEND_CF: {
            if constexpr (kFull)
                on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double& e, double& f) {
                    sbend_cf_op(a, b, c, d, e, f, op.d, op.steps, op.flags);
                });
            break;
        }
        case OP_SOLENOID:
            if constexpr (kFull)
                on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double& e, double& f) {
                    solenoid_op(a, b, c, d, e, f, op.d, op.flags);
                });
            break;
        case OP_RFCAVITY:
            if constexpr (kFull)
                on_copies(x, xp, y, yp, cdt, dpop, [&](double& a, double& b, double& c, double& d, double& e, double& f) {
                    rfcavity_op(a, b, c, d, e, f, op.d, op.steps, op.flags);
                });
            break;
        case OP_SC_KICK:
            if (p.efield32)
                sc_kick<float>(p, P, op.d[0], op.d[1]);
            else
                sc_kick<double>(p, P, op.d[0], op.d[1]);
            break;
        default:
            break;
        }
}

// PPT particles per thread travel through the op list together, so their
// independent load and arithmetic chains overlap (more bytes in flight per
// thread for the memory-bound passes).
// Raw values of one particle as loaded: six coordinates and the mask.
struct RawPart {
    double c[6];
    uint8_t m;
};

// The mask and the six columns are loaded together (no load waits on the
// mask), so all seven requests of a particle are in flight at once; lost
// particles' values are read and ignored.
template <int PPT>
__device__ __forceinline__ void load_tile(const TrackParams& p, int64_t base, RawPart* r)
{
    const int64_t n = p.n, S = p.stride;
#pragma unroll
    for (int q = 0; q < PPT; ++q) {
        const int64_t i = base + q * blockDim.x + threadIdx.x;
        r[q].m = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) r[q].c[j] = 0.0;
        if (i < n) {
            r[q].m = p.masks[i];
#pragma unroll
            for (int j = 0; j < 6; ++j) r[q].c[j] = p.parts[i + j * S];
        }
    }
}

// PF: the next tile's loads are issued before the current tile is computed
// (memory-bound passes: the loads of one tile overlap the arithmetic of the
// previous one).
// The pass over the particles of one bunch by the vg blocks of a grid
// (vb: this block among them): a launch for one bunch uses the whole grid,
// a work-list launch (track_list_kernel) a range of blocks per bunch.
template <int VARIANT, int PPT, bool PF>
__device__ __forceinline__ void track_body(const TrackParams& p, const int vb, const int vg)
{
    __shared__ int s_counts[kMaxOpsPerPass];
    __shared__ double s_mom[6][kTrackThreads]; // per-thread moment sums
    for (int i = threadIdx.x; i < kMaxOpsPerPass; i += blockDim.x) s_counts[i] = 0;
    for (int j = 0; j < 6; ++j) s_mom[j][threadIdx.x] = 0.0;
    __syncthreads();
    double* s_mom_col = &s_mom[0][threadIdx.x];

    const int64_t n = p.n;
    const int64_t S = p.stride;
    const int64_t tile = (int64_t)blockDim.x * PPT;
    const int64_t gstride = (int64_t)vg * tile;
    RawPart nxt[PPT];
    if (PF && (int64_t)vb * tile < n) load_tile<PPT>(p, (int64_t)vb * tile, nxt);
    for (int64_t base = (int64_t)vb * tile; base < n; base += gstride) {
        RawPart cur[PPT];
        if (PF) {
#pragma unroll
            for (int q = 0; q < PPT; ++q) cur[q] = nxt[q];
            if (base + gstride < n) load_tile<PPT>(p, base + gstride, nxt);
        } else {
            load_tile<PPT>(p, base, cur);
        }
        Part P[PPT];
        bool in[PPT];
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            P[q].x = cur[q].c[0];
            P[q].xp = cur[q].c[1];
            P[q].y = cur[q].c[2];
            P[q].yp = cur[q].c[3];
            P[q].cdt = cur[q].c[4];
            P[q].dpop = cur[q].c[5];
            P[q].alive = cur[q].m != 0;
            in[q] = P[q].alive;
            P[q].disc = 0;
            P[q].idx = base + q * blockDim.x + threadIdx.x;
        }
        for (int o = 0; o < p.nops; ++o) {
            const MapOp& op = p.ops[o];
#pragma unroll
            for (int q = 0; q < PPT; ++q) apply_op<VARIANT>(p, op, P[q], s_counts, s_mom_col);
        }
#pragma unroll
        for (int q = 0; q < PPT; ++q) {
            const int64_t i = base + q * blockDim.x + threadIdx.x;
            if (i >= n) continue;
            if (in[q]) {
                p.parts[i] = P[q].x;
                p.parts[i + S] = P[q].xp;
                p.parts[i + 2 * S] = P[q].y;
                p.parts[i + 3 * S] = P[q].yp;
                p.parts[i + 4 * S] = P[q].cdt;
                p.parts[i + 5 * S] = P[q].dpop;
                if (!P[q].alive) p.masks[i] = 0;
            }
            if (p.write_discards && p.discards) p.discards[i] = (uint8_t)P[q].disc;
        }
    }

    // per-aperture discard counts
    __syncthreads();
    for (int s = threadIdx.x; s < kMaxOpsPerPass; s += blockDim.x)
        if (s_counts[s]) atomicAdd(&p.ap_counts[p.slot_base + s], s_counts[s]);

    // moments: fixed-order block reduction -> one partial per block
    bool any_mom = false;
    for (int o = 0; o < p.nops; ++o) any_mom |= (p.ops[o].kind == OP_MOMENTS);
    if (any_mom && p.moment_partials) {
        for (int w = kTrackThreads / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
                for (int j = 0; j < 6; ++j) s_mom[j][threadIdx.x] += s_mom[j][threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x < 6) p.moment_partials[vb * 6 + threadIdx.x] = s_mom[threadIdx.x][0];
    }
}

template <int VARIANT, int PPT, bool PF>
__global__ void __launch_bounds__(kTrackThreads, PF ? SB2_LIGHT_OCC : TrackOcc<VARIANT, PPT>::value)
    track_kernel(const __grid_constant__ TrackParams p)
{
    track_body<VARIANT, PPT, PF>(p, blockIdx.x, gridDim.x);
}

// Block range of the work list: item i owns blocks [first[i], first[i+1]).
__device__ __forceinline__ int list_item(const int* __restrict__ first, int nitems)
{
    int lo = 0, hi = nitems;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= (int)blockIdx.x)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// A block's bunch parameters (header and its nops ops) copied from global
// memory into dynamic shared memory: the op loop reads its descriptors
// thousands of times per block, which from global memory costs an L1 round
// trip each and from shared memory a broadcast.
__device__ __forceinline__ const TrackParams& stage_params(const TrackParams* src)
{
    extern __shared__ __align__(16) unsigned char s_params[];
    const int nops = src->nops;
    const int words = (int)((offsetof(TrackParams, ops) + sizeof(MapOp) * (size_t)nops + 15) / 16);
    const int4* from = (const int4*)src;
    int4* to = (int4*)s_params;
    for (int w = threadIdx.x; w < words; w += blockDim.x) to[w] = from[w];
    __syncthreads();
    return *(const TrackParams*)s_params;
}

// One launch for the passes of many bunches (a batch advanced in lockstep):
// items[i] points at bunch i's parameters (only its nops ops are present;
// the dynamic shared memory of the launch holds the largest of them).
template <int VARIANT, int PPT, bool PF>
__global__ void __launch_bounds__(kTrackThreads, PF ? SB2_LIGHT_OCC : TrackOcc<VARIANT, PPT>::value)
    track_list_kernel(const TrackParams* const* __restrict__ items, const int* __restrict__ first, int nitems)
{
    const int it = list_item(first, nitems);
    const TrackParams& p = stage_params(items[it]);
    track_body<VARIANT, PPT, PF>(p, (int)blockIdx.x - first[it], first[it + 1] - first[it]);
}

// Light pass with the next tile's coordinates prefetched into shared memory
// by per-thread asynchronous copies (cp.async, 8 bytes each) instead of
// registers: each thread copies only its own particle's six values and reads
// back only its own slots, so no block barrier is needed; two buffers, the
// copy of tile k+1 goes to the buffer whose values tile k-1 already consumed.
// The mask byte is prefetched in a register.
__device__ __forceinline__ void cp_async8(void* dst, const void* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

template <int VARIANT>
__device__ __forceinline__ void track_body_lds(const TrackParams& p, const int vb, const int vg)
{
    __shared__ int s_counts[kMaxOpsPerPass];
    __shared__ double s_mom[6][kTrackThreads]; // per-thread moment sums
    __shared__ __align__(16) double s_pf[2][6][kTrackThreads];
    for (int i = threadIdx.x; i < kMaxOpsPerPass; i += blockDim.x) s_counts[i] = 0;
    for (int j = 0; j < 6; ++j) s_mom[j][threadIdx.x] = 0.0;
    __syncthreads();
    double* s_mom_col = &s_mom[0][threadIdx.x];

    const int64_t n = p.n;
    const int64_t S = p.stride;
    const int64_t tile = kTrackThreads;
    const int64_t gstride = (int64_t)vg * tile;
    auto issue = [&](int buf, int64_t i) {
        if (i < n)
#pragma unroll
            for (int j = 0; j < 6; ++j) cp_async8(&s_pf[buf][j][threadIdx.x], p.parts + i + j * S);
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    int64_t base = (int64_t)vb * tile;
    uint8_t m_next = 0;
    if (base < n) {
        issue(0, base + threadIdx.x);
        if (base + threadIdx.x < n) m_next = p.masks[base + threadIdx.x];
    }
    for (int it = 0; base < n; base += gstride, ++it) {
        const int b = it & 1;
        const int64_t i = base + threadIdx.x;
        asm volatile("cp.async.wait_all;" ::: "memory");
        RawPart cur;
        cur.m = m_next;
#pragma unroll
        for (int j = 0; j < 6; ++j) cur.c[j] = i < n ? s_pf[b][j][threadIdx.x] : 0.0;
        const int64_t nb = base + gstride;
        if (nb < n) {
            issue(b ^ 1, nb + threadIdx.x);
            m_next = nb + threadIdx.x < n ? p.masks[nb + threadIdx.x] : 0;
        }
        Part P;
        P.x = cur.c[0];
        P.xp = cur.c[1];
        P.y = cur.c[2];
        P.yp = cur.c[3];
        P.cdt = cur.c[4];
        P.dpop = cur.c[5];
        P.alive = cur.m != 0;
        const bool in = P.alive;
        P.disc = 0;
        P.idx = i;
        for (int o = 0; o < p.nops; ++o) apply_op<VARIANT>(p, p.ops[o], P, s_counts, s_mom_col);
        if (i < n) {
            if (in) {
                p.parts[i] = P.x;
                p.parts[i + S] = P.xp;
                p.parts[i + 2 * S] = P.y;
                p.parts[i + 3 * S] = P.yp;
                p.parts[i + 4 * S] = P.cdt;
                p.parts[i + 5 * S] = P.dpop;
                if (!P.alive) p.masks[i] = 0;
            }
            if (p.write_discards && p.discards) p.discards[i] = (uint8_t)P.disc;
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");

    __syncthreads();
    for (int s = threadIdx.x; s < kMaxOpsPerPass; s += blockDim.x)
        if (s_counts[s]) atomicAdd(&p.ap_counts[p.slot_base + s], s_counts[s]);
    bool any_mom = false;
    for (int o = 0; o < p.nops; ++o) any_mom |= (p.ops[o].kind == OP_MOMENTS);
    if (any_mom && p.moment_partials) {
        for (int w = kTrackThreads / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
                for (int j = 0; j < 6; ++j) s_mom[j][threadIdx.x] += s_mom[j][threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x < 6) p.moment_partials[vb * 6 + threadIdx.x] = s_mom[threadIdx.x][0];
    }
}

template <int VARIANT>
__global__ void __launch_bounds__(kTrackThreads, SB2_LIGHT_OCC) track_kernel_lds(const __grid_constant__ TrackParams p)
{
    track_body_lds<VARIANT>(p, blockIdx.x, gridDim.x);
}

template <int VARIANT>
__global__ void __launch_bounds__(kTrackThreads, SB2_LIGHT_OCC)
    track_list_kernel_lds(const TrackParams* const* __restrict__ items, const int* __restrict__ first, int nitems)
{
    const int it = list_item(first, nitems);
    const TrackParams& p = stage_params(items[it]);
    track_body_lds<VARIANT>(p, (int)blockIdx.x - first[it], first[it + 1] - first[it]);
}

// true when the pass needs no integrator beyond the pure-quadrupole Yoshida
// and the pure-dipole sector bend (FODO and ring lattices)
static bool track_quad_only(const MapOp* ops, int n)
{
    for (int i = 0; i < n; ++i) {
        int k = ops[i].kind;
        if (k == OP_QUAD_CF || k == OP_SEXT_YOSHIDA || k == OP_OCT_YOSHIDA || k == OP_KICK_YOSHIDA ||
            k == OP_SBEND_CF || k == OP_SOLENOID || k == OP_RFCAVITY)
            return false;
    }
    return true;
}

bool track_needs_full(const MapOp* ops, int n)
{
    for (int i = 0; i < n; ++i) {
        int k = ops[i].kind;
        if (k == OP_QUAD || k == OP_QUAD_CF || k == OP_SEXT_YOSHIDA || k == OP_OCT_YOSHIDA || k == OP_KICK_YOSHIDA ||
            k == OP_SBEND || k == OP_SBEND_CF || k == OP_SOLENOID || k == OP_RFCAVITY)
            return true;
    }
    return false;
}

// Kernel of a pass (the launch_pass dispatch below as a number): 0..3 light
// shapes (lds, 1 with prefetch, 2 with prefetch, 2 without), 4/5 quadrupole
// variant with 1/2 particles per thread, 6/7 wide full variant with 1/2,
// 8 full variant at 3 CTAs/SM.
int pass_choice(const TrackParams& p, const TrackTune& t)
{
    if (!track_needs_full(p.ops, p.nops))
        return t.light_shape == 3 ? 0 : t.light_shape == 1 ? 1 : t.light_shape == 2 ? 2 : 3;
    if (t.quad_variant && track_quad_only(p.ops, p.nops)) return t.quad_variant == 2 ? 5 : 4;
    if (t.full_occ != 3) return t.full_ppt == 2 ? 7 : 6;
    return 8;
}

// Work-list launch of passes that share a kernel choice: items[i] runs on
// blocks [first[i], first[i+1]) of an nblocks grid.
template <typename KERN>
static cudaError_t list_launch(KERN* k, int nblocks, int smem, const TrackParams* const* items, const int* first,
                               int nitems, cudaStream_t s)
{
    static cudaError_t once =
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrackParams) + 16);
    if (once) return once;
    k<<<nblocks, kTrackThreads, smem, s>>>(items, first, nitems);
    return cudaGetLastError();
}

// max_ops: the largest op count among the items (sizes the staged parameters)
cudaError_t launch_pass_list(int choice, const TrackParams* const* items, const int* first, int nitems, int nblocks,
                             int max_ops, cudaStream_t s)
{
    const int smem = (int)((offsetof(TrackParams, ops) + sizeof(MapOp) * (size_t)max_ops + 15) / 16 * 16);
    switch (choice) {
    case 0: return list_launch(track_list_kernel_lds<TRACK_LIGHT>, nblocks, smem, items, first, nitems, s);
    case 1: return list_launch(track_list_kernel<TRACK_LIGHT, 1, true>, nblocks, smem, items, first, nitems, s);
    case 2: return list_launch(track_list_kernel<TRACK_LIGHT, 2, true>, nblocks, smem, items, first, nitems, s);
    case 3: return list_launch(track_list_kernel<TRACK_LIGHT, 2, false>, nblocks, smem, items, first, nitems, s);
    case 4: return list_launch(track_list_kernel<TRACK_QUAD, 1, false>, nblocks, smem, items, first, nitems, s);
    case 5: return list_launch(track_list_kernel<TRACK_QUAD, 2, false>, nblocks, smem, items, first, nitems, s);
    case 6: return list_launch(track_list_kernel<TRACK_FULL_WIDE, 1, false>, nblocks, smem, items, first, nitems, s);
    case 7: return list_launch(track_list_kernel<TRACK_FULL_WIDE, 2, false>, nblocks, smem, items, first, nitems, s);
    default: return list_launch(track_list_kernel<TRACK_FULL, 1, false>, nblocks, smem, items, first, nitems, s);
    }
}

// The launch shape comes from the propagator's TrackTune (the measured
// defaults of track_tune_defaults, or what its autotuner chose).
cudaError_t launch_pass(const TrackParams& p, const TrackTune& t, cudaStream_t s)
{
    const int nb = track_grid_blocks(t.ctas_per_sm);
    if (!track_needs_full(p.ops, p.nops)) {
        if (t.light_shape == 3)
            track_kernel_lds<TRACK_LIGHT><<<nb, kTrackThreads, 0, s>>>(p);
        else if (t.light_shape == 1)
            track_kernel<TRACK_LIGHT, 1, true><<<nb, kTrackThreads, 0, s>>>(p);
        else if (t.light_shape == 2)
            track_kernel<TRACK_LIGHT, 2, true><<<nb, kTrackThreads, 0, s>>>(p);
        else
            track_kernel<TRACK_LIGHT, 2, false><<<nb, kTrackThreads, 0, s>>>(p);
    } else if (t.quad_variant && track_quad_only(p.ops, p.nops)) {
        if (t.quad_variant == 2)
            track_kernel<TRACK_QUAD, 2, false><<<nb, kTrackThreads, 0, s>>>(p);
        else
            track_kernel<TRACK_QUAD, 1, false><<<nb, kTrackThreads, 0, s>>>(p);
    } else if (t.full_occ != 3) {
        if (t.full_ppt == 2)
            track_kernel<TRACK_FULL_WIDE, 2, false><<<nb, kTrackThreads, 0, s>>>(p);
        else
            track_kernel<TRACK_FULL_WIDE, 1, false><<<nb, kTrackThreads, 0, s>>>(p);
    } else {
        track_kernel<TRACK_FULL, 1, false><<<nb, kTrackThreads, 0, s>>>(p);
    }
    return cudaGetLastError();
}

} // namespace SB2_TRACK_NS
} // namespace sb2
