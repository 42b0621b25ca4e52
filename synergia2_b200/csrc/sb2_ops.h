// Device-side operation descriptors shared by the host runtime (host.cc) and
// the particle kernels (track.cu).  One MapOp is one particle-local step of a
// half-step: an element slice map, an aperture, the space-charge kick or the
// spatial-moment accumulation.  The host fills every field from the element
// attributes and the design reference particle exactly as the corresponding
// libFF apply() does on the host side of the reference (libFF/ff_*.h), so the
// device only runs the per-particle arithmetic.
#pragma once
#include <cstdint>

namespace sb2 {

enum OpKind : int32_t {
    OP_NONE = 0,
    OP_DRIFT = 1,          // ff_drift.h:31-66
    OP_QUAD = 2,           // ff_quadrupole.h:165-213 (yoshida6, pure quad kick)
    OP_QUAD_CF = 3,        // ff_quadrupole.h:215-260 (yoshida6, cf_kick)
    OP_THIN_QUAD = 4,      // ff_quadrupole.h:59-93
    OP_SBEND = 5,          // ff_sbend.h:127-215
    OP_MPOLE = 6,          // ff_multipole.h:28-78
    OP_THIN_SEXT = 7,      // ff_patterned_propagator.h:21-53 with ff_sextupole kick
    OP_SEXT_YOSHIDA = 8,   // ff_patterned_propagator.h:110-150
    OP_THIN_OCT = 9,       // ff_patterned_propagator.h:21-53 with ff_octupole kick
    OP_OCT_YOSHIDA = 10,   // ff_patterned_propagator.h:110-150 with ff_octupole kick
    OP_THIN_KICK = 11,     // ff_patterned_propagator.h:21-53 with ff_kicker kick
    OP_KICK_YOSHIDA = 12,  // ff_patterned_propagator.h:110-150 with ff_kicker kick
    OP_KICK_SIMPLE = 13,   // ff_patterned_propagator.h:57-100 (drift-kick-drift)
    OP_SOLENOID = 14,      // ff_solenoid.h:160-248 (edge kicks, solenoid_unit)
    OP_RFCAVITY = 15,      // ff_rfcavity.h:23-132 (thin, or half drift - kick - half drift)
    OP_SBEND_CF = 16,      // ff_sbend.h:221-339 (bend_yoshida6 with thin_cf_kick_5)
    OP_THIN_NLLENS = 17,   // ff_nllens.h:9-50 with nllens_unit ff_algorithm.h:1180-1270
    OP_DIPEDGE = 18,       // ff_dipedge.h:196-330 with dipedge_unit ff_algorithm.h:1284-1316
    OP_MATRIX = 19,        // ff_matrix.h:140-515 with matrix_unit ff_algorithm.h:2439-2700
    OP_AP_FINITE = 20,     // aperture_operation.h:54-86
    OP_AP_CIRCULAR = 21,   // aperture_operation.h:92-116
    OP_AP_ELLIPTICAL = 22, // aperture_operation.h:123-151
    OP_AP_RECTANGULAR = 23,// aperture_operation.h:158-183
    OP_SC_KICK = 30,       // space_charge_3d_kernels.h:91-215 (zyx::alg_kicker)
    OP_MOMENTS = 31,       // core_diagnostics.cc:141-153 (spatial_mean_stddev sums)
};

// Field layout per kind (all FP64, indices into d[]):
//  DRIFT:        0 length, 1 ref_p, 2 mass, 3 ref_cdt
//  QUAD/QUAD_CF/SEXT_YOSHIDA (steps in `steps`):
//                0 xoff, 1 yoff, 2 ref_p, 3 mass, 4 substep ref_cdt,
//                5..8 c1..c4 * step_length, 9.. kick strengths:
//                QUAD/SEXT: k1[2] k2[2] k3[2] k4[2] at 9,11,13,15
//                QUAD_CF:   k1[16] k2[16] k3[16] k4[16] at 9,25,41,57
//  THIN_QUAD:    0 xoff, 1 yoff, 2 k0, 3 k1
//  THIN_SEXT:    2 k0, 3 k1
//  THIN_NLLENS:  2 1/cnll, 3 -knll/cnll
//  DIPEDGE:      0 re_2_1, 1 re_4_3, 2..11 te[10]
//  MATRIX:       0..5 kick, 6..41 rm (row major); flags bit0: second-order
//                tensor (216 doubles, [i][j][l]) at the device address whose
//                bits are stored in d[42]
//  SBEND:        flags bit0 ledge, bit1 redge; 0 ce1 1 se1 2 ce2 3 se2
//                4 us_kx 5 us_ky 6 ds_kx 7 ds_ky 8 dphi 9 phase_r 10 phase_i
//                11 term_r 12 term_i 13 strength 14 pref_b 15 m_b 16 ref_cdt
//                17-18 BendConst (igib2, cs) of (pref_b, m_b, strength)
//  SBEND_CF:     flags as SBEND; steps = Yoshida steps; 0 ce1 1 se1 2 ce2
//                3 se2 4 us_kx 5 us_ky 6 ds_kx 7 ds_ky 8 e1 9 e2 10-11 entry
//                face phase 12-13 exit face phase 14 strength 15 pref_b
//                16 m_b 17 substep ref_cdt 18 r0 19-22 dphi[4] 23-30
//                phase[4] 31-38 term[4] 39-70 k1..k4 (8 strengths each)
//                71-72 BendConst (igib2, cs) of (pref_b, m_b, strength)
//  MPOLE:        flags = bitmask of active orders (bit n: order n+1),
//                kl[16] at 0..15
//  AP_CIRCULAR:  0 r2, 1 xoff, 2 yoff
//  AP_ELLIPTICAL:0 h2, 1 v2, 2 xoff, 3 yoff
//  AP_RECTANGULAR: 0 width, 1 height, 2 xoff, 3 yoff
//  apertures:    `slot` = discard-counter slot of this aperture
constexpr int kOpDoubles = 73;

struct MapOp {
    int32_t kind;
    int32_t steps;
    int32_t flags;
    int32_t slot;
    double d[kOpDoubles];
};

// Maximum ops carried in one particle-pass launch (passed by value as a
// __grid_constant__ kernel parameter; longer op lists are split over several
// launches).
constexpr int kMaxOpsPerPass = 40;

// Device-resident space-charge state written by the domain kernel and read
// by the deposit, Green-function and kick kernels.
struct ScState {
    double left[3];   // original-domain left edge
    double h[3];      // original-domain cell size
    double ih[3];     // 1/h (kick/deposit), as 1.0/h
    double dh[3];     // doubled-domain cell size (Green function, E field)
    double w0;        // deposit weight (deposit.cc:608-610)
    double fn_norm;   // get_normalization_force
    double factor;    // apply_kick factor
    double mean_std[6];
    double G000;
    int32_t error;    // 1: degenerate domain
    int32_t valid;
};

// Device-resident bunch bookkeeping (bunch.h:363-370 update_total_num,
// bunch_particles.h:510-524 apply_aperture counts).
struct BunchCounters {
    int32_t n_valid;
    int32_t n_total;
    double real_num;
};

// Bookkeeping program executed after a particle pass: the independent
// operators it contained, in order, each with its aperture slots.
constexpr int kMaxOperatorsPerPass = 64;
constexpr int kMaxSlotsPerPass = 256;
struct PassBook {
    int32_t n_operators;
    int32_t slot_begin[kMaxOperatorsPerPass];
    int32_t slot_end[kMaxOperatorsPerPass];
    int32_t slot_elem[kMaxSlotsPerPass];  // lattice element index per slot (or -1)
    // per-step count record written after this operator (the last one of a
    // step), or -1
    int32_t op_record[kMaxOperatorsPerPass];
};

} // namespace sb2
