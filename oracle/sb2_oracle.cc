// ORACLE — test infrastructure only.
//
// A CPU, FP64, scalar restatement of Synergia's space-charge + libFF tracking
// step, written from the reference sources (paths relative to the synergia2
// project root).  It exists to check the CUDA path: only tests/, the smoke
// check of __graft_entry__.py and bench.py's cpu_baseline leg may load it.
// Nothing in the product links or calls it.
//
// Parity pins: the libFF MAD-X golden tracks
// (src/synergia/libFF/tests/lattices/madx_*.out), the zero-particle tests
// (src/synergia/libFF/tests/test_zeroparticle_propagate.cc), the one-particle
// deposit test (src/synergia/collective/tests/test_deposit.cc:42-97), the rod
// bunch line-charge kick (src/synergia/collective/tests/
// test_space_charge_3d_open_hockney_mpi.cc:8-107) and the Gaussian-sphere
// potential of docs/devel/solvers/3d_open_hockney.py:10-22.  The FFT has no
// golden vectors in the reference; it is pinned against a direct DFT and
// numpy.fft by the tests.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off -fopenmp -shared).
// -ffp-contract=off keeps every a*b+c as two IEEE roundings, as the reference
// (no -ffast-math in effect, CMakeLists.txt:338) does.

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <limits>
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// ---------------------------------------------------------------------------
// constants: src/synergia/foundation/physical_constants.h (PDG 2012)
// ---------------------------------------------------------------------------
namespace pc {
constexpr double pi = 3.14159265358979323846;
constexpr double mp = 0.938272046;
constexpr double e = 1.602176565e-19;
constexpr double c = 299792458.0;
constexpr double mu0 = 4 * pi * 1.0e-7;
constexpr double epsilon0 = 1.0 / (c * c * mu0);
constexpr double rp = e / (4 * pi * epsilon0 * mp * 1.0e9);
} // namespace pc

thread_local std::string g_err;

// ---------------------------------------------------------------------------
// FP64 operation counting: the algorithmic flops per particle of each
// operation, counted by running the oracle's own per-particle code on a
// counting scalar.  CD is a double that tallies every add or subtract,
// multiply, divide, square root and elementary function (asin, sin, cos,
// log, exp) it takes part in; sign changes, comparisons, floor and fabs are
// not counted.  The particle loops below write their per-particle work as a
// body generic in the scalar type; with counting on, count_particle() runs
// that body once more on CD copies of one chosen particle (its results are
// discarded), so the particles' doubles are exactly those of a run without
// counting.  Counts are kept per operation category and cut into one record
// per operator of a step (first half, collective, second half).
// ---------------------------------------------------------------------------
enum FlopCat { FC_DRIFT, FC_QUAD, FC_SBEND, FC_THIN, FC_THICK_OTHER, FC_APERTURE, FC_DOMAIN, FC_DEPOSIT, FC_KICK, FC_N };
enum FlopOp { FO_ADD, FO_MUL, FO_DIV, FO_SQRT, FO_FN, FO_N };

struct FlopRecord {
    int step;
    char kind; // 'I' independent operator, 'C' collective operator
    int64_t n[FC_N][FO_N];
};

struct FlopState {
    bool on = false;
    bool uncounted = false; // an element kind whose particle loop is not instrumented ran
    int64_t index = -1;     // the particle whose work is counted
    int cat = 0;
    int64_t n[FC_N][FO_N] = {};
    std::vector<FlopRecord> records;

    void mark(int step, char kind)
    {
        if (!on) return;
        FlopRecord r{step, kind, {}};
        std::memcpy(r.n, n, sizeof(n));
        std::memset(n, 0, sizeof(n));
        records.push_back(r);
    }
};
inline FlopState g_flops;

struct CD {
    double v;
    CD() : v(0.0) {}
    CD(double a) : v(a) {}
};
inline void tally(int op) { ++g_flops.n[g_flops.cat][op]; }
inline CD operator+(CD a, CD b) { tally(FO_ADD); return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { tally(FO_ADD); return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { tally(FO_MUL); return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { tally(FO_DIV); return CD(a.v / b.v); }
inline CD operator-(CD a) { return CD(-a.v); }
inline CD& operator+=(CD& a, CD b) { return a = a + b; }
inline CD& operator-=(CD& a, CD b) { return a = a - b; }
inline CD& operator*=(CD& a, CD b) { return a = a * b; }
inline CD& operator/=(CD& a, CD b) { return a = a / b; }
inline bool operator<(CD a, CD b) { return a.v < b.v; }
inline bool operator>(CD a, CD b) { return a.v > b.v; }
inline bool operator<=(CD a, CD b) { return a.v <= b.v; }
inline bool operator>=(CD a, CD b) { return a.v >= b.v; }
inline CD sqrt(CD a) { tally(FO_SQRT); return CD(std::sqrt(a.v)); }
inline CD asin(CD a) { tally(FO_FN); return CD(std::asin(a.v)); }
inline CD sin(CD a) { tally(FO_FN); return CD(std::sin(a.v)); }
inline CD cos(CD a) { tally(FO_FN); return CD(std::cos(a.v)); }
inline CD log(CD a) { tally(FO_FN); return CD(std::log(a.v)); }
inline CD floor(CD a) { return CD(std::floor(a.v)); }
inline CD fabs(CD a) { return CD(std::fabs(a.v)); }
inline bool isfinite(CD a) { return std::isfinite(a.v); }
inline double val(double a) { return a; }
inline double val(CD a) { return a.v; }
using std::asin;
using std::cos;
using std::fabs;
using std::floor;
using std::isfinite;
using std::log;
using std::sin;
using std::sqrt;

// ---------------------------------------------------------------------------
// Four_momentum / Reference_particle (foundation/four_momentum.cc:8-16,
// foundation/reference_particle.cc)
// ---------------------------------------------------------------------------
struct Refpart {
    int charge = 1;
    double mass = pc::mp;
    double gamma = 1, beta = 0, p = 0, energy = 0;
    std::array<double, 6> state{0, 0, 0, 0, 0, 0};
    double s_n = 0;

    void set_gamma(double g)
    { // four_momentum.cc:8-16 update_from_gamma
        if (g < 1.0) throw std::range_error("Four_momentum: gamma not >= 1.0");
        gamma = g;
        energy = gamma * mass;
        beta = std::sqrt(1.0 - 1.0 / (gamma * gamma));
        p = gamma * beta * mass;
    }
    void set_total_energy(double E) { set_gamma(E / mass); }
    void set_kinetic_energy(double K) { set_gamma((mass + K) / mass); } // four_momentum.cc:84-88
    // kind: 0 total energy, 1 momentum, 2 kinetic energy
    void set_by(int kind, double v)
    {
        if (kind == 0)
            set_total_energy(v);
        else if (kind == 1)
            set_momentum(v);
        else
            set_kinetic_energy(v);
    }
    void set_momentum(double mom)
    { // four_momentum.cc:90-95 then set_beta
        double r2 = mom * mom / (mass * mass);
        double b = std::sqrt(r2 / (1 + r2));
        if (b < 0.0 || b >= 1.0) throw std::range_error("beta out of range");
        set_gamma(1.0 / std::sqrt(1.0 - b * b));
    }
};

// ---------------------------------------------------------------------------
// Lattice_element / Lattice_element_slice (lattice/lattice_element*.cc)
// ---------------------------------------------------------------------------
struct Element {
    std::string type, name;
    std::map<std::string, double> d;
    std::map<std::string, std::string> s;
    std::map<std::string, std::vector<double>> v;

    double get(const std::string& k, double def) const
    {
        auto it = d.find(k);
        return it == d.end() ? def : it->second;
    }
    double get(const std::string& k) const
    {
        auto it = d.find(k);
        if (it == d.end())
            throw std::runtime_error("Lattice_element::get_double_attribute: element " +
                                     name + " of type " + type +
                                     " has no double attribute '" + k + "'");
        return it->second;
    }
    bool has_s(const std::string& k) const { return s.count(k) > 0; }
    std::string gets(const std::string& k, const std::string& def) const
    {
        auto it = s.find(k);
        return it == s.end() ? def : it->second;
    }
    double length() const { return get("l", 0.0); }
};

struct Lattice {
    std::vector<Element> elements;
    Refpart ref;
    double length() const
    { // lattice.cc:195-201
        double L = 0.0;
        for (auto const& e : elements) L += e.length();
        return L;
    }
};

// lattice_element_slice.cc:9-47 (split_element_tolerance 1e-9)
struct Slice {
    const Element* e = nullptr;
    double left = 0, right = 0;
    bool ledge = true, redge = true;
    Slice() = default;
    explicit Slice(const Element& el) : e(&el), left(0), right(el.length()) {}
    Slice(const Element& el, double l, double r) : e(&el), left(l), right(r)
    {
        const double tol = 1.0e-9;
        if (left < 0.0) throw std::range_error("Lattice_element_slice: left must be >= 0.0");
        if (left < tol) {
            ledge = true;
            left = 0.0;
        } else
            ledge = false;
        double L = el.length();
        if (right > L + tol)
            throw std::range_error("Lattice_element_slice: right must be no greater than the length of the element");
        bool eq;
        if (std::abs(right) < tol)
            eq = std::abs(right - L) < tol;
        else
            eq = std::abs((right - L) / right) < tol;
        if (eq) {
            redge = true;
            right = L;
        } else
            redge = false;
    }
};

// ---------------------------------------------------------------------------
// Bunch (bunch/bunch.h, bunch_particles.h): N x 7 column-major FP64, masks.
// ---------------------------------------------------------------------------
struct Bunch {
    int n_active = 0, n_valid = 0, n_total = 0;
    int64_t cap = 0;
    double real_num = 1.0;
    std::vector<double> parts;
    std::vector<uint8_t> masks, discards;
    Refpart ref;    // bunch reference particle
    Refpart design; // design reference particle
    double& P(int64_t i, int j) { return parts[j * cap + i]; }

    void update_total_num()
    { // bunch.h:363-370
        int old_total = n_total;
        n_total = n_valid;
        real_num = old_total ? n_total * real_num / old_total : 0.0;
    }
};

// Counting mode: runs `body` once on CD copies of the counted particle's six
// coordinates, the tallies going to category `cat`; the copies are dropped.
template <class F>
inline void count_particle(int cat, Bunch& b, F&& body)
{
    if (!g_flops.on) return;
    const int64_t i = g_flops.index;
    if (i < 0 || i >= b.n_active || !b.masks[i]) return;
    CD p[6];
    for (int j = 0; j < 6; ++j) p[j] = CD(b.P(i, j));
    const int saved = g_flops.cat;
    g_flops.cat = cat;
    body(p[0], p[1], p[2], p[3], p[4], p[5]);
    g_flops.cat = saved;
}

// ---------------------------------------------------------------------------
// ff_algorithm.h units, generic in the scalar type R (double, or CD when
// counting)
// ---------------------------------------------------------------------------
inline bool close_to_zero(double v) { return std::fabs(v) < 1e-13; } // :18-22

// drift_unit ff_algorithm.h:47-79
template <class R>
inline void drift_unit(R& x, R xp, R& y, R yp, R& cdt, R dpop,
                       double length, double reference_momentum, double m, double reference_cdt)
{
    double uni = 1.0;
    double sig = (double)((0.0 < length) - (length < 0.0));
    R vl = length, vm = m, vrm = reference_momentum, vrc = reference_cdt;
    R dp = dpop + uni;
    R inv_npz = uni / sqrt(dp * dp - xp * xp - yp * yp);
    R lxpr = xp * vl * inv_npz;
    R lypr = yp * vl * inv_npz;
    R D2 = lxpr * lxpr + vl * vl + lypr * lypr;
    R p = dp * vrm;
    R E2 = p * p + vm * vm;
    R ibeta2 = E2 / (p * p);
    x = x + lxpr;
    y = y + lypr;
    cdt = cdt + sig * sqrt(D2 * ibeta2) - vrc;
}

// slot_unit ff_algorithm.h:83-129
template <class R>
inline void slot_unit(R& x, R& xp, R& y, R& yp, R& cdt, R& dpop,
                      double ct, double st, double pref, double m)
{
    const double uni = 1.0;
    R r0 = x, r1 = y, r2 = 0.0;
    R zp = sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    R p = (dpop + uni) * pref;
    R e = sqrt(p * p + m * m);
    R b0 = xp * pref / e;
    R b1 = yp * pref / e;
    R b2 = zp * pref / e;
    R bp = st * b0 + ct * b2;
    R tau = -x * st / bp;
    r0 = x + tau * b0;
    r1 = y + tau * b1;
    r2 = tau * b2;
    x = r0 * ct - r2 * st;
    y = r1;
    cdt = cdt + tau;
    xp = xp * ct - zp * st;
}

// edge_unit (ref particle angle form) ff_algorithm.h:139-148
template <class R>
inline void edge_unit(R y, R& xp, R& yp, double kx, double ky)
{
    yp = yp - kx * y;
    xp = xp + ky * y;
}

// bend_complete ff_algorithm.h:191-251 (host, complex arithmetic)
inline void bend_complete(double& x, double& xp, double& y, double& yp, double& cdt, double dpop,
                          double dphi, double strength, double p_ref, double m, double cdt_ref,
                          std::complex<double> phase, std::complex<double> term)
{
    typedef std::complex<double> CT;
    const double uni = 1.0;
    double p0 = p_ref;
    double p = p_ref * (dpop + 1.0);
    double E0 = std::sqrt(p0 * p0 + m * m);
    double E = std::sqrt(p * p + m * m);
    double igamma = m / E0;
    double ibeta = uni / std::sqrt(uni - igamma * igamma);
    double csq = pc::c * pc::c * 1e-9;
    double psq = (dpop + 1.0) * (dpop + 1.0);
    double Ef = uni / std::sqrt(psq + igamma * igamma * ibeta * ibeta);
    double beta1 = Ef * xp;
    double beta2 = Ef * yp;
    double beta3 = Ef * std::sqrt((dpop + 1.0) * (dpop + 1.0) - xp * xp - yp * yp);
    CT ui = CT(0.0, x);
    CT vui = CT(pc::c * beta3, pc::c * beta1);
    double iomega = E / (csq * strength);
    CT bi = CT(0.0, 1.0) * vui * iomega - ui;
    CT bf = bi * phase + term;
    double rho = pc::c * std::sqrt(beta1 * beta1 + beta3 * beta3) * iomega;
    double dthmphi = std::asin(bi.real() / rho) - std::asin(bf.real() / rho);
    CT expf = std::exp(CT(0.0, dthmphi));
    CT vuf = vui * expf;
    CT uf = (ui + bi) * expf - bf;
    double dtheta = dthmphi + dphi;
    double ncdt = -pc::c * dtheta * iomega;
    x = uf.imag();
    y += beta2 * ncdt;
    cdt += ncdt - cdt_ref;
    xp = vuf.imag() / (Ef * pc::c);
}

// bend_unit ff_algorithm.h:255-343 (device form, real arithmetic)
template <class R>
inline void bend_unit(R& x, R& xp, R& y, R& yp, R& cdt, R dpop,
                      double theta, double strength, double p_ref, double m, double cdt_ref,
                      std::complex<double> phase, std::complex<double> term)
{
    const double uni = 1.0;
    const double tc = pc::c;
    R p0 = p_ref;
    R p = p_ref * (dpop + uni);
    R E0 = sqrt(p0 * p0 + m * m);
    R E = sqrt(p * p + m * m);
    R igamma = m / E0;
    R ibeta = uni / sqrt(uni - igamma * igamma);
    R csq = pc::c * pc::c * 1e-9;
    R psq = (dpop + uni) * (dpop + uni);
    R Ef = uni / sqrt(psq + igamma * igamma * ibeta * ibeta);
    R beta1 = Ef * xp;
    R beta2 = Ef * yp;
    R beta3 = Ef * sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    R ui_r = 0.0, ui_i = x;
    R vui_r = tc * beta3, vui_i = tc * beta1;
    R iomega = E / (csq * strength);
    R bi_r = -vui_i * iomega - ui_r;
    R bi_i = vui_r * iomega - ui_i;
    double phase_r = phase.real(), phase_i = phase.imag();
    R bf_r = bi_r * phase_r - bi_i * phase_i + term.real();
    R bf_i = bi_r * phase_i + bi_i * phase_r + term.imag();
    R rho = tc * sqrt(beta1 * beta1 + beta3 * beta3) * iomega;
    R dthmphi = asin(bi_r / rho) - asin(bf_r / rho);
    R expf_r = cos(dthmphi);
    R expf_i = sin(dthmphi);
    R vuf_i = vui_r * expf_i + vui_i * expf_r;
    R uf_i = (ui_r + bi_r) * expf_i + (ui_i + bi_i) * expf_r - bf_i;
    R dtheta = dthmphi + theta;
    R ncdt = -tc * dtheta * iomega;
    x = uf_i;
    xp = vuf_i / (Ef * tc);
    y = y + beta2 * ncdt;
    cdt = cdt + ncdt - cdt_ref;
}

// bend_edge ff_algorithm.h:366-450: a pole face of angle e as a pure
// rotation of the particle's circle (bend_unit with term = 0, the face angle
// in place of the bend angle, no reference-time subtraction)
inline void bend_edge(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double e,
                      std::complex<double> phase, double strength, double p_ref, double m)
{
    const double tc = pc::c;
    double p = p_ref * (dpop + 1.0);
    double E0 = std::sqrt(p_ref * p_ref + m * m);
    double E = std::sqrt(p * p + m * m);
    double igamma = m / E0;
    double ibeta = 1.0 / std::sqrt(1.0 - igamma * igamma);
    double csq = pc::c * pc::c * 1e-9;
    double psq = (dpop + 1.0) * (dpop + 1.0);
    double Ef = 1.0 / std::sqrt(psq + igamma * igamma * ibeta * ibeta);
    double beta1 = Ef * xp, beta2 = Ef * yp;
    double beta3 = Ef * std::sqrt((dpop + 1.0) * (dpop + 1.0) - xp * xp - yp * yp);
    double vui_r = tc * beta3, vui_i = tc * beta1;
    double iomega = E / (csq * strength);
    double bi_r = -vui_i * iomega - 0.0;
    double bi_i = vui_r * iomega - x;
    double bf_r = bi_r * phase.real() - bi_i * phase.imag();
    double bf_i = bi_r * phase.imag() + bi_i * phase.real();
    double rho = tc * std::sqrt(beta1 * beta1 + beta3 * beta3) * iomega;
    double dthmphi = std::asin(bi_r / rho) - std::asin(bf_r / rho);
    double cr = std::cos(dthmphi), ci = std::sin(dthmphi);
    double vuf_i = vui_r * ci + vui_i * cr;
    double uf_i = (0.0 + bi_r) * ci + (x + bi_i) * cr - bf_i;
    double ncdt = -tc * (dthmphi + e) * iomega;
    x = uf_i;
    xp = vuf_i / (Ef * tc);
    y = y + beta2 * ncdt;
    cdt = cdt + ncdt;
}

// Sector-magnet multipole potentials (Zolkin, PRAB 20, 043501 (2017),
// table XII; ff_algorithm.h:596-733): for order n the normal (N) and skew
// (S) field components in the cylindrical variables rho = 1 + x/r0,
// v = y/r0.  fr_* is the rho derivative (the y kick), fy_* the v
// derivative (the x kick).
namespace zolkin {
inline double fr_n2(double r, double v) { return -1.0 * (v / r); }
inline double fr_n3(double r, double v) { return -0.5 * (v / r) * (r * r - 1.0); }
inline double fr_n4(double r, double v)
{
    return (-1.0 / 6.0) * (v / r) * ((-3.0 / 2.0) * (r * r - 1.0) - v * v + 3.0 * r * r * std::log(r));
}
inline double fr_n5(double r, double v)
{
    return (-1.0 / 12.0) * (v / r) * ((r * r - 1.0) * ((3.0 / 4.0) * (r * r + 1.0) - v * v) - 3.0 * r * r * std::log(r));
}
inline double fy_n2(double r, double) { return std::log(r); }
inline double fy_n3(double r, double v) { return 0.5 * (0.5 * (r * r - 1.0) - v * v - std::log(r)); }
inline double fy_n4(double r, double v)
{
    return -0.25 * (r * r - 1.0) + 0.5 * (0.5 * (r * r + 1.0) - v * v) * std::log(r);
}
inline double fy_n5(double r, double v)
{
    return 0.125 * (0.125 * (r * r * r * r + 4.0 * r * r - 5.0) - (r * r - 1.0) * v * v + v * v * v * v -
                    (0.5 + r * r - 2.0 * v * v) * std::log(r));
}
inline double fr_s2(double r, double) { return 0.5 / r * (r * r - 1.0); }
inline double fr_s3(double r, double v) { return 0.5 / r * (-0.5 * (r * r - 1.0) - v * v + r * r * std::log(r)); }
inline double fr_s4(double r, double v)
{
    return 0.25 / r * (0.25 * (r * r * r * r - 1.0) - (r * r - 1.0) * v * v - r * r * std::log(r));
}
inline double fr_s5(double r, double v)
{
    return 0.125 / r *
           (-0.625 * r * r * r * r + 0.5 * r * r + 0.125 + (r * r - 1.0) * v * v + v * v * v * v / 3.0 +
            (1.0 + 0.5 * r * r - 2.0 * v * v) * r * r * std::log(r));
}
inline double fy_s2(double, double v) { return v; }
inline double fy_s3(double r, double v) { return v * std::log(r); }
inline double fy_s4(double r, double v) { return 0.5 * v * (0.5 * (r * r - 1.0) - v * v / 3.0 - std::log(r)); }
inline double fy_s5(double r, double v)
{
    return -0.25 * v * (r * r - 1.0) + (1.0 / 6.0) * v * (1.5 * (r * r + 1.0) - v * v) * std::log(r);
}
} // namespace zolkin

// thin_cf_kick_5 ff_algorithm.h:736-800: orders 2..5 of a combined-function
// sector bend; prefactor k rho r0^(n-1) multiplied left to right
inline void thin_cf_kick_5(double x, double& xp, double y, double& yp, double r0, const double* kL)
{
    using namespace zolkin;
    typedef double (*F)(double, double);
    static const F FYN[4] = {fy_n2, fy_n3, fy_n4, fy_n5}, FYS[4] = {fy_s2, fy_s3, fy_s4, fy_s5};
    static const F FRN[4] = {fr_n2, fr_n3, fr_n4, fr_n5}, FRS[4] = {fr_s2, fr_s3, fr_s4, fr_s5};
    double rho = 1.0 + x / r0;
    double v = y / r0;
    for (int o = 0; o < 4; ++o) {
        double kn = kL[2 * o], ks = kL[2 * o + 1];
        if (!(kn || ks)) continue;
        double an = kn * rho, as = ks * rho;
        for (int i = 0; i <= o; ++i) {
            an = an * r0;
            as = as * r0;
        }
        xp = xp - an * FYN[o](rho, v) + as * FYS[o](rho, v);
        yp = yp - an * FRN[o](rho, v) + as * FRS[o](rho, v);
    }
}

// bend_yoshida6 ff_algorithm.h:2194-2440: per step 10 bend pieces of angle
// c_j * step angle around 9 cf kicks of d_j * step strength
inline void bend_yoshida6(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double pref,
                          double m, double step_ref_cdt, const double* step_kl, const double* dphi,
                          const std::complex<double>* phase, const std::complex<double>* term, double r0,
                          double strength, int steps)
{
    const double d[4] = {1.58722492772224294589251207526, -1.99977809735512250728995471397,
                         -1.82324266348482825773733634154, 2.29714181079092974648453380998};
    double k[4][10];
    for (int j = 0; j < 4; ++j)
        for (int i = 0; i < 10; ++i) k[j][i] = d[j] * step_kl[i];
    double sub = step_ref_cdt * 0.1;
    static const int bseq[10] = {0, 1, 1, 2, 3, 3, 2, 1, 1, 0};
    static const int kseq[9] = {0, 1, 0, 2, 3, 2, 0, 1, 0};
    for (int s = 0; s < steps; ++s)
        for (int u = 0; u < 10; ++u) {
            int j = bseq[u];
            bend_unit(x, xp, y, yp, cdt, dpop, dphi[j], strength, pref, m, sub, phase[j], term[j]);
            if (u < 9) thin_cf_kick_5(x, xp, y, yp, r0, k[kseq[u]]);
        }
}

// thin kicks ff_algorithm.h:919-963
template <class R>
inline void thin_dipole_unit(R, R& xp, R, R& yp, const double* kL)
{
    xp = xp - kL[0];
    yp = yp + kL[1];
}
template <class R>
inline void thin_quadrupole_unit(R x, R& xp, R y, R& yp, const double* kL)
{
    double vk0 = kL[0], vk1 = kL[1];
    xp = xp - vk0 * x + vk1 * y;
    yp = yp + vk0 * y + vk1 * x;
}
template <class R>
inline void thin_sextupole_unit(R x, R& xp, R y, R& yp, const double* kL)
{
    double vk0 = kL[0], vk1 = kL[1];
    xp = xp - 0.5 * vk0 * (x * x - y * y) + vk1 * x * y;
    yp = yp + vk0 * x * y + 0.5 * vk1 * (x * x - y * y);
}
template <class R>
inline void thin_octupole_unit(R x, R& xp, R y, R& yp, const double* kL)
{
    double vk0 = kL[0], vk1 = kL[1];
    double n1 = 0.5, n2 = 1.0 / 3.0;
    xp = xp - n1 * vk0 * (x * x * x * n2 - x * y * y) + n1 * vk1 * (x * x * y - y * y * y * n2);
    yp = yp - n1 * vk0 * (y * y * y * n2 - x * x * y) + n1 * vk1 * (x * x * x * n2 - x * y * y);
}

inline double factorial(int n)
{ // ff_algorithm.h:1108-1117
    if (n == 0) return 1.0;
    double r = 1;
    for (int i = 1; i <= n; ++i) r *= i;
    return r;
}
template <class R>
inline R qpow(R x, int i)
{ // utils/kokkos_types.h:89-95
    R r = 1.0;
    while (i--) r = r * x;
    return r;
}

// thin_magnet_unit ff_algorithm.h:1122-1168
template <class R>
inline void thin_magnet_unit(R x, R& xp, R y, R& yp, const double* kL, int n)
{
    for (int k = 0; k < n; k += 4)
        xp = xp - (kL[0] * (n - k)) * qpow(x, n - k - 1) * qpow(y, k) / (factorial(n - k) * factorial(k));
    for (int k = 2; k < n; k += 4)
        xp = xp + (kL[0] * (n - k)) * qpow(x, n - k - 1) * qpow(y, k) / (factorial(n - k) * factorial(k));
    for (int k = 1; k < n; k += 4)
        xp = xp + (kL[1] * (n - k)) * qpow(x, n - k - 1) * qpow(y, k) / (factorial(n - k) * factorial(k));
    for (int k = 3; k < n; k += 4)
        xp = xp - (kL[1] * (n - k)) * qpow(x, n - k - 1) * qpow(y, k) / (factorial(n - k) * factorial(k));
    for (int k = 4; k <= n; k += 4)
        yp = yp - (kL[0] * k) * qpow(x, n - k) * qpow(y, k - 1) / (factorial(n - k) * factorial(k));
    for (int k = 2; k <= n; k += 4)
        yp = yp + (kL[0] * k) * qpow(x, n - k) * qpow(y, k - 1) / (factorial(n - k) * factorial(k));
    for (int k = 1; k <= n; k += 4)
        yp = yp + (kL[1] * k) * qpow(x, n - k) * qpow(y, k - 1) / (factorial(n - k) * factorial(k));
    for (int k = 3; k <= n; k += 4)
        yp = yp - (kL[1] * k) * qpow(x, n - k) * qpow(y, k - 1) / (factorial(n - k) * factorial(k));
}

// Kick functor forms used by the integrators.
using kick_fn = void (*)(double, double&, double, double&, double, const double*);

struct QuadKick { // ff_quadrupole.h:16-19
    template <class R>
    void operator()(R x, R& xp, R y, R& yp, R, const double* kL) const
    {
        thin_quadrupole_unit(x, xp, y, yp, kL);
    }
};
struct QuadCFKick { // ff_quadrupole.h:22-35
    template <class R>
    void operator()(R x, R& xp, R y, R& yp, R, const double* kL) const
    {
        thin_quadrupole_unit(x, xp, y, yp, kL);
        if (kL[2] || kL[3]) thin_quadrupole_unit(x, xp, y, yp, kL + 2);
        if (kL[4] || kL[5]) thin_sextupole_unit(x, xp, y, yp, kL + 4);
        if (kL[6] || kL[7]) thin_octupole_unit(x, xp, y, yp, kL + 6);
        if (kL[8] || kL[9]) thin_magnet_unit(x, xp, y, yp, kL + 8, 5);
        if (kL[10] || kL[11]) thin_magnet_unit(x, xp, y, yp, kL + 10, 6);
        if (kL[12] || kL[13]) thin_magnet_unit(x, xp, y, yp, kL + 12, 7);
        if (kL[14] || kL[15]) thin_magnet_unit(x, xp, y, yp, kL + 14, 8);
    }
};
struct SextKick { // ff_sextupole.h:11-13
    template <class R>
    void operator()(R x, R& xp, R y, R& yp, R, const double* kL) const
    {
        thin_sextupole_unit(x, xp, y, yp, kL);
    }
};
inline void quad_cf_kick(double x, double& xp, double y, double& yp, double c, const double* kL)
{
    QuadCFKick{}(x, xp, y, yp, c, kL);
}
inline void sext_kick(double x, double& xp, double y, double& yp, double c, const double* kL)
{
    SextKick{}(x, xp, y, yp, c, kL);
}

// yoshida6 ff_algorithm.h:1834-2008 (hardwired 6th order, 10 drifts/step)
template <class R, class K>
inline void yoshida6(R& x, R& xp, R& y, R& yp, R& cdt, R dpop,
                     double reference_momentum, double m, double step_reference_cdt,
                     double step_length, const double* step_strength, int steps, K kf,
                     int components)
{
    const double c1 = 0.79361246386112147294625603763;
    const double c2 = -0.206276584816439780698721319354;
    const double c3 = -0.118008867881292655922412133144;
    const double c4 = 0.236949573653050744373598734219;
    const double d1 = 1.58722492772224294589251207526;
    const double d2 = -1.99977809735512250728995471397;
    const double d3 = -1.82324266348482825773733634154;
    const double d4 = 2.29714181079092974648453380998;
    double sub = step_reference_cdt * 0.1;
    double k1[16], k2[16], k3[16], k4[16];
    for (int i = 0; i < components; ++i)
        for (int j = 0; j < 2; ++j) {
            k1[i * 2 + j] = d1 * step_strength[i * 2 + j];
            k2[i * 2 + j] = d2 * step_strength[i * 2 + j];
            k3[i * 2 + j] = d3 * step_strength[i * 2 + j];
            k4[i * 2 + j] = d4 * step_strength[i * 2 + j];
        }
    auto D = [&](double c) { drift_unit(x, xp, y, yp, cdt, dpop, c * step_length, reference_momentum, m, sub); };
    for (int i = 0; i < steps; ++i) {
        D(c1); kf(x, xp, y, yp, cdt, k1);
        D(c2); kf(x, xp, y, yp, cdt, k2);
        D(c2); kf(x, xp, y, yp, cdt, k1);
        D(c3); kf(x, xp, y, yp, cdt, k3);
        D(c4); kf(x, xp, y, yp, cdt, k4);
        D(c4); kf(x, xp, y, yp, cdt, k3);
        D(c3); kf(x, xp, y, yp, cdt, k1);
        D(c2); kf(x, xp, y, yp, cdt, k2);
        D(c2); kf(x, xp, y, yp, cdt, k1);
        D(c1);
    }
}

// general n-th order yoshida, ff_algorithm.h:1481-1646 (used only for the
// design particle of thick sextupoles through FF_patterned_propagator)
inline double yx1(int nn) { return 1.0 / (2.0 - std::pow(2.0, 1.0 / (2 * nn + 1))); }
inline double yx0(int nn) { return 1.0 - 2.0 * yx1(nn); }
inline void yoshida_element(int n, double& x, double& xp, double& y, double& yp, double& cdt,
                            double dpop, double pref, double m, double step_ref_cdt,
                            double step_length, const double* step_strength, double c,
                            kick_fn kf, int components)
{
    if (n == 0) {
        double sub = step_ref_cdt / 2.0;
        double kl[16];
        for (int i = 0; i < components * 2; ++i) kl[i] = step_strength[i] * c;
        drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * c * step_length, pref, m, sub);
        kf(x, xp, y, yp, cdt, kl);
        drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * c * step_length, pref, m, sub);
        return;
    }
    double sub = step_ref_cdt / 3.0;
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, step_strength, c * yx1(n), kf, components);
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, step_strength, c * yx0(n), kf, components);
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, step_strength, c * yx1(n), kf, components);
}
inline void yoshida_general(int order, double& x, double& xp, double& y, double& yp, double& cdt,
                            double dpop, double pref, double m, double step_ref_cdt,
                            double step_length, const double* step_strength, int steps,
                            kick_fn kf, int components)
{
    const int n = (order - 2) / 2;
    for (int i = 0; i < steps; ++i)
        yoshida_element(n, x, xp, y, yp, cdt, dpop, pref, m, step_ref_cdt, step_length, step_strength, 1.0, kf, components);
}

// ---------------------------------------------------------------------------
// Element maps (host part + particle loop), libFF/ff_*.h
// ---------------------------------------------------------------------------
static void drift_apply(const Slice& slice, Bunch& b)
{ // ff_drift.h:95-152
    const double length = slice.right - slice.left;
    const double mass = b.ref.mass;
    if (close_to_zero(length)) {
        b.design.state[4] = 0.0;
        return;
    }
    Refpart& ref_l = b.design;
    const double ref_p = b.ref.p * (1.0 + b.ref.state[5]);
    // get_reference_cdt ff_drift.h:69-88
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
    double cdt = 0.0, dpop = 0.0;
    drift_unit(x, xp, y, yp, cdt, dpop, length, ref_l.p, ref_l.mass, 0.0);
    ref_l.state = {x, xp, y, yp, cdt, dpop};
    const double ref_cdt = cdt;
    auto body = [&](auto& x, auto& xp, auto& y, auto& yp, auto& cdt, auto& dpop) {
        drift_unit(x, xp, y, yp, cdt, dpop, length, ref_p, mass, ref_cdt);
    };
    if (b.n_valid) {
        count_particle(FC_DRIFT, b, body);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i)
            if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
    }
    b.ref.s_n += length;
}

static void quad_apply(const Slice& slice, Bunch& b)
{ // ff_quadrupole.h:310-565
    const Element& ele = *slice.e;
    double length = slice.right - slice.left;
    const double xoff = ele.get("hoffset", 0.0);
    const double yoff = ele.get("voffset", 0.0);
    double tilt = ele.get("tilt", 0.0);
    double kn[16] = {0};
    kn[0] = ele.get("k1", 0.0);
    kn[1] = ele.get("k1s", 0.0);
    double quad_str = kn[0];
    std::complex<double> ck1(kn[0], -kn[1]);
    double rot = std::arg(ck1) / 2.0 + tilt;
    if (tilt != 0.0) {
        std::complex<double> ck2(kn[0], kn[1]);
        ck2 = ck2 * std::exp(std::complex<double>(0.0, -2.0 * tilt));
        kn[0] = ck2.real();
        kn[1] = ck2.imag();
    }
    bool has_mp = false;
    for (int i = 1; i < 8; ++i) {
        std::string a = "a0", bb = "b0";
        a[1] = '0' + i;
        bb[1] = '0' + i;
        kn[i * 2 + 0] = ele.get(bb, 0.0);
        kn[i * 2 + 1] = ele.get(a, 0.0);
        if (kn[i * 2 + 0] || kn[i * 2 + 1]) {
            has_mp = true;
            double coeff = factorial(i);
            kn[i * 2 + 0] *= quad_str * coeff;
            kn[i * 2 + 1] *= quad_str * coeff;
            if (rot || tilt) {
                auto ck = std::complex<double>(kn[i * 2 + 0], kn[i * 2 + 1]);
                ck *= std::exp(std::complex<double>(0.0, -(i + 1) * tilt));
                ck *= std::exp(std::complex<double>(0.0, -(i + 1) * rot));
                kn[i * 2 + 0] = ck.real();
                kn[i * 2 + 1] = ck.imag();
            }
        }
    }
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    double brho_l = ref_l.p / ref_l.charge;
    double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    double scale = brho_l / brho_b;
    for (auto& k : kn) k *= scale;

    auto ref_cdt_fn = [&](int steps) {
        // get_reference_cdt ff_quadrupole.h:263-303
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double cdt = 0.0, dpop = 0.0;
        x -= xoff;
        y -= yoff;
        if (close_to_zero(length))
            thin_quadrupole_unit(x, xp, y, yp, kn);
        else
            yoshida6(x, xp, y, yp, cdt, dpop, ref_l.p, ref_l.mass, 0.0, length / steps, kn, steps, quad_cf_kick, 8);
        x += xoff;
        y += yoff;
        ref_l.state = {x, xp, y, yp, cdt, dpop};
        return cdt;
    };

    if (close_to_zero(length)) {
        ref_cdt_fn(0);
        double k2[2] = {kn[0], kn[1]};
        auto body = [&](auto& x, auto& xp, auto& y, auto& yp, auto&, auto&) {
            auto xr = x - xoff;
            auto yr = y - yoff;
            thin_quadrupole_unit(xr, xp, yr, yp, k2);
        };
        if (b.n_valid) {
            count_particle(FC_THIN, b, body);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i)
                if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
        }
    } else {
        int steps = (int)ele.get("yoshida_steps", 4.0);
        for (auto& k : kn) k *= length / steps;
        double ref_p = ref_b.p, ref_m = ref_b.mass;
        double ref_t = ref_cdt_fn(steps);
        double step_ref_t = ref_t / steps, step_l = length / steps;
        auto body = [&](auto& x, auto& xp, auto& y, auto& yp, auto& cdt, auto& dpop) {
            auto p0 = x - xoff, p2 = y - yoff;
            if (has_mp)
                yoshida6(p0, xp, p2, yp, cdt, dpop, ref_p, ref_m, step_ref_t, step_l, kn, steps, QuadCFKick{}, 8);
            else
                yoshida6(p0, xp, p2, yp, cdt, dpop, ref_p, ref_m, step_ref_t, step_l, kn, steps, QuadKick{}, 1);
            x = p0 + xoff;
            y = p2 + yoff;
        };
        if (b.n_valid) {
            count_particle(FC_QUAD, b, body);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i)
                if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
        }
        b.ref.s_n += length;
    }
}

struct SbendParams { // ff_sbend.h:14-53
    bool ledge, redge;
    double length, angle, r0;
    int steps;
    double k_l[10];
    double scale, strength, pref_b, m_b, ref_cdt;
    double e1, e2, ce1, se1, ce2, se2;
    double us_edge_k, ds_edge_k, us_edge_k_p, ds_edge_k_p;
    double us_edge_k_x, us_edge_k_y, ds_edge_k_x, ds_edge_k_y;
};

static void sbend_cf_apply(SbendParams& sp, Bunch& b);

static void sbend_apply(const Slice& slice, Bunch& b)
{ // ff_sbend.h:741-969
    const Element& ele = *slice.e;
    SbendParams sp{};
    double a = ele.get("angle");
    double l = ele.get("l");
    sp.length = slice.right - slice.left;
    sp.angle = (sp.length / l) * a;
    sp.r0 = l / a;
    sp.steps = 6;
    sp.ledge = slice.ledge;
    sp.redge = slice.redge;
    sp.e1 = ele.get("e1", 0.0);
    sp.e2 = ele.get("e2", 0.0);
    static const char* kn_names[10] = {"k1", "k1s", "k2", "k2s", "k3", "k3s", "k4", "k4s", "k5", "k5s"};
    int cf = 0;
    for (int i = 0; i < 10; ++i) {
        sp.k_l[i] = ele.get(kn_names[i], 0.0);
        if (sp.k_l[i] != 0.0) cf = 1 + i / 2;
    }
    bool has_mp = false; // ff_sbend.h:790-828: b_i, a_i -> k_l of order i+1
    for (int i = 1; i < 5; ++i) {
        std::string an = "a0", bn = "b0";
        an[1] = '0' + i;
        bn[1] = '0' + i;
        double knv = ele.get(bn, 0.0), ksv = ele.get(an, 0.0);
        if (knv || ksv) {
            has_mp = true;
            double coeff = factorial(i);
            knv *= a * coeff;
            ksv *= a * coeff;
            if (sp.k_l[(i - 1) * 2 + 0] || sp.k_l[(i - 1) * 2 + 1])
                throw std::runtime_error("having both kn/ks and a/b coefficents are forbidden in sbends");
            sp.k_l[(i - 1) * 2 + 0] = knv;
            sp.k_l[(i - 1) * 2 + 1] = ksv;
        }
    }
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    sp.scale = ref_l.p / (ref_b.p * (1.0 + ref_b.state[5]));
    if (!sp.redge) sp.e2 = 0;
    if (!sp.ledge) sp.e1 = 0;
    const double brho_cnv = 1.0e-9 * pc::c;
    double pref_l = ref_l.p;
    double brho_l = pref_l / brho_cnv;
    int charge_l = ref_l.charge;
    double pref_b = ref_b.p;
    double brho_b = pref_b / brho_cnv;
    double m_b = b.ref.mass;
    sp.strength = brho_l * a / l;
    sp.pref_b = pref_b;
    sp.m_b = m_b;
    sp.ce1 = std::cos(-sp.e1);
    sp.se1 = std::sin(-sp.e1);
    sp.ce2 = std::cos(-sp.e2);
    sp.se2 = std::sin(-sp.e2);
    double sgn = (charge_l > 0) ? 1.0 : -1.0;
    sp.us_edge_k = sgn * sp.strength * std::tan(sp.e1) / brho_b;
    sp.ds_edge_k = -sgn * sp.strength * std::tan(-sp.e2) / brho_b;
    sp.us_edge_k_p = sgn * sp.strength / brho_b;
    sp.ds_edge_k_p = -sgn * sp.strength / brho_b;
    sp.us_edge_k_x = sp.us_edge_k_y = sp.ds_edge_k_x = sp.ds_edge_k_y = 0.0;
    if (cf != 0 || has_mp) {
        sbend_cf_apply(sp, b);
        return;
    }

    // prop_reference ff_sbend.h:478-566
    {
        double m_l = ref_l.mass;
        double x_l = ref_l.state[0], xp_l = ref_l.state[1], y_l = ref_l.state[2], yp_l = ref_l.state[3];
        double cdt_l = 0.0, dpop_l = 0.0;
        double dphi = -(sp.angle - (sp.e1 + sp.e2));
        std::complex<double> phase = std::exp(std::complex<double>(0.0, -dphi));
        std::complex<double> term = std::complex<double>(0.0, sp.length / sp.angle) *
                                    std::complex<double>(1.0 - std::cos(sp.angle), -std::sin(sp.angle)) *
                                    std::complex<double>(std::cos(sp.e2), -std::sin(sp.e2));
        if (sp.ledge) {
            slot_unit(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.ce1, sp.se1, pref_l, m_l);
            double p_l = 1.0 + dpop_l;
            double zp_l = std::sqrt(p_l * p_l - xp_l * xp_l - yp_l * yp_l);
            sp.us_edge_k_x = sp.us_edge_k_p * (xp_l / zp_l);
            sp.us_edge_k_y = sp.us_edge_k_p * (yp_l / zp_l);
            edge_unit(y_l, xp_l, yp_l, sp.us_edge_k_x / sp.scale, sp.us_edge_k_y / sp.scale);
        }
        bend_complete(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, dphi, sp.strength, pref_l, m_l, 0.0, phase, term);
        if (sp.redge) {
            double p_l = 1.0 + dpop_l;
            double zp_l = std::sqrt(p_l * p_l - xp_l * xp_l - yp_l * yp_l);
            sp.ds_edge_k_x = sp.ds_edge_k_p * (xp_l / zp_l);
            sp.ds_edge_k_y = sp.ds_edge_k_p * (yp_l / zp_l);
            edge_unit(y_l, xp_l, yp_l, sp.ds_edge_k_x / sp.scale, sp.ds_edge_k_y / sp.scale);
            slot_unit(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.ce2, sp.se2, pref_l, m_l);
        }
        ref_l.state = {x_l, xp_l, y_l, yp_l, cdt_l, dpop_l};
        sp.ref_cdt = cdt_l;
    }

    // PropSbendSimd ff_sbend.h:127-215
    const double dphi = -(sp.angle - (sp.e1 + sp.e2));
    const std::complex<double> phase = std::exp(std::complex<double>(0.0, -dphi));
    const std::complex<double> term = std::complex<double>(0.0, sp.length / sp.angle) *
                                      std::complex<double>(1.0 - std::cos(sp.angle), -std::sin(sp.angle)) *
                                      std::complex<double>(std::cos(sp.e2), -std::sin(sp.e2));
    auto body = [&](auto& p0, auto& p1, auto& p2, auto& p3, auto& p4, auto& p5) {
        if (sp.ledge) {
            slot_unit(p0, p1, p2, p3, p4, p5, sp.ce1, sp.se1, sp.pref_b, sp.m_b);
            edge_unit(p2, p1, p3, sp.us_edge_k_x, sp.us_edge_k_y);
        }
        bend_unit(p0, p1, p2, p3, p4, p5, dphi, sp.strength, sp.pref_b, sp.m_b, sp.ref_cdt, phase, term);
        if (sp.redge) {
            edge_unit(p2, p1, p3, sp.ds_edge_k_x, sp.ds_edge_k_y);
            slot_unit(p0, p1, p2, p3, p4, p5, sp.ce2, sp.se2, sp.pref_b, sp.m_b);
        }
    };
    if (b.n_valid) {
        count_particle(FC_SBEND, b, body);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i)
            if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
    }
    b.ref.s_n += sp.length;
}

// Combined-function bend: prop_reference_cf ff_sbend.h:568-660 for the
// design particle, then PropSbendCF ff_sbend.h:221-339 on every particle.
static void sbend_cf_apply(SbendParams& sp, Bunch& b)
{
    if (g_flops.on) g_flops.uncounted = true; // no instrumented particle loop

    const double c[4] = {0.79361246386112147294625603763, -0.206276584816439780698721319354,
                         -0.118008867881292655922412133144, 0.236949573653050744373598734219};
    Refpart& ref_l = b.design;
    const std::complex<double> phase_e1 = std::exp(std::complex<double>(0.0, -sp.e1));
    const std::complex<double> phase_e2 = std::exp(std::complex<double>(0.0, -sp.e2));
    const double step_angle = sp.angle / sp.steps;
    std::complex<double> step_phase[4], step_term[4];
    double step_dphi[4];
    for (int j = 0; j < 4; ++j) {
        double th = c[j] * step_angle;
        step_phase[j] = std::exp(std::complex<double>(0.0, th));
        step_term[j] = std::complex<double>(0.0, sp.r0) * std::complex<double>(1.0 - std::cos(th), -std::sin(th));
        step_dphi[j] = -c[j] * step_angle;
    }
    {
        double pref_l = ref_l.p, m_l = ref_l.mass;
        double x_l = ref_l.state[0], xp_l = ref_l.state[1], y_l = ref_l.state[2], yp_l = ref_l.state[3];
        double cdt_l = 0.0, dpop_l = 0.0;
        double step_length = sp.length / sp.steps;
        double step_kl[10];
        for (int i = 0; i < 10; ++i) step_kl[i] = sp.k_l[i] * step_length;
        if (sp.ledge) {
            slot_unit(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.ce1, sp.se1, pref_l, m_l);
            double p_l = 1.0 + dpop_l;
            double zp_l = std::sqrt(p_l * p_l - xp_l * xp_l - yp_l * yp_l);
            sp.us_edge_k_x = sp.us_edge_k_p * (xp_l / zp_l);
            sp.us_edge_k_y = sp.us_edge_k_p * (yp_l / zp_l);
            edge_unit(y_l, xp_l, yp_l, sp.us_edge_k_x / sp.scale, sp.us_edge_k_y / sp.scale);
            bend_edge(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.e1, phase_e1, sp.strength, pref_l, m_l);
        }
        bend_yoshida6(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, pref_l, m_l, 0.0, step_kl, step_dphi, step_phase,
                      step_term, sp.r0, sp.strength, sp.steps);
        if (sp.redge) {
            bend_edge(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.e2, phase_e2, sp.strength, pref_l, m_l);
            double p_l = 1.0 + dpop_l;
            double zp_l = std::sqrt(p_l * p_l - xp_l * xp_l - yp_l * yp_l);
            sp.ds_edge_k_x = sp.ds_edge_k_p * (xp_l / zp_l);
            sp.ds_edge_k_y = sp.ds_edge_k_p * (yp_l / zp_l);
            edge_unit(y_l, xp_l, yp_l, sp.ds_edge_k_x / sp.scale, sp.ds_edge_k_y / sp.scale);
            slot_unit(x_l, xp_l, y_l, yp_l, cdt_l, dpop_l, sp.ce2, sp.se2, pref_l, m_l);
        }
        ref_l.state = {x_l, xp_l, y_l, yp_l, cdt_l, dpop_l};
        sp.ref_cdt = cdt_l;
    }
    const double step_ref_cdt = sp.ref_cdt / sp.steps;
    double step_kl[10];
    for (int i = 0; i < 10; ++i) step_kl[i] = sp.k_l[i] * sp.scale * sp.length / sp.steps;
    if (b.n_valid) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i) {
            if (!b.masks[i]) continue;
            double p0 = b.P(i, 0), p1 = b.P(i, 1), p2 = b.P(i, 2), p3 = b.P(i, 3), p4 = b.P(i, 4), p5 = b.P(i, 5);
            if (sp.ledge) {
                slot_unit(p0, p1, p2, p3, p4, p5, sp.ce1, sp.se1, sp.pref_b, sp.m_b);
                edge_unit(p2, p1, p3, sp.us_edge_k_x, sp.us_edge_k_y);
                bend_edge(p0, p1, p2, p3, p4, p5, sp.e1, phase_e1, sp.strength, sp.pref_b, sp.m_b);
            }
            bend_yoshida6(p0, p1, p2, p3, p4, p5, sp.pref_b, sp.m_b, step_ref_cdt, step_kl, step_dphi, step_phase,
                          step_term, sp.r0, sp.strength, sp.steps);
            if (sp.redge) {
                bend_edge(p0, p1, p2, p3, p4, p5, sp.e2, phase_e2, sp.strength, sp.pref_b, sp.m_b);
                edge_unit(p2, p1, p3, sp.ds_edge_k_x, sp.ds_edge_k_y);
                slot_unit(p0, p1, p2, p3, p4, p5, sp.ce2, sp.se2, sp.pref_b, sp.m_b);
            }
            b.P(i, 0) = p0; b.P(i, 1) = p1; b.P(i, 2) = p2; b.P(i, 3) = p3; b.P(i, 4) = p4; b.P(i, 5) = p5;
        }
    }
    b.ref.s_n += sp.length;
}

static void multipole_apply(const Slice& slice, Bunch& b)
{ // ff_multipole.h:85-210
    if (slice.right - slice.left > 0.0)
        throw std::runtime_error("FF_multipole::apply() cannot deal with thick elements");
    const int max_order = 8;
    bool kn_on[8] = {false};
    double kl[16] = {0};
    std::vector<double> knl, ksl, tn;
    const Element& element = *slice.e;
    if (element.v.count("knl") || element.v.count("ksl")) {
        std::vector<double> k0(1, 0.0);
        knl = element.v.count("knl") ? element.v.at("knl") : k0;
        ksl = element.v.count("ksl") ? element.v.at("ksl") : k0;
        if (knl.size() > ksl.size())
            ksl.resize(knl.size(), 0.0);
        else if (knl.size() < ksl.size())
            knl.resize(ksl.size(), 0.0);
        double tilt = element.get("tilt", 0.0);
        tn.resize(knl.size(), tilt);
    } else {
        for (int i = 0; i < 6; ++i) {
            std::string skn = "k0l", stn = "t0";
            skn[1] = '0' + i;
            stn[1] = '0' + i;
            knl.push_back(element.get(skn, 0.0));
            tn.push_back(element.get(stn, 0.0));
        }
        int tail = (int)knl.size() - 1;
        while (tail && knl[tail] == 0.0) --tail;
        knl.resize(tail + 1);
        ksl.resize(knl.size(), 0.0);
        tn.resize(knl.size(), 0.0);
    }
    if ((int)knl.size() > max_order) throw std::runtime_error("oracle: multipole order above 8");
    for (size_t i = 0; i < knl.size(); ++i) {
        if (tn[i] != 0.0) {
            std::complex<double> ck2(knl[i], ksl[i]);
            ck2 = ck2 * std::exp(std::complex<double>(0.0, -(double)(i + 1) * tn[i]));
            knl[i] = ck2.real();
            ksl[i] = ck2.imag();
        }
    }
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    double brho_l = ref_l.p / ref_l.charge;
    double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    double scale = brho_l / brho_b;
    for (size_t i = 0; i < knl.size(); ++i) {
        knl[i] *= scale;
        ksl[i] *= scale;
    }
    for (size_t i = 0; i < knl.size(); ++i) {
        if (knl[i] || ksl[i]) kn_on[i] = true;
        kl[i * 2 + 0] = knl[i];
        kl[i * 2 + 1] = ksl[i];
    }
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], dpop = ref_l.state[5];
    for (int n = 0; n < max_order; ++n)
        if (kn_on[n]) thin_magnet_unit(x, xp, y, yp, &kl[n * 2], n + 1);
    ref_l.state = {x, xp, y, yp, 0.0, dpop};
    auto body = [&](auto& p0, auto& p1, auto& p2, auto& p3, auto&, auto&) {
        if (kn_on[0]) thin_dipole_unit(p0, p1, p2, p3, &kl[0]);
        if (kn_on[1]) thin_quadrupole_unit(p0, p1, p2, p3, &kl[2]);
        if (kn_on[2]) thin_sextupole_unit(p0, p1, p2, p3, &kl[4]);
        if (kn_on[3]) thin_octupole_unit(p0, p1, p2, p3, &kl[6]);
        for (int n = 4; n < max_order; ++n)
            if (kn_on[n]) thin_magnet_unit(p0, p1, p2, p3, &kl[n * 2], n + 1);
    };
    if (b.n_valid) {
        count_particle(FC_THIN, b, body);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i)
            if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
    }
}

static void sextupole_apply(const Slice& slice, Bunch& b)
{ // ff_sextupole.h:18-92 with ff_patterned_propagator.h
    const Element& element = *slice.e;
    double length = slice.right - slice.left;
    double k[2] = {element.get("k2", 0.0), element.get("k2s", 0.0)};
    double tilt = element.get("tilt", 0.0);
    if (tilt != 0.0) {
        std::complex<double> ck2(k[0], k[1]);
        ck2 = ck2 * std::exp(std::complex<double>(0.0, -3.0 * tilt));
        k[0] = ck2.real();
        k[1] = ck2.imag();
    }
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    double brho_l = ref_l.p / ref_l.charge;
    double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    double scale = brho_l / brho_b;
    k[0] *= scale;
    k[1] *= scale;
    if (close_to_zero(length)) {
        // get_reference_cdt_zero ff_patterned_propagator.h:227-244
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double dpop = 0.0;
        sext_kick(x, xp, y, yp, dpop, k);
        ref_l.state[1] = xp;
        ref_l.state[3] = yp;
        ref_l.state[4] = 0.0;
        auto body = [&](auto& x, auto& xp, auto& y, auto& yp, auto&, auto&) { thin_sextupole_unit(x, xp, y, yp, k); };
        if (b.n_valid) {
            count_particle(FC_THIN, b, body);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i)
                if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
        }
    } else {
        double pref = b.ref.p, mass = b.ref.mass;
        int steps = (int)element.get("yoshida_steps", 4.0);
        // get_reference_cdt_yoshida ff_patterned_propagator.h:275-316
        double cdt = 0.0;
        auto st = ref_l.state;
        st[5] = 0.0;
        double step_len = length / steps;
        double step_str[2] = {k[0] * step_len, k[1] * step_len};
        yoshida_general(6, st[0], st[1], st[2], st[3], cdt, st[5], ref_l.p, ref_l.mass, 0.0, step_len, step_str, steps, sext_kick, 1);
        st[4] = cdt;
        ref_l.state = st;
        double ref_cdt = cdt;
        // apply_yoshida_kick ff_patterned_propagator.h:199-225
        double step_ref_cdt = ref_cdt / steps;
        double ss[2] = {k[0] * step_len, k[1] * step_len};
        auto body = [&](auto& p0, auto& p1, auto& p2, auto& p3, auto& p4, auto& p5) {
            yoshida6(p0, p1, p2, p3, p4, p5, pref, mass, step_ref_cdt, step_len, ss, steps, SextKick{}, 1);
        };
        if (b.n_valid) {
            count_particle(FC_THICK_OTHER, b, body);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i)
                if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
        }
        b.ref.s_n += length;
    }
}

inline void oct_kick(double x, double& xp, double y, double& yp, double, const double* kL)
{ // ff_octupole.h:12-14
    thin_octupole_unit(x, xp, y, yp, kL);
}
inline void kicker_kick(double, double& xp, double, double& yp, double, const double* kL)
{ // ff_kicker.h:12-14, thin_kicker_unit ff_algorithm.h:994-1000
    xp = xp + kL[0];
    yp = yp + kL[1];
}

// nllens_unit ff_algorithm.h:1180-1270: thin nonlinear lens (Danilov-
// Nagaitsev potential) with k = {1/cnll, -knll/cnll}; the derivative of the
// complex potential F(z) is evaluated with z = (x + i y)/cnll as
// z/(1 - z^2) + arcsin(z)/(1 - z^2), taking the square root of 1 - z^2 with a
// non-negative imaginary part and arcsin(z) = -i log(i z + sqrt(1 - z^2)),
// as the reference's arithmetic does.  On the cut (y = 0, |x| >= cnll) the
// angles become NaN.
inline void nllens_kick(double x, double& xp, double y, double& yp, double, const double* k)
{
    const double zr = x * k[0], zi = y * k[0];
    if (zi == 0 && (zr >= 1.0 || zr <= -1.0)) {
        xp = std::numeric_limits<double>::quiet_NaN();
        yp = std::numeric_limits<double>::quiet_NaN();
        return;
    }
    std::complex<double> c(1.0 - zr * zr + zi * zi, -2.0 * zr * zi);   // 1 - z^2
    const double mod = std::sqrt(c.real() * c.real() + c.imag() * c.imag());
    std::complex<double> root(std::sqrt(0.5 * (c.real() + mod)), std::sqrt(0.5 * (-c.real() + mod)));
    std::complex<double> co(root.real() - zi, root.imag() + zr);         // i z + root
    const double r = std::sqrt(co.real() * co.real() + co.imag() * co.imag());
    const double theta = (co.real() > 0) ? std::atan(co.imag() / co.real()) + 0.0
                                         : std::atan(co.imag() / co.real()) + 3.14159265358979323846;
    const double asin_r = theta, asin_i = -std::log(r);                  // -i log(co)
    const double c2r = root.real() * root.real() - root.imag() * root.imag();
    const double c2i = 2.0 * root.real() * root.imag();
    const double den = c2r * c2r + c2i * c2i;
    const double d1r = (c2r * zr + c2i * zi) / den, d1i = (c2r * zi - c2i * zr) / den;
    const double d2r = (c2r * asin_r + c2i * asin_i) / den, d2i = (c2r * asin_i - c2i * asin_r) / den;
    xp = xp + k[1] * (d1r + d2r);
    yp = yp + -k[1] * (d1i + d2i);
}

// FF_patterned_propagator (ff_patterned_propagator.h) for one slice: the
// design particle follows k_design, the particles k_parts; thin slices kick,
// thick ones run yoshida6 (or drift-kick-drift when `simple`); use_drift
// takes the design particle's time from a plain drift.
static void patterned_apply(const Slice& slice, Bunch& b, const double* k_design, const double* k_parts, kick_fn kf,
                            bool thin, bool simple, bool use_drift, int steps)
{
    const double length = slice.right - slice.left;
    Refpart& ref_l = b.design;
    if (thin) {
        // get_reference_cdt_zero :227-244
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double dpop = 0.0;
        kf(x, xp, y, yp, dpop, k_design);
        ref_l.state[1] = xp;
        ref_l.state[3] = yp;
        ref_l.state[4] = 0.0;
        if (b.n_valid) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i) {
                if (!b.masks[i]) continue;
                double p1 = b.P(i, 1), p3 = b.P(i, 3), p5 = b.P(i, 5);
                kf(b.P(i, 0), p1, b.P(i, 2), p3, p5, k_parts);
                b.P(i, 1) = p1;
                b.P(i, 3) = p3;
            }
        }
        return;
    }
    const double pref = b.ref.p, mass = b.ref.mass;
    if (simple) {
        // get_reference_cdt_simple :246-273
        double cdt = 0.0;
        auto st = ref_l.state;
        st[5] = 0.0;
        double str[2] = {k_design[0] * length, k_design[1] * length};
        drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length * 0.5, ref_l.p, ref_l.mass, 0.0);
        kf(st[0], st[1], st[2], st[3], st[5], str);
        drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length * 0.5, ref_l.p, ref_l.mass, 0.0);
        st[4] = cdt;
        ref_l.state = st;
        const double ref_cdt = cdt;
        // simple_kicker :57-100 (the kick takes the strength per unit length as is)
        if (b.n_valid) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < b.n_active; ++i) {
                if (!b.masks[i]) continue;
                double p0 = b.P(i, 0), p1 = b.P(i, 1), p2 = b.P(i, 2), p3 = b.P(i, 3), p4 = b.P(i, 4), p5 = b.P(i, 5);
                drift_unit(p0, p1, p2, p3, p4, p5, length * 0.5, pref, mass, ref_cdt * 0.5);
                kf(p0, p1, p2, p3, p5, k_parts);
                drift_unit(p0, p1, p2, p3, p4, p5, length * 0.5, pref, mass, ref_cdt * 0.5);
                b.P(i, 0) = p0; b.P(i, 1) = p1; b.P(i, 2) = p2; b.P(i, 3) = p3; b.P(i, 4) = p4;
            }
        }
        b.ref.s_n += length;
        return;
    }
    // get_reference_cdt_yoshida :275-316
    double cdt = 0.0;
    auto st = ref_l.state;
    st[5] = 0.0;
    const double step_len = length / steps;
    double step_str[2] = {k_design[0] * step_len, k_design[1] * step_len};
    if (use_drift)
        drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length, ref_l.p, ref_l.mass, 0.0);
    else
        yoshida_general(6, st[0], st[1], st[2], st[3], cdt, st[5], ref_l.p, ref_l.mass, 0.0, step_len, step_str, steps,
                        kf, 1);
    st[4] = cdt;
    ref_l.state = st;
    // apply_yoshida_kick :199-225
    const double step_ref_cdt = cdt / steps;
    double ss[2] = {k_parts[0] * step_len, k_parts[1] * step_len};
    if (b.n_valid) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i) {
            if (!b.masks[i]) continue;
            double p0 = b.P(i, 0), p1 = b.P(i, 1), p2 = b.P(i, 2), p3 = b.P(i, 3), p4 = b.P(i, 4), p5 = b.P(i, 5);
            yoshida6(p0, p1, p2, p3, p4, p5, pref, mass, step_ref_cdt, step_len, ss, steps, kf, 1);
            b.P(i, 0) = p0; b.P(i, 1) = p1; b.P(i, 2) = p2; b.P(i, 3) = p3; b.P(i, 4) = p4;
        }
    }
    b.ref.s_n += length;
}

// dipedge_unit ff_algorithm.h:1284-1316 (MAD-X tmfrng): linear edge
// focusing re_2_1, re_4_3 and the optional second-order terms te[10]
inline void dipedge_unit(double& x, double& xp, double& y, double& yp, double re21, double re43, const double* te)
{
    double nx, nxp, ny, nyp;
    nxp = xp + re21 * x;
    nyp = yp + re43 * y;
    nx = x + te[0] * x * x + te[1] * y * y;
    nxp = nxp + te[2] * x * x + te[4] * y * y + te[3] * x * xp * 2.0 + te[5] * y * yp * 2.0;
    ny = y + te[6] * x * y * 2.0;
    nyp = nyp + te[7] * x * y * 2.0 + te[8] * x * yp * 2.0 + te[9] * y * xp * 2.0;
    x = nx;
    xp = nxp;
    y = ny;
    yp = nyp;
}

static void dipedge_apply(const Slice& slice, Bunch& b)
{ // ff_dipedge.h:196-330
    const Element& ele = *slice.e;
    const double sig = 1.0, he = 0.0, sk1 = 0.0;
    const double edge = ele.get("e1", 0.0);
    const double h = ele.get("h", 0.0);
    const double fint = ele.get("fint", 0.0);
    const double hgap = ele.get("hgap", 0.0);
    const double corr = (h + h) * hgap * fint;
    const double tanedg = std::tan(edge);
    const double secedg = 1.0 / std::cos(edge);
    const double sn = std::sin(edge);
    const double psip = edge - corr * secedg * (1.0 + sn * sn);
    const double re21 = h * tanedg;
    const double re43 = -h * std::tan(psip);
    double te[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (ele.get("second_order", 0.0) != 0.0) {
        const double hh = sig * (h / 2.0);
        te[0] = -hh * tanedg * tanedg;
        te[1] = hh * secedg * secedg;
        te[2] = (h / 2.0) * he * (secedg * secedg * secedg) + sk1 * tanedg;
        te[3] = -te[0];
        te[4] = hh * h * (tanedg * tanedg * tanedg) - te[2];
        te[5] = te[0];
        te[6] = -te[0];
        te[7] = -te[2];
        te[8] = te[0];
        te[9] = -te[1];
        te[4] += (h * secedg) * (h * secedg) * (tanedg / 2.0); // sig > 0
    }
    if (b.n_valid) { // prop_reference runs inside the per-group apply (:300-318)
        Refpart& ref_l = b.design;
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        dipedge_unit(x, xp, y, yp, re21, re43, te);
        ref_l.state = {x, xp, y, yp, 0.0, ref_l.state[5]};
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i) {
            if (!b.masks[i]) continue;
            dipedge_unit(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), re21, re43, te);
        }
    }
}

// matrix_unit ff_algorithm.h:2439-2700 and FF_matrix::apply
// ff_matrix.h:140-515: the design particle's image is computed but never
// stored by the reference, so it stays; a non-zero length throws (with
// valid particles).
static void matrix_apply(const Slice& slice, Bunch& b)
{
    const Element& ele = *slice.e;
    double k[6], rm[6][6], tm[6][6][6];
    for (int i = 0; i < 6; ++i) k[i] = ele.get("kick" + std::to_string(i + 1), 0.0);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            rm[i][j] = ele.get("rm" + std::to_string(i + 1) + std::to_string(j + 1), i == j ? 1.0 : 0.0);
            for (int l = 0; l < 6; ++l)
                tm[i][j][l] = ele.get("tm" + std::to_string(i + 1) + std::to_string(j + 1) + std::to_string(l + 1), 0.0);
        }
    if (!b.n_valid) return;
    if (ele.get("l", 0.0) != 0) throw std::runtime_error("error, matrix element has non-zero length");
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < b.n_active; ++p) {
        if (!b.masks[p]) continue;
        double v[6];
        for (int i = 0; i < 6; ++i) v[i] = b.P(p, i);
        double out[6];
        for (int i = 0; i < 6; ++i) {
            double a = k[i];
            for (int j = 0; j < 6; ++j) a = a + rm[i][j] * v[j];
            out[i] = a;
        }
        for (int i = 0; i < 6; ++i) {
            double a = out[i];
            for (int j = 0; j < 6; ++j)
                for (int l = 0; l < 6; ++l) a = a + tm[i][j][l] * v[j] * v[l];
            out[i] = a;
        }
        for (int i = 0; i < 6; ++i) b.P(p, i) = out[i];
    }
}

static void nllens_apply(const Slice& slice, Bunch& b)
{ // ff_nllens.h:9-50
    const Element& element = *slice.e;
    const double l = element.get("l", 0.0);
    const double knll = element.get("knll");
    const double cnll = element.get("cnll");
    if (!close_to_zero(l)) throw std::runtime_error("nonlinear lens has non-zero length");
    const double icnll = 1.0 / cnll;
    const double k[2] = {icnll, -knll * icnll};
    patterned_apply(slice, b, k, k, nllens_kick, true, false, false, 1);
    if (std::isnan(b.design.state[1]) || std::isnan(b.design.state[3]))
        throw std::runtime_error("the bunch reference particle hits the sigularity region "
                                 "when propagating through a nonlinearlens");
}

static void octupole_apply(const Slice& slice, Bunch& b)
{ // ff_octupole.h:16-88
    const Element& element = *slice.e;
    const double length = slice.right - slice.left;
    double k[2] = {element.get("k3", 0.0), element.get("k3s", 0.0)};
    const double tilt = element.get("tilt", 0.0);
    if (tilt != 0.0) {
        std::complex<double> ck2(k[0], k[1]);
        ck2 = ck2 * std::exp(std::complex<double>(0.0, -4.0 * tilt));
        k[0] = ck2.real();
        k[1] = ck2.imag();
    }
    const Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    const double brho_l = ref_l.p / ref_l.charge;
    const double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    const double scale = brho_l / brho_b;
    k[0] *= scale;
    k[1] *= scale;
    const int steps = (int)element.get("yoshida_steps", 4.0);
    patterned_apply(slice, b, k, k, oct_kick, close_to_zero(length), false, false, steps);
}

static void kicker_apply(const Slice& slice, Bunch& b)
{ // ff_kicker.h:17-127, attributes as Lattice_element_processor hkicker / vkicker / kicker
    const Element& elem = *slice.e;
    const double length = slice.right - slice.left;
    const std::string& t = elem.type;
    double hk0 = elem.get("hkick", 0.0), vk0 = elem.get("vkick", 0.0);
    if (t == "hkicker") {
        if (elem.d.count("kick")) hk0 = elem.get("kick", 0.0);
        vk0 = 0.0;
    } else if (t == "vkicker") {
        if (elem.d.count("kick")) vk0 = elem.get("kick", 0.0);
        hk0 = 0.0;
    }
    const double l = elem.get("l", 0.0);
    const double tilt = elem.get("tilt", 0.0);
    const double hk = cos(tilt) * hk0 - sin(tilt) * vk0;
    const double vk = sin(tilt) * hk0 + cos(tilt) * vk0;
    const double scale = b.design.p / b.ref.p;
    const double q = (double)b.ref.charge / b.design.charge;
    double k[2] = {hk, vk};
    double sk[2] = {hk * q * scale, vk * q * scale};
    const bool thin = close_to_zero(length);
    if (!thin) {
        k[0] = k[0] / l;
        k[1] = k[1] / l;
        sk[0] = sk[0] / l;
        sk[1] = sk[1] / l;
    }
    const bool simple = std::fabs(elem.get("simple", 0.0)) > 1e-16;
    const int steps = (int)elem.get("yoshida_steps", 4.0);
    const bool use_drift = (int)elem.get("cdt_use_drift", 0.0) != 0;
    patterned_apply(slice, b, k, sk, kicker_kick, thin, simple, use_drift, steps);
}

// solenoid_unit ff_algorithm.h:1317-1356 (the map's callers pass ks*L in
// the `ks` slot and ks in the `ksl` slot, ff_solenoid.h:130-131,231-236;
// kept as is), edge kicks :1358-1372
inline void solenoid_unit(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double ks,
                          double ksl, double length, double ref_p, double mass, double ref_cdt)
{
    const double uni = 1.0;
    double p2 = (uni + dpop) * (uni + dpop);
    double zp = std::sqrt(p2 - xp * xp - yp * yp);
    double dtheta = ksl / zp;
    double sn = std::sin(dtheta);
    double cs = std::cos(dtheta);
    double xpi = xp, ypi = yp;
    xp = cs * xpi + sn * ypi;
    yp = (-sn) * xpi + cs * ypi;
    cs = cs - uni;
    x = x + (cs * (-ypi) + sn * xpi) / ks;
    y = y + ((-sn) * (-ypi) + cs * xpi) / ks;
    double en = std::sqrt(p2 * ref_p * ref_p + mass * mass);
    double duration = length / (zp * ref_p / en);
    cdt = cdt + duration - ref_cdt;
}

static void solenoid_apply(const Slice& slice, Bunch& b)
{ // ff_solenoid.h:160-248
    const double length = slice.right - slice.left;
    const double mass = b.ref.mass;
    const bool in_edge = slice.ledge, out_edge = slice.redge;
    double ks = slice.e->get("ks", 0.0);
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    const double ref_p = ref_b.p * (1.0 + ref_b.state[5]);
    if (std::fabs(ks) < 1e-12) {
        drift_apply(slice, b);
        return;
    }
    const double brho_l = ref_l.p * (1.0 + ref_l.state[5]) / ref_l.charge;
    const double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    ks = ks * (brho_l / brho_b);
    const double ksl = ks * length;
    const double kse = ks * 0.5;
    // get_reference_cdt_solenoid :125-155
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], cdt = 0.0, dpop = 0.0;
    if (in_edge) { xp = xp + kse * y; yp = yp - kse * x; }
    solenoid_unit(x, xp, y, yp, cdt, dpop, ksl, ks, length, ref_l.p * (1 + dpop), ref_l.mass, 0.0);
    if (out_edge) { xp = xp - kse * y; yp = yp + kse * x; }
    ref_l.state = {x, xp, y, yp, cdt, dpop};
    const double ref_cdt = cdt;
    if (b.n_valid) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i) {
            if (!b.masks[i]) continue;
            double p0 = b.P(i, 0), p1 = b.P(i, 1), p2 = b.P(i, 2), p3 = b.P(i, 3), p4 = b.P(i, 4), p5 = b.P(i, 5);
            if (in_edge) { p1 = p1 + kse * p2; p3 = p3 - kse * p0; }
            solenoid_unit(p0, p1, p2, p3, p4, p5, ksl, ks, length, ref_p, mass, ref_cdt);
            if (out_edge) { p1 = p1 - kse * p2; p3 = p3 + kse * p0; }
            b.P(i, 0) = p0; b.P(i, 1) = p1; b.P(i, 2) = p2; b.P(i, 3) = p3; b.P(i, 4) = p4;
        }
    }
    b.ref.s_n += length;
}

// thin_rfcavity_pnew / thin_rfcavity_unit ff_algorithm.h:1017-1082
inline double thin_rfcavity_pnew(double pref, double m, double volt, double phi_s)
{
    double E0 = std::sqrt(pref * pref + m * m);
    double E1 = E0 + volt * std::sin(phi_s);
    return std::sqrt(E1 * E1 - m * m);
}
inline void thin_rfcavity_unit(double& px, double& py, double cdt, double& dpop, double w_rf, double volt,
                               double phi_s, double m, double old_ref_p, double new_ref_p, const double* mhp, int nh)
{
    if (volt == 0.0) return;
    const double anh_phase = 0.0;
    double phase_slip_argument = (cdt * (w_rf / pc::c)) + anh_phase;
    double strength_factor = 0.0;
    for (int i = 0; i < nh; ++i)
        strength_factor = strength_factor + mhp[i * 3 + 1] * std::sin(mhp[i * 3] * (phi_s + phase_slip_argument) +
                                                                      mhp[i * 3 + 2]);
    double p = old_ref_p * (dpop + 1.0);
    double E = std::sqrt(p * p + m * m);
    E = E + volt * strength_factor;
    px = px * (old_ref_p / new_ref_p);
    py = py * (old_ref_p / new_ref_p);
    dpop = std::sqrt((E - m) * (E + m)) / new_ref_p - 1.0;
}

static void rfcavity_apply(const Slice& slice, Bunch& b)
{ // ff_rfcavity.h:134-330
    const Element& elm = *slice.e;
    const double length = slice.right - slice.left;
    const double volt = elm.get("volt", 0.0);
    double lag = elm.get("lag", 0.0);
    const double freq = elm.get("freq", -1.0);
    const double delta_freq = elm.get("delta_freq", 0.0);
    int nh = 1;
    double mhp[12] = {1.0, 1.0, 0.0};
    for (int h = 2; h <= 4; ++h) {
        const std::string sk = "h" + std::to_string(h) + "_str", pk = "h" + std::to_string(h) + "_phase";
        if (elm.d.count(sk)) {
            mhp[nh * 3 + 0] = h;
            mhp[nh * 3 + 1] = elm.get(sk, 0.0);
            mhp[nh * 3 + 2] = elm.get(pk, 0.0);
            ++nh;
        }
    }
    const double str = volt * 1.0e-3;
    while (lag < 0.0) lag += 1.0;
    while (lag >= 1.0) lag -= 1.0;
    const double phi_s = 2.0 * M_PI * lag;
    const double w_rf = 2.0 * M_PI * (freq + delta_freq) * 1.0e6;
    Refpart& ref_l = b.design;
    const double pref_b = b.ref.p, m_b = b.ref.mass;
    const double new_pref_b = thin_rfcavity_pnew(pref_b, m_b, str, phi_s);
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], cdt = 0.0, dpop = 0.0;
    const double lp = ref_l.p, lm = ref_l.mass;
    drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * length, lp, lm, 0.0);
    double total = cdt;
    const double ref_cdt_1 = cdt;
    cdt = 0.0;
    thin_rfcavity_unit(xp, yp, cdt, dpop, w_rf, str, phi_s, lm, lp, lp, mhp, nh);
    drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * length, lp, lm, 0.0);
    total += cdt;
    const double ref_cdt_2 = cdt;
    ref_l.state = {x, xp, y, yp, total, 0.0};
    const bool thin = close_to_zero(length);
    if (b.n_valid) {
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i) {
            if (!b.masks[i]) continue;
            double p0 = b.P(i, 0), p1 = b.P(i, 1), p2 = b.P(i, 2), p3 = b.P(i, 3), p4 = b.P(i, 4), p5 = b.P(i, 5);
            if (!thin) drift_unit(p0, p1, p2, p3, p4, p5, 0.5 * length, pref_b, m_b, ref_cdt_1);
            thin_rfcavity_unit(p1, p3, p4, p5, w_rf, str, phi_s, m_b, pref_b, new_pref_b, mhp, nh);
            if (!thin) drift_unit(p0, p1, p2, p3, p4, p5, 0.5 * length, pref_b, m_b, ref_cdt_2);
            b.P(i, 0) = p0; b.P(i, 1) = p1; b.P(i, 2) = p2; b.P(i, 3) = p3; b.P(i, 4) = p4; b.P(i, 5) = p5;
        }
    }
    b.ref.set_momentum(new_pref_b);
    b.ref.s_n += length;
}

static void element_apply(const Slice& slice, Bunch& b)
{ // ff_element.h:25-67
    const std::string& t = slice.e->type;
    if (g_flops.on && !(t == "drift" || t == "monitor" || t == "hmonitor" || t == "vmonitor" || t == "marker" ||
                        t == "instrument" || t == "rcollimator" || t == "sbend" || t == "quadrupole" ||
                        t == "multipole" || t == "sextupole"))
        g_flops.uncounted = true; // no instrumented particle loop for this kind
    if (t == "drift" || t == "monitor" || t == "hmonitor" || t == "vmonitor" || t == "marker" ||
        t == "instrument" || t == "rcollimator")
        drift_apply(slice, b);
    else if (t == "sbend")
        sbend_apply(slice, b);
    else if (t == "quadrupole")
        quad_apply(slice, b);
    else if (t == "multipole")
        multipole_apply(slice, b);
    else if (t == "sextupole")
        sextupole_apply(slice, b);
    else if (t == "octupole")
        octupole_apply(slice, b);
    else if (t == "nllens")
        nllens_apply(slice, b);
    else if (t == "dipedge")
        dipedge_apply(slice, b);
    else if (t == "matrix")
        matrix_apply(slice, b);
    else if (t == "hkicker" || t == "vkicker" || t == "kicker")
        kicker_apply(slice, b);
    else if (t == "solenoid")
        solenoid_apply(slice, b);
    else if (t == "rfcavity")
        rfcavity_apply(slice, b);
    else
        throw std::runtime_error("FF_element::apply() unknown element type = " + t + ", element name = " + slice.e->name);
}

// ---------------------------------------------------------------------------
// Apertures: simulation/aperture_operation.h, bunch_particles.h:484-524
// ---------------------------------------------------------------------------
enum { AP_FINITE = 0, AP_CIRCULAR = 1, AP_ELLIPTICAL = 2, AP_RECTANGULAR = 3 };

struct Aperture {
    int kind = AP_FINITE;
    double r2 = 1e6, xoff = 0, yoff = 0, h2 = 1, v2 = 1, width = 0, height = 0;
    const Element* elem = nullptr;
};

static Aperture make_aperture(const std::string& type, const Slice& slice)
{ // operation_extractor.cc:55-75
    Aperture ap;
    const Element& ele = *slice.e;
    ap.elem = &ele;
    if (type == "finite") {
        ap.kind = AP_FINITE;
    } else if (type == "circular") {
        ap.kind = AP_CIRCULAR;
        ap.xoff = ele.get("hoffset", 0.0);
        ap.yoff = ele.get("voffset", 0.0);
        double r = ele.get("circular_aperture_radius", 1000.0);
        ap.r2 = r * r;
    } else if (type == "elliptical") {
        ap.kind = AP_ELLIPTICAL;
        ap.xoff = ele.get("hoffset", 0.0);
        ap.yoff = ele.get("voffset", 0.0);
        double hr = ele.get("elliptical_aperture_horizontal_radius");
        double vr = ele.get("elliptical_aperture_vertical_radius");
        ap.h2 = hr * hr;
        ap.v2 = vr * vr;
    } else if (type == "rectangular") {
        ap.kind = AP_RECTANGULAR;
        ap.width = ele.get("rectangular_aperture_width");
        ap.height = ele.get("rectangular_aperture_height");
        ap.xoff = ele.get("hoffset", 0.0);
        ap.yoff = ele.get("voffset", 0.0);
    } else {
        throw std::runtime_error("unknown aperture_type " + type);
    }
    return ap;
}

static int aperture_apply(const Aperture& ap, Bunch& b)
{
    auto decide = [&](auto& x, auto& xp, auto& y, auto& yp, auto& cdt, auto& dpop) -> bool {
        bool discard = false;
        switch (ap.kind) {
        case AP_FINITE: {
            if (!isfinite(x) || !isfinite(xp) || !isfinite(y) || !isfinite(yp) || !isfinite(cdt) || !isfinite(dpop))
                discard = true;
            else {
                auto pt = 1.0 + dpop;
                discard = pt * pt - xp * xp - yp * yp < 0.0;
            }
            break;
        }
        case AP_CIRCULAR: {
            auto xr = x - ap.xoff, yr = y - ap.yoff;
            discard = (xr * xr + yr * yr) > ap.r2;
            break;
        }
        case AP_ELLIPTICAL: {
            auto xr = x - ap.xoff, yr = y - ap.yoff;
            discard = (xr * xr / ap.h2 + yr * yr / ap.v2) > 1.0;
            break;
        }
        case AP_RECTANGULAR: {
            auto xr = x - ap.xoff, yr = y - ap.yoff;
            discard = (fabs(xr) > 0.5 * ap.width) || (fabs(yr) > 0.5 * ap.height);
            break;
        }
        }
        return discard;
    };
    count_particle(FC_APERTURE, b, decide);
    int nd = 0;
#pragma omp parallel for reduction(+ : nd) schedule(static)
    for (int64_t i = 0; i < b.n_active; ++i) {
        b.discards[i] = 0;
        if (!b.masks[i]) continue;
        const bool discard = decide(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
        if (discard) {
            b.discards[i] = 1;
            b.masks[i] = 0;
            ++nd;
        }
    }
    b.n_valid -= nd;
    return nd;
}

// ---------------------------------------------------------------------------
// FFT (project-written; radix-2 iterative, direct DFT for other lengths).
// Pinned against a direct DFT and numpy.fft by the tests.
// ---------------------------------------------------------------------------
typedef std::complex<double> cplx;

static void fft1d(cplx* a, int n, int sign, std::vector<cplx>& scratch)
{
    if (n <= 1) return;
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) std::swap(a[i], a[j]);
        }
        for (int len = 2; len <= n; len <<= 1) {
            double ang = sign * 2.0 * pc::pi / len;
            for (int k = 0; k < len / 2; ++k) {
                cplx w(std::cos(ang * k), std::sin(ang * k));
                for (int i = 0; i < n; i += len) {
                    cplx u = a[i + k], v = a[i + k + len / 2] * w;
                    a[i + k] = u + v;
                    a[i + k + len / 2] = u - v;
                }
            }
        }
    } else {
        scratch.assign(a, a + n);
        for (int k = 0; k < n; ++k) {
            cplx s(0, 0);
            for (int j = 0; j < n; ++j) {
                double ang = sign * 2.0 * pc::pi * (double)((int64_t)j * k % n) / n;
                s += scratch[j] * cplx(std::cos(ang), std::sin(ang));
            }
            a[k] = s;
        }
    }
}

// In-place 3D complex FFT of a (nz, ny, nx) array, x fastest.  sign=-1 is
// forward (FFTW/cuFFT convention), unnormalised.
static void fft3d(cplx* a, int nx, int ny, int nz, int sign)
{
#pragma omp parallel
    {
        std::vector<cplx> buf, scr;
        buf.resize(std::max(nx, std::max(ny, nz)));
#pragma omp for schedule(static)
        for (int64_t r = 0; r < (int64_t)ny * nz; ++r) fft1d(a + r * nx, nx, sign, scr);
#pragma omp for schedule(static)
        for (int64_t r = 0; r < (int64_t)nx * nz; ++r) {
            int64_t z = r / nx, x = r % nx;
            for (int y = 0; y < ny; ++y) buf[y] = a[(z * ny + y) * nx + x];
            fft1d(buf.data(), ny, sign, scr);
            for (int y = 0; y < ny; ++y) a[(z * ny + y) * nx + x] = buf[y];
        }
#pragma omp for schedule(static)
        for (int64_t r = 0; r < (int64_t)nx * ny; ++r) {
            for (int z = 0; z < nz; ++z) buf[z] = a[z * (int64_t)nx * ny + r];
            fft1d(buf.data(), nz, sign, scr);
            for (int z = 0; z < nz; ++z) a[z * (int64_t)nx * ny + r] = buf[z];
        }
    }
}

// ---------------------------------------------------------------------------
// Space_charge_3d_open_hockney (collective/space_charge_3d_open_hockney.cc)
// ---------------------------------------------------------------------------
struct SCOptions { // simulation/implemented_collective_options.h:67-126
    int shape[3] = {32, 32, 64};
    int doubled_shape[3] = {64, 64, 128};
    double size[3] = {0, 0, 0};
    double offset[3] = {0, 0, 0};
    int green_fn = 1; // 0 pointlike, 1 linear
    int periodic_z = 0;
    double z_period = 0.0;
    int grid_entire_period = 0;
    double n_sigma = 8.0;
    double kick_scale = 1.0;
    int domain_fixed = 0;
};

struct Domain { // rectangular_grid_domain.h:20-36
    int g[3];
    double size[3], offset[3], left[3], h[3];
    void set(const int* shape, const double* sz, const double* off)
    {
        for (int i = 0; i < 3; ++i) {
            g[i] = shape[i];
            size[i] = sz[i];
            offset[i] = off[i];
            left[i] = off[i] - sz[i] / 2.0;
            h[i] = sz[i] / (1.0 * shape[i]);
        }
    }
};

static double smallest_non_tiny(double val, double o1, double o2, double tiny)
{ // space_charge_3d_open_hockney.cc:94-109
    if (val > tiny) return val;
    if (o1 > tiny && o2 > tiny) return std::min(o1, o2);
    return std::max(o1, o2);
}

// collective/utils.h:9-18
template <class R>
inline void leftmost_index_offset(R pos, double left, double inv_cell, int& idx, R& off)
{
    R s = (pos - left) * inv_cell - 0.5;
    idx = (int)std::floor(val(s));
    off = s - idx;
}

struct SC3D {
    SCOptions o;
    Domain dom, ddom;
    int ng = 0; // doubled grid points
    std::vector<cplx> rho, gr, phi; // full complex doubled grids (z, y, x)
    std::vector<double> enx, eny, enz, rho_real, phi_real;
    double fn_norm = 0, last_factor = 0;
    std::array<double, 6> last_mean_std{};

    explicit SC3D(const SCOptions& opt) : o(opt)
    {
        double one[3] = {1, 1, 1}, zero[3] = {0, 0, 0};
        dom.set(o.shape, one, zero);
        ddom.set(o.doubled_shape, one, zero);
        if (o.domain_fixed) {
            double ds[3] = {o.size[0] * 2.0, o.size[1] * 2.0, o.size[2] * 2.0};
            dom.set(o.shape, o.size, o.offset);
            ddom.set(o.doubled_shape, ds, o.offset);
        }
        ng = o.doubled_shape[0] * o.doubled_shape[1] * o.doubled_shape[2];
    }

    void update_domain(Bunch& b)
    { // :494-540 with core_diagnostics.cc:422-460
        if (o.domain_fixed) return;
        auto acc = [](auto* s, auto x, auto y, auto z) {
            s[0] += x; s[1] += y; s[2] += z;
            s[3] += x * x; s[4] += y * y; s[5] += z * z;
        };
        count_particle(FC_DOMAIN, b, [&](auto& x, auto&, auto& y, auto&, auto& z, auto&) {
            CD cs[6];
            acc(cs, x, y, z);
        });
        double s[6] = {0, 0, 0, 0, 0, 0};
        for (int64_t i = 0; i < b.n_active; ++i)
            if (b.masks[i]) acc(s, b.P(i, 0), b.P(i, 2), b.P(i, 4));
        double ms[6];
        for (int j = 0; j < 3; ++j) {
            ms[j] = s[j] / b.n_total;
            ms[j + 3] = std::sqrt(s[j + 3] / b.n_total - std::pow(ms[j], 2));
        }
        for (int j = 0; j < 6; ++j) last_mean_std[j] = ms[j];
        const double tiny = 1.0e-10;
        if (ms[3] < tiny && ms[4] < tiny && ms[5] < tiny)
            throw std::runtime_error("Space_charge_3d_open_hockney_eigen::update_domain: all three spatial dimensions have neglible extent");
        double off[3] = {ms[0], ms[1], ms[2]};
        double sz[3] = {o.n_sigma * smallest_non_tiny(ms[3], ms[4], ms[5], tiny),
                        o.n_sigma * smallest_non_tiny(ms[4], ms[3], ms[5], tiny),
                        o.n_sigma * smallest_non_tiny(ms[5], ms[3], ms[4], tiny)};
        if (o.grid_entire_period) {
            off[2] = 0.0;
            sz[2] = o.z_period;
        }
        double ds[3] = {sz[0] * 2.0, sz[1] * 2.0, sz[2] * 2.0};
        dom.set(o.shape, sz, off);
        ddom.set(o.doubled_shape, ds, off);
    }

    // deposit_charge_rectangular_3d_omp_reduce deposit.cc:853-1031, into a
    // dense (gz, gy, gx) grid; edges excluded (deposit.cc:23-30)
    void deposit(Bunch& b)
    {
        int gx = dom.g[0], gy = dom.g[1], gz = dom.g[2];
        double w0 = (b.real_num / b.n_total) * b.ref.charge * pc::e / (dom.h[0] * dom.h[1] * dom.h[2]);
        double lx = dom.left[0], ly = dom.left[1], lz = dom.left[2];
        double ihx = 1.0 / dom.h[0], ihy = 1.0 / dom.h[1], ihz = 1.0 / dom.h[2];
        int64_t nc = (int64_t)gx * gy * gz;
        rho_real.assign(nc, 0.0);
        int nt = 1;
#ifdef _OPENMP
        nt = omp_get_max_threads();
#endif
        std::vector<double> rl((size_t)nt * nc, 0.0);
        auto ingrid = [&](int ix, int iy, int iz) {
            return ix > 0 && ix < gx - 1 && iy > 0 && iy < gy - 1 && iz > 0 && iz < gz - 1;
        };
        // one particle's CIC weights, add(cell, w) for each interior corner
        auto dep = [&](auto px, auto py, auto pz, auto&& add) {
            int ix, iy, iz;
            decltype(px) ox, oy, oz;
            leftmost_index_offset(px, lx, ihx, ix, ox);
            leftmost_index_offset(py, ly, ihy, iy, oy);
            leftmost_index_offset(pz, lz, ihz, iz, oz);
            int64_t base = (int64_t)iz * gx * gy;
            if (ingrid(ix, iy, iz)) add(base + iy * gx + ix, w0 * (1 - ox) * (1 - oy) * (1 - oz));
            if (ingrid(ix + 1, iy, iz)) add(base + iy * gx + ix + 1, w0 * (ox) * (1 - oy) * (1 - oz));
            if (ingrid(ix, iy + 1, iz)) add(base + (iy + 1) * gx + ix, w0 * (1 - ox) * (oy) * (1 - oz));
            if (ingrid(ix + 1, iy + 1, iz)) add(base + (iy + 1) * gx + ix + 1, w0 * (ox) * (oy) * (1 - oz));
            base = (int64_t)(iz + 1) * gx * gy;
            if (ingrid(ix, iy, iz + 1)) add(base + iy * gx + ix, w0 * (1 - ox) * (1 - oy) * (oz));
            if (ingrid(ix + 1, iy, iz + 1)) add(base + iy * gx + ix + 1, w0 * (ox) * (1 - oy) * (oz));
            if (ingrid(ix, iy + 1, iz + 1)) add(base + (iy + 1) * gx + ix, w0 * (1 - ox) * (oy) * (oz));
            if (ingrid(ix + 1, iy + 1, iz + 1)) add(base + (iy + 1) * gx + ix + 1, w0 * (ox) * (oy) * (oz));
        };
        count_particle(FC_DEPOSIT, b, [&](auto& x, auto&, auto& y, auto&, auto& z, auto&) {
            CD sink; // the grid accumulation: one add per deposited corner
            dep(x, y, z, [&](int64_t, CD w) { sink += w; });
        });
#pragma omp parallel num_threads(nt)
        {
            int it = 0, ntt = 1;
#ifdef _OPENMP
            it = omp_get_thread_num();
            ntt = omp_get_num_threads();
#endif
            int64_t le = b.n_active / ntt;
            int64_t ps = it * le, pe = (it == ntt - 1) ? b.n_active : (it + 1) * le;
            double* r = rl.data() + (size_t)it * nc;
            for (int64_t n = ps; n < pe; ++n) {
                if (!b.masks[n]) continue;
                dep(b.P(n, 0), b.P(n, 2), b.P(n, 4), [&](int64_t c, double w) { r[c] += w; });
            }
        }
#pragma omp parallel for schedule(static)
        for (int64_t c = 0; c < nc; ++c) {
            double w = 0.0;
            for (int n = 0; n < nt; ++n) w += rl[(size_t)n * nc + c];
            rho_real[c] = w;
        }
    }

    // alg_g2_linear :230-348 / alg_g2_pointlike :136-228 into a full complex
    // (dgz, dgy, dgx) grid
    void green(std::vector<cplx>& g2)
    {
        if (o.periodic_z)
            throw std::runtime_error("Space_charge_3d_open_hockney::get_green_fn2: periodic_z not yet implemented");
        const int dgx = ddom.g[0], dgy = ddom.g[1], dgz = ddom.g[2];
        const double hx = ddom.h[0], hy = ddom.h[1], hz = ddom.h[2];
        g2.assign(ng, cplx(0, 0));
        auto at = [&](int z, int y, int x) -> cplx& { return g2[((int64_t)z * dgy + y) * dgx + x]; };
        if (o.green_fn == 0) {
            const int gx = dom.g[0] + 1, gy = dom.g[1] + 1, gz = dom.g[2] + 1;
            double G000 = 2.8 / std::min(hx, std::min(hy, hz));
            for (int iz = 0; iz < gz; ++iz)
                for (int iy = 0; iy < gy; ++iy)
                    for (int ix = 0; ix < gx; ++ix) {
                        double dx = ix * hx, dy = iy * hy, dz = iz * hz;
                        double G = (ix == 0 && iy == 0 && iz == 0) ? G000 : 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
                        int mix = dgx - ix; if (mix == dgx) mix = 0;
                        int miy = dgy - iy; if (miy == dgy) miy = 0;
                        int miz = dgz - iz; if (miz == dgz) miz = 0;
                        at(iz, iy, ix) = G; at(iz, miy, ix) = G; at(iz, iy, mix) = G; at(iz, miy, mix) = G;
                        at(miz, iy, ix) = G; at(miz, miy, ix) = G; at(miz, iy, mix) = G; at(miz, miy, mix) = G;
                    }
            return;
        }
        const int gx0 = dom.g[0], gy0 = dom.g[1], gz0 = dom.g[2];
        double rr0 = hx * hx + hy * hy;
        double r10 = std::sqrt(hx * hx + hy * hy + hz * hz);
        double G000 = (2.0 / rr0) * (hz * r10 + rr0 * std::log((hz + r10) / std::sqrt(rr0)) - hz * hz);
        const double epsz = 1e-12 * hz;
        for (int iz = 0; iz < dgz; ++iz)
            for (int iy = 0; iy <= gy0; ++iy)
                for (int ix = 0; ix <= gx0; ++ix) {
                    double z = (iz > gz0) ? (dgz - iz) * hz : iz * hz;
                    double y = iy * hy, x = ix * hx;
                    double rr = x * x + y * y;
                    double s0 = std::sqrt(rr + z * z);
                    double sn = std::sqrt(rr + (z - hz) * (z - hz));
                    double sp = std::sqrt(rr + (z + hz) * (z + hz));
                    double G = 2.0 * s0 - sn - sp;
                    double T1, T2, r1, r2;
                    if (z < -hz) {
                        r1 = (sn - z + hz) / (s0 - z);
                        T1 = (hz - z) * std::log(r1);
                        r2 = (s0 - z) / (sp - z - hz);
                        T2 = (hz + z) * std::log(r2);
                        G += T1 + T2;
                    } else if (std::abs(z + hz) < epsz) {
                        r1 = (sn - z + hz) / (s0 - z);
                        T1 = (hz - z) * std::log(r1);
                        G += T1;
                    } else if (std::abs(z) < epsz) {
                        if (std::abs(x) + std::abs(y) < 2. * epsz) {
                            G += hz * G000;
                        } else {
                            r1 = (std::sqrt(hz * hz + rr) + hz) / std::sqrt(rr);
                            G += 2.0 * hz * std::log(r1);
                        }
                    } else if (std::abs(z - hz) < epsz) {
                        r1 = (sp + z + hz) / (s0 + z);
                        T1 = (hz + z) * std::log(r1);
                        G += T1;
                    } else if (z > hz) {
                        r1 = (s0 + z) / (sn + z - hz);
                        T1 = (hz - z) * std::log(r1);
                        r2 = (sp + z + hz) / (s0 + z);
                        T2 = (hz + z) * std::log(r2);
                        G += T1 + T2;
                    }
                    int miy = dgy - iy, mix = dgx - ix;
                    if (mix == dgx) mix = 0;
                    if (miy == dgy) miy = 0;
                    at(iz, iy, ix) = G;
                    if (iy != gy0) {
                        at(iz, miy, ix) = G;
                        if (ix != gx0) at(iz, miy, mix) = G;
                    }
                    if (ix != gx0) at(iz, iy, mix) = G;
                }
    }

    // get_local_phi2 :642-676, get_normalization_force :708-735,
    // alg_force_extractor_doubled_domain space_charge_3d_kernels.h:217-307
    void solve()
    {
        const int dgx = ddom.g[0], dgy = ddom.g[1], dgz = ddom.g[2];
        const int gx = dom.g[0], gy = dom.g[1], gz = dom.g[2];
        rho.assign(ng, cplx(0, 0));
        for (int z = 0; z < gz; ++z)
            for (int y = 0; y < gy; ++y)
                for (int x = 0; x < gx; ++x)
                    rho[((int64_t)z * dgy + y) * dgx + x] = rho_real[((int64_t)z * gy + y) * gx + x];
        green(gr);
        fft3d(rho.data(), dgx, dgy, dgz, -1);
        fft3d(gr.data(), dgx, dgy, dgz, -1);
        phi.resize(ng);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < ng; ++i) {
            double ar = rho[i].real(), ai = rho[i].imag(), br = gr[i].real(), bi = gr[i].imag();
            phi[i] = cplx(ar * br - ai * bi, ar * bi + ai * br);
        }
        fft3d(phi.data(), dgx, dgy, dgz, +1);
        double hx = dom.h[0], hy = dom.h[1], hz = dom.h[2];
        double norm = hx * hy * hz;
        norm *= 1.0 / (4.0 * pc::pi * pc::epsilon0);
        norm *= 1.0;
        if (o.green_fn == 1) norm *= 1.0 / (hz * hz);
        norm *= 1.0 / (dgx * dgy * dgz);
        fn_norm = norm;
        phi_real.assign((int64_t)gx * gy * gz, 0.0);
        for (int z = 0; z < gz; ++z)
            for (int y = 0; y < gy; ++y)
                for (int x = 0; x < gx; ++x)
                    phi_real[((int64_t)z * gy + y) * gx + x] = phi[((int64_t)z * dgy + y) * dgx + x].real();
        int64_t G = (int64_t)gx * gy * gz;
        enx.assign(G, 0.0);
        eny.assign(G, 0.0);
        enz.assign(G, 0.0);
        double ihx = 0.5 / ddom.h[0], ihy = 0.5 / ddom.h[1], ihz = 0.5 / ddom.h[2];
        auto ph = [&](int z, int y, int x) { return phi[((int64_t)z * dgy + y) * dgx + x].real(); };
#pragma omp parallel for schedule(static)
        for (int iz = 1; iz < gz - 1; ++iz)
            for (int iy = 1; iy < gy - 1; ++iy)
                for (int ix = 1; ix < gx - 1; ++ix) {
                    int64_t i = ((int64_t)iz * gy + iy) * gx + ix;
                    enx[i] = -(ph(iz, iy, ix + 1) - ph(iz, iy, ix - 1)) * ihx;
                    eny[i] = -(ph(iz, iy + 1, ix) - ph(iz, iy - 1, ix)) * ihy;
                    enz[i] = -(ph(iz + 1, iy, ix) - ph(iz - 1, iy, ix)) * ihz;
                }
    }

    // apply_kick :753-784 + zyx::alg_kicker space_charge_3d_kernels.h:91-215
    void kick(Bunch& b, double time_step)
    {
        double q = b.ref.charge * pc::e;
        double m = b.ref.mass;
        double gamma = b.ref.gamma, beta = b.ref.beta, pref = b.ref.p;
        double unit_conversion = pc::c / (1e9 * pc::e);
        double factor = o.kick_scale * unit_conversion * q * time_step * fn_norm / (pref * gamma * gamma * beta);
        last_factor = factor;
        const int gx = dom.g[0], gy = dom.g[1], gz = dom.g[2];
        double ihx = 1.0 / dom.h[0], ihy = 1.0 / dom.h[1], ihz = 1.0 / dom.h[2];
        double lx = dom.left[0], ly = dom.left[1], lz = dom.left[2];
        auto body = [&](auto& x, auto& xp, auto& y, auto& yp, auto& cdt, auto& dpop) {
            typedef std::remove_reference_t<decltype(x)> R;
            int ix, iy, iz;
            R ox, oy, oz;
            leftmost_index_offset(x, lx, ihx, ix, ox);
            leftmost_index_offset(y, ly, ihy, iy, oy);
            leftmost_index_offset(cdt, lz, ihz, iz, oz);
            R aox = 1.0 - ox, aoy = 1.0 - oy, aoz = 1.0 - oz;
            if (!((ix >= 0 && ix < gx - 1) && (iy >= 0 && iy < gy - 1) && (iz >= 0 && iz < gz - 1))) return;
            auto interp = [&](const std::vector<double>& e) {
                int64_t base = ((int64_t)iz * gy + iy) * gx + ix;
                R a = aoz * aoy * aox * e[base];
                a += aoz * aoy * ox * e[base + 1];
                a += aoz * oy * aox * e[base + gx];
                a += aoz * oy * ox * e[base + gx + 1];
                base = ((int64_t)(iz + 1) * gy + iy) * gx + ix;
                a += oz * aoy * aox * e[base];
                a += oz * aoy * ox * e[base + 1];
                a += oz * oy * aox * e[base + gx];
                a += oz * oy * ox * e[base + gx + 1];
                return a;
            };
            R v = interp(enz);
            R p = pref + dpop * pref;
            R Eoc_i = sqrt(p * p + m * m);
            R Eoc_f = Eoc_i + factor * (-pref) * v;
            R ddp = (sqrt(Eoc_f * Eoc_f - m * m) - sqrt(Eoc_i * Eoc_i - m * m)) / pref;
            dpop += ddp;
            v = interp(eny);
            yp += factor * v;
            v = interp(enx);
            xp += factor * v;
        };
        count_particle(FC_KICK, b, body);
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < b.n_active; ++i)
            if (b.masks[i]) body(b.P(i, 0), b.P(i, 1), b.P(i, 2), b.P(i, 3), b.P(i, 4), b.P(i, 5));
    }

    void apply(Bunch& b, double time_step)
    { // apply_bunch :423-453
        if (!o.domain_fixed) update_domain(b);
        deposit(b);
        solve();
        kick(b, time_step);
    }
};

// ---------------------------------------------------------------------------
// Steps and operators: split_operator_stepper.cc, independent_operator.cc,
// independent_stepper_elements.cc, split_operator_stepper_elements.cc, step.cc
// ---------------------------------------------------------------------------
struct IndepOp {
    std::vector<Slice> slices;
    // operations: 'L' = libff group, 'A' = aperture
    struct Opn {
        char kind;
        std::vector<Slice> group;
        Aperture ap;
    };
    std::vector<Opn> ops;

    void create_operations()
    { // independent_operator.cc:25-91
        ops.clear();
        std::string aperture_type;
        bool need_left = false, need_right = false;
        std::string extractor_type, last_extractor_type;
        std::vector<Slice> group;
        for (auto const& slice : slices) {
            const Element& el = *slice.e;
            if (el.has_s("aperture_type")) {
                aperture_type = el.gets("aperture_type", "");
                need_left = slice.ledge;
                need_right = slice.redge;
            } else {
                need_left = need_right = false;
            }
            extractor_type = el.gets("extractor_type", "default");
            if (extractor_type != "default" && extractor_type != "libff")
                throw std::runtime_error("unknown extractor_type: " + extractor_type);
            if (((extractor_type != last_extractor_type) || need_left) && !group.empty()) {
                ops.push_back({'L', group, {}});
                group.clear();
            }
            if (need_left) ops.push_back({'A', {}, make_aperture(aperture_type, slice)});
            group.push_back(slice);
            last_extractor_type = extractor_type;
            if (need_right) {
                ops.push_back({'L', group, {}});
                ops.push_back({'A', {}, make_aperture(aperture_type, slice)});
                group.clear();
            }
        }
        if (!group.empty()) ops.push_back({'L', group, {}});
        ops.push_back({'A', {}, make_aperture("finite", slices.back())});
        ops.push_back({'A', {}, make_aperture("circular", slices.back())});
    }

    void apply(Bunch& b, std::vector<int64_t>& lost_per_step)
    {
        for (auto& op : ops) {
            if (op.kind == 'L') {
                for (auto& s : op.group) element_apply(s, b);
            } else {
                int nd = aperture_apply(op.ap, b);
                lost_per_step.push_back(nd);
            }
        }
        b.update_total_num();
    }
};

struct Step {
    double length = 0;
    // sequence of operators: 'I' independent, 'C' collective
    std::vector<char> kinds;
    std::vector<IndepOp> indeps;
};

template <typename IT>
static std::vector<Slice> fixed_step_slices(IT& it, const IT& end, double& left, double step_length,
                                            double& offset_fudge)
{ // split_operator_stepper.cc:14-82 (force_diagnostics not supported)
    const double tol = 1.0e-8;
    std::vector<Slice> slices;
    double length = offset_fudge;
    bool complete = false;
    while (!complete) {
        double right = it->length();
        if (length + (right - left) - tol <= step_length) {
            Slice slice(*it, left, right);
            slices.push_back(slice);
            length += (right - left);
            ++it;
            left = 0.0;
            if (std::abs(length - step_length) < tol) {
                if ((it == end) || (it->length() != 0.0)) complete = true;
            } else {
                if (it == end) throw std::runtime_error("get_step stepped beyond end of lattice");
            }
        } else {
            bool end_within_error = false;
            double old_right = right;
            right = step_length - length + left;
            if (std::abs(old_right - right) < tol) {
                right = old_right;
                end_within_error = true;
            }
            Slice slice(*it, left, right);
            slices.push_back(slice);
            length += (right - left);
            if (end_within_error) {
                ++it;
                left = 0.0;
            } else {
                left = right;
            }
            complete = true;
        }
    }
    offset_fudge = length - step_length;
    return slices;
}

enum { STEPPER_SPLIT = 0, STEPPER_SPLIT_ELEMENTS = 1, STEPPER_INDEP_ELEMENTS = 2 };

static std::vector<Step> make_steps(const Lattice& lat, int kind, int num, bool has_collective)
{
    std::vector<Step> steps;
    auto add_indep = [](Step& st, std::vector<Slice> sl) {
        IndepOp op;
        op.slices = std::move(sl);
        op.create_operations();
        st.kinds.push_back('I');
        st.indeps.push_back(std::move(op));
    };
    if (kind == STEPPER_SPLIT) {
        // split_operator_stepper.cc:132-261 (no force_diagnostics)
        double step_length = lat.length() / num;
        double half = 0.5 * step_length;
        auto it = lat.elements.begin();
        auto end = lat.elements.end();
        if (it == end) return steps;
        double left = 0.0, fudge = 0.0;
        for (int i = 0; i < num; ++i) {
            auto s1 = fixed_step_slices(it, end, left, half, fudge);
            auto s2 = fixed_step_slices(it, end, left, half, fudge);
            Step st;
            st.length = step_length;
            add_indep(st, s1);
            if (has_collective) st.kinds.push_back('C');
            add_indep(st, s2);
            steps.push_back(std::move(st));
        }
        if (it != end)
            throw std::runtime_error("internal error: split_operator_stepper did not make it to the end of the lattice\n");
    } else {
        if (num < 1) throw std::runtime_error("Split_operator_stepper_elements: steps_per_element must be >= 1");
        for (auto const& ele : lat.elements) {
            double length = ele.length();
            if (length == 0.0) {
                Step st;
                st.length = 0.0;
                add_indep(st, {Slice(ele)});
                steps.push_back(std::move(st));
                continue;
            }
            double sl = length / num;
            for (int i = 0; i < num; ++i) {
                double left = i * sl, right = (i + 1) * sl;
                Step st;
                st.length = sl;
                if (kind == STEPPER_INDEP_ELEMENTS) {
                    add_indep(st, {Slice(ele, left, right)});
                } else {
                    double middle = left + 0.5 * sl;
                    add_indep(st, {Slice(ele, left, middle)});
                    if (has_collective) st.kinds.push_back('C');
                    add_indep(st, {Slice(ele, middle, right)});
                }
                steps.push_back(std::move(st));
            }
        }
    }
    return steps;
}

struct Sim {
    Lattice lat;
    Bunch b;
    std::vector<Step> steps;
    std::unique_ptr<SC3D> sc;
    bool started = false;
    std::vector<int64_t> losses;

    void propagate(int turns)
    { // propagator.cc:157-283 (single bunch, no diagnostics)
        if (!started) {
            b.design = lat.ref; // do_before_start: set_lattice_reference_particle
            started = true;
        }
        for (int t = 0; t < turns; ++t) {
            b.ref.s_n = 0.0;
            for (auto& st : steps) {
                if (b.n_active == 0) throw std::runtime_error("Step::apply() unable to proceed. no bunch in the simulator");
                double time = st.length / (b.ref.beta * pc::c); // step.cc:44-53
                size_t ii = 0;
                for (char k : st.kinds) {
                    if (k == 'I')
                        st.indeps[ii++].apply(b, losses);
                    else if (sc)
                        sc->apply(b, time * 1.0);
                }
            }
        }
    }
};

} // namespace orc

// ===========================================================================
// C API used by the tests (ctypes)
// ===========================================================================
using namespace orc;

#define ORC_TRY try {
#define ORC_CATCH                                                                                  \
    }                                                                                              \
    catch (std::exception & ex)                                                                    \
    {                                                                                              \
        g_err = ex.what();                                                                         \
        return 1;                                                                                  \
    }                                                                                              \
    return 0;

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

int orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Reference particle given as (charge, mass, value, kind) with kind 0 =
// total energy, 1 = momentum, 2 = kinetic energy [GeV].
void* orc_lattice_new(int charge, double mass, double value, int kind)
{
    auto* L = new Lattice();
    L->ref.charge = charge;
    L->ref.mass = mass;
    L->ref.set_by(kind, value);
    return L;
}
void orc_lattice_free(void* l) { delete (Lattice*)l; }
int orc_lattice_append(void* l, const char* type, const char* name)
{
    auto* L = (Lattice*)l;
    Element e;
    e.type = type;
    e.name = name;
    L->elements.push_back(e);
    return (int)L->elements.size() - 1;
}
void orc_lattice_set_double(void* l, int idx, const char* k, double v) { ((Lattice*)l)->elements[idx].d[k] = v; }
void orc_lattice_set_string(void* l, int idx, const char* k, const char* v) { ((Lattice*)l)->elements[idx].s[k] = v; }
void orc_lattice_set_vector(void* l, int idx, const char* k, const double* v, int n)
{
    ((Lattice*)l)->elements[idx].v[k] = std::vector<double>(v, v + n);
}
double orc_lattice_length(void* l) { return ((Lattice*)l)->length(); }

// Bunch reference particle given by (charge, mass, value, kind) as for
// orc_lattice_new; sc_opts may be NULL (no collective operator).
int orc_sim_new(void* lattice, int stepper_kind, int num, const SCOptions* sc_opts, int charge,
                double mass, double value, int kind, int64_t n, double real_num, void** out)
{
    ORC_TRY
    auto* s = new Sim();
    s->lat = *(Lattice*)lattice;
    s->b.ref.charge = charge;
    s->b.ref.mass = mass;
    s->b.ref.set_by(kind, value);
    s->b.n_active = s->b.n_valid = s->b.n_total = (int)n;
    s->b.cap = n;
    s->b.real_num = real_num;
    s->b.parts.assign(7 * n, 0.0);
    for (int64_t i = 0; i < n; ++i) s->b.P(i, 6) = (double)i;
    s->b.masks.assign(n, 1);
    s->b.discards.assign(n, 0);
    if (sc_opts) s->sc.reset(new SC3D(*sc_opts));
    s->steps = make_steps(s->lat, stepper_kind, num, sc_opts != nullptr);
    *out = s;
    ORC_CATCH
}
void orc_sim_free(void* s) { delete (Sim*)s; }
int orc_sim_num_steps(void* s) { return (int)((Sim*)s)->steps.size(); }

// Step structure: returns per step the list of slices (element index, left,
// right) so the tests can compare slicing with the product.
int orc_sim_step_slices(void* sp, int step, int op, double* out, int cap)
{
    auto* s = (Sim*)sp;
    auto& st = s->steps[step];
    if (op >= (int)st.indeps.size()) return -1;
    auto& sl = st.indeps[op].slices;
    int n = 0;
    for (auto& x : sl) {
        if (n >= cap) break;
        out[n * 3 + 0] = (double)(x.e - s->lat.elements.data());
        out[n * 3 + 1] = x.left;
        out[n * 3 + 2] = x.right;
        ++n;
    }
    return n;
}

int orc_sim_set_particles(void* sp, const double* parts, const uint8_t* masks)
{
    auto* s = (Sim*)sp;
    auto& b = s->b;
    std::memcpy(b.parts.data(), parts, sizeof(double) * 7 * b.cap);
    int nv = 0;
    for (int64_t i = 0; i < b.n_active; ++i) {
        b.masks[i] = masks ? masks[i] : 1;
        nv += b.masks[i] ? 1 : 0;
    }
    b.n_valid = b.n_total = nv;
    return 0;
}
int orc_sim_get_particles(void* sp, double* parts, uint8_t* masks, uint8_t* discards)
{
    auto* s = (Sim*)sp;
    auto& b = s->b;
    std::memcpy(parts, b.parts.data(), sizeof(double) * 7 * b.cap);
    if (masks) std::memcpy(masks, b.masks.data(), b.n_active);
    if (discards) std::memcpy(discards, b.discards.data(), b.n_active);
    return 0;
}
int orc_sim_counts(void* sp, int* n_valid, int* n_total, double* real_num)
{
    auto* s = (Sim*)sp;
    *n_valid = s->b.n_valid;
    *n_total = s->b.n_total;
    *real_num = s->b.real_num;
    return 0;
}
int orc_sim_design_state(void* sp, double* state6, double* s_n)
{
    auto* s = (Sim*)sp;
    for (int i = 0; i < 6; ++i) state6[i] = s->b.design.state[i];
    *s_n = s->b.ref.s_n;
    return 0;
}
int orc_sim_propagate(void* sp, int turns)
{
    ORC_TRY((Sim*)sp)->propagate(turns);
    ORC_CATCH
}
int orc_sim_propagate_steps(void* sp, int first, int count)
{ // partial turn (bench CPU sample): steps [first, first+count)
    ORC_TRY
    auto* s = (Sim*)sp;
    if (!s->started) {
        s->b.design = s->lat.ref;
        s->started = true;
    }
    for (int k = first; k < first + count; ++k) {
        auto& st = s->steps[k % s->steps.size()];
        double time = st.length / (s->b.ref.beta * pc::c);
        size_t ii = 0;
        for (char kk : st.kinds) {
            if (kk == 'I')
                st.indeps[ii++].apply(s->b, s->losses);
            else if (s->sc)
                s->sc->apply(s->b, time);
            g_flops.mark(k, kk);
        }
    }
    ORC_CATCH
}

// LibFF_operation::apply_impl (simulation/independent_operation.h:45-60) on
// explicit slices of the Sim's lattice: triples (element index, left, right),
// each through FF_element::apply (ff_element.h:25-67) in order.  The design
// reference particle starts from the lattice's on first use, as
// Propagator::do_before_start sets it.
int orc_sim_libff_apply(void* sp, const double* slices, int nslices)
{
    ORC_TRY
    auto* s = (Sim*)sp;
    if (!s->started) {
        s->b.design = s->lat.ref;
        s->started = true;
    }
    for (int i = 0; i < nslices; ++i) {
        const int ei = (int)slices[3 * i];
        if (ei < 0 || ei >= (int)s->lat.elements.size()) throw std::runtime_error("slice element out of range");
        element_apply(Slice(s->lat.elements[ei], slices[3 * i + 1], slices[3 * i + 2]), s->b);
    }
    ORC_CATCH
}

// Aperture_operation<AP>::apply_impl (simulation/aperture_operation.h:14-24)
// with the attributes of element `index` (operation_extractor.cc:55-75):
// Bunch::apply_aperture alone, so n_valid drops by the discards and n_total
// is left to the next update_total_num.
int orc_sim_aperture_apply(void* sp, int index, const char* type, int* ndiscarded)
{
    ORC_TRY
    auto* s = (Sim*)sp;
    if (index < 0 || index >= (int)s->lat.elements.size()) throw std::runtime_error("element index out of range");
    const Slice whole(s->lat.elements[index]);
    *ndiscarded = aperture_apply(make_aperture(type, whole), s->b);
    ORC_CATCH
}

// Operation counting (see FlopState): counts the algorithmic FP64 work of
// particle `index` through the oracle's own particle code while the Sim
// runs as usual; one record per operator of each step run.
int orc_flops_begin(int64_t index)
{
    g_flops = FlopState();
    g_flops.on = true;
    g_flops.index = index;
    return 0;
}
int orc_flops_end(int* uncounted)
{
    g_flops.on = false;
    *uncounted = g_flops.uncounted ? 1 : 0;
    return (int)g_flops.records.size();
}
// record r: its step and operator kind ('I' or 'C'), counts[FC_N][FO_N]
int orc_flops_record(int r, int* step, int* kind, int64_t* counts)
{
    if (r < 0 || r >= (int)g_flops.records.size()) return 1;
    const auto& rec = g_flops.records[r];
    *step = rec.step;
    *kind = rec.kind;
    std::memcpy(counts, rec.n, sizeof(rec.n));
    return 0;
}

// Last space-charge solve of a Sim: domain (left[3], h[3]), rho, phi and E on
// the original grid (gz, gy, gx), and fn_norm / kick factor.
int orc_sim_sc_last(void* sp, double* left, double* h, double* rho, double* phi, double* ex, double* ey,
                    double* ez, double* scalars)
{
    auto* s = (Sim*)sp;
    if (!s->sc) return 1;
    auto& sc = *s->sc;
    for (int i = 0; i < 3; ++i) {
        left[i] = sc.dom.left[i];
        h[i] = sc.dom.h[i];
    }
    size_t G = sc.rho_real.size();
    if (rho) std::memcpy(rho, sc.rho_real.data(), G * 8);
    if (phi) std::memcpy(phi, sc.phi_real.data(), G * 8);
    if (ex) std::memcpy(ex, sc.enx.data(), G * 8);
    if (ey) std::memcpy(ey, sc.eny.data(), G * 8);
    if (ez) std::memcpy(ez, sc.enz.data(), G * 8);
    if (scalars) {
        scalars[0] = sc.fn_norm;
        scalars[1] = sc.last_factor;
        for (int j = 0; j < 6; ++j) scalars[2 + j] = sc.last_mean_std[j];
    }
    return 0;
}

// One standalone space-charge kick on host particle arrays (the collective
// operator alone, as the reference's own SC tests drive it).
int orc_sc_apply(const SCOptions* opts, int charge, double mass, double value, int kind, int64_t n,
                 double real_num, int n_total, double* parts, const uint8_t* masks, double time_step,
                 double* left, double* h, double* rho, double* phi, double* ex, double* ey, double* ez,
                 double* scalars)
{
    ORC_TRY
    Bunch b;
    b.ref.charge = charge;
    b.ref.mass = mass;
    b.ref.set_by(kind, value);
    b.n_active = (int)n;
    b.cap = n;
    b.parts.assign(parts, parts + 7 * n);
    b.masks.assign(n, 1);
    int nv = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (masks) b.masks[i] = masks[i];
        nv += b.masks[i] ? 1 : 0;
    }
    b.n_valid = nv;
    b.n_total = n_total > 0 ? n_total : nv;
    b.real_num = real_num;
    SC3D sc(*opts);
    sc.apply(b, time_step);
    std::memcpy(parts, b.parts.data(), sizeof(double) * 7 * n);
    for (int i = 0; i < 3; ++i) {
        left[i] = sc.dom.left[i];
        h[i] = sc.dom.h[i];
    }
    size_t G = sc.rho_real.size();
    if (rho) std::memcpy(rho, sc.rho_real.data(), G * 8);
    if (phi) std::memcpy(phi, sc.phi_real.data(), G * 8);
    if (ex) std::memcpy(ex, sc.enx.data(), G * 8);
    if (ey) std::memcpy(ey, sc.eny.data(), G * 8);
    if (ez) std::memcpy(ez, sc.enz.data(), G * 8);
    if (scalars) {
        scalars[0] = sc.fn_norm;
        scalars[1] = sc.last_factor;
        for (int j = 0; j < 6; ++j) scalars[2 + j] = sc.last_mean_std[j];
    }
    ORC_CATCH
}

// Deposit alone into a dense (gz, gy, gx) grid for a given domain.
int orc_deposit(const int* shape, const double* size, const double* offset, int charge, double real_num,
                int n_total, int64_t n, const double* parts, const uint8_t* masks, double* rho_out)
{
    ORC_TRY
    SCOptions o;
    for (int i = 0; i < 3; ++i) {
        o.shape[i] = shape[i];
        o.doubled_shape[i] = 2 * shape[i];
        o.size[i] = size[i];
        o.offset[i] = offset[i];
    }
    o.domain_fixed = 1;
    SC3D sc(o);
    Bunch b;
    b.ref.charge = charge;
    b.n_active = (int)n;
    b.cap = n;
    b.parts.assign(parts, parts + 7 * n);
    b.masks.assign(n, 1);
    if (masks) std::memcpy(b.masks.data(), masks, n);
    b.n_total = n_total;
    b.real_num = real_num;
    sc.deposit(b);
    std::memcpy(rho_out, sc.rho_real.data(), sc.rho_real.size() * 8);
    ORC_CATCH
}

// The oracle FFT on a (nz, ny, nx) complex array (interleaved re/im).
int orc_fft3d(double* data, int nx, int ny, int nz, int sign)
{
    fft3d((cplx*)data, nx, ny, nz, sign);
    return 0;
}

// Green function on the full doubled grid (real part), for a given domain.
int orc_green(const int* shape, const int* dshape, const double* size, int green_fn, double* out)
{
    ORC_TRY
    SCOptions o;
    for (int i = 0; i < 3; ++i) {
        o.shape[i] = shape[i];
        o.doubled_shape[i] = dshape[i];
        o.size[i] = size[i];
        o.offset[i] = 0;
    }
    o.green_fn = green_fn;
    o.domain_fixed = 1;
    SC3D sc(o);
    std::vector<cplx> g;
    sc.green(g);
    for (size_t i = 0; i < g.size(); ++i) out[i] = g[i].real();
    ORC_CATCH
}

} // extern "C"
