// Host runtime of the B200 space-charge + tracking step and its C ABI
// (include/sb2.h).
//
// What lives here: reference-particle kinematics, the lattice and its
// slicing by the three steppers, the host half of every libFF element map
// (attribute lookup, strength scaling and design-reference-particle
// propagation, done exactly as the reference does on the host), the fused
// pass executor that turns one step into device launches, and the
// space-charge operator's workspaces.
//
// Compiled with -ffp-contract=off: the host-side design-particle arithmetic
// must round exactly as the reference's (no -ffast-math is in effect there,
// CMakeLists.txt:338).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <array>
#include <cmath>
#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sb2.h"
#include "sb2_kernels.h"

namespace sb2 {

// ---------------------------------------------------------------------------
// constants: foundation/physical_constants.h (PDG 2012)
// ---------------------------------------------------------------------------
namespace pc {
constexpr double pi = 3.14159265358979323846;
constexpr double c = 299792458.0;
constexpr double e = 1.602176565e-19;
} // namespace pc

struct Error : std::runtime_error {
    sb2_status code;
    Error(sb2_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

static void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        cudaGetLastError(); // clear a non-sticky error so later launch checks do not see it
        throw Error(e == cudaErrorMemoryAllocation ? SB2_ERR_NOMEM : SB2_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e));
    }
}

// Device memory comes from the stream-ordered allocator.  Objects are freed
// only at rest (no kernel of theirs in flight: every propagate, batch job
// and operator call ends by synchronising its own stream), so a free is
// ordered on the legacy stream and never waits for the device as cudaFree
// would -- a request loop retiring one job does not stall the jobs still
// running on other streams.
template <typename T>
static T* dalloc(size_t count, const char* what)
{
    void* p = nullptr;
    cuda_check(cudaMallocAsync(&p, std::max<size_t>(count, 1) * sizeof(T), 0), what);
    cuda_check(cudaStreamSynchronize(0), what);
    return (T*)p;
}
static void dfree(void* p)
{
    if (p) cudaFreeAsync(p, 0);
}

// ---------------------------------------------------------------------------
// Reference particle (foundation/four_momentum.cc, reference_particle.cc)
// ---------------------------------------------------------------------------
struct Refpart {
    int charge = 1;
    double mass = 0.938272046;
    double gamma = 1, beta = 0, p = 0, energy = 0;
    std::array<double, 6> state{0, 0, 0, 0, 0, 0};
    double s = 0, s_n = 0;
    int repetition = 0;

    void set_gamma(double g)
    { // four_momentum.cc:8-16
        if (g < 1.0) throw Error(SB2_ERR_INVALID, "Four_momentum: gamma not >= 1.0");
        gamma = g;
        energy = gamma * mass;
        beta = std::sqrt(1.0 - 1.0 / (gamma * gamma));
        p = gamma * beta * mass;
    }
    void set(int chg, double m, double value, int kind)
    {
        charge = chg;
        mass = m;
        if (kind == SB2_REF_TOTAL_ENERGY)
            set_gamma(value / mass);
        else if (kind == SB2_REF_KINETIC_ENERGY)
            set_gamma((mass + value) / mass);
        else if (kind == SB2_REF_MOMENTUM) { // four_momentum.cc:90-110
            double r2 = value * value / (mass * mass);
            double b = std::sqrt(r2 / (1 + r2));
            if ((b < 0.0) || (b >= 1.0))
                throw Error(SB2_ERR_INVALID, "Four_momentum: beta not in range 0.0 <= beta < 1.0");
            set_gamma(1.0 / std::sqrt(1.0 - b * b));
        } else
            throw Error(SB2_ERR_INVALID, "unknown reference particle kind");
    }
    void start_repetition()
    { // reference_particle.cc:231-237
        if (s == 0.0) s = s_n;
        if (s_n > 0.0) repetition += 1;
        s_n = 0.0;
    }
};

// ---------------------------------------------------------------------------
// Lattice (lattice/lattice_element.h, lattice.cc)
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
            throw Error(SB2_ERR_RUNTIME, "Lattice_element::get_double_attribute: element " + name +
                                             " of type " + type + " has no double attribute '" + k + "'");
        return it->second;
    }
    bool has(const std::string& k) const { return d.count(k) > 0; }
    bool has_string(const std::string& k) const { return s.count(k) > 0; }
    std::string get_string(const std::string& k, const std::string& def) const
    {
        auto it = s.find(k);
        return it == s.end() ? def : it->second;
    }
    double length() const { return get("l", 0.0); }
};

struct Lattice {
    std::string name;
    std::vector<Element> elements;
    Refpart ref;
    bool has_ref = false;
    // device copies of the second-order tensors of matrix elements (216
    // doubles each), by element index; made with the propagator
    std::map<int, std::shared_ptr<double>> matrix_tensors;

    double length() const
    { // lattice.cc:195-201
        double L = 0.0;
        for (auto const& e : elements) L += e.length();
        return L;
    }
};

// lattice_element_slice.cc:9-47
struct Slice {
    int elem = -1;
    double left = 0, right = 0;
    bool ledge = true, redge = true;
};

static Slice make_slice(const Lattice& lat, int ei, double l, double r)
{
    const double tol = 1.0e-9;
    Slice s;
    s.elem = ei;
    s.left = l;
    s.right = r;
    if (l < 0.0) throw Error(SB2_ERR_RUNTIME, "Lattice_element_slice: left must be >= 0.0");
    if (l < tol) {
        s.ledge = true;
        s.left = 0.0;
    } else
        s.ledge = false;
    double L = lat.elements[ei].length();
    if (r > L + tol)
        throw Error(SB2_ERR_RUNTIME,
                    "Lattice_element_slice: right must be no greater than the length of the element");
    bool eq = (std::abs(r) < tol) ? (std::abs(r - L) < tol) : (std::abs((r - L) / r) < tol); // floating_point_equal
    if (eq) {
        s.redge = true;
        s.right = L;
    } else
        s.redge = false;
    return s;
}

static Slice whole_slice(const Lattice& lat, int ei)
{
    Slice s;
    s.elem = ei;
    s.left = 0;
    s.right = lat.elements[ei].length();
    s.ledge = s.redge = true;
    return s;
}

// ---------------------------------------------------------------------------
// Host copies of the libFF units used for the design reference particle
// (ff_algorithm.h; same operation order)
// ---------------------------------------------------------------------------
namespace hostff {
inline bool close_to_zero(double v) { return std::fabs(v) < 1e-13; }

inline void drift_unit(double& x, double xp, double& y, double yp, double& cdt, double dpop, double length,
                       double ref_p, double m, double ref_cdt)
{
    const double uni = 1.0;
    const double sig = (double)((0.0 < length) - (length < 0.0));
    double dp = dpop + uni;
    double inv_npz = uni / std::sqrt(dp * dp - xp * xp - yp * yp);
    double lxpr = xp * length * inv_npz;
    double lypr = yp * length * inv_npz;
    double D2 = lxpr * lxpr + length * length + lypr * lypr;
    double p = dp * ref_p;
    double E2 = p * p + m * m;
    double ibeta2 = E2 / (p * p);
    x = x + lxpr;
    y = y + lypr;
    cdt = cdt + sig * std::sqrt(D2 * ibeta2) - ref_cdt;
}
inline void thin_quad(double x, double& xp, double y, double& yp, const double* k)
{
    xp = xp - k[0] * x + k[1] * y;
    yp = yp + k[0] * y + k[1] * x;
}
inline void thin_sext(double x, double& xp, double y, double& yp, const double* k)
{
    xp = xp - 0.5 * k[0] * (x * x - y * y) + k[1] * x * y;
    yp = yp + k[0] * x * y + 0.5 * k[1] * (x * x - y * y);
}
inline void thin_oct(double x, double& xp, double y, double& yp, const double* k)
{
    const double n1 = 0.5, n2 = 1.0 / 3.0;
    xp = xp - n1 * k[0] * (x * x * x * n2 - x * y * y) + n1 * k[1] * (x * x * y - y * y * y * n2);
    yp = yp - n1 * k[0] * (y * y * y * n2 - x * x * y) + n1 * k[1] * (x * x * x * n2 - x * y * y);
}
inline double factorial(int n)
{
    if (n == 0) return 1.0;
    double r = 1;
    for (int i = 1; i <= n; ++i) r *= i;
    return r;
}
inline double qpow(double x, int i)
{
    double r = 1;
    while (i--) r = r * x;
    return r;
}
inline void thin_magnet(double x, double& xp, double y, double& yp, const double* kL, int n)
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
inline void cf_kick(double x, double& xp, double y, double& yp, const double* kL)
{ // ff_quadrupole.h:22-35
    thin_quad(x, xp, y, yp, kL);
    if (kL[2] || kL[3]) thin_quad(x, xp, y, yp, kL + 2);
    if (kL[4] || kL[5]) thin_sext(x, xp, y, yp, kL + 4);
    if (kL[6] || kL[7]) thin_oct(x, xp, y, yp, kL + 6);
    if (kL[8] || kL[9]) thin_magnet(x, xp, y, yp, kL + 8, 5);
    if (kL[10] || kL[11]) thin_magnet(x, xp, y, yp, kL + 10, 6);
    if (kL[12] || kL[13]) thin_magnet(x, xp, y, yp, kL + 12, 7);
    if (kL[14] || kL[15]) thin_magnet(x, xp, y, yp, kL + 14, 8);
}

constexpr double Y_C1 = 0.79361246386112147294625603763;
constexpr double Y_C2 = -0.206276584816439780698721319354;
constexpr double Y_C3 = -0.118008867881292655922412133144;
constexpr double Y_C4 = 0.236949573653050744373598734219;
constexpr double Y_D1 = 1.58722492772224294589251207526;
constexpr double Y_D2 = -1.99977809735512250728995471397;
constexpr double Y_D3 = -1.82324266348482825773733634154;
constexpr double Y_D4 = 2.29714181079092974648453380998;

using kick_fn = void (*)(double, double&, double, double&, const double*);

// yoshida6 ff_algorithm.h:1834-2008
inline void yoshida6(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double pref,
                     double m, double step_ref_cdt, double step_length, const double* step_strength, int steps,
                     kick_fn kf, int components)
{
    double sub = step_ref_cdt * 0.1;
    double k1[16], k2[16], k3[16], k4[16];
    for (int i = 0; i < components * 2; ++i) {
        k1[i] = Y_D1 * step_strength[i];
        k2[i] = Y_D2 * step_strength[i];
        k3[i] = Y_D3 * step_strength[i];
        k4[i] = Y_D4 * step_strength[i];
    }
    auto D = [&](double cc) { drift_unit(x, xp, y, yp, cdt, dpop, cc * step_length, pref, m, sub); };
    for (int i = 0; i < steps; ++i) {
        D(Y_C1); kf(x, xp, y, yp, k1);
        D(Y_C2); kf(x, xp, y, yp, k2);
        D(Y_C2); kf(x, xp, y, yp, k1);
        D(Y_C3); kf(x, xp, y, yp, k3);
        D(Y_C4); kf(x, xp, y, yp, k4);
        D(Y_C4); kf(x, xp, y, yp, k3);
        D(Y_C3); kf(x, xp, y, yp, k1);
        D(Y_C2); kf(x, xp, y, yp, k2);
        D(Y_C2); kf(x, xp, y, yp, k1);
        D(Y_C1);
    }
}

// general 6th-order yoshida, ff_algorithm.h:1481-1646
inline double yx1(int nn) { return 1.0 / (2.0 - std::pow(2.0, 1.0 / (2 * nn + 1))); }
inline double yx0(int nn) { return 1.0 - 2.0 * yx1(nn); }
inline void yoshida_element(int n, double& x, double& xp, double& y, double& yp, double& cdt, double dpop,
                            double pref, double m, double step_ref_cdt, double step_length, const double* ss,
                            double c, kick_fn kf, int comps)
{
    if (n == 0) {
        double sub = step_ref_cdt / 2.0;
        double kl[16];
        for (int i = 0; i < comps * 2; ++i) kl[i] = ss[i] * c;
        drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * c * step_length, pref, m, sub);
        kf(x, xp, y, yp, kl);
        drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * c * step_length, pref, m, sub);
        return;
    }
    double sub = step_ref_cdt / 3.0;
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, ss, c * yx1(n), kf, comps);
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, ss, c * yx0(n), kf, comps);
    yoshida_element(n - 1, x, xp, y, yp, cdt, dpop, pref, m, sub, step_length, ss, c * yx1(n), kf, comps);
}

// slot_unit ff_algorithm.h:83-129
inline void slot_unit(double& x, double& xp, double& y, double& yp, double& cdt, double& dpop, double ct,
                      double st, double pref, double m)
{
    const double uni = 1.0;
    double zp = std::sqrt((dpop + uni) * (dpop + uni) - xp * xp - yp * yp);
    double p = (dpop + uni) * pref;
    double e = std::sqrt(p * p + m * m);
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

// bend_complete ff_algorithm.h:191-251 (complex arithmetic form)
inline void bend_complete(double& x, double& xp, double& y, double& yp, double& cdt, double dpop, double dphi,
                          double strength, double p_ref, double m, double cdt_ref, std::complex<double> phase,
                          std::complex<double> term)
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

void quad_kick_cb(double x, double& xp, double y, double& yp, const double* k) { cf_kick(x, xp, y, yp, k); }
void sext_kick_cb(double x, double& xp, double y, double& yp, const double* k) { thin_sext(x, xp, y, yp, k); }
void oct_kick_cb(double x, double& xp, double y, double& yp, const double* k) { thin_oct(x, xp, y, yp, k); }
// solenoid_unit ff_algorithm.h:1317-1356 (reference argument order)
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
void kicker_kick_cb(double, double& xp, double, double& yp, const double* k)
{ // thin_kicker_unit ff_algorithm.h:994-1000
    xp = xp + k[0];
    yp = yp + k[1];
}
// bend_unit, bend_edge, cf_kick5, bend_yoshida6 (ff_algorithm.h), shared
// with the particle kernels
#define SB2_FF inline
#define SB2_FF_SINCOS 0
#include "ff_bend.h"
#include "ff_nllens.h"
#undef SB2_FF
#undef SB2_FF_SINCOS
} // namespace hostff

// ---------------------------------------------------------------------------
// Bunch
// ---------------------------------------------------------------------------
struct Bunch {
    int device = 0;
    // arrays the kernels work on: the home arrays, or the working copy
    double* parts = nullptr;
    int64_t stride = 0;
    uint8_t* masks = nullptr;
    uint8_t* discards = nullptr;
    int64_t n = 0;
    bool owns = false;
    BunchCounters* counters = nullptr; // device
    BunchCounters host_counters{};     // last value read back
    Refpart ref;
    Refpart design;
    bool design_set = false;
    int turns_done = 0;
    int next_step = 0; // step of the stepper the bunch is at (0 after whole turns)

    // Home arrays: the ones the caller handed over or reads back, in the
    // caller's particle order.
    double* home_parts = nullptr;
    int64_t home_stride = 0;
    uint8_t* home_masks = nullptr;
    uint8_t* home_discards = nullptr;
    // Cell-ordered working copy used by space-charge propagation.  It
    // outlives a propagate call, so consecutive calls keep the particles in
    // (nearly) cell order; the home arrays are brought up to date by
    // settle() before anything reads or writes them in the caller's order.
    SortBuffers wc{};
    BunchCounters* snap_counters = nullptr; // pinned: counts of the last snapshot
    bool permuted = false;    // current data is the working copy
    int kicks_since_sort = 0; // kicks since the working copy was last sorted

    void set_home()
    {
        home_parts = parts;
        home_stride = stride;
        home_masks = masks;
        home_discards = discards;
    }
    void free_work()
    {
        dfree(wc.parts);
        dfree(wc.masks);
        dfree(wc.discards);
        dfree(wc.perm);
        dfree(wc.parts2);
        dfree(wc.masks2);
        dfree(wc.discards2);
        dfree(wc.perm2);
        wc = SortBuffers{};
        perm_valid = false;
    }
    // home -> working copy: the first time in the caller's order (identity
    // permutation), later in the order the bunch last left its working copy
    void enter_work(cudaStream_t s)
    {
        if (permuted) return;
        const bool again = perm_valid;
        enter_work_host();
        if (again) // the order the bunch last left: nearly cell-ordered
            cuda_check(launch_sort_gather_perm(home_parts, home_stride, home_masks, home_discards, wc, s),
                       "sort gather");
        else
            cuda_check(launch_sort_gather_in(home_parts, home_stride, home_masks, home_discards, wc, s),
                       "sort gather");
        perm_valid = true;
    }
    bool perm_valid = false; // wc.perm holds the last working copy's order
    // enter_work's host side: the working copy's buffers and the switch to
    // them (without the gather, which enter_work launches)
    void enter_work_host()
    {
        if (!wc.parts) {
            // a multiple of 32 particles: every column starts 256-byte
            // aligned, and the sort's 16-byte staging copies of the last
            // tile stay inside the arrays
            const int64_t cap = (std::max<int64_t>(n, 1) + 31) / 32 * 32;
            wc.n = n;
            wc.stride = cap;
            wc.parts = dalloc<double>((size_t)7 * cap, "working copy");
            wc.parts2 = dalloc<double>((size_t)7 * cap, "working copy");
            wc.masks = dalloc<uint8_t>(cap, "working copy");
            wc.masks2 = dalloc<uint8_t>(cap, "working copy");
            wc.discards = dalloc<uint8_t>(cap, "working copy");
            wc.discards2 = dalloc<uint8_t>(cap, "working copy");
            wc.perm = dalloc<int32_t>(cap, "working copy");
            wc.perm2 = dalloc<int32_t>(cap, "working copy");
        }
        parts = wc.parts;
        stride = wc.stride;
        masks = wc.masks;
        discards = wc.discards;
        permuted = true;
        kicks_since_sort = 0;
    }
    // home arrays brought up to date from the working copy, which stays in
    // use (a snapshot for I/O reads the home arrays)
    void sync_home(cudaStream_t s)
    {
        if (!permuted) return;
        cuda_check(launch_sort_scatter_out(wc, home_parts, home_stride, home_masks, home_discards, s), "sort scatter");
    }
    // working copy -> home arrays, back in the caller's order
    void settle(cudaStream_t s)
    {
        if (!permuted) return;
        cuda_check(launch_sort_scatter_out(wc, home_parts, home_stride, home_masks, home_discards, s), "sort scatter");
        drop_work();
    }
    // settle() with the caller's copy made at the same time: each array is
    // put back in the caller's order and copied to the host while the next
    // one is being put back (host arrays as sb2_bunch_get_particles takes
    // them; null ones are skipped).  Returns when the copies are done.
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t col_done[9] = {};
    void settle_to_host(double* host_parts, uint8_t* host_masks, uint8_t* host_discards)
    {
        if (!copy_stream) {
            cuda_check(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking), "stream");
            for (auto& e : col_done) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
        }
        cudaStream_t s = 0;
        cuda_check(launch_sort_invert(wc, s), "sort invert");
        for (int c = 0; c < 9; ++c) {
            void* host = nullptr;
            const void* dev = nullptr;
            size_t bytes = 0;
            if (c < 7) {
                cuda_check(launch_sort_scatter_out_col(wc, c, home_parts + c * home_stride, s), "sort scatter");
                host = host_parts ? host_parts + c * n : nullptr;
                dev = home_parts + c * home_stride;
                bytes = sizeof(double) * n;
            } else if (c == 7) {
                cuda_check(launch_sort_scatter_out_bytes(wc.masks, wc, home_masks, s), "sort scatter");
                host = host_masks;
                dev = home_masks;
                bytes = n;
            } else if (home_discards) {
                cuda_check(launch_sort_scatter_out_bytes(wc.discards, wc, home_discards, s), "sort scatter");
                host = host_discards;
                dev = home_discards;
                bytes = n;
            }
            if (!host || !bytes) continue;
            cuda_check(cudaEventRecord(col_done[c], s), "event");
            cuda_check(cudaStreamWaitEvent(copy_stream, col_done[c], 0), "event");
            cuda_check(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, copy_stream), "checkout");
        }
        cuda_check(cudaStreamSynchronize(copy_stream), "checkout");
        cuda_check(cudaStreamSynchronize(s), "checkout");
        drop_work();
    }
    // forget the working copy (the home arrays are about to be overwritten)
    void drop_work()
    {
        permuted = false;
        parts = home_parts;
        stride = home_stride;
        masks = home_masks;
        discards = home_discards;
    }
    // the working copy after a sort (sort.cu writes into the second buffers)
    void swap_work()
    {
        std::swap(wc.parts, wc.parts2);
        std::swap(wc.masks, wc.masks2);
        std::swap(wc.discards, wc.discards2);
        std::swap(wc.perm, wc.perm2);
        parts = wc.parts;
        masks = wc.masks;
        discards = wc.discards;
    }

    ~Bunch()
    {
        if (owns) {
            dfree(home_parts);
            dfree(home_masks);
            dfree(home_discards);
        }
        free_work();
        dfree(counters);
        if (snap_counters) cudaFreeHost(snap_counters);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        for (auto e : col_done)
            if (e) cudaEventDestroy(e);
    }
    void sync_counters(cudaStream_t s)
    {
        cuda_check(cudaMemcpyAsync(&host_counters, counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost, s),
                   "counters");
        cuda_check(cudaStreamSynchronize(s), "sync");
    }
};

// ---------------------------------------------------------------------------
// Operations of one independent operator (independent_operator.cc:25-91)
// ---------------------------------------------------------------------------
struct Operation {
    bool aperture = false;
    std::vector<Slice> group; // libFF group
    std::string ap_type;
    Slice ap_slice;
};

static std::vector<Operation> create_operations(const Lattice& lat, const std::vector<Slice>& slices)
{
    std::vector<Operation> ops;
    std::string aperture_type;
    bool need_left = false, need_right = false;
    std::string extractor_type, last_extractor_type;
    std::vector<Slice> group;
    auto push_group = [&]() {
        Operation o;
        o.group = group;
        ops.push_back(o);
    };
    auto push_ap = [&](const std::string& t, const Slice& s) {
        if (t != "finite" && t != "circular" && t != "elliptical" && t != "rectangular")
            throw Error(t == "polygon" ? SB2_ERR_UNSUPPORTED : SB2_ERR_RUNTIME, "unknown aperture_type " + t);
        Operation o;
        o.aperture = true;
        o.ap_type = t;
        o.ap_slice = s;
        ops.push_back(o);
    };
    for (auto const& slice : slices) {
        const Element& el = lat.elements[slice.elem];
        if (el.has_string("aperture_type")) {
            aperture_type = el.get_string("aperture_type", "");
            need_left = slice.ledge;
            need_right = slice.redge;
        } else {
            need_left = need_right = false;
        }
        extractor_type = el.get_string("extractor_type", "default");
        if (extractor_type != "default" && extractor_type != "libff")
            throw Error(SB2_ERR_UNSUPPORTED, "unknown extractor_type: " + extractor_type);
        if (((extractor_type != last_extractor_type) || need_left) && !group.empty()) {
            push_group();
            group.clear();
        }
        if (need_left) push_ap(aperture_type, slice);
        group.push_back(slice);
        last_extractor_type = extractor_type;
        if (need_right) {
            push_group();
            push_ap(aperture_type, slice);
            group.clear();
        }
    }
    if (!group.empty()) push_group();
    push_ap("finite", slices.back());
    push_ap("circular", slices.back());
    return ops;
}

struct IndepOperator {
    std::vector<Slice> slices;
    std::vector<Operation> ops;
};

struct Step {
    double length = 0;
    std::vector<char> items; // 'I' independent, 'C' collective
    std::vector<IndepOperator> indeps;
};

// get_fixed_step_slices split_operator_stepper.cc:14-82 (no force_diagnostics)
static std::vector<Slice> fixed_step_slices(const Lattice& lat, size_t& it, double& left, double step_length,
                                            double& offset_fudge)
{
    const double tol = 1.0e-8;
    std::vector<Slice> slices;
    double length = offset_fudge;
    bool complete = false;
    const size_t end = lat.elements.size();
    while (!complete) {
        double right = lat.elements[it].length();
        if (length + (right - left) - tol <= step_length) {
            slices.push_back(make_slice(lat, (int)it, left, right));
            length += (right - left);
            ++it;
            left = 0.0;
            if (std::abs(length - step_length) < tol) {
                if ((it == end) || (lat.elements[it].length() != 0.0)) complete = true;
            } else {
                if (it == end) throw Error(SB2_ERR_RUNTIME, "get_step stepped beyond end of lattice");
            }
        } else {
            bool end_within_error = false;
            double old_right = right;
            right = step_length - length + left;
            if (std::abs(old_right - right) < tol) {
                right = old_right;
                end_within_error = true;
            }
            slices.push_back(make_slice(lat, (int)it, left, right));
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

static std::vector<Step> make_steps(const Lattice& lat, int kind, int num, bool collective)
{
    std::vector<Step> steps;
    auto add_indep = [&](Step& st, std::vector<Slice> sl) {
        IndepOperator op;
        op.slices = std::move(sl);
        op.ops = create_operations(lat, op.slices);
        st.items.push_back('I');
        st.indeps.push_back(std::move(op));
    };
    if (kind == SB2_STEPPER_SPLIT_OPERATOR) {
        // Split_operator_stepper::apply_impl split_operator_stepper.cc:132-261
        if (num < 1) throw Error(SB2_ERR_INVALID, "Split_operator_stepper: num_steps must be >= 1");
        double step_length = lat.length() / num;
        double half = 0.5 * step_length;
        if (lat.elements.empty()) return steps;
        size_t it = 0;
        double left = 0.0, fudge = 0.0;
        for (int i = 0; i < num; ++i) {
            for (auto const& el : lat.elements)
                if (el.has_string("force_diagnostics"))
                    throw Error(SB2_ERR_UNSUPPORTED, "force_diagnostics substeps are not supported");
            auto s1 = fixed_step_slices(lat, it, left, half, fudge);
            auto s2 = fixed_step_slices(lat, it, left, half, fudge);
            Step st;
            st.length = step_length;
            add_indep(st, s1);
            if (collective) st.items.push_back('C');
            add_indep(st, s2);
            steps.push_back(std::move(st));
        }
        if (it != lat.elements.size())
            throw Error(SB2_ERR_RUNTIME,
                        "internal error: split_operator_stepper did not make it to the end of the lattice\n");
    } else if (kind == SB2_STEPPER_SPLIT_OPERATOR_ELEMENTS || kind == SB2_STEPPER_INDEPENDENT_ELEMENTS) {
        // split_operator_stepper_elements.cc:4-47, independent_stepper_elements.cc:3-36
        if (num < 1) throw Error(SB2_ERR_INVALID, "Split_operator_stepper_elements: steps_per_element must be >= 1");
        for (size_t ei = 0; ei < lat.elements.size(); ++ei) {
            double length = lat.elements[ei].length();
            if (length == 0.0) {
                Step st;
                st.length = 0.0;
                add_indep(st, {whole_slice(lat, (int)ei)});
                steps.push_back(std::move(st));
                continue;
            }
            double sl = length / num;
            for (int i = 0; i < num; ++i) {
                double left = i * sl, right = (i + 1) * sl;
                Step st;
                st.length = sl;
                if (kind == SB2_STEPPER_INDEPENDENT_ELEMENTS) {
                    add_indep(st, {make_slice(lat, (int)ei, left, right)});
                } else {
                    double middle = left + 0.5 * sl;
                    add_indep(st, {make_slice(lat, (int)ei, left, middle)});
                    if (collective) st.items.push_back('C');
                    add_indep(st, {make_slice(lat, (int)ei, middle, right)});
                }
                steps.push_back(std::move(st));
            }
        }
    } else {
        throw Error(SB2_ERR_INVALID, "unknown stepper kind");
    }
    return steps;
}

// ---------------------------------------------------------------------------
// Host half of the element maps -> MapOps
// ---------------------------------------------------------------------------
static MapOp new_op(int kind)
{
    MapOp o;
    std::memset(&o, 0, sizeof(o));
    o.kind = kind;
    return o;
}

static double brho_scale(const Bunch& b)
{
    const Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    double brho_l = ref_l.p / ref_l.charge;
    double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    return brho_l / brho_b;
}

// FF_drift::apply ff_drift.h:95-152
static void ops_drift(const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const double length = sl.right - sl.left;
    if (hostff::close_to_zero(length)) {
        b.design.state[4] = 0.0;
        return;
    }
    Refpart& ref_l = b.design;
    const double ref_p = b.ref.p * (1.0 + b.ref.state[5]);
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
    double cdt = 0.0, dpop = 0.0;
    hostff::drift_unit(x, xp, y, yp, cdt, dpop, length, ref_l.p, ref_l.mass, 0.0);
    ref_l.state = {x, xp, y, yp, cdt, dpop};
    MapOp o = new_op(OP_DRIFT);
    o.d[0] = length;
    o.d[1] = ref_p;
    o.d[2] = b.ref.mass;
    o.d[3] = cdt;
    out.push_back(o);
    b.ref.s_n += length;
}

// FF_quadrupole::apply ff_quadrupole.h:310-565
static void ops_quad(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const Element& ele = lat.elements[sl.elem];
    double length = sl.right - sl.left;
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
        a[1] = (char)('0' + i);
        bb[1] = (char)('0' + i);
        kn[i * 2 + 0] = ele.get(bb, 0.0);
        kn[i * 2 + 1] = ele.get(a, 0.0);
        if (kn[i * 2 + 0] || kn[i * 2 + 1]) {
            has_mp = true;
            double coeff = hostff::factorial(i);
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
    double scale = brho_scale(b);
    for (auto& k : kn) k *= scale;

    auto ref_cdt = [&](int steps) { // get_reference_cdt ff_quadrupole.h:263-303
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double cdt = 0.0, dpop = 0.0;
        x -= xoff;
        y -= yoff;
        if (hostff::close_to_zero(length))
            hostff::thin_quad(x, xp, y, yp, kn);
        else
            hostff::yoshida6(x, xp, y, yp, cdt, dpop, ref_l.p, ref_l.mass, 0.0, length / steps, kn, steps,
                             hostff::quad_kick_cb, 8);
        x += xoff;
        y += yoff;
        ref_l.state = {x, xp, y, yp, cdt, dpop};
        return cdt;
    };

    if (hostff::close_to_zero(length)) {
        ref_cdt(0);
        MapOp o = new_op(OP_THIN_QUAD);
        o.d[0] = xoff;
        o.d[1] = yoff;
        o.d[2] = kn[0];
        o.d[3] = kn[1];
        out.push_back(o);
        return;
    }
    int steps = (int)ele.get("yoshida_steps", 4.0);
    for (auto& k : kn) k *= length / steps;
    double ref_p = b.ref.p, ref_m = b.ref.mass;
    double ref_t = ref_cdt(steps);
    double step_ref_t = ref_t / steps, step_l = length / steps;
    MapOp o = new_op(has_mp ? OP_QUAD_CF : OP_QUAD);
    o.steps = steps;
    o.d[0] = xoff;
    o.d[1] = yoff;
    o.d[2] = ref_p;
    o.d[3] = ref_m;
    o.d[4] = step_ref_t * 0.1;
    o.d[5] = hostff::Y_C1 * step_l;
    o.d[6] = hostff::Y_C2 * step_l;
    o.d[7] = hostff::Y_C3 * step_l;
    o.d[8] = hostff::Y_C4 * step_l;
    const int comps = has_mp ? 8 : 1;
    const int KS = has_mp ? 16 : 2;
    for (int i = 0; i < comps * 2; ++i) {
        o.d[9 + i] = hostff::Y_D1 * kn[i];
        o.d[9 + KS + i] = hostff::Y_D2 * kn[i];
        o.d[9 + 2 * KS + i] = hostff::Y_D3 * kn[i];
        o.d[9 + 3 * KS + i] = hostff::Y_D4 * kn[i];
    }
    out.push_back(o);
    b.ref.s_n += length;
}

// FF_sbend::apply ff_sbend.h:741-969.  Pure dipoles run PropSbendSimd
// (one exact bend unit); k1..k5(s) or a_n/b_n multipoles select the
// combined-function path (prop_reference_cf + PropSbendCF).
static void ops_sbend_cf(const Slice& sl, Bunch& b, std::vector<MapOp>& out, double a, double l, double length,
                         double angle, const double* k_l, double e1, double e2);

static void ops_sbend(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const Element& ele = lat.elements[sl.elem];
    double a = ele.get("angle");
    double l = ele.get("l");
    double length = sl.right - sl.left;
    double angle = (length / l) * a;
    bool ledge = sl.ledge, redge = sl.redge;
    double e1 = ele.get("e1", 0.0), e2 = ele.get("e2", 0.0);
    static const char* kn_names[10] = {"k1", "k1s", "k2", "k2s", "k3", "k3s", "k4", "k4s", "k5", "k5s"};
    double k_l[10];
    bool cf = false;
    for (int i = 0; i < 10; ++i) {
        k_l[i] = ele.get(kn_names[i], 0.0);
        if (k_l[i] != 0.0) cf = true;
    }
    // b_n / a_n multipole moments become the k_l of order n+1, scaled by
    // angle * n! (ff_sbend.h:790-828)
    bool has_mp = false;
    for (int i = 1; i < 5; ++i) {
        std::string an = "a0", bn = "b0";
        an[1] = (char)('0' + i);
        bn[1] = (char)('0' + i);
        double kn = ele.get(bn, 0.0), ks = ele.get(an, 0.0);
        if (kn != 0.0 || ks != 0.0) {
            has_mp = true;
            double coeff = hostff::factorial(i);
            kn *= a * coeff;
            ks *= a * coeff;
            if (k_l[(i - 1) * 2 + 0] != 0.0 || k_l[(i - 1) * 2 + 1] != 0.0)
                throw Error(SB2_ERR_RUNTIME, "having both kn/ks and a/b coefficents are forbidden in sbends");
            k_l[(i - 1) * 2 + 0] = kn;
            k_l[(i - 1) * 2 + 1] = ks;
        }
    }
    if (cf || has_mp) {
        ops_sbend_cf(sl, b, out, a, l, length, angle, k_l, e1, e2);
        return;
    }
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    double scale = ref_l.p / (ref_b.p * (1.0 + ref_b.state[5]));
    if (!redge) e2 = 0;
    if (!ledge) e1 = 0;
    const double cnv = 1.0e-9 * pc::c;
    double pref_l = ref_l.p;
    double brho_l = pref_l / cnv;
    int charge_l = ref_l.charge;
    double pref_b = ref_b.p;
    double brho_b = pref_b / cnv;
    double m_b = b.ref.mass;
    double strength = brho_l * a / l;
    double ce1 = std::cos(-e1), se1 = std::sin(-e1), ce2 = std::cos(-e2), se2 = std::sin(-e2);
    double sgn = (charge_l > 0) ? 1.0 : -1.0;
    double us_edge_k_p = sgn * strength / brho_b;
    double ds_edge_k_p = -sgn * strength / brho_b;
    double us_kx = 0, us_ky = 0, ds_kx = 0, ds_ky = 0;
    double dphi = -(angle - (e1 + e2));
    std::complex<double> phase = std::exp(std::complex<double>(0.0, -dphi));
    std::complex<double> term = std::complex<double>(0.0, length / angle) *
                                std::complex<double>(1.0 - std::cos(angle), -std::sin(angle)) *
                                std::complex<double>(std::cos(e2), -std::sin(e2));
    { // prop_reference ff_sbend.h:478-566
        double m_l = ref_l.mass;
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double cdt = 0.0, dpop = 0.0;
        if (ledge) {
            hostff::slot_unit(x, xp, y, yp, cdt, dpop, ce1, se1, pref_l, m_l);
            double p_l = 1.0 + dpop;
            double zp = std::sqrt(p_l * p_l - xp * xp - yp * yp);
            us_kx = us_edge_k_p * (xp / zp);
            us_ky = us_edge_k_p * (yp / zp);
            double kx = us_kx / scale, ky = us_ky / scale;
            yp = yp - kx * y;
            xp = xp + ky * y;
        }
        hostff::bend_complete(x, xp, y, yp, cdt, dpop, dphi, strength, pref_l, m_l, 0.0, phase, term);
        if (redge) {
            double p_l = 1.0 + dpop;
            double zp = std::sqrt(p_l * p_l - xp * xp - yp * yp);
            ds_kx = ds_edge_k_p * (xp / zp);
            ds_ky = ds_edge_k_p * (yp / zp);
            double kx = ds_kx / scale, ky = ds_ky / scale;
            yp = yp - kx * y;
            xp = xp + ky * y;
            hostff::slot_unit(x, xp, y, yp, cdt, dpop, ce2, se2, pref_l, m_l);
        }
        ref_l.state = {x, xp, y, yp, cdt, dpop};
        MapOp o = new_op(OP_SBEND);
        o.flags = (ledge ? 1 : 0) | (redge ? 2 : 0);
        o.d[0] = ce1; o.d[1] = se1; o.d[2] = ce2; o.d[3] = se2;
        o.d[4] = us_kx; o.d[5] = us_ky; o.d[6] = ds_kx; o.d[7] = ds_ky;
        o.d[8] = dphi; o.d[9] = phase.real(); o.d[10] = phase.imag();
        o.d[11] = term.real(); o.d[12] = term.imag();
        o.d[13] = strength; o.d[14] = pref_b; o.d[15] = m_b; o.d[16] = cdt;
        const hostff::BendConst bk = hostff::bend_const(pref_b, m_b, strength);
        o.d[17] = bk.igib2;
        o.d[18] = bk.cs;
        out.push_back(o);
    }
    b.ref.s_n += length;
}

// Combined-function sector bend (ff_sbend.h:568-660 prop_reference_cf,
// then PropSbendCF :221-339 on the particles).
static void ops_sbend_cf(const Slice& sl, Bunch& b, std::vector<MapOp>& out, double a, double l, double length,
                         double angle, const double* k_l, double e1, double e2)
{
    const bool ledge = sl.ledge, redge = sl.redge;
    const double r0 = l / a;
    const int steps = 6; // FF_algorithm::default_steps
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    const double scale = ref_l.p / (ref_b.p * (1.0 + ref_b.state[5]));
    if (!redge) e2 = 0;
    if (!ledge) e1 = 0;
    const double cnv = 1.0e-9 * pc::c;
    const double pref_l = ref_l.p;
    const double brho_l = pref_l / cnv;
    const double m_l = ref_l.mass;
    const int charge_l = ref_l.charge;
    const double pref_b = ref_b.p;
    const double brho_b = pref_b / cnv;
    const double m_b = b.ref.mass;
    const double strength = brho_l * a / l;
    const double ce1 = std::cos(-e1), se1 = std::sin(-e1), ce2 = std::cos(-e2), se2 = std::sin(-e2);
    const double sgn = (charge_l > 0) ? 1.0 : -1.0;
    const double us_edge_k_p = sgn * strength / brho_b;
    const double ds_edge_k_p = -sgn * strength / brho_b;
    // bend_edge_phase(e) = exp(-i e); sbend_unit_phase(c, d) = exp(i c d);
    // sbend_unit_term(c, d, r0) = i r0 (1 - cos(c d) - i sin(c d));
    // sbend_dphi(c, d) = -c d  (ff_algorithm.h:346-362, 2143-2175)
    const double pe1_r = std::cos(-e1), pe1_i = std::sin(-e1);
    const double pe2_r = std::cos(-e2), pe2_i = std::sin(-e2);
    const double step_angle = angle / steps;
    double dphi[4], phase[8], term[8];
    for (int j = 0; j < 4; ++j) {
        const double th = hostff::kBY6_C[j] * step_angle;
        phase[2 * j] = std::cos(th);
        phase[2 * j + 1] = std::sin(th);
        const double re = 1.0 - std::cos(th), im = -std::sin(th);
        term[2 * j] = 0.0 * re - r0 * im;
        term[2 * j + 1] = 0.0 * im + r0 * re;
        dphi[j] = -hostff::kBY6_C[j] * step_angle;
    }
    double us_kx = 0, us_ky = 0, ds_kx = 0, ds_ky = 0;
    { // prop_reference_cf: the design particle, from dp/p = 0, strengths unscaled
        const hostff::BendConst bk_l = hostff::bend_const(pref_l, m_l, strength);
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        double cdt = 0.0, dpop = 0.0;
        const double step_length = length / steps;
        double kr[4][8];
        for (int i = 0; i < 8; ++i) {
            const double skl = k_l[i] * step_length;
            for (int j = 0; j < 4; ++j) kr[j][i] = hostff::kBY6_D[j] * skl;
        }
        if (ledge) {
            hostff::slot_unit(x, xp, y, yp, cdt, dpop, ce1, se1, pref_l, m_l);
            double p_l = 1.0 + dpop;
            double zp = std::sqrt(p_l * p_l - xp * xp - yp * yp);
            us_kx = us_edge_k_p * (xp / zp);
            us_ky = us_edge_k_p * (yp / zp);
            double kx = us_kx / scale, ky = us_ky / scale;
            yp = yp - kx * y;
            xp = xp + ky * y;
            hostff::bend_edge(x, xp, y, yp, cdt, dpop, e1, pe1_r, pe1_i, bk_l, pref_l, m_l);
        }
        hostff::bend_yoshida6(x, xp, y, yp, cdt, dpop, pref_l, m_l, 0.0 * 0.1, kr[0], kr[1], kr[2], kr[3], dphi, phase,
                              term, r0, bk_l, steps);
        if (redge) {
            hostff::bend_edge(x, xp, y, yp, cdt, dpop, e2, pe2_r, pe2_i, bk_l, pref_l, m_l);
            double p_l = 1.0 + dpop;
            double zp = std::sqrt(p_l * p_l - xp * xp - yp * yp);
            ds_kx = ds_edge_k_p * (xp / zp);
            ds_ky = ds_edge_k_p * (yp / zp);
            double kx = ds_kx / scale, ky = ds_ky / scale;
            yp = yp - kx * y;
            xp = xp + ky * y;
            hostff::slot_unit(x, xp, y, yp, cdt, dpop, ce2, se2, pref_l, m_l);
        }
        ref_l.state = {x, xp, y, yp, cdt, dpop};
    }
    const double ref_cdt = ref_l.state[4];
    MapOp o = new_op(OP_SBEND_CF);
    o.flags = (ledge ? 1 : 0) | (redge ? 2 : 0);
    o.steps = steps;
    o.d[0] = ce1; o.d[1] = se1; o.d[2] = ce2; o.d[3] = se2;
    o.d[4] = us_kx; o.d[5] = us_ky; o.d[6] = ds_kx; o.d[7] = ds_ky;
    o.d[8] = e1; o.d[9] = e2;
    o.d[10] = pe1_r; o.d[11] = pe1_i; o.d[12] = pe2_r; o.d[13] = pe2_i;
    o.d[14] = strength; o.d[15] = pref_b; o.d[16] = m_b;
    o.d[17] = (ref_cdt / steps) * 0.1;
    o.d[18] = r0;
    for (int j = 0; j < 4; ++j) o.d[19 + j] = dphi[j];
    for (int j = 0; j < 8; ++j) {
        o.d[23 + j] = phase[j];
        o.d[31 + j] = term[j];
    }
    for (int i = 0; i < 8; ++i) { // PropSbendCF step strengths, d_j-scaled
        const double skl = k_l[i] * scale * length / steps;
        for (int j = 0; j < 4; ++j) o.d[39 + 8 * j + i] = hostff::kBY6_D[j] * skl;
    }
    const hostff::BendConst bk_b = hostff::bend_const(pref_b, m_b, strength);
    o.d[71] = bk_b.igib2;
    o.d[72] = bk_b.cs;
    out.push_back(o);
    b.ref.s_n += length;
}

// FF_multipole::apply ff_multipole.h:85-210
static void ops_multipole(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    if (sl.right - sl.left > 0.0) throw Error(SB2_ERR_RUNTIME, "FF_multipole::apply() cannot deal with thick elements");
    const Element& el = lat.elements[sl.elem];
    const int max_order = 8;
    std::vector<double> knl, ksl, tn;
    if (el.v.count("knl") || el.v.count("ksl")) {
        std::vector<double> k0(1, 0.0);
        knl = el.v.count("knl") ? el.v.at("knl") : k0;
        ksl = el.v.count("ksl") ? el.v.at("ksl") : k0;
        if (knl.size() > ksl.size())
            ksl.resize(knl.size(), 0.0);
        else if (knl.size() < ksl.size())
            knl.resize(ksl.size(), 0.0);
        tn.resize(knl.size(), el.get("tilt", 0.0));
    } else {
        for (int i = 0; i < 6; ++i) {
            std::string skn = "k0l", stn = "t0";
            skn[1] = (char)('0' + i);
            stn[1] = (char)('0' + i);
            knl.push_back(el.get(skn, 0.0));
            tn.push_back(el.get(stn, 0.0));
        }
        int tail = (int)knl.size() - 1;
        while (tail && knl[tail] == 0.0) --tail;
        knl.resize(tail + 1);
        ksl.resize(knl.size(), 0.0);
        tn.resize(knl.size(), 0.0);
    }
    if ((int)knl.size() > max_order) throw Error(SB2_ERR_UNSUPPORTED, "multipole order above 8");
    for (size_t i = 0; i < knl.size(); ++i)
        if (tn[i] != 0.0) {
            std::complex<double> ck2(knl[i], ksl[i]);
            ck2 = ck2 * std::exp(std::complex<double>(0.0, -(double)(i + 1) * tn[i]));
            knl[i] = ck2.real();
            ksl[i] = ck2.imag();
        }
    double scale = brho_scale(b);
    for (size_t i = 0; i < knl.size(); ++i) {
        knl[i] *= scale;
        ksl[i] *= scale;
    }
    MapOp o = new_op(OP_MPOLE);
    for (size_t i = 0; i < knl.size(); ++i) {
        if (knl[i] || ksl[i]) o.flags |= (1 << i);
        o.d[i * 2 + 0] = knl[i];
        o.d[i * 2 + 1] = ksl[i];
    }
    Refpart& ref_l = b.design;
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], dpop = ref_l.state[5];
    for (int n = 0; n < max_order; ++n)
        if (o.flags & (1 << n)) hostff::thin_magnet(x, xp, y, yp, &o.d[n * 2], n + 1);
    ref_l.state = {x, xp, y, yp, 0.0, dpop};
    out.push_back(o);
}

// FF_sextupole::apply ff_sextupole.h:18-92 + ff_patterned_propagator.h
static void ops_sextupole(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const Element& el = lat.elements[sl.elem];
    double length = sl.right - sl.left;
    double k[2] = {el.get("k2", 0.0), el.get("k2s", 0.0)};
    double tilt = el.get("tilt", 0.0);
    if (tilt != 0.0) {
        std::complex<double> ck2(k[0], k[1]);
        ck2 = ck2 * std::exp(std::complex<double>(0.0, -3.0 * tilt));
        k[0] = ck2.real();
        k[1] = ck2.imag();
    }
    double scale = brho_scale(b);
    k[0] *= scale;
    k[1] *= scale;
    Refpart& ref_l = b.design;
    if (hostff::close_to_zero(length)) {
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        hostff::thin_sext(x, xp, y, yp, k);
        ref_l.state[1] = xp;
        ref_l.state[3] = yp;
        ref_l.state[4] = 0.0;
        MapOp o = new_op(OP_THIN_SEXT);
        o.d[2] = k[0];
        o.d[3] = k[1];
        out.push_back(o);
        return;
    }
    int steps = (int)el.get("yoshida_steps", 4.0);
    double cdt = 0.0;
    auto st = ref_l.state;
    st[5] = 0.0;
    double step_len = length / steps;
    double step_str[2] = {k[0] * step_len, k[1] * step_len};
    // yoshida<double, kf, 6, 1> ff_algorithm.h:1622-1646: n = (6 - 2) / 2
    for (int i = 0; i < steps; ++i)
        hostff::yoshida_element(2, st[0], st[1], st[2], st[3], cdt, st[5], ref_l.p, ref_l.mass, 0.0, step_len,
                                step_str, 1.0, hostff::sext_kick_cb, 1);
    st[4] = cdt;
    ref_l.state = st;
    double step_ref_cdt = cdt / steps;
    MapOp o = new_op(OP_SEXT_YOSHIDA);
    o.steps = steps;
    o.d[2] = b.ref.p;
    o.d[3] = b.ref.mass;
    o.d[4] = step_ref_cdt * 0.1;
    o.d[5] = hostff::Y_C1 * step_len;
    o.d[6] = hostff::Y_C2 * step_len;
    o.d[7] = hostff::Y_C3 * step_len;
    o.d[8] = hostff::Y_C4 * step_len;
    for (int i = 0; i < 2; ++i) {
        o.d[9 + i] = hostff::Y_D1 * step_str[i];
        o.d[11 + i] = hostff::Y_D2 * step_str[i];
        o.d[13 + i] = hostff::Y_D3 * step_str[i];
        o.d[15 + i] = hostff::Y_D4 * step_str[i];
    }
    out.push_back(o);
    b.ref.s_n += length;
}

// Patterned element slice (FF_patterned_propagator, ff_patterned_propagator.h)
// with kick kf: the design particle follows k_design (get_reference_cdt_*),
// the particles k_parts.  Thin slices kick; thick ones run yoshida6 (or a
// drift-kick-drift with `simple`); use_drift times the design particle by a
// plain drift.
static void ops_patterned(const Slice& sl, Bunch& b, std::vector<MapOp>& out, const double* k_design,
                          const double* k_parts, hostff::kick_fn kf, int thin_kind, int yoshida_kind, bool thin,
                          bool simple, bool use_drift, int steps)
{
    const double length = sl.right - sl.left;
    Refpart& ref_l = b.design;
    if (thin) { // get_reference_cdt_zero :227-244
        double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
        kf(x, xp, y, yp, k_design);
        ref_l.state[1] = xp;
        ref_l.state[3] = yp;
        ref_l.state[4] = 0.0;
        MapOp o = new_op(thin_kind);
        o.d[2] = k_parts[0];
        o.d[3] = k_parts[1];
        out.push_back(o);
        return;
    }
    if (simple) { // get_reference_cdt_simple :246-273, simple_kicker :57-100
        double cdt = 0.0;
        auto st = ref_l.state;
        st[5] = 0.0;
        double str[2] = {k_design[0] * length, k_design[1] * length};
        hostff::drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length * 0.5, ref_l.p, ref_l.mass, 0.0);
        kf(st[0], st[1], st[2], st[3], str);
        hostff::drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length * 0.5, ref_l.p, ref_l.mass, 0.0);
        st[4] = cdt;
        ref_l.state = st;
        MapOp o = new_op(OP_KICK_SIMPLE);
        o.d[0] = length * 0.5;
        o.d[1] = b.ref.p;
        o.d[2] = b.ref.mass;
        o.d[3] = cdt * 0.5;
        o.d[4] = k_parts[0]; // the reference kicks with the per-length strength as is
        o.d[5] = k_parts[1];
        out.push_back(o);
        b.ref.s_n += length;
        return;
    }
    // get_reference_cdt_yoshida :275-316, apply_yoshida_kick :199-225
    double cdt = 0.0;
    auto st = ref_l.state;
    st[5] = 0.0;
    const double step_len = length / steps;
    double dstr[2] = {k_design[0] * step_len, k_design[1] * step_len};
    if (use_drift)
        hostff::drift_unit(st[0], st[1], st[2], st[3], cdt, st[5], length, ref_l.p, ref_l.mass, 0.0);
    else
        for (int i = 0; i < steps; ++i)
            hostff::yoshida_element(2, st[0], st[1], st[2], st[3], cdt, st[5], ref_l.p, ref_l.mass, 0.0, step_len, dstr,
                                    1.0, kf, 1);
    st[4] = cdt;
    ref_l.state = st;
    const double step_ref_cdt = cdt / steps;
    const double pstr[2] = {k_parts[0] * step_len, k_parts[1] * step_len};
    MapOp o = new_op(yoshida_kind);
    o.steps = steps;
    o.d[2] = b.ref.p;
    o.d[3] = b.ref.mass;
    o.d[4] = step_ref_cdt * 0.1;
    o.d[5] = hostff::Y_C1 * step_len;
    o.d[6] = hostff::Y_C2 * step_len;
    o.d[7] = hostff::Y_C3 * step_len;
    o.d[8] = hostff::Y_C4 * step_len;
    for (int i = 0; i < 2; ++i) {
        o.d[9 + i] = hostff::Y_D1 * pstr[i];
        o.d[11 + i] = hostff::Y_D2 * pstr[i];
        o.d[13 + i] = hostff::Y_D3 * pstr[i];
        o.d[15 + i] = hostff::Y_D4 * pstr[i];
    }
    out.push_back(o);
    b.ref.s_n += length;
}

static void ops_octupole(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{ // ff_octupole.h:16-88
    const Element& el = lat.elements[sl.elem];
    double k[2] = {el.get("k3", 0.0), el.get("k3s", 0.0)};
    const double tilt = el.get("tilt", 0.0);
    if (tilt != 0.0) {
        std::complex<double> ck2(k[0], k[1]);
        ck2 = ck2 * std::exp(std::complex<double>(0.0, -4.0 * tilt));
        k[0] = ck2.real();
        k[1] = ck2.imag();
    }
    const double scale = brho_scale(b);
    k[0] *= scale;
    k[1] *= scale;
    ops_patterned(sl, b, out, k, k, hostff::oct_kick_cb, OP_THIN_OCT, OP_OCT_YOSHIDA,
                  hostff::close_to_zero(sl.right - sl.left), false, false, (int)el.get("yoshida_steps", 4.0));
}

// FF_matrix::apply ff_matrix.h:140-515: MAD-X MATRIX element, kick + linear
// map + second-order tensor (matrix_unit ff_algorithm.h:2439-2700).  The
// reference computes the design particle's image but never stores it, so
// the design particle is unchanged; a non-zero length is an error.
static void ops_matrix(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const Element& ele = lat.elements[sl.elem];
    if (ele.get("l", 0.0) != 0) throw Error(SB2_ERR_RUNTIME, "error, matrix element has non-zero length");
    MapOp o = new_op(OP_MATRIX);
    for (int i = 0; i < 6; ++i) o.d[i] = ele.get("kick" + std::to_string(i + 1), 0.0);
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j)
            o.d[6 + i * 6 + j] = ele.get("rm" + std::to_string(i + 1) + std::to_string(j + 1), i == j ? 1.0 : 0.0);
    auto it = lat.matrix_tensors.find(sl.elem);
    if (it != lat.matrix_tensors.end()) {
        o.flags = 1;
        const uint64_t bits = (uint64_t)(uintptr_t)it->second.get();
        std::memcpy(&o.d[42], &bits, sizeof(bits));
    }
    out.push_back(o);
    (void)b;
}

// FF_dipedge::apply ff_dipedge.h:196-330: MAD-X tmfrng edge focusing
// (linear, or with the second-order terms when `second_order` is set); the
// design particle takes the same map with its cdt zeroed.  (The reference
// propagates it inside the per-particle-group loop, so a bunch without valid
// particles leaves it alone; here it always moves, which changes nothing
// for a design particle on the axis.)
static void ops_dipedge(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const Element& ele = lat.elements[sl.elem];
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
    MapOp o = new_op(OP_DIPEDGE);
    o.d[0] = h * tanedg;
    o.d[1] = -h * std::tan(psip);
    double* te = o.d + 2;
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
    Refpart& ref_l = b.design;
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3];
    double nxp = xp + o.d[0] * x, nyp = yp + o.d[1] * y;
    double nx = x + te[0] * x * x + te[1] * y * y;
    nxp = nxp + te[2] * x * x + te[4] * y * y + te[3] * x * xp * 2.0 + te[5] * y * yp * 2.0;
    double ny = y + te[6] * x * y * 2.0;
    nyp = nyp + te[7] * x * y * 2.0 + te[8] * x * yp * 2.0 + te[9] * y * xp * 2.0;
    ref_l.state = {nx, nxp, ny, nyp, 0.0, ref_l.state[5]};
    out.push_back(o);
}

static void nllens_kick_cb(double x, double& xp, double y, double& yp, const double* k)
{
    hostff::nllens_unit(x, xp, y, yp, k);
}

static void ops_nllens(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{ // ff_nllens.h:9-50: thin only, through FF_patterned_propagator's thin kick
    const Element& el = lat.elements[sl.elem];
    const double l = el.get("l", 0.0);
    const double knll = el.get("knll");
    const double cnll = el.get("cnll");
    if (!hostff::close_to_zero(l)) throw Error(SB2_ERR_RUNTIME, "nonlinear lens has non-zero length");
    const double icnll = 1.0 / cnll;
    const double k[2] = {icnll, -knll * icnll};
    ops_patterned(sl, b, out, k, k, nllens_kick_cb, OP_THIN_NLLENS, -1, true, false, false, 1);
    if (std::isnan(b.design.state[1]) || std::isnan(b.design.state[3]))
        throw Error(SB2_ERR_RUNTIME, "the bunch reference particle hits the sigularity region "
                                     "when propagating through a nonlinearlens");
}

static void ops_kicker(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{ // ff_kicker.h:17-127; attributes as Lattice_element_processor::hkicker / vkicker / kicker
  // (lattice_element_processor.cc:86-159)
    const Element& el = lat.elements[sl.elem];
    const double length = sl.right - sl.left;
    double hk0 = el.get("hkick", 0.0), vk0 = el.get("vkick", 0.0);
    if (el.type == "hkicker") {
        if (el.has("kick")) hk0 = el.get("kick", 0.0);
        vk0 = 0.0;
    } else if (el.type == "vkicker") {
        if (el.has("kick")) vk0 = el.get("kick", 0.0);
        hk0 = 0.0;
    }
    const double l = el.get("l", 0.0);
    const double tilt = el.get("tilt", 0.0);
    const double hk = std::cos(tilt) * hk0 - std::sin(tilt) * vk0;
    const double vk = std::sin(tilt) * hk0 + std::cos(tilt) * vk0;
    const double scale = b.design.p / b.ref.p;
    const double q = (double)b.ref.charge / b.design.charge;
    double k[2] = {hk, vk};
    double sk[2] = {hk * q * scale, vk * q * scale};
    const bool thin = hostff::close_to_zero(length);
    if (!thin) {
        k[0] = k[0] / l;
        k[1] = k[1] / l;
        sk[0] = sk[0] / l;
        sk[1] = sk[1] / l;
    }
    ops_patterned(sl, b, out, k, sk, hostff::kicker_kick_cb, OP_THIN_KICK, OP_KICK_YOSHIDA, thin,
                  std::fabs(el.get("simple", 0.0)) > 1e-16, (int)el.get("cdt_use_drift", 0.0) != 0,
                  (int)el.get("yoshida_steps", 4.0));
}

static void ops_solenoid(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{ // ff_solenoid.h:160-248
    const Element& el = lat.elements[sl.elem];
    const double length = sl.right - sl.left;
    double ks = el.get("ks");
    Refpart& ref_l = b.design;
    const Refpart& ref_b = b.ref;
    if (std::fabs(ks) < 1e-12) {
        ops_drift(sl, b, out);
        return;
    }
    const double ref_p = ref_b.p * (1.0 + ref_b.state[5]);
    const double brho_l = ref_l.p * (1.0 + ref_l.state[5]) / ref_l.charge;
    const double brho_b = ref_b.p * (1.0 + ref_b.state[5]) / ref_l.charge;
    ks = ks * (brho_l / brho_b);
    const double ksl = ks * length;
    const double kse = ks * 0.5;
    // get_reference_cdt_solenoid :125-155
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], cdt = 0.0, dpop = 0.0;
    if (sl.ledge) {
        xp = xp + kse * y;
        yp = yp - kse * x;
    }
    hostff::solenoid_unit(x, xp, y, yp, cdt, dpop, ksl, ks, length, ref_l.p * (1 + dpop), ref_l.mass, 0.0);
    if (sl.redge) {
        xp = xp - kse * y;
        yp = yp + kse * x;
    }
    ref_l.state = {x, xp, y, yp, cdt, dpop};
    MapOp o = new_op(OP_SOLENOID);
    o.flags = (sl.ledge ? 1 : 0) | (sl.redge ? 2 : 0);
    o.d[0] = ksl; // passed as `ks`, as the reference does
    o.d[1] = ks;  // passed as `ksl`
    o.d[2] = length;
    o.d[3] = ref_p;
    o.d[4] = b.ref.mass;
    o.d[5] = cdt;
    o.d[6] = kse;
    out.push_back(o);
    b.ref.s_n += length;
}

static void ops_rfcavity(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{ // ff_rfcavity.h:134-330; the bunch reference momentum changes to the new one
    const Element& elm = lat.elements[sl.elem];
    const double length = sl.right - sl.left;
    const double volt = elm.get("volt", 0.0);
    double lag = elm.get("lag", 0.0);
    const double freq = elm.get("freq", -1.0);
    const double delta_freq = elm.get("delta_freq", 0.0);
    int nh = 1;
    double mhp[12] = {1.0, 1.0, 0.0};
    for (int h = 2; h <= 4; ++h) {
        const std::string sk = "h" + std::to_string(h) + "_str", pk = "h" + std::to_string(h) + "_phase";
        if (elm.has(sk)) {
            mhp[nh * 3 + 0] = h;
            mhp[nh * 3 + 1] = elm.get(sk, 0.0);
            mhp[nh * 3 + 2] = elm.get(pk, 0.0);
            ++nh;
        }
    }
    const double str = volt * 1.0e-3;
    while (lag < 0.0) lag += 1.0;
    while (lag >= 1.0) lag -= 1.0;
    const double pi = 3.14159265358979323846;
    const double phi_s = 2.0 * pi * lag;
    const double w_rf = 2.0 * pi * (freq + delta_freq) * 1.0e6;
    Refpart& ref_l = b.design;
    const double pref_b = b.ref.p, m_b = b.ref.mass;
    // thin_rfcavity_pnew ff_algorithm.h:1016-1022
    const double E0 = std::sqrt(pref_b * pref_b + m_b * m_b);
    const double E1 = E0 + str * std::sin(phi_s);
    const double new_pref_b = std::sqrt(E1 * E1 - m_b * m_b);
    // design particle: half drift, cavity at its own momentum, half drift
    double x = ref_l.state[0], xp = ref_l.state[1], y = ref_l.state[2], yp = ref_l.state[3], cdt = 0.0, dpop = 0.0;
    const double lp = ref_l.p, lm = ref_l.mass;
    hostff::drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * length, lp, lm, 0.0);
    double total = cdt;
    const double ref_cdt_1 = cdt;
    cdt = 0.0;
    if (str != 0.0) { // thin_rfcavity_unit with old = new = the design momentum
        double phase_slip_argument = (cdt * (w_rf / pc::c)) + 0.0;
        double strength_factor = 0.0;
        for (int i = 0; i < nh; ++i)
            strength_factor = strength_factor + mhp[i * 3 + 1] * std::sin(mhp[i * 3] * (phi_s + phase_slip_argument) +
                                                                          mhp[i * 3 + 2]);
        double p = lp * (dpop + 1.0);
        double E = std::sqrt(p * p + lm * lm);
        E = E + str * strength_factor;
        xp = xp * (lp / lp);
        yp = yp * (lp / lp);
        dpop = std::sqrt((E - lm) * (E + lm)) / lp - 1.0;
    }
    hostff::drift_unit(x, xp, y, yp, cdt, dpop, 0.5 * length, lp, lm, 0.0);
    total += cdt;
    const double ref_cdt_2 = cdt;
    ref_l.state = {x, xp, y, yp, total, 0.0};
    MapOp o = new_op(OP_RFCAVITY);
    o.steps = nh;
    o.flags = hostff::close_to_zero(length) ? 1 : 0;
    o.d[0] = 0.5 * length;
    o.d[1] = pref_b;
    o.d[2] = m_b;
    o.d[3] = ref_cdt_1;
    o.d[4] = ref_cdt_2;
    o.d[5] = w_rf;
    o.d[6] = str;
    o.d[7] = phi_s;
    o.d[8] = new_pref_b;
    for (int i = 0; i < 12; ++i) o.d[9 + i] = mhp[i];
    out.push_back(o);
    b.ref.set(b.ref.charge, b.ref.mass, new_pref_b, SB2_REF_MOMENTUM);
    b.ref.s_n += length;
}

// FF_element::apply ff_element.h:25-67
static void ops_slice(const Lattice& lat, const Slice& sl, Bunch& b, std::vector<MapOp>& out)
{
    const std::string& t = lat.elements[sl.elem].type;
    if (t == "drift" || t == "monitor" || t == "hmonitor" || t == "vmonitor" || t == "marker" || t == "instrument" ||
        t == "rcollimator")
        ops_drift(sl, b, out);
    else if (t == "sbend")
        ops_sbend(lat, sl, b, out);
    else if (t == "quadrupole")
        ops_quad(lat, sl, b, out);
    else if (t == "multipole")
        ops_multipole(lat, sl, b, out);
    else if (t == "sextupole")
        ops_sextupole(lat, sl, b, out);
    else if (t == "octupole")
        ops_octupole(lat, sl, b, out);
    else if (t == "hkicker" || t == "vkicker" || t == "kicker")
        ops_kicker(lat, sl, b, out);
    else if (t == "solenoid")
        ops_solenoid(lat, sl, b, out);
    else if (t == "rfcavity")
        ops_rfcavity(lat, sl, b, out);
    else if (t == "nllens")
        ops_nllens(lat, sl, b, out);
    else if (t == "dipedge")
        ops_dipedge(lat, sl, b, out);
    else if (t == "matrix")
        ops_matrix(lat, sl, b, out);
    else if (t == "elens" || t == "foil")
        throw Error(SB2_ERR_UNSUPPORTED, "element type " + t + " is not on the GPU path of this build (element " +
                                             lat.elements[sl.elem].name + ")");
    else
        throw Error(SB2_ERR_RUNTIME, "FF_element::apply() unknown element type = " + t + ", element name = " +
                                         lat.elements[sl.elem].name);
}

// Aperture_operation constructors (aperture_operation.h)
static MapOp op_aperture(const Lattice& lat, const std::string& type, const Slice& sl)
{
    const Element& el = lat.elements[sl.elem];
    if (type == "finite") return new_op(OP_AP_FINITE);
    if (type == "circular") {
        MapOp o = new_op(OP_AP_CIRCULAR);
        double r = el.get("circular_aperture_radius", 1000.0);
        o.d[0] = r * r;
        o.d[1] = el.get("hoffset", 0.0);
        o.d[2] = el.get("voffset", 0.0);
        return o;
    }
    if (type == "elliptical") {
        MapOp o = new_op(OP_AP_ELLIPTICAL);
        double hr = el.get("elliptical_aperture_horizontal_radius");
        double vr = el.get("elliptical_aperture_vertical_radius");
        o.d[0] = hr * hr;
        o.d[1] = vr * vr;
        o.d[2] = el.get("hoffset", 0.0);
        o.d[3] = el.get("voffset", 0.0);
        return o;
    }
    if (type == "rectangular") {
        MapOp o = new_op(OP_AP_RECTANGULAR);
        o.d[0] = el.get("rectangular_aperture_width");
        o.d[1] = el.get("rectangular_aperture_height");
        o.d[2] = el.get("hoffset", 0.0);
        o.d[3] = el.get("voffset", 0.0);
        return o;
    }
    throw Error(SB2_ERR_RUNTIME, "unknown aperture_type " + type);
}


// ---------------------------------------------------------------------------
// Launch signature: while a turn is captured into a CUDA graph or re-derived
// on the host, every flush and solve appends the bytes that determine its
// launches (op lists, bookkeeping program, time step, Ghat refresh).  In
// dry-run mode nothing is launched; the host state still advances.
// ---------------------------------------------------------------------------
struct LaunchSig {
    bool dry = false;
    std::vector<unsigned char>* sig = nullptr;
};
static thread_local LaunchSig g_sig;
static void sig_append(const void* p, size_t n)
{
    if (!g_sig.sig) return;
    const unsigned char* c = (const unsigned char*)p;
    g_sig.sig->insert(g_sig.sig->end(), c, c + n);
}

// ---------------------------------------------------------------------------
// Kernel-category timing with CUDA events on the launching stream (the
// reference's scoped_simple_timer labels, utils/simple_timer.h:50-66).
// Off unless sb2_profile_enable(1) is called.
// ---------------------------------------------------------------------------
enum ProfCat {
    PROF_TRACK = 0, // particle passes without Yoshida integrators or bends
    PROF_DOMAIN,
    PROF_DEPOSIT,
    PROF_GREEN,
    PROF_SOLVE,
    PROF_EFIELD,
    PROF_SORT,
    PROF_TRACK_FULL, // particle passes with Yoshida integrators or sector bends
    PROF_NCAT
};
static const char* kProfNames[PROF_NCAT] = {"track", "domain", "deposit", "green", "solve", "efield", "sort",
                                            "track_full"};

// A particle pass runs the full kernel variant when it holds a Yoshida
// integrator or a sector bend (track_impl.cuh makes the same choice).
static bool pass_is_full(const MapOp* ops, int n)
{
    for (int i = 0; i < n; ++i) {
        const int k = ops[i].kind;
        if (k == OP_QUAD || k == OP_QUAD_CF || k == OP_SEXT_YOSHIDA || k == OP_OCT_YOSHIDA || k == OP_KICK_YOSHIDA ||
            k == OP_SBEND || k == OP_SBEND_CF || k == OP_SOLENOID || k == OP_RFCAVITY)
            return true;
    }
    return false;
}

struct Profiler {
    bool on = false;
    struct Rec {
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs[PROF_NCAT];
    std::vector<cudaEvent_t> pool;
    double total_ms[PROF_NCAT] = {0};
    int64_t count[PROF_NCAT] = {0};

    cudaEvent_t ev()
    {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "event");
        return e;
    }
    Rec begin(int cat, cudaStream_t s)
    {
        (void)cat;
        Rec r{ev(), nullptr};
        cuda_check(cudaEventRecord(r.a, s), "event");
        return r;
    }
    void end(int cat, Rec r, cudaStream_t s)
    {
        r.b = ev();
        cuda_check(cudaEventRecord(r.b, s), "event");
        recs[cat].push_back(r);
    }
    void collect()
    {
        for (int c = 0; c < PROF_NCAT; ++c) {
            for (auto& r : recs[c]) {
                cuda_check(cudaEventSynchronize(r.b), "event");
                float ms = 0;
                cuda_check(cudaEventElapsedTime(&ms, r.a, r.b), "event");
                total_ms[c] += ms;
                count[c] += 1;
                pool.push_back(r.a);
                pool.push_back(r.b);
            }
            recs[c].clear();
        }
    }
    void reset()
    {
        collect();
        for (int c = 0; c < PROF_NCAT; ++c) {
            total_ms[c] = 0;
            count[c] = 0;
        }
    }
};
static Profiler g_prof;

struct ProfScope {
    int cat;
    cudaStream_t s;
    Profiler::Rec r{};
    ProfScope(int c, cudaStream_t st) : cat(c), s(st)
    {
        if (g_prof.on && !g_sig.sig) r = g_prof.begin(cat, s);
    }
    ~ProfScope()
    {
        if (g_prof.on && r.a) g_prof.end(cat, r, s);
    }
};

// ---------------------------------------------------------------------------
// Launch recording for a batch in lockstep: while g_rec is set, the launch
// sites of one bunch's step append what they would launch to it instead of
// launching; Batch::run_lockstep then issues the records of all bunches as
// work-list launches, one per kernel kind (and grid shape).
// ---------------------------------------------------------------------------
struct LaunchRec {
    enum Kind { TRACK, DOMAIN, ZERO, DEPOSIT, GREEN, CONV, EFIELD, SORT } kind = TRACK;
    std::vector<unsigned char> tp; // TRACK: TrackParams header and its nops ops
    int choice = 0, ctas_per_sm = 8;
    bool fast = false, has_mom = false;
    int64_t n = 0;
    DomainParams dp;   // DOMAIN
    ZeroItem z{};      // ZERO
    DepositItem dep{}; // DEPOSIT
    bool f32 = false;
    ConvItem ci{}; // GREEN, CONV, EFIELD
    Dims d{};
    int linear = 0, mode = 0;
    const double2* tw64[3] = {nullptr, nullptr, nullptr};
    const float2* tw32[3] = {nullptr, nullptr, nullptr};
    SortItem sort{}; // SORT
};
static thread_local std::vector<LaunchRec>* g_rec = nullptr;

// ---------------------------------------------------------------------------
// Space-charge operator: options, workspaces, solve
// ---------------------------------------------------------------------------
static bool is_pow2(int v) { return v > 1 && (v & (v - 1)) == 0; }
static int ilog2(int v)
{
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

// Sum over the ranks of a bunch split by particle range (the reference's
// MPI_Allreduce of the moment sums, core_diagnostics.cc:444, of the charge
// density, space_charge_3d_open_hockney.cc:572, and of the valid counts in
// update_total_num).  The caller's function sums `count` doubles in place
// and returns 0; the library has finished its own work on the stream before
// the call.  With on_host the data is staged through pinned host memory (a
// host-side collective such as gloo or MPI), otherwise the function gets the
// device pointer (NCCL).
// stream of the exchange a sum-allreduce callback is running for
static thread_local cudaStream_t g_hook_stream = nullptr;

struct AllreduceHook {
    sb2_allreduce_fn fn = nullptr;
    sb2_allreduce_typed_fn tfn = nullptr; // typed: FP32 buffers too
    void* ctx = nullptr;
    int on_host = 0;
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    ~AllreduceHook()
    {
        if (pinned) cudaFreeHost(pinned);
    }
    explicit operator bool() const { return fn != nullptr || tfn != nullptr; }
    bool typed() const { return tfn != nullptr; }
    // Host buffers: the stream is drained, the data staged through pinned
    // memory, summed by the callback and copied back.  Device buffers: the
    // callback is called at once with the device pointer and must order its
    // collective on the library's stream (sb2_allreduce_stream() inside the
    // callback), so nothing waits on the host.
    void run(double* dev, int64_t n, cudaStream_t s) { run_bytes(dev, n, 0, s); }
    void run(float* dev, int64_t n, cudaStream_t s)
    {
        if (!tfn) throw Error(SB2_ERR_RUNTIME, "FP32 exchange without a typed allreduce");
        run_bytes(dev, n, 1, s);
    }

  private:
    int32_t call(void* data, int64_t n, int dtype, int host)
    {
        return tfn ? tfn(ctx, data, n, dtype, host) : fn(ctx, (double*)data, n, host);
    }
    void run_bytes(void* dev, int64_t n, int dtype, cudaStream_t s)
    {
        struct StreamScope {
            cudaStream_t prev;
            explicit StreamScope(cudaStream_t st) : prev(g_hook_stream) { g_hook_stream = st; }
            ~StreamScope() { g_hook_stream = prev; }
        } scope(s);
        const size_t bytes = (size_t)n * (dtype ? sizeof(float) : sizeof(double));
        int32_t rc;
        if (on_host) {
            cuda_check(cudaStreamSynchronize(s), "allreduce");
            if (pinned_bytes < bytes) {
                if (pinned) cudaFreeHost(pinned);
                pinned = nullptr;
                pinned_bytes = 0;
                cuda_check(cudaMallocHost(&pinned, bytes), "allreduce staging");
                pinned_bytes = bytes;
            }
            cuda_check(cudaMemcpy(pinned, dev, bytes, cudaMemcpyDeviceToHost), "allreduce staging");
            rc = call(pinned, n, dtype, 1);
            cuda_check(cudaMemcpy(dev, pinned, bytes, cudaMemcpyHostToDevice), "allreduce staging");
        } else {
            rc = call(dev, n, dtype, 0);
        }
        if (rc != 0) throw Error(SB2_ERR_RUNTIME, "allreduce callback failed");
    }
};

struct SpaceCharge {
    AllreduceHook* hook = nullptr; // bunch split over ranks
    sb2_sc3d_options o;
    Dims d{};
    int64_t G = 0;
    bool mixed = false;
    double* rho = nullptr;
    double2* S = nullptr;
    double* ghat = nullptr;
    double* phi = nullptr;
    double2* E = nullptr;
    double2 *tw_x = nullptr, *tw_y = nullptr, *tw_z = nullptr;
    // mixed precision: FP32 charge grid (FP64 when the charge is exchanged
    // between ranks), spectrum, potential and field; FP64 butterflies.
    // SB2_MIXED_BUTTERFLIES=fp32 selects FP32 butterflies: 3% faster on the
    // 4M-particle FODO step but 1.0e-5 / 1.8e-5 field error at 64^2 x 128 /
    // 128^2 x 256 (the finite-difference field magnifies the transforms'
    // rounding about 100x), against 4.4e-6 / 7.0e-6 with FP64 butterflies
    float* rho32 = nullptr;
    float2* S32 = nullptr;
    float* phi32 = nullptr;
    float4* E32 = nullptr;
    float2 *tw32_x = nullptr, *tw32_y = nullptr, *tw32_z = nullptr;
    int fp32_butterflies = 0;
    bool last_rho32 = false; // the last solve's charge is in rho32
    int deposit_chunk = deposit_default_chunk(); // particles per thread of the tile deposit (0: warp groups)
    ScState* state = nullptr;
    double* mom_partials = nullptr;
    int n_partials = 0;
    bool ghat_valid = false;

    // Option checks done at construction, before any device allocation.
    static void validate(const sb2_sc3d_options& o)
    {
        for (int i = 0; i < 3; ++i) {
            if (o.shape[i] < 3) throw Error(SB2_ERR_INVALID, "space-charge grid shape must be >= 3 in each dimension");
            if (o.doubled_shape[i] != 2 * o.shape[i])
                throw Error(SB2_ERR_UNSUPPORTED, "doubled_shape must be 2 * shape on the GPU path");
            if (!is_pow2(o.doubled_shape[i]) || o.doubled_shape[i] < 8 || o.doubled_shape[i] > 2048)
                throw Error(SB2_ERR_UNSUPPORTED, "doubled grid sizes must be powers of two in [8, 2048] on the GPU path");
        }
        if (o.periodic_z)
            throw Error(SB2_ERR_RUNTIME, "Space_charge_3d_open_hockney::get_green_fn2_linear: periodic_z not yet implemented");
        if (o.precision != SB2_PRECISION_FP64 && o.precision != SB2_PRECISION_MIXED)
            throw Error(SB2_ERR_INVALID, "unknown precision");
        if (o.domain_fixed)
            for (int i = 0; i < 3; ++i)
                if (!(o.size[i] > 0.0)) throw Error(SB2_ERR_INVALID, "fixed domain size must be > 0");
    }

    explicit SpaceCharge(const sb2_sc3d_options& opts) : o(opts)
    {
        validate(o);
        d.gx = o.shape[0];
        d.gy = o.shape[1];
        d.gz = o.shape[2];
        d.nx = o.doubled_shape[0];
        d.ny = o.doubled_shape[1];
        d.nz = o.doubled_shape[2];
        d.nkx = d.nx / 2 + 1;
        d.nkxp = (d.nkx + 1) & ~1;
        d.lx = ilog2(d.nx);
        d.ly = ilog2(d.ny);
        d.lz = ilog2(d.nz);
        G = (int64_t)d.gx * d.gy * d.gz;
        mixed = o.precision == SB2_PRECISION_MIXED;
        if (mixed) {
            rho32 = dalloc<float>(G, "rho");
            phi32 = dalloc<float>(G, "phi");
            E32 = dalloc<float4>(G, "E");
            S32 = dalloc<float2>((size_t)d.nz * d.ny * d.nkxp, "spectrum");
            cuda_check(cudaMemset(E32, 0, sizeof(float4) * G), "memset");
        } else {
            rho = dalloc<double>(G, "rho");
            phi = dalloc<double>(G, "phi");
            E = dalloc<double2>(2 * G, "E");
            S = dalloc<double2>((size_t)d.nz * d.ny * d.nkxp, "spectrum");
            cuda_check(cudaMemset(E, 0, sizeof(double2) * 2 * G), "memset");
        }
        ghat = dalloc<double>((size_t)(d.nx / 2 + 1) * (d.ny / 2 + 1) * (d.nz / 2 + 1), "ghat");
        state = dalloc<ScState>(1, "sc state");
        n_partials = track_grid_blocks();
        mom_partials = dalloc<double>((size_t)track_grid_blocks(kMaxCtasPerSm) * 6, "moments"); // any tuned grid
        cuda_check(cudaMemset(state, 0, sizeof(ScState)), "memset");
        tw_x = twiddles(d.nx);
        tw_y = twiddles(d.ny);
        tw_z = twiddles(d.nz);
        if (mixed) {
            tw32_x = twiddles32(d.nx);
            tw32_y = twiddles32(d.ny);
            tw32_z = twiddles32(d.nz);
            const char* e = getenv("SB2_MIXED_BUTTERFLIES");
            if (e && !strcmp(e, "fp32")) fp32_butterflies = 1;
        }
    }
    ~SpaceCharge()
    {
        dfree(rho);
        dfree(phi);
        dfree(E);
        dfree(S);
        dfree(ghat);
        dfree(state);
        dfree(mom_partials);
        dfree(tw_x);
        dfree(tw_y);
        dfree(tw_z);
        dfree(S32);
        dfree(phi32);
        dfree(E32);
        dfree(rho32);
        dfree(tw32_x);
        dfree(tw32_y);
        dfree(tw32_z);
    }
    // exp(-2 pi i k / L), k < L, from long-double sin/cos
    static double2* twiddles(int L)
    {
        std::vector<double2> h(L);
        for (int k = 0; k < L; ++k) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * k / L;
            h[k] = make_double2((double)std::cos(a), (double)std::sin(a));
        }
        double2* dp = dalloc<double2>(L, "twiddles");
        cuda_check(cudaMemcpy(dp, h.data(), sizeof(double2) * L, cudaMemcpyHostToDevice), "twiddles");
        return dp;
    }
    // the same in FP32, each rounded once from the long-double value
    static float2* twiddles32(int L)
    {
        std::vector<float2> h(L);
        for (int k = 0; k < L; ++k) {
            long double a = -2.0L * 3.14159265358979323846264338327950288L * k / L;
            h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        float2* dp = dalloc<float2>(L, "twiddles");
        cuda_check(cudaMemcpy(dp, h.data(), sizeof(float2) * L, cudaMemcpyHostToDevice), "twiddles");
        return dp;
    }

    DomainParams domain_params(const Bunch& b, double time_step) const
    {
        DomainParams p;
        std::memset(&p, 0, sizeof(p));
        p.counters = b.counters;
        p.moment_partials = mom_partials;
        p.n_partials = n_partials;
        p.compute_domain = 1;
        p.sc = state;
        for (int i = 0; i < 3; ++i) {
            p.g[i] = o.shape[i];
            p.dg[i] = o.doubled_shape[i];
            p.fixed_size[i] = o.size[i];
            p.fixed_offset[i] = o.offset[i];
        }
        p.domain_fixed = o.domain_fixed;
        p.grid_entire_period = o.grid_entire_period;
        p.green_linear = o.green_fn == SB2_GREEN_LINEAR;
        p.n_sigma = o.n_sigma;
        p.z_period = o.z_period;
        p.kick_scale = o.kick_scale;
        p.charge = b.ref.charge;
        p.pref = b.ref.p;
        p.gamma = b.ref.gamma;
        p.beta = b.ref.beta;
        p.time_step = time_step;
        return p;
    }

    // deposit -> Ghat (if needed) -> convolution -> E; the domain is already
    // in `state`.
    void solve(const Bunch& b, cudaStream_t s)
    {
        const bool refresh = !o.domain_fixed || !ghat_valid;
        sig_append(&refresh, sizeof(refresh));
        const void* arrays[2] = {b.parts, b.masks};
        sig_append(arrays, sizeof(arrays));
        if (g_sig.dry) {
            if (refresh) ghat_valid = true;
            return;
        }
        const bool exchange = hook && *hook;
        // an FP32 charge grid is exchanged as float through a typed callback
        last_rho32 = mixed && (!exchange || hook->typed());
        if (g_rec) {
            record_solve(b);
            return;
        }
        {
            ProfScope ps(PROF_DEPOSIT, s);
            if (last_rho32) {
                cuda_check(cudaMemsetAsync(rho32, 0, sizeof(float) * G, s), "memset rho");
                cuda_check(launch_deposit_f32_k(deposit_chunk, b.parts, b.stride, b.masks, b.n, state, rho32, d.gx,
                                                d.gy, d.gz, s),
                           "deposit");
            } else {
                if (!rho) rho = dalloc<double>(G, "rho"); // mixed precision with an exchange: FP64 charge
                cuda_check(cudaMemsetAsync(rho, 0, sizeof(double) * G, s), "memset rho");
                cuda_check(launch_deposit_k(deposit_chunk, b.parts, b.stride, b.masks, b.n, state, rho, d.gx, d.gy,
                                            d.gz, s),
                           "deposit");
            }
        }
        if (exchange) { // charge of all ranks
            if (last_rho32)
                hook->run(rho32, G, s);
            else
                hook->run(rho, G, s);
        }
        if (!o.domain_fixed || !ghat_valid) {
            ProfScope ps(PROF_GREEN, s);
            cuda_check(launch_green(state, ghat, d, o.green_fn == SB2_GREEN_LINEAR, tw_x, tw_y, tw_z, s), "green");
            ghat_valid = true;
        }
        {
            ProfScope ps(PROF_SOLVE, s);
            if (mixed) {
                MixedConv m;
                m.rho32 = last_rho32 ? rho32 : nullptr;
                m.rho64 = last_rho32 ? nullptr : rho;
                m.tw64[0] = tw_x;
                m.tw64[1] = tw_y;
                m.tw64[2] = tw_z;
                m.tw32[0] = tw32_x;
                m.tw32[1] = tw32_y;
                m.tw32[2] = tw32_z;
                m.fp32_butterflies = fp32_butterflies;
                cuda_check(launch_convolve_mixed(m, S32, ghat, phi32, d, state, s), "convolve");
            } else
                cuda_check(launch_convolve(rho, S, ghat, phi, d, tw_x, tw_y, tw_z, state, s), "convolve");
        }
        {
            ProfScope ps(PROF_EFIELD, s);
            if (mixed)
                cuda_check(launch_efield_f32(phi32, E32, d.gx, d.gy, d.gz, state, s), "efield");
            else
                cuda_check(launch_efield(phi, E, d.gx, d.gy, d.gz, state, s), "efield");
        }
    }

    // solve() recorded for a batch in lockstep (the same launches)
    void record_solve(const Bunch& b)
    {
        if (!last_rho32 && !rho) rho = dalloc<double>(G, "rho");
        LaunchRec z;
        z.kind = LaunchRec::ZERO;
        z.z.ptr = last_rho32 ? (void*)rho32 : (void*)rho;
        z.z.bytes = (last_rho32 ? (int64_t)sizeof(float) : (int64_t)sizeof(double)) * G;
        g_rec->push_back(z);
        LaunchRec dep;
        dep.kind = LaunchRec::DEPOSIT;
        dep.dep = DepositItem{b.parts, b.stride, b.masks, b.n, state, z.z.ptr};
        dep.f32 = last_rho32;
        dep.d = d;
        g_rec->push_back(dep);
        ConvItem ci{};
        ci.rho = z.z.ptr;
        ci.S = mixed ? (void*)S32 : (void*)S;
        ci.ghat = ghat;
        ci.phi = mixed ? (void*)phi32 : (void*)phi;
        ci.E = mixed ? (void*)E32 : (void*)E;
        ci.sc = state;
        if (!o.domain_fixed || !ghat_valid) {
            LaunchRec g;
            g.kind = LaunchRec::GREEN;
            g.ci = ci;
            g.d = d;
            g.linear = o.green_fn == SB2_GREEN_LINEAR;
            g.tw64[0] = tw_x;
            g.tw64[1] = tw_y;
            g.tw64[2] = tw_z;
            g_rec->push_back(g);
            ghat_valid = true;
        }
        LaunchRec c;
        c.kind = LaunchRec::CONV;
        c.ci = ci;
        c.d = d;
        c.mode = !mixed ? 0 : last_rho32 ? (fp32_butterflies ? 1 : 3) : (fp32_butterflies ? 2 : 4);
        c.tw64[0] = tw_x;
        c.tw64[1] = tw_y;
        c.tw64[2] = tw_z;
        c.tw32[0] = tw32_x;
        c.tw32[1] = tw32_y;
        c.tw32[2] = tw32_z;
        g_rec->push_back(c);
        LaunchRec e;
        e.kind = LaunchRec::EFIELD;
        e.ci = ci;
        e.d = d;
        e.f32 = mixed;
        g_rec->push_back(e);
    }

    void copy_last(double* left, double* h, double* rho_o, double* phi_o, double* ex, double* ey, double* ez,
                   double* scalars)
    {
        ScState st;
        cuda_check(cudaMemcpy(&st, state, sizeof(st), cudaMemcpyDeviceToHost), "state");
        if (left)
            for (int i = 0; i < 3; ++i) left[i] = st.left[i];
        if (h)
            for (int i = 0; i < 3; ++i) h[i] = st.h[i];
        if (rho_o) {
            if (last_rho32) {
                std::vector<float> f(G);
                cuda_check(cudaMemcpy(f.data(), rho32, sizeof(float) * G, cudaMemcpyDeviceToHost), "rho");
                for (int64_t i = 0; i < G; ++i) rho_o[i] = f[i];
            } else if (rho) {
                cuda_check(cudaMemcpy(rho_o, rho, sizeof(double) * G, cudaMemcpyDeviceToHost), "rho");
            }
        }
        if (phi_o) {
            if (mixed) {
                std::vector<float> f(G);
                cuda_check(cudaMemcpy(f.data(), phi32, sizeof(float) * G, cudaMemcpyDeviceToHost), "phi");
                for (int64_t i = 0; i < G; ++i) phi_o[i] = f[i];
            } else
                cuda_check(cudaMemcpy(phi_o, phi, sizeof(double) * G, cudaMemcpyDeviceToHost), "phi");
        }
        if (ex || ey || ez) {
            if (mixed) {
                std::vector<float4> e(G);
                cuda_check(cudaMemcpy(e.data(), E32, sizeof(float4) * G, cudaMemcpyDeviceToHost), "E");
                for (int64_t i = 0; i < G; ++i) {
                    if (ex) ex[i] = e[i].x;
                    if (ey) ey[i] = e[i].y;
                    if (ez) ez[i] = e[i].z;
                }
            } else {
                std::vector<double2> e(2 * G);
                cuda_check(cudaMemcpy(e.data(), E, sizeof(double2) * 2 * G, cudaMemcpyDeviceToHost), "E");
                for (int64_t i = 0; i < G; ++i) {
                    if (ex) ex[i] = e[2 * i].x;
                    if (ey) ey[i] = e[2 * i].y;
                    if (ez) ez[i] = e[2 * i + 1].x;
                }
            }
        }
        if (scalars) {
            scalars[0] = st.fn_norm;
            scalars[1] = st.factor;
            for (int j = 0; j < 6; ++j) scalars[2 + j] = st.mean_std[j];
        }
    }

    void check_error()
    {
        ScState st;
        cuda_check(cudaMemcpy(&st, state, sizeof(st), cudaMemcpyDeviceToHost), "state");
        if (st.error == 1)
            throw Error(SB2_ERR_RUNTIME, "Space_charge_3d_open_hockney_eigen::update_domain: all three spatial "
                                         "dimensions have neglible extent");
    }
};


// ---------------------------------------------------------------------------
// Engine: accumulates the particle-local ops of consecutive operators and
// launches them as fused particle passes (one read + one write of the
// particle array per pass), followed by the bookkeeping/domain kernel.
// ---------------------------------------------------------------------------
struct Engine {
    int32_t* ap_counts = nullptr;
    std::vector<MapOp> ops;
    PassBook book{};
    int nslots = 0;
    AllreduceHook* hook = nullptr; // bunch split over ranks
    double* xchg = nullptr;        // [6 moment sums][discards per slot]
    // Diagnostics_loss: lost-particle records on the device, and per
    // aperture the (repetition, s, s_n) of the bunch reference at it
    double* loss_buf = nullptr;
    int32_t* loss_count = nullptr;
    int32_t loss_cap = 0;
    std::vector<std::array<double, 3>>* loss_tags = nullptr;
    // Per-step count records (the counts Bunch_simulator::reg_diag_per_step
    // would see): the bookkeeping writes the counters after each step's last
    // operator into rec_dev; every flush copies the records it completed to
    // the caller's host buffer in stream order.
    BunchCounters* rec_dev = nullptr;
    BunchCounters* rec_host = nullptr;
    int32_t* rec_cursor = nullptr; // device cursor when rec_host is pinned (written by the device directly)
    TrackTune tune = track_tune_defaults(); // launch shape of the particle passes
    int32_t rec_cap = 0, rec_next = 0;
    int32_t rec_first = -1, rec_count = 0; // records completed by the pending book

    Engine()
    {
        ap_counts = dalloc<int32_t>(kMaxSlotsPerPass, "aperture counters");
        cuda_check(cudaMemset(ap_counts, 0, sizeof(int32_t) * kMaxSlotsPerPass), "memset");
        reset();
    }
    ~Engine()
    {
        dfree(ap_counts);
        dfree(xchg);
    }
    void reset()
    {
        ops.clear();
        std::memset(&book, 0, sizeof(book));
        for (int o = 0; o < kMaxOperatorsPerPass; ++o) book.op_record[o] = -1;
        nslots = 0;
        rec_first = -1;
        rec_count = 0;
    }

    // End of a step: an empty operator whose bookkeeping writes the next
    // count record (when records are enabled and capacity is left).
    void mark_step_end(Bunch& b, SpaceCharge* sc, double* elem_charge, cudaStream_t s)
    {
        if (!rec_cap || rec_next >= rec_cap) return;
        if (book.n_operators == kMaxOperatorsPerPass) flush(b, sc, elem_charge, false, 0.0, s);
        const int o = book.n_operators++;
        book.slot_begin[o] = book.slot_end[o] = nslots;
        book.op_record[o] = rec_cursor ? 0 : rec_next; // with the device cursor a flag, so turns stay alike
        if (rec_first < 0) rec_first = rec_next;
        ++rec_count;
        ++rec_next;
    }

    // One independent operator: its libFF groups and apertures, then
    // update_total_num (independent_operator.cc:94-133).
    void add_operator(const Lattice& lat, const IndepOperator& op, Bunch& b, SpaceCharge* sc, double* elem_charge,
                      cudaStream_t s)
    {
        int naps = 0;
        for (auto const& o : op.ops) naps += o.aperture ? 1 : 0;
        if (naps > kMaxSlotsPerPass) throw Error(SB2_ERR_UNSUPPORTED, "too many apertures in one operator");
        if (book.n_operators == kMaxOperatorsPerPass || nslots + naps > kMaxSlotsPerPass)
            flush(b, sc, elem_charge, false, 0.0, s);
        int first = nslots;
        for (auto const& o : op.ops) {
            if (o.aperture) {
                MapOp m = op_aperture(lat, o.ap_type, o.ap_slice);
                m.slot = nslots;
                if (loss_tags) {
                    m.d[10] = (double)loss_tags->size();
                    loss_tags->push_back({(double)b.ref.repetition, b.ref.repetition * b.ref.s + b.ref.s_n, b.ref.s_n});
                }
                book.slot_elem[nslots] = o.ap_slice.elem;
                ++nslots;
                ops.push_back(m);
            } else {
                for (auto const& sl : o.group) ops_slice(lat, sl, b, ops);
            }
        }
        book.slot_begin[book.n_operators] = first;
        book.slot_end[book.n_operators] = nslots;
        ++book.n_operators;
    }

    // the kick uses the bunch's reference momentum at the kick (an rf
    // cavity later in the same pass changes it)
    void add_kick(const Bunch& b)
    {
        MapOp o = new_op(OP_SC_KICK);
        o.d[0] = b.ref.p;
        o.d[1] = b.ref.mass;
        ops.push_back(o);
    }

    // Launch the pending ops.  with_domain: append the moment sums and run
    // the domain computation for a space-charge kick of `time_step`.
    void flush(Bunch& b, SpaceCharge* sc, double* elem_charge, bool with_domain, double time_step, cudaStream_t s)
    {
        if (with_domain && !sc->o.domain_fixed) ops.push_back(new_op(OP_MOMENTS));
        if (sc) sc->n_partials = track_grid_blocks(tune.ctas_per_sm); // one moment partial per pass block
        if (g_sig.sig) {
            // a replayed graph reads the arrays it was captured with
            const void* arrays[5] = {b.parts, b.masks, b.discards, b.counters, (const void*)(intptr_t)b.n};
            sig_append(arrays, sizeof(arrays));
            uint64_t nops = ops.size();
            sig_append(&nops, sizeof(nops));
            if (nops) sig_append(ops.data(), sizeof(MapOp) * nops);
            sig_append(&book, sizeof(book));
            sig_append(&tune, sizeof(tune));
            sig_append(&with_domain, sizeof(with_domain));
            sig_append(&time_step, sizeof(time_step));
        }
        if (g_sig.dry) {
            reset();
            return;
        }
        size_t i = 0;
        while (i < ops.size()) {
            size_t n = std::min<size_t>(kMaxOpsPerPass, ops.size() - i);
            TrackParams tp;
            std::memset(&tp, 0, offsetof(TrackParams, ops));
            tp.parts = b.parts;
            tp.stride = b.stride;
            tp.masks = b.masks;
            tp.discards = b.discards;
            tp.n = b.n;
            tp.ap_counts = ap_counts;
            tp.nops = (int32_t)n;
            tp.slot_base = -1;
            bool has_mom = false;
            for (size_t k = 0; k < n; ++k) {
                const MapOp& m = ops[i + k];
                tp.ops[k] = m;
                if (m.kind >= OP_AP_FINITE && m.kind <= OP_AP_RECTANGULAR) {
                    tp.write_discards = 1;
                    if (tp.slot_base < 0) tp.slot_base = m.slot;
                }
                if (m.kind == OP_MOMENTS) has_mom = true;
            }
            if (tp.slot_base < 0) tp.slot_base = 0;
            if (sc) {
                tp.sc = sc->state;
                tp.efield = sc->E;
                tp.efield32 = sc->E32;
                tp.fast_maps = sc->mixed ? 1 : 0;
                tp.gx = sc->d.gx;
                tp.gy = sc->d.gy;
                tp.gz = sc->d.gz;
                if (has_mom) tp.moment_partials = sc->mom_partials;
            }
            if (loss_buf) {
                tp.loss_buf = loss_buf;
                tp.loss_count = loss_count;
                tp.loss_cap = loss_cap;
            }
            if (g_rec) {
                LaunchRec r;
                r.kind = LaunchRec::TRACK;
                const size_t bytes = offsetof(TrackParams, ops) + sizeof(MapOp) * (size_t)tp.nops;
                r.tp.assign((const unsigned char*)&tp, (const unsigned char*)&tp + bytes);
                r.choice = track_pass_choice(tp, tune);
                r.ctas_per_sm = tune.ctas_per_sm;
                r.fast = tp.fast_maps != 0;
                r.has_mom = tp.moment_partials != nullptr;
                r.n = tp.n;
                g_rec->push_back(std::move(r));
            } else {
                ProfScope ps(pass_is_full(tp.ops, tp.nops) ? PROF_TRACK_FULL : PROF_TRACK, s);
                cuda_check(launch_track(tp, tune, s), "track kernel");
            }
            i += n;
        }
        if (book.n_operators > 0 || with_domain) {
            DomainParams dp;
            if (with_domain)
                dp = sc->domain_params(b, time_step);
            else {
                std::memset(&dp, 0, sizeof(dp));
                dp.counters = b.counters;
            }
            dp.ap_counts = ap_counts;
            dp.elem_charge = elem_charge;
            dp.book = book;
            dp.xchg = nullptr;
            dp.step_records = rec_count ? (rec_cursor ? rec_host : rec_dev) : nullptr;
            dp.rec_cursor = rec_count ? rec_cursor : nullptr;
            dp.rec_cap = rec_cap;
            if (hook && *hook) {
                if (!xchg) xchg = dalloc<double>(6 + kMaxSlotsPerPass, "exchange");
                cuda_check(launch_shard_pack(dp, nslots, xchg, s), "shard pack");
                hook->run(xchg, 6 + nslots, s);
                dp.xchg = xchg;
            }
            if (g_rec) {
                LaunchRec r;
                r.kind = LaunchRec::DOMAIN;
                r.dp = dp;
                g_rec->push_back(std::move(r));
            } else {
                ProfScope ps(PROF_DOMAIN, s);
                cuda_check(launch_book_domain(dp, s), "domain kernel");
            }
            if (rec_count && !rec_cursor) // pageable buffer: copied in stream order
                cuda_check(cudaMemcpyAsync(rec_host + rec_first, rec_dev + rec_first, sizeof(BunchCounters) * rec_count,
                                           cudaMemcpyDeviceToHost, s),
                           "step records");
        }
        reset();
    }
};

// ---------------------------------------------------------------------------
// Propagator
// ---------------------------------------------------------------------------
struct Propagator {
    Lattice lat;
    int stepper = 0, num = 1;
    std::vector<Step> steps;
    bool has_sc = false;
    sb2_sc3d_options sc_opts{};
    // device resources, allocated on first propagate
    std::unique_ptr<SpaceCharge> sc;
    std::unique_ptr<Engine> engine_;
    double* elem_charge = nullptr;
    // cell-ordered working copy of the bunch (space-charge runs only)
    bool cell_sort = true;
    int sort_interval = 4; // re-sort before every k-th space-charge kick (measured best of 1, 2, 4, 8 at 4M particles)
    TrackTune tune = track_tune_defaults(); // launch shape of the particle passes
    // space-charge launch shapes: FFT radix plan of the line passes, particles
    // per thread of the tile deposit
    struct SolveTune {
        int fft_plan = 0;
        int deposit_chunk = deposit_default_chunk();
        bool operator==(const SolveTune& o) const { return fft_plan == o.fft_plan && deposit_chunk == o.deposit_chunk; }
    } solve_tune;
    int32_t* sort_scratch = nullptr; // histogram, offsets (the scatter's cursors) and block sums of the counting sort

    Propagator(const Lattice& l, int stepper_kind, int n, const sb2_sc3d_options* opts)
        : lat(l), stepper(stepper_kind), num(n)
    {
        if (!lat.has_ref) throw Error(SB2_ERR_INVALID, "lattice has no reference particle");
        if (opts) {
            SpaceCharge::validate(*opts);
            sc_opts = *opts;
            has_sc = true;
        }
        steps = make_steps(lat, stepper, num, has_sc);
        for (size_t i = 0; i < lat.elements.size(); ++i) { // FF_matrix second-order terms, on the device
            const Element& e = lat.elements[i];
            if (e.type != "matrix") continue;
            std::vector<double> tm(216);
            bool any = false;
            for (int a = 0; a < 6; ++a)
                for (int j = 0; j < 6; ++j)
                    for (int l = 0; l < 6; ++l) {
                        const std::string k = "tm" + std::to_string(a + 1) + std::to_string(j + 1) + std::to_string(l + 1);
                        tm[(a * 6 + j) * 6 + l] = e.get(k, 0.0);
                        any |= tm[(a * 6 + j) * 6 + l] != 0.0;
                    }
            if (!any) continue;
            double* dev = dalloc<double>(216, "matrix tensor");
            cuda_check(cudaMemcpy(dev, tm.data(), sizeof(double) * 216, cudaMemcpyHostToDevice), "matrix tensor");
            lat.matrix_tensors[(int)i] = std::shared_ptr<double>(dev, [](double* p) { dfree(p); });
        }
        const char* e = getenv("SB2_CELL_SORT");
        if (e && atoi(e) == 0) cell_sort = false;
        const char* k = getenv("SB2_SORT_INTERVAL");
        if (k && atoi(k) > 0) sort_interval = atoi(k);
    }
    ~Propagator()
    {
        drop_graphs();
        if (own_stream) cudaStreamDestroy(own_stream);
        dfree(elem_charge);
        dfree(sort_scratch);
        dfree(diag_records);
        dfree(diag_count);
        dfree(diag_partials);
        dfree(diag_tmp);
        dfree(loss_buf);
        dfree(step_rec_dev);
        dfree(step_rec_cursor);
        dfree(loss_count);
    }

    bool sorting(const Bunch& b) const { return has_sc && cell_sort && b.n >= 64; }

    // Start of a propagate call: space-charge runs work on the bunch's
    // cell-ordered working copy (entered from the home arrays if the bunch
    // is not already there).
    void enter_sorted(Bunch& b, cudaStream_t s)
    {
        sort_active = false;
        if (!sorting(b)) return;
        if (!sort_scratch) {
            const int64_t G = (int64_t)sc_opts.shape[0] * sc_opts.shape[1] * sc_opts.shape[2];
            sort_scratch = dalloc<int32_t>(sort_scratch_ints(G), "sort scratch");
        }
        if (!b.permuted) {
            ProfScope ps(PROF_SORT, s);
            b.enter_work(s);
        }
        sort_active = true;
    }
    // End of a propagate call: a bunch over caller-owned arrays is brought
    // back to them at once (the caller may read them directly); an owned
    // bunch stays in the working copy until the caller next touches it.
    void leave_sorted(Bunch& b, cudaStream_t s)
    {
        sort_active = false;
        if (b.permuted && !b.owns) {
            ProfScope ps(PROF_SORT, s);
            b.settle(s);
        }
    }

    // Re-sort the working copy by the cells of the current domain.
    void resort(Bunch& b, cudaStream_t s)
    {
        if (g_rec) {
            LaunchRec r;
            r.kind = LaunchRec::SORT;
            r.sort.sb = b.wc;
            r.sort.sc = sc->state;
            r.sort.scratch = sort_scratch;
            r.sort.gx = sc->d.gx;
            r.sort.gy = sc->d.gy;
            r.sort.gz = sc->d.gz;
            g_rec->push_back(std::move(r));
        } else if (!g_sig.dry) {
            ProfScope ps(PROF_SORT, s);
            cuda_check(launch_cell_sort(b.wc, sort_scratch, sc->state, sc->d.gx, sc->d.gy, sc->d.gz, s), "cell sort");
        }
        b.swap_work();
    }

    AllreduceHook hook; // set when the bunch is split over ranks

    void ensure_device()
    {
        if (!engine_) engine_.reset(new Engine());
        if (has_sc && !sc) {
            sc.reset(new SpaceCharge(sc_opts));
            sc->d.plan = solve_tune.fft_plan;
            sc->deposit_chunk = solve_tune.deposit_chunk;
        }
        engine_->hook = &hook;
        engine_->tune = tune;
        if (sc) sc->hook = &hook;
        wire_loss();
        wire_step_counts(false);
        if (!elem_charge) {
            elem_charge = dalloc<double>(lat.elements.size(), "element charge");
            cuda_check(cudaMemset(elem_charge, 0, sizeof(double) * std::max<size_t>(1, lat.elements.size())), "memset");
        }
    }

    void begin(Bunch& b, cudaStream_t s)
    { // do_before_start propagator.cc:8-23
        ensure_device();
        if (hook) { // the bunch's total number is the sum of the ranks' valid counts
            if (!engine_->xchg) engine_->xchg = dalloc<double>(6 + kMaxSlotsPerPass, "exchange");
            cuda_check(launch_shard_count(b.counters, engine_->xchg, s), "shard count");
            hook.run(engine_->xchg, 1, s);
            cuda_check(launch_shard_total(b.counters, engine_->xchg, s), "shard total");
        }
        if (b.turns_done == 0 && !b.design_set) {
            b.design = lat.ref;
            b.design_set = true;
        }
    }

    void run_step(Bunch& b, const Step& st, cudaStream_t s)
    { // Step::apply step.cc:44-79
        double time = st.length / (b.ref.beta * pc::c);
        size_t ii = 0;
        for (char item : st.items) {
            if (item == 'I') {
                engine_->add_operator(lat, st.indeps[ii++], b, sc.get(), elem_charge, s);
            } else if (sc) {
                engine_->flush(b, sc.get(), elem_charge, true, time * 1.0, s);
                if (sort_active && (b.kicks_since_sort++ % sort_interval) == 0) resort(b, s);
                sc->solve(b, s);
                engine_->add_kick(b);
            }
        }
        engine_->mark_step_end(b, sc.get(), elem_charge, s);
    }

    void finish(Bunch& b, cudaStream_t s)
    {
        engine_->flush(b, sc.get(), elem_charge, false, 0.0, s);
        b.sync_counters(s);
        if (sc) sc->check_error();
    }

    bool sort_active = false;

    // ----- CUDA-graph turns ------------------------------------------------
    // A turn's launches are captured once and replayed while the host-side
    // re-derivation of the turn gives the same launch signature.
    bool use_graphs = false;
    cudaStream_t own_stream = nullptr; // capture needs a non-legacy stream
    cudaStream_t graph_stream(cudaStream_t s)
    {
        if (s) return s;
        if (!own_stream) cuda_check(cudaStreamCreate(&own_stream), "stream");
        return own_stream;
    }
    struct CachedGraph {
        std::vector<unsigned char> sig;
        cudaGraphExec_t exec = nullptr;
        uint64_t last_use = 0;
    };
    std::vector<CachedGraph> graphs;
    uint64_t graph_clock = 0;
    int64_t graph_captures = 0, graph_replays = 0;

    struct HostSnap {
        Refpart ref, design;
        bool design_set;
        int turns_done;
        std::vector<MapOp> ops;
        PassBook book;
        int nslots;
        bool ghat_valid;
        // working-copy buffers swap at every sort
        double* parts;
        uint8_t* masks;
        uint8_t* discards;
        SortBuffers wc;
        int kicks_since_sort;
        size_t ndiag; // host-side diagnostic entries
        int32_t rec_next, rec_first, rec_count; // per-step count records
    };
    HostSnap snap(const Bunch& b) const
    {
        HostSnap h{b.ref, b.design, b.design_set, b.turns_done, engine_->ops, engine_->book, engine_->nslots,
                   sc ? sc->ghat_valid : false, b.parts, b.masks, b.discards, b.wc, b.kicks_since_sort,
                   diag_s.size(), engine_->rec_next, engine_->rec_first, engine_->rec_count};
        return h;
    }
    void restore(Bunch& b, const HostSnap& h)
    {
        b.ref = h.ref;
        b.design = h.design;
        b.design_set = h.design_set;
        b.turns_done = h.turns_done;
        b.parts = h.parts;
        b.masks = h.masks;
        b.discards = h.discards;
        b.wc = h.wc;
        b.kicks_since_sort = h.kicks_since_sort;
        diag_s.resize(h.ndiag);
        diag_turn.resize(h.ndiag);
        engine_->ops = h.ops;
        engine_->book = h.book;
        engine_->nslots = h.nslots;
        engine_->rec_next = h.rec_next;
        engine_->rec_first = h.rec_first;
        engine_->rec_count = h.rec_count;
        if (sc) sc->ghat_valid = h.ghat_valid;
    }
    // ----- per-turn diagnostics (Diagnostics_full2 at turn ends) ----------
    int diag_cap = 0;
    double* diag_records = nullptr; // [diag_cap][kDiagRecord]
    int32_t* diag_count = nullptr;  // records appended so far (device)
    double* diag_partials = nullptr;
    double* diag_tmp = nullptr;
    std::vector<double> diag_s;     // path length s of each record (host: known at launch)
    std::vector<int> diag_turn;     // turns completed at each record

    // ----- Diagnostics_loss ------------------------------------------------
    int loss_cap = 0;
    double* loss_buf = nullptr;
    int32_t* loss_count = nullptr;
    std::vector<std::array<double, 3>> loss_tags;

    // ----- autotuning -------------------------------------------------------
    // Coordinate descent over the particle-pass launch shapes, the re-sort
    // interval, the FFT radix plan and the deposit tile chunk: every
    // candidate propagates `steps` untimed steps of a scratch copy of the
    // bunch and then `steps` more timed with CUDA events, and the fastest is
    // kept.  The bunch, the diagnostics, the loss and step records and the
    // per-element lost charge are left as they were.  Each trial appends (light_shape,
    // full_occ, full_ppt, quad_variant, ctas_per_sm, sort_interval, fft_plan,
    // deposit_chunk, ms).
    void apply_tune(const TrackTune& t, int si, const SolveTune& st)
    {
        tune = t;
        sort_interval = si;
        solve_tune = st;
        if (engine_) engine_->tune = t;
        if (sc) {
            sc->d.plan = st.fft_plan;
            sc->deposit_chunk = st.deposit_chunk;
        }
        drop_graphs();
    }
    void autotune(Bunch& b, int steps, std::vector<std::array<double, 9>>& log)
    {
        if (hook) throw Error(SB2_ERR_UNSUPPORTED, "autotuning is not available on a sharded propagator");
        if (steps < 1) throw Error(SB2_ERR_INVALID, "autotune: steps must be >= 1");
        ensure_device();
        b.sync_home(0);
        Bunch t;
        t.device = b.device;
        t.n = b.n;
        t.stride = std::max<int64_t>(b.n, 1);
        t.owns = true;
        t.parts = dalloc<double>((size_t)7 * t.stride, "autotune bunch");
        t.masks = dalloc<uint8_t>(t.stride, "autotune bunch");
        t.discards = dalloc<uint8_t>(t.stride, "autotune bunch");
        t.counters = dalloc<BunchCounters>(1, "autotune bunch");
        t.set_home();
        const size_t ne = std::max<size_t>(1, lat.elements.size());
        double* keep_charge = dalloc<double>(ne, "autotune");
        cuda_check(cudaMemcpy(keep_charge, elem_charge, sizeof(double) * ne, cudaMemcpyDeviceToDevice), "autotune");
        const int keep_diag = diag_cap, keep_loss = loss_cap, keep_rec = step_rec_cap;
        const bool keep_graphs = use_graphs;
        const TrackTune t0 = tune;
        const int si0 = sort_interval;
        const SolveTune st0 = solve_tune;
        diag_cap = 0;
        loss_cap = 0;
        step_rec_cap = 0;
        use_graphs = false;
        wire_loss();
        wire_step_counts(false);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        auto restore = [&]() {
            diag_cap = keep_diag;
            loss_cap = keep_loss;
            step_rec_cap = keep_rec;
            use_graphs = keep_graphs;
            wire_loss();
            wire_step_counts(false);
            cudaMemcpy(elem_charge, keep_charge, sizeof(double) * ne, cudaMemcpyDeviceToDevice);
            dfree(keep_charge);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        };
        try {
            cuda_check(cudaEventCreate(&e0), "event");
            cuda_check(cudaEventCreate(&e1), "event");
            auto trial = [&](const TrackTune& tt, int si, const SolveTune& st) -> double {
                apply_tune(tt, si, st);
                t.drop_work();
                t.kicks_since_sort = 0;
                if (b.n) {
                    cuda_check(cudaMemcpy2D(t.parts, sizeof(double) * t.stride, b.home_parts,
                                            sizeof(double) * b.home_stride, sizeof(double) * b.n, 7,
                                            cudaMemcpyDeviceToDevice),
                               "autotune copy");
                    cuda_check(cudaMemcpy(t.masks, b.home_masks, b.n, cudaMemcpyDeviceToDevice), "autotune copy");
                    if (b.home_discards)
                        cuda_check(cudaMemcpy(t.discards, b.home_discards, b.n, cudaMemcpyDeviceToDevice),
                                   "autotune copy");
                }
                cuda_check(cudaMemcpy(t.counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToDevice),
                           "autotune copy");
                t.host_counters = b.host_counters;
                t.ref = b.ref;
                t.design = b.design;
                t.design_set = b.design_set;
                t.turns_done = b.turns_done;
                // an untimed lead-in of the same length brings the scratch
                // copy to the state the timed steps see in a long run (its
                // cell order aged as the re-sort interval lets it).  Both
                // continue from the bunch's own step: started elsewhere in
                // the lattice the beam is mismatched to the optics, its size
                // and density change, and so do the costs being compared.
                const int first = b.next_step;
                propagate_steps(t, first, steps, 0);
                cuda_check(cudaEventRecord(e0, 0), "event");
                propagate_steps(t, first + steps, steps, 0);
                cuda_check(cudaEventRecord(e1, 0), "event");
                cuda_check(cudaEventSynchronize(e1), "event");
                float ms = 0.f;
                cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
                log.push_back({(double)tt.light_shape, (double)tt.full_occ, (double)tt.full_ppt,
                               (double)tt.quad_variant, (double)tt.ctas_per_sm, (double)si, (double)st.fft_plan,
                               (double)st.deposit_chunk, (double)ms});
                return ms;
            };
            trial(t0, si0, st0); // warm-up: allocations of the scratch working copy
            log.clear();
            TrackTune best = t0;
            int best_si = si0;
            SolveTune best_st = st0;
            double best_ms = trial(best, best_si, best_st);
            auto consider = [&](TrackTune c, int si, SolveTune st) {
                if (!std::memcmp(&c, &best, sizeof(c)) && si == best_si && st == best_st) return;
                const double ms = trial(c, si, st);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = c;
                    best_si = si;
                    best_st = st;
                }
            };
            for (int v : {1, 3, 2, 0}) {
                TrackTune c = best;
                c.light_shape = v;
                consider(c, best_si, best_st);
            }
            const int fulls[3][2] = {{2, 1}, {2, 2}, {3, 1}};
            for (auto& f : fulls) {
                TrackTune c = best;
                c.full_occ = f[0];
                c.full_ppt = f[1];
                consider(c, best_si, best_st);
            }
            for (int v : {1, 2, 0}) {
                TrackTune c = best;
                c.quad_variant = v;
                consider(c, best_si, best_st);
            }
            for (int v : {4, 8, 12}) {
                TrackTune c = best;
                c.ctas_per_sm = v;
                consider(c, best_si, best_st);
            }
            if (has_sc && cell_sort)
                for (int v : {2, 4, 8}) consider(best, v, best_st);
            if (has_sc) {
                for (int v : {0, 1}) { // FFT radix plans
                    SolveTune st = best_st;
                    st.fft_plan = v;
                    consider(best, best_si, st);
                }
                for (int v : {4, 8}) { // deposit tile: particles per thread
                    SolveTune st = best_st;
                    st.deposit_chunk = v;
                    consider(best, best_si, st);
                }
            }
            apply_tune(best, best_si, best_st);
        } catch (...) {
            apply_tune(t0, si0, st0);
            restore();
            throw;
        }
        restore();
    }

    // ----- per-step count records -----------------------------------------
    // A pinned (page-locked, device-addressable) caller buffer is written by
    // the pass bookkeeping directly, at a device-side cursor: the launches of
    // a turn are then the same every turn, and CUDA-graph turns can replay
    // them.  A pageable buffer gets the records by stream-ordered copies of a
    // device array, and CUDA-graph turns are refused.
    int step_rec_cap = 0;
    BunchCounters* step_rec_dev = nullptr;
    BunchCounters* step_rec_host = nullptr;
    int32_t* step_rec_cursor = nullptr; // pinned buffer: the device-side record cursor
    bool step_rec_pinned() const { return step_rec_cursor != nullptr; }
    void set_step_counts(BunchCounters* host, int capacity)
    {
        dfree(step_rec_dev);
        step_rec_dev = nullptr;
        dfree(step_rec_cursor);
        step_rec_cursor = nullptr;
        step_rec_host = capacity > 0 ? host : nullptr;
        step_rec_cap = capacity > 0 ? capacity : 0;
        if (step_rec_cap) {
            cudaPointerAttributes a{};
            const bool pinned = cudaPointerGetAttributes(&a, host) == cudaSuccess &&
                                a.type == cudaMemoryTypeHost && a.devicePointer == (void*)host;
            cudaGetLastError(); // a pageable pointer may leave an error behind
            if (pinned) {
                step_rec_cursor = dalloc<int32_t>(1, "step record cursor");
                cuda_check(cudaMemset(step_rec_cursor, 0, sizeof(int32_t)), "step record cursor");
            } else {
                step_rec_dev = dalloc<BunchCounters>((size_t)step_rec_cap, "step records");
            }
        }
        wire_step_counts(true);
    }
    void wire_step_counts(bool restart)
    {
        if (!engine_) return;
        engine_->rec_dev = step_rec_dev;
        engine_->rec_host = step_rec_host;
        engine_->rec_cap = step_rec_cap;
        engine_->rec_cursor = step_rec_cursor;
        if (restart) engine_->rec_next = 0;
    }

    void set_loss_diagnostics(int capacity)
    {
        dfree(loss_buf);
        dfree(loss_count);
        loss_buf = nullptr;
        loss_count = nullptr;
        loss_tags.clear();
        loss_cap = capacity;
        if (capacity > 0) {
            loss_buf = dalloc<double>((size_t)capacity * 8, "loss diagnostics");
            loss_count = dalloc<int32_t>(1, "loss diagnostics");
            cuda_check(cudaMemset(loss_count, 0, sizeof(int32_t)), "loss diagnostics");
        }
        wire_loss();
    }
    void wire_loss()
    {
        if (!engine_) return;
        engine_->loss_buf = loss_buf;
        engine_->loss_count = loss_count;
        engine_->loss_cap = loss_cap;
        engine_->loss_tags = loss_cap > 0 ? &loss_tags : nullptr;
    }

    void set_diagnostics(int capacity)
    {
        drop_graphs(); // captured turns change shape
        dfree(diag_records);
        dfree(diag_count);
        dfree(diag_partials);
        dfree(diag_tmp);
        diag_records = diag_partials = diag_tmp = nullptr;
        diag_count = nullptr;
        diag_s.clear();
        diag_turn.clear();
        diag_cap = capacity;
        if (capacity <= 0) return;
        diag_records = dalloc<double>((size_t)capacity * kDiagRecord, "diagnostics");
        diag_count = dalloc<int32_t>(1, "diagnostics");
        diag_partials = dalloc<double>((size_t)track_grid_blocks() * 27, "diagnostics");
        diag_tmp = dalloc<double>(12, "diagnostics");
        cuda_check(cudaMemset(diag_count, 0, sizeof(int32_t)), "diagnostics");
    }

    // Flushes the pending maps (a record sees the bunch at the end of the
    // turn) and appends one record on the device.
    void record_diagnostics(Bunch& b, cudaStream_t s)
    {
        if (!diag_cap) return;
        engine_->flush(b, sc.get(), elem_charge, false, 0.0, s);
        diag_s.push_back(b.ref.repetition * b.ref.s + b.ref.s_n); // Reference_particle::get_s
        diag_turn.push_back(b.turns_done);
        if (g_sig.dry) return;
        cuda_check(launch_diagnostics(b.parts, b.stride, b.masks, b.n, b.counters, diag_partials, track_grid_blocks(),
                                      diag_tmp, diag_records, diag_count, diag_cap, s),
                   "diagnostics");
    }

    void run_turn(Bunch& b, cudaStream_t s)
    {
        b.ref.start_repetition();
        for (auto const& st : steps) run_step(b, st, s);
        b.turns_done += 1;
        record_diagnostics(b, s);
    }
    void drop_graphs()
    {
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        graphs.clear();
    }

    void propagate_graph_turn(Bunch& b, cudaStream_t s)
    {
        graph_run(b, s, [&] { run_turn(b, s); });
    }
    // Steps [k0, k1) of one turn as one graph (propagate_steps).
    void graph_segment(Bunch& b, int k0, int k1, cudaStream_t s)
    {
        graph_run(b, s, [&] {
            for (int k = k0; k < k1; ++k) plain_step(b, k, s);
        });
    }
    // The launches of run() from a cached graph with the same signature, or
    // captured into a new one.
    template <class F>
    void graph_run(Bunch& b, cudaStream_t s, F&& run)
    {
        HostSnap s0 = snap(b);
        std::vector<unsigned char> sig;
        g_sig.dry = true;
        g_sig.sig = &sig;
        try {
            run();
        } catch (...) {
            g_sig = LaunchSig{};
            throw;
        }
        g_sig = LaunchSig{};
        ++graph_clock;
        for (auto& g : graphs)
            if (g.sig == sig) {
                g.last_use = graph_clock;
                ++graph_replays;
                cuda_check(cudaGraphLaunch(g.exec, s), "graph launch");
                return;
            }
        restore(b, s0);
        cuda_check(cudaGraphLaunch(capture(b, s, run), s), "graph launch");
    }

    // Capture run() into a new cached graph (the host state advances as if
    // it ran; nothing runs on the GPU) and return it.
    template <class F>
    cudaGraphExec_t capture(Bunch& b, cudaStream_t s, F&& run)
    {
        std::vector<unsigned char> sig2;
        cudaGraph_t graph = nullptr;
        cuda_check(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
        g_sig.sig = &sig2;
        try {
            run();
        } catch (...) {
            g_sig = LaunchSig{};
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        g_sig = LaunchSig{};
        cuda_check(cudaStreamEndCapture(s, &graph), "end capture");
        cudaGraphExec_t exec = nullptr;
        cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "graph instantiate");
        if (graphs.size() >= 4) { // evict the least recently used
            size_t lru = 0;
            for (size_t k = 1; k < graphs.size(); ++k)
                if (graphs[k].last_use < graphs[lru].last_use) lru = k;
            cudaGraphExecDestroy(graphs[lru].exec);
            graphs.erase(graphs.begin() + lru);
        }
        graphs.push_back(CachedGraph{sig2, exec, ++graph_clock});
        ++graph_captures;
        return exec;
    }

    // Capture, without running them, the graphs that propagate_steps(b,
    // first, count) will replay: the steps are re-derived on the host only
    // (as the signature check of a graph does), each segment whose
    // signature is not cached yet is captured, and the bunch's host state is
    // put back.  Nothing runs on the GPU (a bunch not yet in its cell-ordered
    // working copy gets the copy's buffers, not its gather).
    void prepare_steps(Bunch& b, int first, int count, cudaStream_t s)
    {
        if (!use_graphs || count <= 0 || steps.empty()) return;
        s = graph_stream(s);
        ensure_device();
        const int ns = (int)steps.size();
        const HostSnap s0 = snap(b);
        const bool keep_sort = sort_active, keep_permuted = b.permuted;
        const int64_t keep_stride = b.stride;
        sort_active = sorting(b);
        if (sort_active && !b.permuted) { // as the call's enter_sorted will (its gather is not launched here)
            if (!sort_scratch) {
                const int64_t G = (int64_t)sc_opts.shape[0] * sc_opts.shape[1] * sc_opts.shape[2];
                sort_scratch = dalloc<int32_t>(sort_scratch_ints(G), "sort scratch");
            }
            b.enter_work_host();
        }
        const SortBuffers entered_wc = b.wc; // before the sorts of the derivation swap its buffers
        auto put_back = [&]() {
            g_sig = LaunchSig{};
            restore(b, s0);
            // buffers allocated here stay, in the order the call will enter
            // them: the captured graphs name them
            if (!keep_permuted && !s0.wc.parts) b.wc = entered_wc;
            b.permuted = keep_permuted;
            b.stride = keep_stride;
            sort_active = keep_sort;
        };
        const bool design_set = b.design_set;
        if (b.turns_done == 0 && !b.design_set) { // as begin() does
            b.design = lat.ref;
            b.design_set = true;
        }
        try {
            if (diag_cap && diag_s.empty()) { // the call's record of the initial state
                std::vector<unsigned char> sig;
                g_sig.dry = true;
                g_sig.sig = &sig;
                record_diagnostics(b, s);
                g_sig = LaunchSig{};
            }
            for (int k = first; k < first + count;) {
                const int k1 = std::min(first + count, k + ns - ((k % ns) + ns) % ns);
                auto run = [&] {
                    for (int j = k; j < k1; ++j) plain_step(b, j, s);
                };
                const HostSnap t0 = snap(b);
                std::vector<unsigned char> sig;
                g_sig.dry = true;
                g_sig.sig = &sig;
                run();
                g_sig = LaunchSig{};
                bool cached = false;
                for (auto& g : graphs)
                    if (g.sig == sig) cached = true;
                if (!cached) {
                    restore(b, t0);
                    capture(b, s, run);
                }
                k = k1;
            }
        } catch (...) {
            put_back();
            b.design_set = design_set;
            throw;
        }
        put_back();
        b.design_set = design_set;
    }

    // Turns without the end-of-call synchronisation (batched jobs): the
    // pending second half of the last step is flushed at the end.
    void propagate_async(Bunch& b, int turns, cudaStream_t s)
    {
        if (use_graphs) s = graph_stream(s);
        begin(b, s);
        enter_sorted(b, s);
        if (diag_cap && diag_s.empty()) record_diagnostics(b, s); // initial state
        for (int t = 0; t < turns; ++t) {
            if (use_graphs)
                propagate_graph_turn(b, s);
            else
                run_turn(b, s);
        }
        if (turns > 0) b.next_step = 0;
        engine_->flush(b, sc.get(), elem_charge, false, 0.0, s);
        leave_sorted(b, s);
    }

    void propagate(Bunch& b, int turns, cudaStream_t s)
    { // Propagator::propagate propagator.cc:157-283 (one bunch, no diagnostics)
        if (use_graphs) s = graph_stream(s);
        propagate_async(b, turns, s);
        finish(b, s);
    }

    // one step of propagate_steps outside a graph turn
    void plain_step(Bunch& b, int k, cudaStream_t s)
    {
        const int ns = (int)steps.size();
        const int si = ((k % ns) + ns) % ns;
        if (si == 0) b.ref.start_repetition();
        run_step(b, steps[si], s);
        if (si == ns - 1) {
            b.turns_done += 1;
            record_diagnostics(b, s);
        }
    }
    // With CUDA-graph turns on, the steps of [first, first + count) that
    // fall in one turn are one graph launch: whole turns (the same start of
    // repetition, steps, turn count and diagnostics as run_turn, so they share
    // graphs with propagate) and the partial turns at either end.
    void propagate_steps(Bunch& b, int first, int count, cudaStream_t s)
    {
        if (use_graphs) s = graph_stream(s);
        begin(b, s);
        enter_sorted(b, s);
        if (diag_cap && diag_s.empty()) record_diagnostics(b, s); // initial state
        const int ns = (int)steps.size();
        for (int k = first; k < first + count;) {
            if (use_graphs && ns > 0) {
                const int k1 = std::min(first + count, k + ns - ((k % ns) + ns) % ns);
                graph_segment(b, k, k1, s);
                k = k1;
            } else {
                plain_step(b, k, s);
                ++k;
            }
        }
        if (count > 0 && ns > 0) b.next_step = (((first + count) % ns) + ns) % ns;
        engine_->flush(b, sc.get(), elem_charge, false, 0.0, s);
        leave_sorted(b, s);
        finish(b, s);
    }
};

// Standalone collective operator (space_charge_3d_open_hockney.cc:400-453)
struct ScOperator {
    SpaceCharge sc;
    Engine engine;
    explicit ScOperator(const sb2_sc3d_options& o) : sc(o) {}
    void apply(Bunch& b, double time_step, cudaStream_t s)
    {
        engine.flush(b, &sc, nullptr, true, time_step, s);
        sc.solve(b, s);
        engine.add_kick(b);
        engine.flush(b, &sc, nullptr, false, 0.0, s);
        cuda_check(cudaStreamSynchronize(s), "sync");
        sc.check_error();
    }
};

// ---------------------------------------------------------------------------
// Batch of independent jobs (propagator + bunch), each on its own stream:
// one call advances the listed jobs concurrently.  With CUDA-graph turns the
// host cost per job and turn is one signature check and one graph launch.
// ---------------------------------------------------------------------------
struct Batch {
    struct Job {
        Propagator* p = nullptr;
        Bunch* b = nullptr;
        cudaStream_t s = nullptr;
        cudaEvent_t done = nullptr; // recorded after the last launched turn
        bool used = false;
        bool pending = false; // launched, not yet collected by query()
    };
    std::vector<Job> jobs;
    ~Batch()
    {
        for (auto& j : jobs) {
            if (j.s) cudaStreamDestroy(j.s);
            if (j.done) cudaEventDestroy(j.done);
        }
        lock_groups.clear();
    }
    Job& job(int slot)
    {
        if (slot < 0 || slot >= (int)jobs.size() || !jobs[slot].used) throw Error(SB2_ERR_INVALID, "bad batch slot");
        return jobs[slot];
    }
    // Enqueue `turns` turns of one job on its stream and return at once.
    void launch(int slot, int turns)
    {
        Job& j = job(slot);
        if (j.pending) throw Error(SB2_ERR_INVALID, "batch slot already has turns in flight");
        if (!j.done) cuda_check(cudaEventCreateWithFlags(&j.done, cudaEventDisableTiming), "event");
        j.p->propagate_async(*j.b, turns, j.s);
        cuda_check(cudaEventRecord(j.done, j.s), "event record");
        j.pending = true;
    }
    // 1 when the job's launched turns have finished (their bookkeeping and
    // error checks done), 0 while they run.
    int query(int slot)
    {
        Job& j = job(slot);
        if (!j.pending) return 1;
        cudaError_t e = cudaEventQuery(j.done);
        if (e == cudaErrorNotReady) {
            cudaGetLastError();
            return 0;
        }
        cuda_check(e, "batch job");
        j.pending = false;
        j.p->finish(*j.b, j.s);
        return 1;
    }
    int add(Propagator* p, Bunch* b)
    {
        for (size_t k = 0; k < jobs.size(); ++k)
            if (!jobs[k].used) {
                jobs[k].p = p;
                jobs[k].b = b;
                jobs[k].used = true;
                return (int)k;
            }
        Job j;
        j.p = p;
        j.b = b;
        j.used = true;
        cuda_check(cudaStreamCreateWithFlags(&j.s, cudaStreamNonBlocking), "stream");
        jobs.push_back(j);
        return (int)jobs.size() - 1;
    }
    void remove(int slot)
    {
        Job& j = job(slot);
        if (j.pending) cuda_check(cudaStreamSynchronize(j.s), "batch remove");
        j.pending = false;
        jobs[slot].used = false;
        jobs[slot].p = nullptr;
        jobs[slot].b = nullptr;
    }
    // ----- lockstep: one work-list launch per kernel kind and step ---------
    // The listed jobs advance `turns` turns together.  Every job runs the
    // host side of its step as usual (its op lists, design particle,
    // bookkeeping programs), with its launches recorded (g_rec); the records
    // of all jobs, position by position, then go out as work-list launches
    // on one stream: the particle passes of all bunches in one launch per
    // pass kernel, the bookkeeping and domain of all bunches in one launch,
    // the charge grids cleared in one, the deposits in one per grid shape,
    // the Green functions, convolutions and fields in one per grid shape.
    // The item arrays of a step travel to the device in one copy.  Jobs must
    // have the same number of steps per turn and the same launch sequence
    // per step (e.g. one lattice with different strengths, or bunch sizes
    // and grids that differ); per-turn diagnostics, step-count records and
    // sharded propagators are not available here.
    // The listed jobs are split into groups of about equal particle count
    // (SB2_LOCKSTEP_GROUPS, default 2), each group's launches on its own
    // stream, so one group's grid work overlaps the other's particle passes.
    // A group stages its item arrays through a ring of three areas.
    struct LockGroup {
        cudaStream_t s = nullptr;
        unsigned char* host[3] = {nullptr, nullptr, nullptr};
        unsigned char* dev[3] = {nullptr, nullptr, nullptr};
        cudaEvent_t done[3] = {nullptr, nullptr, nullptr};
        size_t cap = 0;
        int next = 0;
        void free_arena()
        {
            for (int k = 0; k < 3; ++k) {
                if (host[k]) cudaFreeHost(host[k]);
                if (dev[k]) dfree(dev[k]);
                host[k] = dev[k] = nullptr;
            }
            cap = 0;
        }
        ~LockGroup()
        {
            if (s) cudaStreamSynchronize(s);
            free_arena();
            for (auto& e : done)
                if (e) cudaEventDestroy(e);
            if (s) cudaStreamDestroy(s);
        }
    };
    std::vector<std::unique_ptr<LockGroup>> lock_groups;

    struct Merge {
        std::vector<unsigned char> host; // the step's item arrays, in the order they are used
        size_t add(const void* p, size_t bytes)
        {
            size_t at = (host.size() + 255) & ~(size_t)255;
            host.resize(at + bytes);
            std::memcpy(host.data() + at, p, bytes);
            return at;
        }
    };

    void execute(std::vector<std::vector<LaunchRec>>& recs, LockGroup& G)
    {
        cudaStream_t s = G.s;
        const size_t nj = recs.size();
        const size_t npos = recs[0].size();
        for (size_t j = 1; j < nj; ++j)
            if (recs[j].size() != npos)
                throw Error(SB2_ERR_UNSUPPORTED, "batch jobs are not in lockstep (different launch sequences)");
        for (size_t k = 0; k < npos; ++k)
            for (size_t j = 1; j < nj; ++j)
                if (recs[j][k].kind != recs[0][k].kind)
                    throw Error(SB2_ERR_UNSUPPORTED, "batch jobs are not in lockstep (different launch sequences)");
        // 1. item arrays of every position, laid out in one host block
        Merge m;
        struct Op {
            int kind, variant, max_ops;
            bool f32;
            size_t items, first;
            int nitems, nblocks;
            Dims d;
            int linear, mode;
            const double2* tw64[3];
            const float2* tw32[3];
            int sort_blocks[4], sort_max_m;
        };
        std::vector<Op> ops;
        std::vector<int> mom_blocks(nj, 0);
        for (size_t k = 0; k < npos; ++k) {
            const int kind = recs[0][k].kind;
            if (kind == LaunchRec::SORT) { // every bunch's counting sort in one set of list launches
                std::vector<SortItem> items(nj);
                std::vector<int> first(4 * (nj + 1));
                Op o{};
                o.kind = kind;
                o.nitems = (int)nj;
                for (size_t j = 0; j < nj; ++j) {
                    items[j] = recs[j][k].sort;
                    const SortItem& it = items[j];
                    o.sort_max_m = std::max(o.sort_max_m, it.gx * it.gy * it.gz + 2);
                }
                sort_list_plan(items.data(), (int)nj, first.data(), o.sort_blocks);
                o.items = m.add(items.data(), sizeof(SortItem) * nj);
                o.first = m.add(first.data(), sizeof(int) * first.size());
                ops.push_back(o);
                continue;
            }
            if (kind == LaunchRec::DOMAIN) {
                std::vector<DomainParams> items(nj);
                for (size_t j = 0; j < nj; ++j) {
                    items[j] = recs[j][k].dp;
                    // one moment partial per block the bunch had in the last pass
                    if (items[j].compute_domain && !items[j].domain_fixed && items[j].moment_partials)
                        items[j].n_partials = mom_blocks[j];
                }
                Op o{};
                o.kind = kind;
                o.items = m.add(items.data(), sizeof(DomainParams) * nj);
                o.nitems = (int)nj;
                ops.push_back(o);
                continue;
            }
            if (kind == LaunchRec::ZERO) {
                std::vector<ZeroItem> items(nj);
                for (size_t j = 0; j < nj; ++j) items[j] = recs[j][k].z;
                Op o{};
                o.kind = kind;
                o.items = m.add(items.data(), sizeof(ZeroItem) * nj);
                o.nitems = (int)nj;
                ops.push_back(o);
                continue;
            }
            // grouped kinds: the key decides which jobs share a launch
            std::vector<std::vector<size_t>> groups;
            auto key_of = [&](const LaunchRec& r) {
                std::vector<int> key = {r.kind, r.choice, r.fast ? 1 : 0, r.f32 ? 1 : 0, r.d.gx, r.d.gy, r.d.gz,
                                        r.d.plan, r.linear, r.mode};
                return key;
            };
            {
                std::vector<std::vector<int>> keys;
                for (size_t j = 0; j < nj; ++j) {
                    auto key = key_of(recs[j][k]);
                    size_t g = 0;
                    while (g < keys.size() && keys[g] != key) ++g;
                    if (g == keys.size()) {
                        keys.push_back(key);
                        groups.emplace_back();
                    }
                    groups[g].push_back(j);
                }
            }
            for (auto const& grp : groups) {
                const LaunchRec& r0 = recs[grp[0]][k];
                Op o{};
                o.kind = kind;
                o.nitems = (int)grp.size();
                o.d = r0.d;
                o.linear = r0.linear;
                o.mode = r0.mode;
                o.f32 = r0.f32;
                for (int a = 0; a < 3; ++a) {
                    o.tw64[a] = r0.tw64[a];
                    o.tw32[a] = r0.tw32[a];
                }
                if (kind == LaunchRec::TRACK) {
                    o.variant = r0.choice;
                    o.f32 = r0.fast;
                    std::vector<size_t> at(grp.size());
                    std::vector<int> first(grp.size() + 1, 0);
                    const int tile = track_pass_tile(r0.choice);
                    for (size_t q = 0; q < grp.size(); ++q) {
                        const LaunchRec& r = recs[grp[q]][k];
                        at[q] = m.add(r.tp.data(), r.tp.size());
                        o.max_ops = std::max(o.max_ops, ((const TrackParams*)r.tp.data())->nops);
                        const int64_t need = std::max<int64_t>(1, (r.n + tile - 1) / tile);
                        const int vg = (int)std::min<int64_t>(need, track_grid_blocks(r.ctas_per_sm));
                        first[q + 1] = first[q] + vg;
                        if (r.has_mom) mom_blocks[grp[q]] = vg;
                    }
                    // item pointers are arena offsets here, made device addresses below
                    std::vector<uint64_t> ptrs(at.begin(), at.end());
                    o.items = m.add(ptrs.data(), sizeof(uint64_t) * ptrs.size());
                    o.first = m.add(first.data(), sizeof(int) * first.size());
                    o.nblocks = first.back();
                } else if (kind == LaunchRec::DEPOSIT) {
                    std::vector<DepositItem> items;
                    std::vector<int> first(1, 0);
                    for (size_t j : grp) {
                        items.push_back(recs[j][k].dep);
                        first.push_back(first.back() + std::max(1, deposit_list_blocks(recs[j][k].dep.n)));
                    }
                    o.items = m.add(items.data(), sizeof(DepositItem) * items.size());
                    o.first = m.add(first.data(), sizeof(int) * first.size());
                    o.nblocks = first.back();
                } else {
                    std::vector<ConvItem> items;
                    for (size_t j : grp) items.push_back(recs[j][k].ci);
                    o.items = m.add(items.data(), sizeof(ConvItem) * items.size());
                }
                ops.push_back(o);
            }
        }
        // 2. the block to the device (a ring of three staging areas)
        const size_t bytes = std::max<size_t>(m.host.size(), 256);
        if (bytes > G.cap) {
            cuda_check(cudaStreamSynchronize(s), "lockstep");
            G.free_arena();
            G.cap = bytes * 2;
            for (int k = 0; k < 3; ++k) {
                cuda_check(cudaMallocHost((void**)&G.host[k], G.cap), "lockstep staging");
                G.dev[k] = dalloc<unsigned char>(G.cap, "lockstep items");
                if (!G.done[k]) cuda_check(cudaEventCreateWithFlags(&G.done[k], cudaEventDisableTiming), "event");
            }
        }
        const int slot = G.next;
        G.next = (G.next + 1) % 3;
        cuda_check(cudaEventSynchronize(G.done[slot]), "lockstep staging"); // its last copy has run
        unsigned char* dev = G.dev[slot];
        for (auto const& o : ops) // TRACK item pointers: arena offsets -> device addresses
            if (o.kind == LaunchRec::TRACK) {
                uint64_t* ptrs = (uint64_t*)(m.host.data() + o.items);
                for (int q = 0; q < o.nitems; ++q) ptrs[q] = (uint64_t)(uintptr_t)(dev + ptrs[q]);
            }
        std::memcpy(G.host[slot], m.host.data(), m.host.size());
        cuda_check(cudaMemcpyAsync(dev, G.host[slot], m.host.size(), cudaMemcpyHostToDevice, s), "lockstep items");
        cuda_check(cudaEventRecord(G.done[slot], s), "event");
        // 3. the launches, in the recorded order
        for (auto const& o : ops) {
            const unsigned char* items = dev + o.items;
            const int* first = (const int*)(dev + o.first);
            switch (o.kind) {
            case LaunchRec::TRACK: {
                ProfScope ps(PROF_TRACK, s);
                cuda_check(launch_track_list(o.variant, o.f32, (const TrackParams* const*)items, first, o.nitems,
                                             o.nblocks, o.max_ops, s),
                           "track list");
                break;
            }
            case LaunchRec::DOMAIN: {
                ProfScope ps(PROF_DOMAIN, s);
                cuda_check(launch_book_domain_list((const DomainParams*)items, o.nitems, s), "domain list");
                break;
            }
            case LaunchRec::ZERO: {
                ProfScope ps(PROF_DEPOSIT, s);
                cuda_check(launch_zero_list((const ZeroItem*)items, o.nitems, s), "zero list");
                break;
            }
            case LaunchRec::DEPOSIT: {
                ProfScope ps(PROF_DEPOSIT, s);
                cuda_check(launch_deposit_list(o.f32, (const DepositItem*)items, first, o.nitems, o.nblocks, o.d.gx,
                                               o.d.gy, o.d.gz, s),
                           "deposit list");
                break;
            }
            case LaunchRec::GREEN: {
                ProfScope ps(PROF_GREEN, s);
                cuda_check(launch_green_list((const ConvItem*)items, o.nitems, o.d, o.linear, o.tw64[0], o.tw64[1],
                                             o.tw64[2], s),
                           "green list");
                break;
            }
            case LaunchRec::CONV: {
                ProfScope ps(PROF_SOLVE, s);
                cuda_check(launch_convolve_list(o.mode, (const ConvItem*)items, o.nitems, o.d, o.tw64, o.tw32, s),
                           "convolve list");
                break;
            }
            case LaunchRec::EFIELD: {
                ProfScope ps(PROF_EFIELD, s);
                cuda_check(launch_efield_list(o.f32, (const ConvItem*)items, o.nitems, o.d.gx, o.d.gy, o.d.gz, s),
                           "efield list");
                break;
            }
            case LaunchRec::SORT: {
                ProfScope ps(PROF_SORT, s);
                cuda_check(launch_cell_sort_list((const SortItem*)items, first, o.nitems, o.sort_blocks, o.sort_max_m,
                                                 s),
                           "cell sort list");
                break;
            }
            }
        }
    }

    void run_lockstep(const int32_t* slots, int n, int turns)
    {
        if (n < 1 || turns < 0) throw Error(SB2_ERR_INVALID, "run_lockstep: bad job list");
        std::vector<Job*> js;
        for (int k = 0; k < n; ++k) {
            Job& j = job(slots[k]);
            if (j.pending) throw Error(SB2_ERR_INVALID, "batch slot already has turns in flight");
            for (Job* o : js) {
                if (o == &j) throw Error(SB2_ERR_INVALID, "run_lockstep: a slot is listed twice");
                // the list launches run all jobs at once: one job's grids,
                // scratch and working copy must not be another's
                if (o->p == j.p || o->b == j.b)
                    throw Error(SB2_ERR_UNSUPPORTED, "run_lockstep: jobs must have their own propagator and bunch");
            }
            Propagator& P = *j.p;
            if (P.hook) throw Error(SB2_ERR_UNSUPPORTED, "run_lockstep: sharded propagators are not supported");
            if (P.diag_cap || P.step_rec_cap)
                throw Error(SB2_ERR_UNSUPPORTED, "run_lockstep: per-turn diagnostics and step-count records are not "
                                                 "supported");
            if (!js.empty() && P.steps.size() != js[0]->p->steps.size())
                throw Error(SB2_ERR_UNSUPPORTED, "batch jobs are not in lockstep (different steps per turn)");
            js.push_back(&j);
        }
        // groups of about equal particle count (largest jobs first)
        int ngroups = 2;
        if (const char* e = getenv("SB2_LOCKSTEP_GROUPS")) ngroups = std::max(1, atoi(e));
        ngroups = std::min<int>(ngroups, (int)js.size());
        while ((int)lock_groups.size() < ngroups) {
            lock_groups.emplace_back(new LockGroup());
            cuda_check(cudaStreamCreateWithFlags(&lock_groups.back()->s, cudaStreamNonBlocking), "stream");
        }
        std::vector<std::vector<Job*>> part(ngroups);
        {
            std::vector<Job*> order = js;
            std::stable_sort(order.begin(), order.end(), [](Job* a, Job* b) { return a->b->n > b->b->n; });
            std::vector<int64_t> load(ngroups, 0);
            for (Job* j : order) {
                const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
                part[g].push_back(j);
                load[g] += j->b->n;
            }
        }
        for (int g = 0; g < ngroups; ++g) // work queued on the jobs' own streams comes first
            for (Job* j : part[g]) {
                if (!j->done) cuda_check(cudaEventCreateWithFlags(&j->done, cudaEventDisableTiming), "event");
                cuda_check(cudaEventRecord(j->done, j->s), "event");
                cuda_check(cudaStreamWaitEvent(lock_groups[g]->s, j->done, 0), "event");
            }
        const int ns = (int)js[0]->p->steps.size();
        std::vector<std::vector<std::vector<LaunchRec>>> recs(ngroups);
        for (int g = 0; g < ngroups; ++g) recs[g].resize(part[g].size());
        auto record = [&](auto&& fn) {
            for (int g = 0; g < ngroups; ++g) {
                for (size_t q = 0; q < part[g].size(); ++q) {
                    recs[g][q].clear();
                    g_rec = &recs[g][q];
                    try {
                        fn(*part[g][q], lock_groups[g]->s);
                    } catch (...) {
                        g_rec = nullptr;
                        throw;
                    }
                    g_rec = nullptr;
                }
                execute(recs[g], *lock_groups[g]);
            }
        };
        for (int g = 0; g < ngroups; ++g)
            for (Job* j : part[g]) {
                j->p->begin(*j->b, lock_groups[g]->s);
                j->p->enter_sorted(*j->b, lock_groups[g]->s);
            }
        for (int t = 0; t < turns; ++t)
            for (int si = 0; si < ns; ++si)
                record([&](Job& j, cudaStream_t s) {
                    if (si == 0) j.b->ref.start_repetition();
                    j.p->run_step(*j.b, j.p->steps[si], s);
                    if (si == ns - 1) {
                        j.b->turns_done += 1;
                        j.b->next_step = 0;
                    }
                });
        record([&](Job& j, cudaStream_t s) {
            j.p->engine_->flush(*j.b, j.p->sc.get(), j.p->elem_charge, false, 0.0, s);
        });
        for (int g = 0; g < ngroups; ++g)
            for (Job* j : part[g]) j->p->leave_sorted(*j->b, lock_groups[g]->s);
        for (int g = 0; g < ngroups; ++g) // later work on the jobs' own streams sees the result
            cuda_check(cudaStreamSynchronize(lock_groups[g]->s), "lockstep");
        std::string err;
        sb2_status code = SB2_OK;
        for (Job* j : js) {
            try {
                j->p->finish(*j->b, lock_groups[0]->s);
            } catch (const Error& e) {
                if (code == SB2_OK) {
                    code = e.code;
                    err = e.what();
                }
            }
        }
        if (code != SB2_OK) throw Error(code, err);
    }

    void run(const int32_t* slots, const int32_t* turns, int n)
    {
        std::string err;
        sb2_status code = SB2_OK;
        std::vector<int> launched;
        for (int k = 0; k < n; ++k) {
            int sl = slots[k];
            if (job(sl).pending) throw Error(SB2_ERR_INVALID, "batch slot already has turns in flight");
            try {
                jobs[sl].p->propagate_async(*jobs[sl].b, turns[k], jobs[sl].s);
                launched.push_back(sl);
            } catch (const Error& e) {
                if (code == SB2_OK) {
                    code = e.code;
                    err = e.what();
                }
            }
        }
        for (int sl : launched) {
            try {
                jobs[sl].p->finish(*jobs[sl].b, jobs[sl].s);
            } catch (const Error& e) {
                if (code == SB2_OK) {
                    code = e.code;
                    err = e.what();
                }
            }
        }
        if (code != SB2_OK) throw Error(code, err);
    }
};

// Helpers for the other translation units: option checks and reference
// kinematics without exceptions crossing the boundary.
int check_sc_options(const sb2_sc3d_options& o, std::string* msg)
{
    try {
        SpaceCharge::validate(o);
    } catch (const Error& e) {
        if (msg) *msg = e.what();
        return e.code;
    }
    return SB2_OK;
}

int ref_kinematics(int charge, double mass, double value, int kind, double* gamma, double* beta, double* p,
                   std::string* msg)
{
    try {
        Refpart r;
        r.set(charge, mass, value, kind);
        *gamma = r.gamma;
        *beta = r.beta;
        *p = r.p;
    } catch (const Error& e) {
        if (msg) *msg = e.what();
        return e.code;
    }
    return SB2_OK;
}

void set_last_error(const std::string& m);

} // namespace sb2

// ===========================================================================
// C ABI
// ===========================================================================
using namespace sb2;

struct sb2_bunch {
    Bunch b;
};
struct sb2_lattice {
    Lattice l;
};
struct sb2_propagator {
    std::unique_ptr<Propagator> p;
};
struct sb2_sc3d {
    std::unique_ptr<ScOperator> op;
};
struct sb2_batch {
    Batch q;
};

static thread_local std::string g_last_error;
void sb2::set_last_error(const std::string& m) { g_last_error = m; }

#define SB2_TRY try {
#define SB2_CATCH                                                                                                  \
    }                                                                                                              \
    catch (const Error& ex)                                                                                        \
    {                                                                                                              \
        g_last_error = ex.what();                                                                                  \
        return ex.code;                                                                                            \
    }                                                                                                              \
    catch (const std::bad_alloc&)                                                                                  \
    {                                                                                                              \
        g_last_error = "host allocation failed";                                                                   \
        return SB2_ERR_NOMEM;                                                                                      \
    }                                                                                                              \
    catch (const std::exception& ex)                                                                               \
    {                                                                                                              \
        g_last_error = ex.what();                                                                                  \
        return SB2_ERR_RUNTIME;                                                                                    \
    }                                                                                                              \
    return SB2_OK;

#define SB2_REQUIRE(cond, msg)                                                                                     \
    if (!(cond)) throw Error(SB2_ERR_INVALID, msg)

static cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

extern "C" {

const char* sb2_last_error(void) { return g_last_error.c_str(); }
const char* sb2_version(void) { return "synergia2_b200 0.1 (sm_100a)"; }

sb2_status sb2_set_device(int32_t device)
{
    SB2_TRY
    cuda_check(cudaSetDevice(device), "set device");
    SB2_CATCH
}

sb2_status sb2_profile_enable(int32_t on)
{
    SB2_TRY
    g_prof.on = on != 0;
    SB2_CATCH
}

sb2_status sb2_profile_read(int32_t category, const char** name, double* total_ms, int64_t* launches, int32_t reset)
{
    SB2_TRY
    SB2_REQUIRE(category >= 0 && category < PROF_NCAT, "bad profile category");
    g_prof.collect();
    if (name) *name = kProfNames[category];
    if (total_ms) *total_ms = g_prof.total_ms[category];
    if (launches) *launches = g_prof.count[category];
    if (reset) {
        g_prof.total_ms[category] = 0;
        g_prof.count[category] = 0;
    }
    SB2_CATCH
}

sb2_status sb2_fp64_peak_probe(double* tflops, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(tflops, "null output");
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0, sms = 0;
    cuda_check(cudaGetDevice(&dev), "device");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    const int blocks = sms * 8, iters = 4096;
    double* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&]() {
        if (out) cudaFree(out);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    try {
        cuda_check(cudaMalloc(&out, sizeof(double) * blocks * 256), "probe buffer");
        cuda_check(cudaEventCreate(&e0), "event");
        cuda_check(cudaEventCreate(&e1), "event");
        float best = 0.0f;
        for (int rep = 0; rep < 8; ++rep) {
            cuda_check(cudaEventRecord(e0, s), "event");
            cuda_check(launch_fp64_probe(out, blocks, iters, s), "fp64 probe");
            cuda_check(cudaEventRecord(e1, s), "event");
            cuda_check(cudaEventSynchronize(e1), "event");
            float ms = 0.0f;
            cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event");
            if (rep >= 2 && (best == 0.0f || ms < best)) best = ms; // two warm-up launches
        }
        *tflops = 2.0 * 8.0 * iters * (double)blocks * 256.0 / (best * 1e-3) / 1e12;
    } catch (...) {
        release();
        throw;
    }
    release();
    SB2_CATCH
}

sb2_status sb2_sc3d_options_init(sb2_sc3d_options* o, int gx, int gy, int gz)
{
    SB2_TRY
    SB2_REQUIRE(o, "null options");
    std::memset(o, 0, sizeof(*o));
    o->shape[0] = gx;
    o->shape[1] = gy;
    o->shape[2] = gz;
    o->doubled_shape[0] = gx * 2;
    o->doubled_shape[1] = gy * 2;
    o->doubled_shape[2] = gz * 2;
    o->green_fn = SB2_GREEN_LINEAR;
    o->n_sigma = 8.0;
    o->kick_scale = 1.0;
    o->comm_group_size = 4;
    o->precision = SB2_PRECISION_FP64;
    SB2_CATCH
}

sb2_status sb2_sc3d_options_set_fixed_domain(sb2_sc3d_options* o, const double offset[3], const double size[3])
{ // implemented_collective_options.h:97-108
    SB2_TRY
    SB2_REQUIRE(o && offset && size, "null argument");
    for (int i = 0; i < 3; ++i) {
        o->offset[i] = offset[i];
        o->size[i] = size[i];
    }
    o->domain_fixed = 1;
    SB2_CATCH
}

static void bunch_alloc_counters(Bunch& b, double real_num)
{
    b.counters = dalloc<BunchCounters>(1, "counters");
    b.host_counters.n_valid = (int32_t)b.n;
    b.host_counters.n_total = (int32_t)b.n;
    b.host_counters.real_num = real_num;
    cuda_check(cudaMemcpy(b.counters, &b.host_counters, sizeof(BunchCounters), cudaMemcpyHostToDevice), "counters");
}

sb2_status sb2_bunch_create(int32_t charge, double mass, double value, int32_t kind, int64_t n, double real_num,
                            sb2_bunch** out)
{
    SB2_TRY
    SB2_REQUIRE(out && n >= 0 && n < (int64_t)INT32_MAX, "bad bunch size");
    auto* h = new sb2_bunch();
    std::unique_ptr<sb2_bunch> guard(h);
    Bunch& b = h->b;
    cuda_check(cudaGetDevice(&b.device), "device");
    b.ref.set(charge, mass, value, kind);
    b.n = n;
    b.stride = n;
    b.owns = true;
    const int64_t cap = std::max<int64_t>(n, 1);
    b.parts = dalloc<double>((size_t)7 * cap, "particles");
    b.masks = dalloc<uint8_t>(cap, "masks");
    b.discards = dalloc<uint8_t>(cap, "discards");
    cuda_check(cudaMemset(b.parts, 0, sizeof(double) * 7 * cap), "memset");
    cuda_check(cudaMemset(b.masks, 1, cap), "memset");
    cuda_check(cudaMemset(b.discards, 0, cap), "memset");
    b.set_home();
    if (n) { // ids 0..n-1 (bunch_particles.cc:283-300)
        std::vector<double> ids(n);
        for (int64_t i = 0; i < n; ++i) ids[i] = (double)i;
        cuda_check(cudaMemcpy(b.parts + 6 * n, ids.data(), sizeof(double) * n, cudaMemcpyHostToDevice), "ids");
    }
    bunch_alloc_counters(b, real_num);
    *out = guard.release();
    SB2_CATCH
}

sb2_status sb2_bunch_wrap(int32_t charge, double mass, double value, int32_t kind, double* parts, int64_t stride,
                          uint8_t* masks, uint8_t* discards, int64_t n, double real_num, sb2_bunch** out)
{
    SB2_TRY
    SB2_REQUIRE(out && parts && masks && stride >= n && n >= 0, "bad wrapped bunch");
    auto* h = new sb2_bunch();
    std::unique_ptr<sb2_bunch> guard(h);
    Bunch& b = h->b;
    cuda_check(cudaGetDevice(&b.device), "device");
    b.ref.set(charge, mass, value, kind);
    b.n = n;
    b.stride = stride;
    b.parts = parts;
    b.masks = masks;
    b.discards = discards;
    b.owns = false;
    b.set_home();
    bunch_alloc_counters(b, real_num);
    // count valid particles
    std::vector<uint8_t> m(n);
    if (n) cuda_check(cudaMemcpy(m.data(), masks, n, cudaMemcpyDeviceToHost), "masks");
    int64_t nv = 0;
    for (auto v : m) nv += v ? 1 : 0;
    b.host_counters.n_valid = b.host_counters.n_total = (int32_t)nv;
    cuda_check(cudaMemcpy(b.counters, &b.host_counters, sizeof(BunchCounters), cudaMemcpyHostToDevice), "counters");
    *out = guard.release();
    SB2_CATCH
}

sb2_status sb2_bunch_destroy(sb2_bunch* b)
{
    SB2_TRY
    delete b;
    SB2_CATCH
}

sb2_status sb2_bunch_set_particles(sb2_bunch* h, const double* host_parts, const uint8_t* host_masks)
{
    SB2_TRY
    SB2_REQUIRE(h && host_parts, "null argument");
    Bunch& b = h->b;
    b.settle(0);
    if (b.n == 0) return SB2_OK;
    cuda_check(cudaMemcpy2D(b.parts, sizeof(double) * b.stride, host_parts, sizeof(double) * b.n,
                            sizeof(double) * b.n, 7, cudaMemcpyHostToDevice),
               "checkin");
    if (host_masks) {
        cuda_check(cudaMemcpy(b.masks, host_masks, b.n, cudaMemcpyHostToDevice), "masks");
        cuda_check(launch_count_valid(b.masks, b.n, b.counters, 0), "count valid");
    } else {
        cuda_check(cudaMemset(b.masks, 1, b.n), "masks");
        b.host_counters.n_valid = b.host_counters.n_total = (int32_t)b.n;
        cuda_check(cudaMemcpy(&b.counters->n_valid, &b.host_counters.n_valid, 2 * sizeof(int32_t),
                              cudaMemcpyHostToDevice),
                   "counters");
    }
    cuda_check(cudaMemcpy(&b.host_counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost), "counters");
    SB2_CATCH
}

sb2_status sb2_bunch_get_particles(sb2_bunch* h, double* host_parts, uint8_t* host_masks, uint8_t* host_discards)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    Bunch& b = h->b;
    if (b.permuted && b.n > 0) { // put back in the caller's order and copied out, array by array
        b.settle_to_host(host_parts, host_masks, host_discards);
        if (host_discards && !b.discards) std::memset(host_discards, 0, b.n);
        return SB2_OK;
    }
    b.settle(0);
    if (b.n == 0) return SB2_OK;
    if (host_parts)
        cuda_check(cudaMemcpy2D(host_parts, sizeof(double) * b.n, b.parts, sizeof(double) * b.stride,
                                sizeof(double) * b.n, 7, cudaMemcpyDeviceToHost),
                   "checkout");
    if (host_masks) cuda_check(cudaMemcpy(host_masks, b.masks, b.n, cudaMemcpyDeviceToHost), "masks");
    if (host_discards) {
        if (b.discards)
            cuda_check(cudaMemcpy(host_discards, b.discards, b.n, cudaMemcpyDeviceToHost), "discards");
        else
            std::memset(host_discards, 0, b.n);
    }
    SB2_CATCH
}

sb2_status sb2_bunch_device_arrays(sb2_bunch* h, double** parts, int64_t* stride, uint8_t** masks, uint8_t** discards)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    h->b.settle(0);
    cuda_check(cudaStreamSynchronize(0), "settle");
    if (parts) *parts = h->b.parts;
    if (stride) *stride = h->b.stride;
    if (masks) *masks = h->b.masks;
    if (discards) *discards = h->b.discards;
    SB2_CATCH
}

sb2_status sb2_bunch_counts(sb2_bunch* h, int64_t* n_active, int64_t* n_valid, int64_t* n_total, double* real_num)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    Bunch& b = h->b;
    cuda_check(cudaMemcpy(&b.host_counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost), "counters");
    if (n_active) *n_active = b.n;
    if (n_valid) *n_valid = b.host_counters.n_valid;
    if (n_total) *n_total = b.host_counters.n_total;
    if (real_num) *real_num = b.host_counters.real_num;
    SB2_CATCH
}

sb2_status sb2_bunch_design_state(sb2_bunch* h, double state[6], double* s_n)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    if (state)
        for (int i = 0; i < 6; ++i) state[i] = h->b.design.state[i];
    if (s_n) *s_n = h->b.ref.s_n;
    SB2_CATCH
}

static void export_refpart(const Refpart& r, sb2_refpart_state& o)
{
    o.charge = r.charge;
    o.repetition = r.repetition;
    o.mass = r.mass;
    o.gamma = r.gamma;
    o.beta = r.beta;
    o.momentum = r.p;
    o.energy = r.energy;
    for (int i = 0; i < 6; ++i) o.state[i] = r.state[i];
    o.s = r.s;
    o.s_n = r.s_n;
}

static void import_refpart(const sb2_refpart_state& o, Refpart& r)
{
    r.charge = o.charge;
    r.repetition = o.repetition;
    r.mass = o.mass;
    r.gamma = o.gamma;
    r.beta = o.beta;
    r.p = o.momentum;
    r.energy = o.energy;
    for (int i = 0; i < 6; ++i) r.state[i] = o.state[i];
    r.s = o.s;
    r.s_n = o.s_n;
}

sb2_status sb2_bunch_get_state(sb2_bunch* h, sb2_bunch_state* out)
{
    SB2_TRY
    SB2_REQUIRE(h && out, "null argument");
    Bunch& b = h->b;
    cuda_check(cudaMemcpy(&b.host_counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost), "counters");
    export_refpart(b.ref, out->ref);
    export_refpart(b.design, out->design);
    out->design_set = b.design_set ? 1 : 0;
    out->turns_done = b.turns_done;
    out->n_valid = b.host_counters.n_valid;
    out->n_total = b.host_counters.n_total;
    out->real_num = b.host_counters.real_num;
    SB2_CATCH
}

sb2_status sb2_bunch_set_state(sb2_bunch* h, const sb2_bunch_state* in)
{
    SB2_TRY
    SB2_REQUIRE(h && in, "null argument");
    Bunch& b = h->b;
    SB2_REQUIRE(in->ref.mass == b.ref.mass && in->ref.charge == b.ref.charge,
                "bunch state of a different particle species");
    SB2_REQUIRE(in->n_valid >= 0 && in->n_valid <= b.n && in->n_total >= in->n_valid, "bunch state counts");
    import_refpart(in->ref, b.ref);
    import_refpart(in->design, b.design);
    b.design_set = in->design_set != 0;
    b.turns_done = in->turns_done;
    b.host_counters.n_valid = (int32_t)in->n_valid;
    b.host_counters.n_total = (int32_t)in->n_total;
    b.host_counters.real_num = in->real_num;
    cuda_check(cudaMemcpy(b.counters, &b.host_counters, sizeof(BunchCounters), cudaMemcpyHostToDevice), "counters");
    SB2_CATCH
}

sb2_status sb2_bunch_set_discards(sb2_bunch* h, const uint8_t* host_discards)
{
    SB2_TRY
    SB2_REQUIRE(h && host_discards, "null argument");
    Bunch& b = h->b;
    b.settle(0);
    SB2_REQUIRE(b.discards != nullptr, "bunch has no discard array");
    if (b.n) cuda_check(cudaMemcpy(b.discards, host_discards, b.n, cudaMemcpyHostToDevice), "discards");
    SB2_CATCH
}

sb2_status sb2_bunch_snapshot_async(sb2_bunch* h, double* host_parts, uint8_t* host_masks, uint8_t* host_discards,
                                    void* stream)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    Bunch& b = h->b;
    cudaStream_t s = (cudaStream_t)stream;
    if (!b.snap_counters)
        cuda_check(cudaMallocHost((void**)&b.snap_counters, sizeof(BunchCounters)), "snapshot counts");
    b.sync_home(s);
    if (b.n > 0) {
        if (host_parts)
            cuda_check(cudaMemcpy2DAsync(host_parts, sizeof(double) * b.n, b.home_parts, sizeof(double) * b.home_stride,
                                         sizeof(double) * b.n, 7, cudaMemcpyDeviceToHost, s),
                       "snapshot");
        if (host_masks) cuda_check(cudaMemcpyAsync(host_masks, b.home_masks, b.n, cudaMemcpyDeviceToHost, s), "masks");
        if (host_discards) {
            if (b.home_discards)
                cuda_check(cudaMemcpyAsync(host_discards, b.home_discards, b.n, cudaMemcpyDeviceToHost, s),
                           "discards");
            else
                std::memset(host_discards, 0, b.n);
        }
    }
    cuda_check(cudaMemcpyAsync(b.snap_counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost, s),
               "snapshot counts");
    SB2_CATCH
}

sb2_status sb2_bunch_snapshot_counts(sb2_bunch* h, int64_t* n_valid, int64_t* n_total, double* real_num)
{
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    Bunch& b = h->b;
    SB2_REQUIRE(b.snap_counters != nullptr, "no snapshot taken");
    if (n_valid) *n_valid = b.snap_counters->n_valid;
    if (n_total) *n_total = b.snap_counters->n_total;
    if (real_num) *real_num = b.snap_counters->real_num;
    SB2_CATCH
}

sb2_status sb2_bunch_populate_gaussian(sb2_bunch* h, const double sigma[6], uint64_t seed)
{
    SB2_TRY
    SB2_REQUIRE(h && sigma, "null argument");
    Bunch& b = h->b;
    b.settle(0);
    if (b.n) cuda_check(launch_populate(b.parts, b.stride, b.masks, b.n, sigma, seed, 0), "populate");
    cuda_check(cudaStreamSynchronize(0), "populate");
    b.host_counters.n_valid = b.host_counters.n_total = (int32_t)b.n;
    cuda_check(cudaMemcpy(&b.host_counters.real_num, &b.counters->real_num, sizeof(double), cudaMemcpyDeviceToHost),
               "counters");
    cuda_check(cudaMemcpy(b.counters, &b.host_counters, sizeof(BunchCounters), cudaMemcpyHostToDevice), "counters");
    SB2_CATCH
}

sb2_status sb2_bunch_moments(sb2_bunch* h, double mean[6], double mom2[36], double emit[3])
{ // Core_diagnostics::calculate_mean / calculate_mom2, calculate_emittances
    SB2_TRY
    SB2_REQUIRE(h, "null bunch");
    Bunch& b = h->b;
    b.settle(0);
    const int nb = track_grid_blocks();
    double* part = dalloc<double>((size_t)nb * 27, "moment partials");
    double* dmean = dalloc<double>(6, "mean");
    std::vector<double> hp((size_t)nb * 27);
    cuda_check(cudaMemcpy(&b.host_counters, b.counters, sizeof(BunchCounters), cudaMemcpyDeviceToHost), "counters");
    double nt = b.host_counters.n_total;
    double mu[6] = {0, 0, 0, 0, 0, 0};
    cuda_check(launch_moments(b.parts, b.stride, b.masks, b.n, nullptr, part, nb, 0), "moments");
    cuda_check(cudaMemcpy(hp.data(), part, sizeof(double) * nb * 27, cudaMemcpyDeviceToHost), "moments");
    for (int k = 0; k < nb; ++k)
        for (int j = 0; j < 6; ++j) mu[j] += hp[(size_t)k * 27 + j];
    for (int j = 0; j < 6; ++j) mu[j] /= nt;
    cuda_check(cudaMemcpy(dmean, mu, sizeof(mu), cudaMemcpyHostToDevice), "mean");
    cuda_check(launch_moments(b.parts, b.stride, b.masks, b.n, dmean, part, nb, 0), "moments");
    cuda_check(cudaMemcpy(hp.data(), part, sizeof(double) * nb * 27, cudaMemcpyDeviceToHost), "moments");
    dfree(part);
    dfree(dmean);
    double m2[6][6];
    int t = 6;
    double acc[21] = {0};
    for (int k = 0; k < nb; ++k)
        for (int j = 0; j < 21; ++j) acc[j] += hp[(size_t)k * 27 + 6 + j];
    for (int j = 0; j < 6; ++j)
        for (int k = 0; k <= j; ++k) {
            m2[j][k] = m2[k][j] = acc[t - 6] / nt;
            ++t;
        }
    if (mean)
        for (int j = 0; j < 6; ++j) mean[j] = mu[j];
    if (mom2)
        for (int j = 0; j < 6; ++j)
            for (int k = 0; k < 6; ++k) mom2[j * 6 + k] = m2[j][k];
    if (emit)
        for (int pl = 0; pl < 3; ++pl) {
            double det = m2[2 * pl][2 * pl] * m2[2 * pl + 1][2 * pl + 1] - m2[2 * pl][2 * pl + 1] * m2[2 * pl + 1][2 * pl];
            if (det < 0 && det > -1.0e-15) det = 0; // eliminate_small_negative
            emit[pl] = std::sqrt(det);
        }
    SB2_CATCH
}

sb2_status sb2_lattice_create(const char* name, sb2_lattice** out)
{
    SB2_TRY
    SB2_REQUIRE(out, "null out");
    auto* l = new sb2_lattice();
    l->l.name = name ? name : "";
    *out = l;
    SB2_CATCH
}
sb2_status sb2_lattice_destroy(sb2_lattice* l)
{
    SB2_TRY
    delete l;
    SB2_CATCH
}
sb2_status sb2_lattice_set_reference_particle(sb2_lattice* l, int32_t charge, double mass, double value, int32_t kind)
{
    SB2_TRY
    SB2_REQUIRE(l, "null lattice");
    l->l.ref.set(charge, mass, value, kind);
    l->l.has_ref = true;
    SB2_CATCH
}
sb2_status sb2_lattice_append(sb2_lattice* l, const char* type, const char* name, int32_t* index)
{
    SB2_TRY
    SB2_REQUIRE(l && type, "null argument");
    Element e;
    e.type = type;
    e.name = name ? name : "";
    l->l.elements.push_back(e);
    if (index) *index = (int32_t)l->l.elements.size() - 1;
    SB2_CATCH
}
static Element& elem_at(sb2_lattice* l, int32_t i)
{
    if (!l || i < 0 || i >= (int32_t)l->l.elements.size()) throw Error(SB2_ERR_INVALID, "element index out of range");
    return l->l.elements[i];
}
sb2_status sb2_lattice_set_double(sb2_lattice* l, int32_t i, const char* attr, double v)
{
    SB2_TRY
    SB2_REQUIRE(attr, "null attribute");
    elem_at(l, i).d[attr] = v;
    SB2_CATCH
}
sb2_status sb2_lattice_set_string(sb2_lattice* l, int32_t i, const char* attr, const char* v)
{
    SB2_TRY
    SB2_REQUIRE(attr && v, "null attribute");
    elem_at(l, i).s[attr] = v;
    SB2_CATCH
}
sb2_status sb2_lattice_set_vector(sb2_lattice* l, int32_t i, const char* attr, const double* v, int32_t n)
{
    SB2_TRY
    SB2_REQUIRE(attr && (v || n == 0) && n >= 0, "bad vector attribute");
    elem_at(l, i).v[attr] = std::vector<double>(v, v + n);
    SB2_CATCH
}
sb2_status sb2_lattice_length(sb2_lattice* l, double* length)
{
    SB2_TRY
    SB2_REQUIRE(l && length, "null argument");
    *length = l->l.length();
    SB2_CATCH
}
sb2_status sb2_lattice_num_elements(sb2_lattice* l, int32_t* n)
{
    SB2_TRY
    SB2_REQUIRE(l && n, "null argument");
    *n = (int32_t)l->l.elements.size();
    SB2_CATCH
}


sb2_status sb2_propagator_create(const sb2_lattice* lattice, int32_t stepper, int32_t num_steps,
                                 const sb2_sc3d_options* sc, sb2_propagator** out)
{
    SB2_TRY
    SB2_REQUIRE(lattice && out, "null argument");
    auto* p = new sb2_propagator();
    std::unique_ptr<sb2_propagator> guard(p);
    p->p.reset(new Propagator(lattice->l, stepper, num_steps, sc));
    *out = guard.release();
    SB2_CATCH
}
sb2_status sb2_propagator_destroy(sb2_propagator* p)
{
    SB2_TRY
    delete p;
    SB2_CATCH
}
sb2_status sb2_propagator_num_steps(sb2_propagator* p, int32_t* n)
{
    SB2_TRY
    SB2_REQUIRE(p && n, "null argument");
    *n = (int32_t)p->p->steps.size();
    SB2_CATCH
}
sb2_status sb2_propagator_step_slices(sb2_propagator* p, int32_t step, int32_t op, double* out, int32_t cap, int32_t* n)
{
    SB2_TRY
    SB2_REQUIRE(p && n && step >= 0 && step < (int32_t)p->p->steps.size(), "bad step");
    auto& st = p->p->steps[step];
    if (op < 0 || op >= (int32_t)st.indeps.size()) {
        *n = -1;
        return SB2_OK;
    }
    auto& sl = st.indeps[op].slices;
    int32_t k = 0;
    for (auto& s : sl) {
        if (k >= cap) break;
        out[k * 3 + 0] = s.elem;
        out[k * 3 + 1] = s.left;
        out[k * 3 + 2] = s.right;
        ++k;
    }
    *n = k;
    SB2_CATCH
}

sb2_status sb2_propagator_propagate(sb2_propagator* p, sb2_bunch* b, int32_t turns, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(p && b && turns >= 0, "bad argument");
    p->p->propagate(b->b, turns, as_stream(stream));
    SB2_CATCH
}
sb2_status sb2_propagator_propagate_steps(sb2_propagator* p, sb2_bunch* b, int32_t first, int32_t count, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(p && b && count >= 0, "bad argument");
    p->p->propagate_steps(b->b, first, count, as_stream(stream));
    SB2_CATCH
}
sb2_status sb2_propagator_prepare_steps(sb2_propagator* p, sb2_bunch* b, int32_t first, int32_t count, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(p && b && count >= 0, "bad argument");
    p->p->prepare_steps(b->b, first, count, as_stream(stream));
    SB2_CATCH
}
sb2_status sb2_propagator_set_graphs(sb2_propagator* p, int32_t on)
{
    SB2_TRY
    SB2_REQUIRE(p, "null propagator");
    if (on && p->p->hook) throw Error(SB2_ERR_UNSUPPORTED, "CUDA-graph turns are not available on a sharded propagator");
    if (on && p->p->loss_cap)
        throw Error(SB2_ERR_UNSUPPORTED, "loss diagnostics are not available with CUDA-graph turns");
    if (on && p->p->step_rec_cap && !p->p->step_rec_pinned())
        throw Error(SB2_ERR_UNSUPPORTED, "per-step count records into a pageable buffer are not available with "
                                         "CUDA-graph turns (pass pinned memory)");
    p->p->use_graphs = on != 0;
    if (!on) p->p->drop_graphs();
    SB2_CATCH
}

sb2_status sb2_propagator_graph_stats(sb2_propagator* p, int64_t* captures, int64_t* replays)
{
    SB2_TRY
    SB2_REQUIRE(p, "null propagator");
    if (captures) *captures = p->p->graph_captures;
    if (replays) *replays = p->p->graph_replays;
    SB2_CATCH
}

sb2_status sb2_batch_create(sb2_batch** out)
{
    SB2_TRY
    SB2_REQUIRE(out, "null out");
    *out = new sb2_batch();
    SB2_CATCH
}

sb2_status sb2_batch_destroy(sb2_batch* q)
{
    SB2_TRY
    delete q;
    SB2_CATCH
}

sb2_status sb2_batch_add(sb2_batch* q, sb2_propagator* p, sb2_bunch* b, int32_t* slot)
{
    SB2_TRY
    SB2_REQUIRE(q && p && b && slot, "null argument");
    *slot = q->q.add(p->p.get(), &b->b);
    SB2_CATCH
}

sb2_status sb2_batch_remove(sb2_batch* q, int32_t slot)
{
    SB2_TRY
    SB2_REQUIRE(q, "null batch");
    q->q.remove(slot);
    SB2_CATCH
}

sb2_status sb2_batch_run(sb2_batch* q, const int32_t* slots, const int32_t* turns, int32_t n)
{
    SB2_TRY
    SB2_REQUIRE(q && (n == 0 || (slots && turns)) && n >= 0, "bad argument");
    q->q.run(slots, turns, n);
    SB2_CATCH
}

sb2_status sb2_propagator_set_diagnostics(sb2_propagator* p, int32_t capacity)
{
    SB2_TRY
    SB2_REQUIRE(p && capacity >= 0, "bad argument");
    if (capacity > 0 && p->p->hook)
        throw Error(SB2_ERR_UNSUPPORTED, "per-turn diagnostics are not available on a sharded propagator");
    p->p->set_diagnostics(capacity);
    SB2_CATCH
}

void* sb2_allreduce_stream(void) { return (void*)g_hook_stream; }

sb2_status sb2_propagator_set_allreduce(sb2_propagator* p, sb2_allreduce_fn fn, void* ctx, int32_t on_host)
{
    SB2_TRY
    SB2_REQUIRE(p, "null propagator");
    if (fn && (p->p->use_graphs || p->p->diag_cap))
        throw Error(SB2_ERR_UNSUPPORTED, "a sharded propagator runs without CUDA-graph turns and per-turn diagnostics");
    p->p->hook.fn = fn;
    p->p->hook.tfn = nullptr;
    p->p->hook.ctx = ctx;
    p->p->hook.on_host = on_host != 0;
    SB2_CATCH
}

sb2_status sb2_propagator_set_allreduce_typed(sb2_propagator* p, sb2_allreduce_typed_fn fn, void* ctx,
                                              int32_t on_host)
{
    SB2_TRY
    SB2_REQUIRE(p, "null propagator");
    if (fn && (p->p->use_graphs || p->p->diag_cap))
        throw Error(SB2_ERR_UNSUPPORTED, "a sharded propagator runs without CUDA-graph turns and per-turn diagnostics");
    p->p->hook.fn = nullptr;
    p->p->hook.tfn = fn;
    p->p->hook.ctx = ctx;
    p->p->hook.on_host = on_host != 0;
    SB2_CATCH
}

sb2_status sb2_propagator_read_diagnostics(sb2_propagator* p, int32_t max_records, int32_t* count, double* records,
                                           double* s, int32_t* turns)
{
    SB2_TRY
    SB2_REQUIRE(p && count && max_records >= 0, "bad argument");
    Propagator& P = *p->p;
    *count = 0;
    if (!P.diag_cap) return SB2_OK;
    int32_t dev_count = 0;
    cuda_check(cudaMemcpy(&dev_count, P.diag_count, sizeof(int32_t), cudaMemcpyDeviceToHost), "diagnostics");
    const int n = std::min(std::min(dev_count, P.diag_cap), max_records);
    *count = n;
    if (records && n)
        cuda_check(cudaMemcpy(records, P.diag_records, sizeof(double) * kDiagRecord * n, cudaMemcpyDeviceToHost),
                   "diagnostics");
    for (int i = 0; i < n && i < (int)P.diag_s.size(); ++i) {
        if (s) s[i] = P.diag_s[i];
        if (turns) turns[i] = P.diag_turn[i];
    }
    SB2_CATCH
}

int32_t sb2_diagnostics_record_size(void) { return kDiagRecord; }

sb2_status sb2_propagator_set_loss_diagnostics(sb2_propagator* p, int32_t capacity)
{
    SB2_TRY
    SB2_REQUIRE(p && capacity >= 0, "bad argument");
    if (capacity > 0 && p->p->use_graphs)
        throw Error(SB2_ERR_UNSUPPORTED, "loss diagnostics are not available with CUDA-graph turns");
    p->p->set_loss_diagnostics(capacity);
    SB2_CATCH
}

static void check_tune(const sb2_tune& t)
{
    SB2_REQUIRE(t.light_shape >= 0 && t.light_shape <= 3, "tune: light_shape is 0, 1, 2 or 3");
    SB2_REQUIRE(t.full_occ == 2 || t.full_occ == 3, "tune: full_occ is 2 or 3");
    SB2_REQUIRE(t.full_ppt == 1 || t.full_ppt == 2, "tune: full_ppt is 1 or 2");
    SB2_REQUIRE(t.quad_variant >= 0 && t.quad_variant <= 2, "tune: quad_variant is 0, 1 or 2");
    SB2_REQUIRE(t.ctas_per_sm >= 1 && t.ctas_per_sm <= kMaxCtasPerSm, "tune: ctas_per_sm is 1..12");
    SB2_REQUIRE(t.sort_interval >= 1, "tune: sort_interval >= 1");
    SB2_REQUIRE(t.fft_plan == 0 || t.fft_plan == 1, "tune: fft_plan is 0 or 1");
    SB2_REQUIRE(t.deposit_chunk == 0 || t.deposit_chunk == 4 || t.deposit_chunk == 8,
                "tune: deposit_chunk is 0, 4 or 8");
}

static sb2_tune export_tune(const Propagator& P)
{
    sb2_tune t;
    t.light_shape = P.tune.light_shape;
    t.full_occ = P.tune.full_occ;
    t.full_ppt = P.tune.full_ppt;
    t.quad_variant = P.tune.quad_variant;
    t.ctas_per_sm = P.tune.ctas_per_sm;
    t.sort_interval = P.sort_interval;
    t.fft_plan = P.solve_tune.fft_plan;
    t.deposit_chunk = P.solve_tune.deposit_chunk;
    return t;
}

sb2_status sb2_propagator_get_tune(sb2_propagator* p, sb2_tune* out)
{
    SB2_TRY
    SB2_REQUIRE(p && out, "null argument");
    *out = export_tune(*p->p);
    SB2_CATCH
}

sb2_status sb2_propagator_set_tune(sb2_propagator* p, const sb2_tune* in)
{
    SB2_TRY
    SB2_REQUIRE(p && in, "null argument");
    check_tune(*in);
    TrackTune t{in->light_shape, in->full_occ, in->full_ppt, in->quad_variant, in->ctas_per_sm};
    Propagator::SolveTune st;
    st.fft_plan = in->fft_plan;
    st.deposit_chunk = in->deposit_chunk;
    p->p->apply_tune(t, in->sort_interval, st);
    SB2_CATCH
}

sb2_status sb2_propagator_autotune(sb2_propagator* p, sb2_bunch* b, int32_t steps, sb2_tune* best, double* trials,
                                   int32_t max_trials, int32_t* ntrials)
{
    SB2_TRY
    SB2_REQUIRE(p && b, "null argument");
    std::vector<std::array<double, 9>> log;
    p->p->autotune(b->b, steps, log);
    if (best) *best = export_tune(*p->p);
    const int n = (int)log.size();
    if (ntrials) *ntrials = n;
    if (trials)
        for (int i = 0; i < std::min(n, (int)max_trials); ++i)
            for (int j = 0; j < 9; ++j) trials[9 * i + j] = log[i][j];
    SB2_CATCH
}

sb2_status sb2_propagator_set_step_counts(sb2_propagator* p, sb2_step_counts* host, int32_t capacity)
{
    SB2_TRY
    SB2_REQUIRE(p && capacity >= 0 && (host || capacity == 0), "bad argument");
    static_assert(sizeof(sb2_step_counts) == sizeof(BunchCounters), "step record layout");
    p->p->set_step_counts(reinterpret_cast<BunchCounters*>(host), capacity);
    if (capacity > 0 && p->p->use_graphs && !p->p->step_rec_pinned()) {
        p->p->set_step_counts(nullptr, 0);
        throw Error(SB2_ERR_UNSUPPORTED, "per-step count records into a pageable buffer are not available with "
                                         "CUDA-graph turns (pass pinned memory)");
    }
    p->p->drop_graphs(); // captured launches name the record arrays
    SB2_CATCH
}

sb2_status sb2_propagator_step_counts_written(sb2_propagator* p, int32_t* count)
{
    SB2_TRY
    SB2_REQUIRE(p && count, "bad argument");
    *count = p->p->engine_ ? p->p->engine_->rec_next : 0;
    SB2_CATCH
}

sb2_status sb2_propagator_read_losses(sb2_propagator* p, int32_t max_records, int32_t* count, double* records)
{
    SB2_TRY
    SB2_REQUIRE(p && count && max_records >= 0, "bad argument");
    Propagator& P = *p->p;
    *count = 0;
    if (!P.loss_cap) return SB2_OK;
    int32_t dev = 0;
    cuda_check(cudaMemcpy(&dev, P.loss_count, sizeof(int32_t), cudaMemcpyDeviceToHost), "losses");
    const int n = std::min(std::min(dev, P.loss_cap), max_records);
    std::vector<double> raw((size_t)std::max(n, 1) * 8);
    if (n) cuda_check(cudaMemcpy(raw.data(), P.loss_buf, sizeof(double) * 8 * n, cudaMemcpyDeviceToHost), "losses");
    // appended in atomic order: sort by (aperture, id) for a stable listing
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const double ta = raw[a * 8 + 7], tb = raw[b * 8 + 7];
        return ta != tb ? ta < tb : raw[a * 8 + 6] < raw[b * 8 + 6];
    });
    for (int k = 0; k < n; ++k) {
        const double* r = &raw[(size_t)order[k] * 8];
        double* o = records + (size_t)k * 10;
        for (int j = 0; j < 7; ++j) o[j] = r[j];
        const size_t tag = (size_t)r[7];
        const auto t = tag < P.loss_tags.size() ? P.loss_tags[tag] : std::array<double, 3>{-1.0, -1.0, -1.0};
        o[7] = t[0];
        o[8] = t[1];
        o[9] = t[2];
    }
    *count = n;
    SB2_CATCH
}

sb2_status sb2_batch_run_lockstep(sb2_batch* q, const int32_t* slots, int32_t n, int32_t turns)
{
    SB2_TRY
    SB2_REQUIRE(q && slots, "null argument");
    q->q.run_lockstep(slots, n, turns);
    SB2_CATCH
}

sb2_status sb2_batch_launch(sb2_batch* q, int32_t slot, int32_t turns)
{
    SB2_TRY
    SB2_REQUIRE(q && turns >= 0, "bad argument");
    q->q.launch(slot, turns);
    SB2_CATCH
}

sb2_status sb2_batch_query(sb2_batch* q, int32_t slot, int32_t* done)
{
    SB2_TRY
    SB2_REQUIRE(q && done, "bad argument");
    *done = q->q.query(slot);
    SB2_CATCH
}

sb2_status sb2_propagator_deposited_charge(sb2_propagator* p, int32_t index, double* charge)
{
    SB2_TRY
    SB2_REQUIRE(p && charge && index >= 0 && index < (int32_t)p->p->lat.elements.size(), "bad element index");
    *charge = 0.0;
    if (!p->p->elem_charge) return SB2_OK;
    cuda_check(cudaMemcpy(charge, p->p->elem_charge + index, sizeof(double), cudaMemcpyDeviceToHost), "charge");
    SB2_CATCH
}

sb2_status sb2_propagator_sc_last(sb2_propagator* p, double left[3], double h[3], double* rho, double* phi, double* ex,
                                  double* ey, double* ez, double scalars[8])
{
    SB2_TRY
    SB2_REQUIRE(p, "null propagator");
    if (!p->p->has_sc) throw Error(SB2_ERR_INVALID, "propagator has no space-charge operator");
    if (!p->p->sc) throw Error(SB2_ERR_INVALID, "propagator has not run a space-charge kick yet");
    p->p->sc->copy_last(left, h, rho, phi, ex, ey, ez, scalars);
    SB2_CATCH
}

sb2_status sb2_sc3d_create(const sb2_sc3d_options* opts, sb2_sc3d** out)
{
    SB2_TRY
    SB2_REQUIRE(opts && out, "null argument");
    auto* s = new sb2_sc3d();
    std::unique_ptr<sb2_sc3d> guard(s);
    s->op.reset(new ScOperator(*opts));
    *out = guard.release();
    SB2_CATCH
}
sb2_status sb2_sc3d_destroy(sb2_sc3d* sc)
{
    SB2_TRY
    delete sc;
    SB2_CATCH
}
sb2_status sb2_sc3d_apply(sb2_sc3d* sc, sb2_bunch* b, double time_step, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(sc && b, "null argument");
    b->b.settle(as_stream(stream));
    sc->op->apply(b->b, time_step, as_stream(stream));
    b->b.sync_counters(as_stream(stream));
    SB2_CATCH
}
sb2_status sb2_sc3d_last(sb2_sc3d* sc, double left[3], double h[3], double* rho, double* phi, double* ex, double* ey,
                         double* ez, double scalars[8])
{
    SB2_TRY
    SB2_REQUIRE(sc, "null argument");
    sc->op->sc.copy_last(left, h, rho, phi, ex, ey, ez, scalars);
    SB2_CATCH
}

sb2_status sb2_libff_apply(const sb2_lattice* lattice, const double* slices, int32_t nslices, sb2_bunch* hb, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(lattice && hb && (slices || nslices == 0), "null argument");
    Bunch& b = hb->b;
    b.settle(as_stream(stream));
    const Lattice& lat = lattice->l;
    if (!b.design_set) {
        b.design = lat.ref;
        b.design_set = true;
    }
    Engine eng;
    std::vector<MapOp> ops;
    for (int32_t i = 0; i < nslices; ++i) {
        int ei = (int)slices[3 * i];
        SB2_REQUIRE(ei >= 0 && ei < (int)lat.elements.size(), "slice element out of range");
        Slice sl = make_slice(lat, ei, slices[3 * i + 1], slices[3 * i + 2]);
        ops_slice(lat, sl, b, eng.ops);
    }
    eng.flush(b, nullptr, nullptr, false, 0.0, as_stream(stream));
    cuda_check(cudaStreamSynchronize(as_stream(stream)), "sync");
    SB2_CATCH
}

sb2_status sb2_aperture_apply(const sb2_lattice* lattice, int32_t index, const char* aperture_type, sb2_bunch* hb,
                              int32_t* ndiscarded, void* stream)
{
    SB2_TRY
    SB2_REQUIRE(lattice && hb && aperture_type, "null argument");
    SB2_REQUIRE(index >= 0 && index < (int32_t)lattice->l.elements.size(), "element index out of range");
    Bunch& b = hb->b;
    b.settle(as_stream(stream));
    Engine eng;
    Slice sl = whole_slice(lattice->l, index);
    MapOp m = op_aperture(lattice->l, aperture_type, sl);
    m.slot = 0;
    eng.ops.push_back(m);
    eng.nslots = 1;
    // a lone aperture does not run update_total_num: only n_valid changes
    eng.flush(b, nullptr, nullptr, false, 0.0, as_stream(stream));
    int32_t nd = 0;
    cuda_check(cudaMemcpyAsync(&nd, eng.ap_counts, sizeof(int32_t), cudaMemcpyDeviceToHost, as_stream(stream)), "count");
    cuda_check(cudaMemsetAsync(eng.ap_counts, 0, sizeof(int32_t), as_stream(stream)), "count");
    b.sync_counters(as_stream(stream));
    b.host_counters.n_valid -= nd;
    cuda_check(cudaMemcpy(b.counters, &b.host_counters, sizeof(BunchCounters), cudaMemcpyHostToDevice), "counters");
    if (ndiscarded) *ndiscarded = nd;
    SB2_CATCH
}

} // extern "C"
