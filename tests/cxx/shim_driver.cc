// The per-operator drop-in as a reference-side shim would drive it, written
// against the C ABI only (include/sb2.h).  The reference's
// Independent_operator::apply_impl (simulation/independent_operator.cc:94-133)
// runs, for each half step, one LibFF_operation over the half step's slices
// (independent_operation.h:45-60 -> FF_element::apply) and then the Finite
// and Circular Aperture_operations of the last slice (:80-85,
// aperture_operation.h:14-24).  A LibFF_b200_operation / Aperture_operation
// shim replaces those bodies with sb2_libff_apply and sb2_aperture_apply;
// this driver makes exactly those calls, slice lists taken from the
// stepper's own slicing (sb2_propagator_step_slices).
//
//   shim_driver <lattice: fodo|ring> <particles in> <particles out> <turns> <steps per turn>
//
// Particle files: n (int64) then the n x 7 column-major FP64 array and the n
// mask bytes; the output adds the n discard bytes and, per aperture call,
// the number of discarded particles is printed as one JSON line.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "sb2.h"

static void check(sb2_status s)
{
    if (s != SB2_OK) throw std::runtime_error(sb2_last_error());
}

static void add(sb2_lattice* lat, const char* type, const char* name, double l,
                std::vector<std::pair<const char*, double>> attrs)
{
    int32_t idx = 0;
    check(sb2_lattice_append(lat, type, name, &idx));
    check(sb2_lattice_set_double(lat, idx, "l", l));
    for (auto const& a : attrs) check(sb2_lattice_set_double(lat, idx, a.first, a.second));
}

int main(int argc, char** argv)
{
    try {
        if (argc < 6) throw std::runtime_error("usage: shim_driver fodo|ring in out turns steps");
        const std::string kind = argv[1];
        const int turns = std::atoi(argv[4]), nsteps = std::atoi(argv[5]);
        const double mp = 0.938272046, kinetic = 2.5;

        sb2_lattice* lat = nullptr;
        check(sb2_lattice_create(kind.c_str(), &lat));
        check(sb2_lattice_set_reference_particle(lat, 1, mp, mp + kinetic, SB2_REF_TOTAL_ENERGY));
        if (kind == "fodo") {
            add(lat, "quadrupole", "qf", 0.5, {{"k1", 0.6}});
            add(lat, "drift", "d1", 4.5, {});
            add(lat, "quadrupole", "qd", 0.5, {{"k1", -0.6}});
            add(lat, "drift", "d2", 4.5, {});
        } else {
            // one cell of the 24-cell ring with a 6 mm circular aperture on
            // every element (particles are lost)
            const double ang = 2 * M_PI / 48, r = 0.006;
            add(lat, "quadrupole", "qf", 0.5, {{"k1", 0.55}, {"circular_aperture_radius", r}});
            add(lat, "sextupole", "sf", 0.0, {{"k2", 0.2}, {"circular_aperture_radius", r}});
            add(lat, "drift", "d1", 0.75, {{"circular_aperture_radius", r}});
            add(lat, "sbend", "b1", 2.0, {{"angle", ang}, {"circular_aperture_radius", r}});
            add(lat, "drift", "d2", 0.75, {{"circular_aperture_radius", r}});
            add(lat, "quadrupole", "qd", 0.5, {{"k1", -0.55}, {"circular_aperture_radius", r}});
            add(lat, "sextupole", "sd", 0.0, {{"k2", -0.2}, {"circular_aperture_radius", r}});
            add(lat, "drift", "d3", 0.75, {{"circular_aperture_radius", r}});
            add(lat, "sbend", "b2", 2.0, {{"angle", ang}, {"circular_aperture_radius", r}});
            add(lat, "drift", "d4", 0.75, {{"circular_aperture_radius", r}});
        }

        // the stepper's slicing (no collective operator: its steps are used
        // only for their slice lists)
        sb2_propagator* stepper = nullptr;
        check(sb2_propagator_create(lat, SB2_STEPPER_SPLIT_OPERATOR, nsteps, nullptr, &stepper));
        int32_t nst = 0;
        check(sb2_propagator_num_steps(stepper, &nst));

        FILE* f = std::fopen(argv[2], "rb");
        if (!f) throw std::runtime_error("cannot open input");
        int64_t n = 0;
        if (std::fread(&n, sizeof n, 1, f) != 1) throw std::runtime_error("short input");
        std::vector<double> parts(7 * n);
        std::vector<uint8_t> masks(n), discards(n);
        if (std::fread(parts.data(), sizeof(double), parts.size(), f) != parts.size() ||
            std::fread(masks.data(), 1, n, f) != (size_t)n)
            throw std::runtime_error("short input");
        std::fclose(f);

        sb2_bunch* bunch = nullptr;
        check(sb2_bunch_create(1, mp, mp + kinetic, SB2_REF_TOTAL_ENERGY, n, 1e11, &bunch));
        check(sb2_bunch_set_particles(bunch, parts.data(), masks.data()));

        std::printf("{\"discards\": [");
        bool first = true;
        std::vector<double> sl(3 * 256);
        for (int t = 0; t < turns; ++t)
            for (int s = 0; s < nst; ++s)
                for (int op = 0; op < 2; ++op) {
                    int32_t ns = 0;
                    check(sb2_propagator_step_slices(stepper, s, op, sl.data(), 256, &ns));
                    if (ns <= 0) continue;
                    // LibFF_b200_operation::apply_impl
                    check(sb2_libff_apply(lat, sl.data(), ns, bunch, nullptr));
                    // Aperture_operation<Finite_aperture>, <Circular_aperture>
                    const int32_t last = (int32_t)sl[3 * (ns - 1)];
                    for (const char* ap : {"finite", "circular"}) {
                        int32_t nd = 0;
                        check(sb2_aperture_apply(lat, last, ap, bunch, &nd, nullptr));
                        std::printf("%s%d", first ? "" : ", ", nd);
                        first = false;
                    }
                }
        std::printf("]}\n");

        check(sb2_bunch_get_particles(bunch, parts.data(), masks.data(), discards.data()));
        FILE* g = std::fopen(argv[3], "wb");
        if (!g) throw std::runtime_error("cannot open output");
        std::fwrite(&n, sizeof n, 1, g);
        std::fwrite(parts.data(), sizeof(double), parts.size(), g);
        std::fwrite(masks.data(), 1, n, g);
        std::fwrite(discards.data(), 1, n, g);
        std::fclose(g);

        check(sb2_bunch_destroy(bunch));
        check(sb2_propagator_destroy(stepper));
        check(sb2_lattice_destroy(lat));
        return 0;
    } catch (std::exception const& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
