// A C++ driver in the shape of the reference's examples/fodo_cxx/fodo_cxx.cc,
// written against the C ABI only (include/sb2.h): FODO lattice, 3D open
// Hockney space charge in a split-operator stepper, a seeded Gaussian bunch,
// N turns, the bunch moments printed as one JSON line.  It is what a C++
// caller of the library compiles against; the test suite builds and runs it.
//
//   g++ -std=c++17 -I include fodo_driver.cc -L synergia2_b200 -lsb2 -o fodo_driver
//   ./fodo_driver <macroparticles> <turns> [mixed]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "sb2.h"

static void check(sb2_status s)
{
    if (s != SB2_OK) throw std::runtime_error(sb2_last_error());
}

int main(int argc, char** argv)
{
    try {
        const long n = argc > 1 ? std::atol(argv[1]) : 1048576;
        const int turns = argc > 2 ? std::atoi(argv[2]) : 1;
        const bool mixed = argc > 3 && std::strcmp(argv[3], "mixed") == 0;
        const double mp = 0.938272046, kinetic = 2.5;

        sb2_lattice* lat = nullptr;
        check(sb2_lattice_create("fodo", &lat));
        check(sb2_lattice_set_reference_particle(lat, 1, mp, kinetic, SB2_REF_KINETIC_ENERGY));
        struct { const char *type, *name; double l, k1; } cell[] = {
            {"quadrupole", "qf", 0.5, 0.6}, {"drift", "d1", 4.5, 0.0},
            {"quadrupole", "qd", 0.5, -0.6}, {"drift", "d2", 4.5, 0.0}};
        for (auto const& e : cell) {
            int32_t idx = 0;
            check(sb2_lattice_append(lat, e.type, e.name, &idx));
            check(sb2_lattice_set_double(lat, idx, "l", e.l));
            if (std::string(e.type) == "quadrupole") check(sb2_lattice_set_double(lat, idx, "k1", e.k1));
        }

        sb2_sc3d_options sc;
        check(sb2_sc3d_options_init(&sc, 32, 32, 64));
        if (mixed) sc.precision = SB2_PRECISION_MIXED;
        sb2_propagator* prop = nullptr;
        check(sb2_propagator_create(lat, SB2_STEPPER_SPLIT_OPERATOR, 8, &sc, &prop));
        check(sb2_lattice_destroy(lat));

        sb2_bunch* bunch = nullptr;
        check(sb2_bunch_create(1, mp, kinetic, SB2_REF_KINETIC_ENERGY, n, 1e11, &bunch));
        const double sigma[6] = {1e-3, 1e-4, 1e-3, 1e-4, 0.3, 1e-4};
        check(sb2_bunch_populate_gaussian(bunch, sigma, 1));
        check(sb2_propagator_propagate(prop, bunch, turns, nullptr));

        double mean[6], mom2[36], emit[3];
        check(sb2_bunch_moments(bunch, mean, mom2, emit));
        int64_t active = 0, valid = 0, total = 0;
        double real = 0.0;
        check(sb2_bunch_counts(bunch, &active, &valid, &total, &real));
        std::printf("{\"n\": %ld, \"turns\": %d, \"total_num\": %lld, \"real_num\": %.17g, \"mean\": [", n, turns,
                    (long long)total, real);
        for (int j = 0; j < 6; ++j) std::printf("%s%.17g", j ? ", " : "", mean[j]);
        std::printf("], \"emit\": [%.17g, %.17g, %.17g]}\n", emit[0], emit[1], emit[2]);

        check(sb2_bunch_destroy(bunch));
        check(sb2_propagator_destroy(prop));
        return 0;
    } catch (std::exception const& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
}
