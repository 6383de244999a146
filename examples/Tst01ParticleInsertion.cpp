// Reference command line of examples/tst_01_particle_insertion.cpp:
// Tst01ParticleInsertion <input.json> <output_folder> --angle=<deg>.  No time stepping: the
// particle set is written, resized to 20 particles stacked 3 r apart moving at +y, written,
// moved by 2 u, written, resized to 15 particles 5 r apart and written again (:100-190), as
// particles_0/10/20/30.csv.  Slices taken before a resize follow the new size here; the
// reference's loop bound after the second resize reads the old slice's size.
#include <cmath>
#include <cstdio>

#include "example_common.hpp"

using namespace examples;

int main(int argc, char *argv[]) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder --angle=<degrees>\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double angle = examples::option_value(argv[3]) / 180. * M_PI;
    const double r = inputs["particle_radius"], v = inputs["velocity_p"];
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 1>>(exec_space(), 1, argv[2]);
    set_material(*particles, inputs);
    auto x = particles->slicePosition();
    auto u = particles->sliceVelocity();
    particles->updateParticles(exec_space{}, [=](const int pid) {
        x(pid, 1) = r + r / 1000000.;
        u(pid, 0) = v * sin(angle);
        u(pid, 1) = -v * cos(angle);
    });
    particles->output(0, 0.);
    particles->resize(20);
    for (int i = 0; i < (int)u.size(); i++) {
        x(i, 0) = 0.;
        x(i, 1) = 3 * i * r + r / 1000000.;
        x(i, 2) = 0.;
        u(i, 0) = 0.;
        u(i, 1) = 1.;
        u(i, 2) = 0.;
    }
    particles->output(10, 0.1);
    for (int i = 0; i < (int)u.size(); i++)
        for (int d = 0; d < 3; ++d) x(i, d) += 2. * u.get(i, d);
    particles->output(20, 0.2);
    particles->resize(15);
    for (int i = 0; i < (int)u.size(); i++) {
        x(i, 0) = 0.;
        x(i, 1) = 5 * i * r + r / 1000000.;
        x(i, 2) = 0.;
        u(i, 0) = 0.;
        u(i, 1) = 1.;
        u(i, 2) = 0.;
    }
    particles->output(30, 0.3);
    return 0;
}
