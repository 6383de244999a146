// Reference command line of examples/tst_03_multiple_particles_contacts.cpp:
// Tst03MultipleParticlesContacts <input.json> <output_folder>.  Sphere 0 at x = -r moving at
// +v into two spheres at rest, placed at (r/2 + r/100, +-3r/2) (:103-140); the one wall at
// y = -3 r has a zero normal, as in the reference (:151-190); cutoff 3 r.
#include <cstdio>

#include "example_common.hpp"

using namespace examples;

int main(int argc, char *argv[]) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double r = inputs["particle_radius"], v = inputs["velocity_p"];
    auto force = std::make_shared<CabanaDEM::Force<exec_space>>(
        inputs["coefficient_of_restitution_pp"], inputs["coefficient_of_restitution_pw"], inputs["friction_pp"],
        inputs["friction_pw"]);
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 1>>(exec_space(), 3, argv[2]);
    set_material(*particles, inputs);
    auto x = particles->slicePosition();
    auto u = particles->sliceVelocity();
    particles->updateParticles(exec_space{}, [=](const int pid) {
        x(pid, 0) = -r + pid * (2. * r) + pid * r / 100.;
        x(pid, 1) = 0.;
        if (pid == 1) {
            x(pid, 0) = -r + 1 * (1.5 * r) + 1 * r / 100.;
            x(pid, 1) = r + r / 2.;
        }
        if (pid == 2) {
            x(pid, 0) = -r + 1 * (1.5 * r) + 1 * r / 100.;
            x(pid, 1) = -r - r / 2.;
        }
        u(pid, 0) = pid == 0 ? v : 0.;
    });
    const double p[3] = {0., -3. * r, 0.}, zero[3] = {0., 0., 0.};
    auto wall = make_walls(inputs, 1, p, zero);
    CabanaDEM::createSolverDEM<memory_space>(inputs, particles, wall, force, 3. * r)->run();
    return 0;
}
