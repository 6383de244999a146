// Reference command line of examples/01_elastic_normal_impact_of_two_identical_particles.cpp
// (main, :198-222): 01ElasticNormalImpactOfTwoIdenticalParticles <input.json> <output_folder>.
// Two spheres at x = -r and x = r + r/100 moving at +v and -v (:103-129), a wall out of reach at
// y = -3 r (:140-170), neighbour cutoff 3 r; particles_<k>.csv snapshots every output_frequency
// steps.  (01_two_sphere_head_on.cpp records the force at every step instead.)
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
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 1>>(exec_space(), 2, argv[2]);
    set_material(*particles, inputs);
    auto x = particles->slicePosition();
    auto u = particles->sliceVelocity();
    particles->updateParticles(exec_space{}, [=](const int pid) {
        x(pid, 0) = -r + pid * (2. * r) + pid * r / 100.;
        u(pid, 0) = pid == 0 ? v : -v;
    });
    const double p[3] = {0., -3. * r, 0.}, up[3] = {0., 1., 0.};
    auto wall = make_walls(inputs, 1, p, up);
    CabanaDEM::createSolverDEM<memory_space>(inputs, particles, wall, force, 3. * r)->run();
    return 0;
}
