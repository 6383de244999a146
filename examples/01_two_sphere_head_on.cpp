// Two identical spheres colliding head on, through the C++ interface of libb200dem.so.
// Same set-up as the reference's first validation case
// (examples/01_elastic_normal_impact_of_two_identical_particles.cpp): spheres at
// x = -r and x = r + r/100 moving at +v and -v, one wall out of reach, delta = 3 r.
// Usage: 01_two_sphere_head_on <input.json> [output.csv]
// Writes step, time, force on sphere 1 (x) and the overlap for every step to the CSV.
#include <cmath>
#include <cstdio>
#include <memory>

#include "CabanaDEM_B200.hpp"

int main(int argc, char *argv[]) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s input.json [output.csv]\n", argv[0]);
        return 1;
    }
    using exec_space = CabanaDEM::DefaultExecutionSpace;
    using memory_space = exec_space::memory_space;
    CabanaDEM::Inputs inputs(argv[1]);
    const double rho = inputs["particle_density"], r = inputs["particle_radius"];
    const double E = inputs["particle_youngs_modulus"], G = inputs["particle_shear_modulus"];
    const double nu = inputs["particle_poissons_ratio"], v = inputs["velocity_p"];

    auto force = std::make_shared<CabanaDEM::Force<exec_space>>(
        inputs["coefficient_of_restitution_pp"], inputs["coefficient_of_restitution_pw"], inputs["friction_pp"],
        inputs["friction_pw"]);
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 1>>(exec_space(), 2);
    auto x = particles->slicePosition();
    auto u = particles->sliceVelocity();
    auto m = particles->sliceMass();
    auto I = particles->sliceMomentOfInertia();
    auto rad = particles->sliceRadius();
    auto dens = particles->sliceDensity();
    auto Ep = particles->sliceYoungsMod();
    auto Gp = particles->sliceShearMod();
    auto nup = particles->slicePoissonsRatio();
    particles->updateParticles(exec_space{}, [=](const int pid) {
        const double mass = 4. / 3. * M_PI * r * r * r * rho;
        x(pid, 0) = -r + pid * (2. * r) + pid * r / 100.;
        x(pid, 1) = 0.;
        x(pid, 2) = 0.;
        u(pid, 0) = pid == 0 ? v : -v;
        m(pid) = mass;
        I(pid) = 2. / 5. * mass * r * r;
        rad(pid) = r;
        dens(pid) = rho;
        Ep(pid) = E;
        Gp(pid) = G;
        nup(pid) = nu;
    });
    auto wall = std::make_shared<CabanaDEM::Wall<memory_space, 3>>(exec_space(), 1);
    auto xw = wall->slicePosition();
    auto nw = wall->sliceNormal();
    auto Ew = wall->sliceYoungsMod();
    auto Gw = wall->sliceShearMod();
    auto nuw = wall->slicePoissonsRatio();
    const double Ewi = inputs["wall_youngs_modulus"], Gwi = inputs["wall_shear_modulus"];
    const double nuwi = inputs["wall_poissons_ratio"];
    wall->updateParticles(exec_space{}, [=](const int w) {
        xw(w, 1) = -3. * r;
        nw(w, 1) = 1.;
        Ew(w) = Ewi;
        Gw(w) = Gwi;
        nuw(w) = nuwi;
    });
    auto solver = CabanaDEM::createSolverDEM<memory_space>(inputs, particles, wall, force, 3. * r);
    std::FILE *out = argc > 2 ? std::fopen(argv[2], "w") : nullptr;
    if (out) std::fprintf(out, "step,time,force_1x,overlap\n");
    // one step at a time so that every step's force is recorded (the reference writes every
    // output_frequency steps)
    for (int step = 0; step <= solver->num_steps; ++step) {
        solver->run_steps(1);
        if (out) {
            auto f = particles->sliceForce();
            auto xs = particles->slicePosition();
            std::fprintf(out, "%d,%.17g,%.17g,%.17g\n", step, step * solver->dt, f(1, 0),
                         2. * r - (xs(1, 0) - xs(0, 0)));
        }
    }
    if (out) std::fclose(out);
    auto f = particles->sliceVelocity();
    std::printf("final u0 %.17g u1 %.17g\n", f(0, 0), f(1, 0));
    return 0;
}
