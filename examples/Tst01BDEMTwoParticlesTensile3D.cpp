// Reference command line of examples/tst_01_BDEM_two_particles_tensile_3D.cpp (main,
// :318-329): Tst01BDEMTwoParticlesTensile3D [output_folder] (the reference takes no arguments).
// Two bonded spheres (r = 0.5, rho = 2000, E = 1e4, G = 1e3, nu = 0.25) touching at the origin
// are pulled apart by -+1e3 N along x; particle 0's force is zeroed after the bond pass
// (applyBoundaryConditions).  dt = 1e-4 to t = 4, snapshots every 100 steps (:162-306).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "example_common.hpp"

using namespace examples;

int main(int argc, char *argv[]) {
    const std::string folder = argc > 1 ? argv[1] : "tst_01_bdem_output";
    const double radius = 0.5, rho = 2000., E = 1e4, G = 1e3, nu = 0.25;
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 1, 0>>(exec_space(), 2, folder);
    auto x = particles->slicePosition();
    auto m = particles->sliceMass();
    auto I = particles->sliceMomentOfInertia();
    auto rad = particles->sliceRadius();
    auto dens = particles->sliceDensity();
    auto Ep = particles->sliceYoungsMod();
    auto Gp = particles->sliceShearMod();
    auto nup = particles->slicePoissonsRatio();
    particles->updateParticles(exec_space{}, [=](const int i) {
        const double mass = 4. / 3. * M_PI * radius * radius * radius * rho;
        x(i, 0) = -radius + i * (2. * radius);
        m(i) = mass;
        I(i) = 2. / 5. * mass * radius * radius;
        rad(i) = radius;
        dens(i) = rho;
        Ep(i) = E;
        Gp(i) = G;
        nup(i) = nu;
    });
    particles->setExternalForce({-1e3, 0., 0., 1e3, 0., 0.});
    particles->setFixFlags({DEM_FIX_FORCE, 0});
    const double dt = 1e-4, final_time = 4.;
    const int num_steps = final_time / dt, output_frequency = 100;
    // the reference's bond model as written: history indexed by partner, stiffness from E, G
    // and the bond area, the partner velocity read from particle i
    dem_bond_params bp{};
    bp.quirks = DEM_BQ10_INDEX_BY_J | DEM_BQ11_HARDCODED_K | DEM_BQ1_VELJ_USES_UI;
    bp.beta = 0.1;
    bp.radius_factor = 1.0;
    CabanaBondedDEM::BondedDEM<memory_space, 3, 27> bonded(particles, dt, bp);
    bonded.setupBonds(3.0, 4. * radius);
    // steps 0..num_steps; a snapshot after every step divisible by output_frequency
    for (int step = 0; step <= num_steps;) {
        const int stop = step == 0 ? 0 : std::min(num_steps, (step + output_frequency - 1) / output_frequency *
                                                                 output_frequency);
        bonded.run_steps(stop - step + 1);
        if (stop % output_frequency == 0) {
            std::printf("We are at %d / %d\n", stop, num_steps);
            particles->output(stop / output_frequency, stop * dt);
        }
        step = stop + 1;
    }
    auto xs = particles->slicePosition();
    std::printf("final x0 %.17g x1 %.17g broken %ld\n", xs.get(0, 0), xs.get(1, 0), bonded.broken());
    return 0;
}
