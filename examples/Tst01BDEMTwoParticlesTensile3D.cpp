// examples/tst_01_BDEM_two_particles_tensile_3D.cpp on the C++ interface, written as the
// reference's own loop (:295-306): BondedDEMIntegrator stage1, stage2, resetForcesAndTorques,
// the example's applyTensileForce, computeBondedForce, the example's applyBoundaryConditions,
// stage3, a snapshot every 100 steps.  Two bonded spheres (r = 0.5, rho = 2000, E = 1e4,
// G = 1e3, nu = 0.25) touching at the origin are pulled apart by -+1e3 N along x; particle 0's
// force is zeroed after the bond pass.  dt = 1e-4 to t = 4 (:162-306).
//
//   Tst01BDEMTwoParticlesTensile3D [output_folder] [--hooks=slices|device] [--fused]
//
// The reference takes no arguments.  --hooks=slices (the default) writes the two hooks as the
// reference does, through the force slice (host mirrors, uploaded before the next phase);
// --hooks=device runs them on the device (setExternalForce + addExternalForce, setFixFlags +
// applyFixFlags).  --fused runs the whole loop fused (one kernel per step) between snapshots.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "example_common.hpp"

using namespace examples;

#define MAX_BONDS 27

// tst_01_BDEM:19-67: the first particle's force is zeroed (every thread of the reference's
// loop writes the same entry)
template <class ExecutionSpace, class ParticleType>
void applyBoundaryConditions(ParticleType &particles) {
    auto force = particles.sliceForce();
    force(0, 0) = 0.;
    force(0, 1) = 0.;
    force(0, 2) = 0.;
}

// tst_01_BDEM:70-117: F += the external force
template <class ExecutionSpace, class ParticleType>
void applyTensileForce(ParticleType &particles, const std::vector<double> &ext_frc) {
    auto force = particles.sliceForce();
    for (int i = 0; i < static_cast<int>(force.size()); ++i) {
        force(i, 0) += ext_frc[3 * i + 0];
        force(i, 1) += ext_frc[3 * i + 1];
        force(i, 2) += ext_frc[3 * i + 2];
    }
}

int main(int argc, char *argv[]) {
    std::string folder = "tst_01_bdem_output";
    bool device_hooks = false, fused = false;
    for (int a = 1; a < argc; ++a) {
        if (!std::strcmp(argv[a], "--hooks=device")) device_hooks = true;
        else if (!std::strcmp(argv[a], "--hooks=slices")) device_hooks = false;
        else if (!std::strcmp(argv[a], "--fused")) fused = true;
        else folder = argv[a];
    }
    const double radius_p_inp = 0.5, rho_p_inp = 2000., E_p_inp = 1e4, G_p_inp = 1e3, nu_p_inp = 0.25;
    CabanaBondedDEM::ParticlesBondedDEM<memory_space, 3, MAX_BONDS> particles(exec_space(), 2, folder);
    particles.update_mesh_limits({-4. * radius_p_inp, -4. * radius_p_inp, -4. * radius_p_inp},
                                 {4. * radius_p_inp, 4. * radius_p_inp, 4. * radius_p_inp});
    auto x = particles.slicePosition();
    auto u = particles.sliceVelocity();
    auto au = particles.sliceAcceleration();
    auto force = particles.sliceForce();
    auto torque = particles.sliceTorque();
    auto omega = particles.sliceOmega();
    auto m = particles.sliceMass();
    auto rho = particles.sliceDensity();
    auto rad = particles.sliceRadius();
    auto E = particles.sliceYoungsMod();
    auto nu = particles.slicePoissonsRatio();
    auto G = particles.sliceShearMod();
    auto I = particles.sliceMomentOfInertia();
    auto bond_ft_x = particles.sliceBondFtX();
    auto bond_mt_z = particles.sliceBondMtZ();
    auto bond_idx = particles.sliceBondIdx();
    auto bond_init_len = particles.sliceBondInitLen();
    auto total_no_bonds = particles.sliceTotalNoBonds();
    auto particles_init_functor = [=](const int i) {
        const double m_p_i = 4. / 3. * M_PI * radius_p_inp * radius_p_inp * radius_p_inp * rho_p_inp;
        const double I_p_i = 2. / 5. * m_p_i * radius_p_inp * radius_p_inp;
        x(i, 0) = -radius_p_inp + i * (2. * radius_p_inp);
        x(i, 1) = 0.;
        x(i, 2) = 0.;
        for (int j = 0; j < 3; ++j) {
            u(i, j) = 0.;
            au(i, j) = 0.;
            force(i, j) = 0.;
            torque(i, j) = 0.;
            omega(i, j) = 0.;
        }
        m(i) = m_p_i;
        rho(i) = rho_p_inp;
        rad(i) = radius_p_inp;
        E(i) = E_p_inp;
        nu(i) = nu_p_inp;
        G(i) = G_p_inp;
        I(i) = I_p_i;
        for (int j = 0; j < MAX_BONDS; ++j) {
            bond_ft_x(i, j) = 0.;
            bond_mt_z(i, j) = 0.;
            bond_idx(i, j) = -1;
            bond_init_len(i, j) = 0.;
        }
        total_no_bonds(i) = 0;
    };
    particles.updateParticles(exec_space{}, particles_init_functor);
    particles.setupBonds<exec_space>();

    CabanaBondedDEM::BondedDEMIntegrator<exec_space> integrator(1e-4);
    const double dt = 1e-4, final_time = 4.;
    const int num_steps = final_time / dt, output_frequency = 100;
    const std::vector<double> ext_frc = {-1e3, 0., 0., 1e3, 0., 0.};
    if (device_hooks || fused) {
        particles.setExternalForce(ext_frc);
        particles.setFixFlags({DEM_FIX_FORCE, 0});
    }

    if (fused) {
        for (int step = 0; step <= num_steps;) {
            const int stop = step == 0 ? 0 : std::min(num_steps, (step + output_frequency - 1) / output_frequency *
                                                                     output_frequency);
            particles.run_steps(stop - step + 1, dt);
            std::printf("We are at %d / %d\n", stop, num_steps);
            particles.output(stop / output_frequency, stop * dt);
            step = stop + 1;
        }
    } else {
        for (int step = 0; step <= num_steps; step++) {
            integrator.stage1(particles);
            integrator.stage2(particles);
            CabanaBondedDEM::resetForcesAndTorques<exec_space>(particles);
            if (device_hooks) particles.addExternalForce();
            else applyTensileForce<exec_space>(particles, ext_frc);
            CabanaBondedDEM::computeBondedForce<exec_space>(particles, dt);
            if (device_hooks) particles.applyFixFlags();
            else applyBoundaryConditions<exec_space>(particles);
            integrator.stage3(particles);
            if (step % output_frequency == 0) {
                std::printf("We are at %d / %d\n", step, num_steps);
                particles.output(step / output_frequency, step * dt);
            }
        }
    }
    auto xs = particles.slicePosition();
    std::printf("final x0 %.17g x1 %.17g broken %ld\n", xs.get(0, 0), xs.get(1, 0), particles.broken());
    return 0;
}
