// Set-up shared by the example drivers: uniform material from the input file, one plane
// wall, the "--key=value" option of examples 03/04 and the single sphere thrown at a wall
// that examples 02, 03 and 04 share.
#pragma once

#include <cmath>
#include <cstdlib>
#include <memory>
#include <string>

#include "CabanaDEM_B200.hpp"

namespace examples {

using exec_space = CabanaDEM::DefaultExecutionSpace;
using memory_space = exec_space::memory_space;

// every particle gets the input's particle_* material; mass and inertia of a solid sphere in
// the examples' scalar form (examples/02_elastic_normal_impact_of_particle_wall.cpp:99-120)
template <class ParticleType>
void set_material(ParticleType &particles, const CabanaDEM::Inputs &inputs) {
    const double rho = inputs["particle_density"], r = inputs["particle_radius"];
    const double E = inputs["particle_youngs_modulus"], G = inputs["particle_shear_modulus"];
    const double nu = inputs["particle_poissons_ratio"];
    auto m = particles.sliceMass();
    auto I = particles.sliceMomentOfInertia();
    auto rad = particles.sliceRadius();
    auto dens = particles.sliceDensity();
    auto Ep = particles.sliceYoungsMod();
    auto Gp = particles.sliceShearMod();
    auto nup = particles.slicePoissonsRatio();
    particles.updateParticles(exec_space{}, [=](const int pid) {
        const double mass = 4. / 3. * M_PI * r * r * r * rho;
        m(pid) = mass;
        I(pid) = 2. / 5. * mass * r * r;
        rad(pid) = r;
        dens(pid) = rho;
        Ep(pid) = E;
        Gp(pid) = G;
        nup(pid) = nu;
    });
}

// nw walls, all at point p with normal nrm and the input's wall_* material
inline std::shared_ptr<CabanaDEM::Wall<memory_space, 3>> make_walls(const CabanaDEM::Inputs &inputs, int nw,
                                                                    const double p[3], const double nrm[3]) {
    auto wall = std::make_shared<CabanaDEM::Wall<memory_space, 3>>(exec_space(), nw);
    auto xw = wall->slicePosition();
    auto nw_ = wall->sliceNormal();
    auto Ew = wall->sliceYoungsMod();
    auto Gw = wall->sliceShearMod();
    auto nuw = wall->slicePoissonsRatio();
    const double E = inputs["wall_youngs_modulus"], G = inputs["wall_shear_modulus"];
    const double nu = inputs["wall_poissons_ratio"];
    const double px = p[0], py = p[1], pz = p[2], nx = nrm[0], ny = nrm[1], nz = nrm[2];
    wall->updateParticles(exec_space{}, [=](const int w) {
        xw(w, 0) = px;
        xw(w, 1) = py;
        xw(w, 2) = pz;
        nw_(w, 0) = nx;
        nw_(w, 1) = ny;
        nw_(w, 2) = nz;
        Ew(w) = E;
        Gw(w) = G;
        nuw(w) = nu;
    });
    return wall;
}

// "--cor_pw=0.4" -> 0.4: the text after '=' read with atof, as examples/03_normal_particle_wall_different_cor.cpp:37-40 and
// examples/04_oblique_particle_wall_different_angles.cpp:47-52
inline double option_value(const std::string &arg) {
    const auto parts = CabanaDEM::splitString(arg, '=');
    if (parts.size() < 2) throw CabanaDEM::Error("expected --name=value, got " + arg);
    return std::atof(parts[1].c_str());
}

// One sphere just above a wall through the origin with normal +y, thrown at it with velocity
// (ux, uy) (examples/02_elastic_normal_impact_of_particle_wall.cpp:84-180, and the same lines of
// examples 03 and 04): centre at y = r + r/1e6, neighbour
// cutoff 3 r, snapshots every output_frequency steps into `folder`.
inline void run_single_over_wall(const CabanaDEM::Inputs &inputs, const std::string &folder, double ux, double uy,
                                 double cor_pw) {
    auto force = std::make_shared<CabanaDEM::Force<exec_space>>(inputs["coefficient_of_restitution_pp"], cor_pw,
                                                                inputs["friction_pp"], inputs["friction_pw"]);
    auto particles = std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 1>>(exec_space(), 1, folder);
    set_material(*particles, inputs);
    const double r = inputs["particle_radius"];
    auto x = particles->slicePosition();
    auto u = particles->sliceVelocity();
    particles->updateParticles(exec_space{}, [=](const int pid) {
        x(pid, 0) = 0.;
        x(pid, 1) = r + r / 1000000.;
        x(pid, 2) = 0.;
        u(pid, 0) = ux;
        u(pid, 1) = uy;
        u(pid, 2) = 0.;
    });
    const double origin[3] = {0., 0., 0.}, up[3] = {0., 1., 0.};
    auto wall = make_walls(inputs, 1, origin, up);
    auto solver = CabanaDEM::createSolverDEM<memory_space>(inputs, particles, wall, force, 3. * r);
    solver->run();
}

}  // namespace examples
