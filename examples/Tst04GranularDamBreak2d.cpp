// Reference command line of examples/tst_04_granular_dam_break_2d.cpp (main, :271-293):
// Tst04GranularDamBreak2d <input.json> <output_folder> [--walls=box].
// Particles on the reference's zigzag lattice over a 1 x 1 square with spacing 2 r (create_points,
// :14-52: rows and columns int(1 / spacing), odd rows shifted by half a spacing).  The reference
// sets three box walls and then overwrites all of them in its wall functor (:189-248), so every
// wall sits at (0, -3 r, 0) with a zero normal; that is the state run by default, and
// --walls=box keeps the left wall, floor and right wall as first set.  The reference
// declares one wall-history slot per particle for its three walls (:120), which indexes past the
// slot; this library refuses that, so the particles carry three slots.
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "example_common.hpp"

using namespace examples;

int main(int argc, char *argv[]) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double r = inputs["particle_radius"];
    const double length = 1., height = 1., spacing = 2. * r;
    const int cols = static_cast<int>(length / spacing), rows = static_cast<int>(height / spacing);
    std::vector<std::pair<double, double>> pts;
    for (int i = 0; i < rows; ++i) {
        const double off = (i % 2 == 0) ? 0.0 : spacing / 2.0;
        for (int j = 0; j < cols; ++j) {
            const double px = j * spacing + off, py = i * spacing;
            if (px <= length && py <= height) pts.emplace_back(px, py);
        }
    }
    auto force = std::make_shared<CabanaDEM::Force<exec_space>>(
        inputs["coefficient_of_restitution_pp"], inputs["coefficient_of_restitution_pw"], inputs["friction_pp"],
        inputs["friction_pw"]);
    auto particles =
        std::make_shared<CabanaDEM::Particles<memory_space, 3, 6, 3>>(exec_space(), pts.size(), argv[2]);
    set_material(*particles, inputs);
    auto x = particles->slicePosition();
    particles->updateParticles(exec_space{}, [&](const int pid) {
        x(pid, 0) = pts[pid].first;
        x(pid, 1) = pts[pid].second;
        x(pid, 2) = 0.;
    });
    const double p[3] = {0., -3. * r, 0.}, zero[3] = {0., 0., 0.};
    auto wall = make_walls(inputs, 3, p, zero);
    if (argc > 3 && std::string(argv[3]) == "--walls=box") {
        auto xw = wall->slicePosition();
        auto nw = wall->sliceNormal();
        const double bx[3][3] = {{-2. * r, 0.5, 0.}, {0.8, 0., 0.}, {1.4, 0.5, 0.}};
        const double bn[3][3] = {{1., 0., 0.}, {0., 1., 0.}, {-1., 0., 0.}};
        wall->updateParticles(exec_space{}, [&](const int w) {
            for (int d = 0; d < 3; ++d) {
                xw(w, d) = bx[w][d];
                nw(w, d) = bn[w][d];
            }
        });
    }
    CabanaDEM::createSolverDEM<memory_space>(inputs, particles, wall, force, 3. * r)->run();
    return 0;
}
