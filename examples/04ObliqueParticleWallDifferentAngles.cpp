// Reference command line of examples/04_oblique_particle_wall_different_angles.cpp (main,
// :211-235): 04ObliqueParticleWallDifferentAngles <input.json> <output_folder> --angle=<deg>.
// The sphere hits the wall at the incident angle from the wall normal:
// u = (v sin a, -v cos a, 0) (:113-116); the rebound spin omega_z of the last snapshot is what
// the reference's comparison plots against the incident angle.
#include <cmath>
#include <cstdio>

#include "example_common.hpp"

int main(int argc, char *argv[]) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder --angle=<degrees>\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double incident_angle = examples::option_value(argv[3]);
    const double angle = incident_angle / 180. * M_PI;
    const double v = inputs["velocity_p"];
    examples::run_single_over_wall(inputs, argv[2], v * sin(angle), -v * cos(angle),
                                   inputs["coefficient_of_restitution_pw"]);
    return 0;
}
