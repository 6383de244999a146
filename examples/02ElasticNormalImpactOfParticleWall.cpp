// Reference command line of examples/02_elastic_normal_impact_of_particle_wall.cpp (main,
// :184-208): 02ElasticNormalImpactOfParticleWall <input.json> <output_folder>.  One sphere
// dropped normally onto a wall at velocity_p (:99-180); particles_<k>.csv snapshots every
// output_frequency steps.
#include <cstdio>

#include "example_common.hpp"

int main(int argc, char *argv[]) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double v = inputs["velocity_p"];
    examples::run_single_over_wall(inputs, argv[2], 0.0, -v, inputs["coefficient_of_restitution_pw"]);
    return 0;
}
