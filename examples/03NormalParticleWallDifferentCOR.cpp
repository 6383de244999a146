// Reference command line of examples/03_normal_particle_wall_different_cor.cpp (main,
// :192-216): 03NormalParticleWallDifferentCOR <input.json> <output_folder> --cor_pw=<e>.
// As example 02 with the particle-wall restitution coefficient taken from the third argument
// (:37-57); the input file carries no coefficient_of_restitution_pw.
#include <cstdio>

#include "example_common.hpp"

int main(int argc, char *argv[]) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s input_file_name output_folder --cor_pw=<value>\n", argv[0]);
        return 1;
    }
    CabanaDEM::Inputs inputs(argv[1]);
    const double cor_pw = examples::option_value(argv[3]);
    const double v = inputs["velocity_p"];
    examples::run_single_over_wall(inputs, argv[2], 0.0, -v, cor_pw);
    return 0;
}
