// bin/infraga-accel-sph: the name of the reference's MPI build of infraga-sph,
// as `mpirun -np N infraga-accel-sph ...` launches it; the GPU traces the whole
// job in the first process.
#include "cli_common.h"

int main(int argc, char** argv) { return cli::run(argc, argv, cli::Variant::kSph, true); }
