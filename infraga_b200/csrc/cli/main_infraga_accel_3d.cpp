// bin/infraga-accel-3d: the name of the reference's MPI build of infraga-3d,
// as `mpirun -np N infraga-accel-3d ...` launches it; the GPU traces the whole
// job in the first process.
#include "cli_common.h"

int main(int argc, char** argv) { return cli::run(argc, argv, cli::Variant::k3D, true); }
