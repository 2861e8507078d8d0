// bin/infraga-3d-rngdep: GPU drop-in for the reference binary of the same name.
#include "cli_common.h"

int main(int argc, char** argv) { return cli::run(argc, argv, cli::Variant::k3DRngdep); }
