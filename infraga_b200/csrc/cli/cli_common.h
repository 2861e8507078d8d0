// Drop-in command-line front ends (bin/infraga-3d, infraga-sph,
// infraga-3d-rngdep, infraga-sph-rngdep) over libinfraga_gpu.so.
//
// They keep the reference binaries' argv grammar (src/main.infraga.*.cpp:
// option prefix matching in main(), a first pass over key=value tokens for
// the atmosphere options, set_region, then the full pass), their defaults,
// console messages and unknown-key prompt, and write the same output files
// ({id}.arrivals.dat, {id}.raypaths.dat, {id}.caustics-N.dat,
// {id}.terrain.dat, {id}.eigenray-N.dat) with the same header text, column
// order and stream precision.  The rays themselves are traced on the GPU by
// the library, all rays of a run at once.
#pragma once

namespace cli {

enum class Variant { k3D, kSph, k3DRngdep, kSphRngdep };

// main() of one binary: option dispatch as in the reference mains.  accel:
// the infraga-accel-* names the reference gives its MPI builds
// (src/main.infraga.*.mpi.cpp), which run_infraga.py launches as
// `mpirun -np N infraga-accel-* ...` for --cpu-cnt N >= 2.  The GPU traces the
// whole job in the first process; the other processes of such a launch exit
// at once.
int run(int argc, char** argv, Variant v, bool accel = false);

}  // namespace cli
