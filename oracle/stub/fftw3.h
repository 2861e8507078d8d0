/*
 * Declaration-only stand-in for <fftw3.h>, used only to compile the
 * reference solver as a CPU oracle (test infrastructure, never shipped).
 *
 * The reference includes <fftw3.h> in its equation-set and waveform files
 * (geoac.eqset.*.cpp:9, waveforms.cpp:10) but calls FFTW only from the
 * weakly non-linear waveform mode, which is not on the ray-fan / eigenray
 * path.  FFTW is not installed in this image, so every function here aborts
 * if it is ever reached.  No FFTW code is contained or reproduced here.
 */
#ifndef IGA_ORACLE_FFTW3_STUB_H_
#define IGA_ORACLE_FFTW3_STUB_H_

#include <stdio.h>
#include <stdlib.h>

typedef double fftw_complex[2];
typedef struct iga_stub_fftw_plan_s* fftw_plan;

#define FFTW_MEASURE (0U)

static inline void iga_stub_fftw_abort(const char* fn) {
    fprintf(stderr, "oracle build: %s called, but FFTW is stubbed (waveform mode is off-path)\n", fn);
    abort();
}
static inline void* fftw_malloc(size_t) { iga_stub_fftw_abort("fftw_malloc"); return 0; }
static inline void fftw_free(void*) { iga_stub_fftw_abort("fftw_free"); }
static inline fftw_plan fftw_plan_dft_r2c_1d(int, double*, fftw_complex*, unsigned) { iga_stub_fftw_abort("fftw_plan_dft_r2c_1d"); return 0; }
static inline fftw_plan fftw_plan_dft_c2r_1d(int, fftw_complex*, double*, unsigned) { iga_stub_fftw_abort("fftw_plan_dft_c2r_1d"); return 0; }
static inline void fftw_execute(const fftw_plan) { iga_stub_fftw_abort("fftw_execute"); }
static inline void fftw_destroy_plan(fftw_plan) { iga_stub_fftw_abort("fftw_destroy_plan"); }

#endif
