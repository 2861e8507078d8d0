"""The FFT behind oracle/fftshim/fftw3.h (the stand-in that lets the
reference's waveform mode run as the -wnl_wvfrm oracle) against numpy's
real FFT: FFTW's r2c / c2r conventions (unnormalised, the c2r ignoring the
imaginary parts of the DC and Nyquist bins), power-of-two and other lengths."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from tests._cases import ROOT

SRC = r'''
#include <stdio.h>
#include "fftw3.h"
int main(void) {
    int n;
    if (scanf("%d", &n) != 1) return 1;
    double* x = (double*)fftw_malloc(sizeof(double) * n);
    fftw_complex* X = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * (n / 2 + 1));
    fftw_plan f = fftw_plan_dft_r2c_1d(n, x, X, FFTW_MEASURE);
    fftw_plan b = fftw_plan_dft_c2r_1d(n, X, x, FFTW_MEASURE);
    for (int i = 0; i < n; i++) scanf("%lf", &x[i]);
    fftw_execute(f);
    for (int k = 0; k <= n / 2; k++) printf("%.17g %.17g\n", X[k][0], X[k][1]);
    for (int k = 0; k <= n / 2; k++) scanf("%lf %lf", &X[k][0], &X[k][1]);
    fftw_execute(b);
    for (int i = 0; i < n; i++) printf("%.17g\n", x[i]);
    fftw_destroy_plan(f); fftw_destroy_plan(b);
    fftw_free(x); fftw_free(X);
    return 0;
}
'''


@pytest.fixture(scope="module")
def shim_bin():
    d = tempfile.mkdtemp()
    src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
    with open(src, "w") as f:
        f.write(SRC)
    subprocess.run(["gcc", "-O2", "-I", os.path.join(ROOT, "oracle", "fftshim"), src, "-o", exe, "-lm"], check=True)
    return exe


@pytest.mark.parametrize("n", [16, 12, 1000, 1024, 8192])
def test_shim_matches_numpy_rfft(shim_bin, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    Y = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)   # not Hermitian at DC / Nyquist
    inp = f"{n}\n" + "\n".join(f"{v:.17g}" for v in x) + "\n" + \
        "\n".join(f"{c.real:.17g} {c.imag:.17g}" for c in Y) + "\n"
    out = subprocess.run([shim_bin], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    m = n // 2 + 1
    X = np.array([complex(*map(float, ln.split())) for ln in out[:m]])
    y = np.array([float(v) for v in out[m:m + n]])
    ref_X = np.fft.rfft(x)
    tol = 1e-12 * np.max(np.abs(ref_X))
    assert np.max(np.abs(X - ref_X)) <= tol
    ref_y = np.fft.irfft(Y, n) * n
    assert np.max(np.abs(y - ref_y)) <= 1e-12 * np.max(np.abs(ref_y))
