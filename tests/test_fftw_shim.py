"""The FFTW-API shim that the reference's order-4 executor is built against
(``oracle/fftw_shim``): its 2-D transforms match numpy's to FP64 roundoff,
forward and backward, for power-of-two and other sizes, in and out of place.

The shim is compiled here with a small C driver into a temporary folder (gcc,
no GPU): the driver reads n0, n1, sign and the input from stdin, plans with
``fftw_plan_dft_2d`` and writes the unnormalised transform to stdout.
"""

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

SHIM = Path(__file__).resolve().parents[1] / "oracle" / "fftw_shim"

DRIVER = r"""
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"
int main(int argc, char** argv) {
  int n0, n1, sign, inplace, threads;
  if (fread(&n0, 4, 1, stdin) != 1 || fread(&n1, 4, 1, stdin) != 1 || fread(&sign, 4, 1, stdin) != 1 ||
      fread(&inplace, 4, 1, stdin) != 1 || fread(&threads, 4, 1, stdin) != 1) return 2;
  size_t z = (size_t)n0 * n1;
  fftw_complex* a = (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * z);
  fftw_complex* b = inplace ? a : (fftw_complex*)fftw_malloc(sizeof(fftw_complex) * z);
  if (fread(a, sizeof(fftw_complex), z, stdin) != z) return 3;
  if (!fftw_init_threads()) return 4;
  fftw_plan_with_nthreads(threads);
  fftw_plan p = fftw_plan_dft_2d(n0, n1, a, b, sign, FFTW_ESTIMATE);
  if (!p) return 5;
  fftw_execute(p);
  fwrite(b, sizeof(fftw_complex), z, stdout);
  fftw_destroy_plan(p);
  fftw_cleanup_threads();
  if (!inplace) fftw_free(b);
  fftw_free(a);
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not available")
    d = tmp_path_factory.mktemp("fftw_shim")
    (d / "driver.c").write_text(DRIVER)
    exe = d / "driver"
    subprocess.run(["gcc", "-O2", "-fopenmp", f"-I{SHIM}", str(d / "driver.c"),
                    str(SHIM / "fftw3_shim.c"), "-lm", "-o", str(exe)], check=True,
                   capture_output=True)
    return exe


def _run(exe, x, sign, inplace, threads):
    n0, n1 = x.shape
    head = np.array([n0, n1, sign, int(inplace), threads], dtype="<i4").tobytes()
    r = subprocess.run([str(exe)], input=head + np.ascontiguousarray(x, np.complex128).tobytes(),
                       capture_output=True, check=True)
    return np.frombuffer(r.stdout, dtype=np.complex128).reshape(n0, n1)


@pytest.mark.parametrize("n0,n1", [(32, 32), (64, 16), (24, 40), (30, 6), (1, 8)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_shim_matches_numpy(driver, n0, n1, sign):
    rng = np.random.default_rng(n0 * 100 + n1)
    x = rng.standard_normal((n0, n1)) + 1j * rng.standard_normal((n0, n1))
    want = np.fft.fft2(x) if sign == -1 else np.fft.ifft2(x) * (n0 * n1)
    for inplace, threads in ((False, 1), (True, 3)):
        got = _run(driver, x, sign, inplace, threads)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < 1e-14, (n0, n1, sign, inplace, err)
