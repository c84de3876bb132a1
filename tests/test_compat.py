"""The C++ compat header compiles against the C ABI library (CPU) and runs a
reference-style driver on the GPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = r"""
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include "afmm2d_compat.hpp"
int main() {
  const int N = 4096;
  std::vector<double> loc(2 * N), b(N);
  srand(3);
  for (int j = 0; j < N; ++j) {  // column-major N x 2, as Eigen::MatrixXd loc(N, 2)
    loc[j] = 2.0 * rand() / RAND_MAX - 1.0;
    loc[N + j] = 2.0 * rand() / RAND_MAX - 1.0;
    b[j] = 2.0 * rand() / RAND_MAX - 1.0;
  }
  AFMM* afmm = new AFMM(N, 32, 8, loc.data(), AFMM_KERNEL_LOG);
  afmm->assemble();
  std::vector<double> y = afmm->computeMatVecProduct(b);
  double e = afmm->evaluateError(0, 1);
  std::printf("nLevels %u first %.17g err %.3e\n", afmm->nLevels, y[0], e);
  afmm->save("afmm_setup.bin");
  AFMM* again = AFMM::load("afmm_setup.bin");
  std::vector<double> y2 = again->computeMatVecProduct(b);
  bool same = again->N == N && again->nLevels == afmm->nLevels;
  for (int j = 0; j < N; ++j) same = same && y2[j] == y[j];
  std::printf("reload identical: %d\n", (int)same);
  again->autotune();
  std::vector<double> y3 = again->computeMatVecProduct(b);
  for (int j = 0; j < N; ++j) same = same && y3[j] == y[j];
  std::printf("tuned identical: %d\n", (int)same);
  delete again;
  delete afmm;
  try {
    AFMM bad(100, 64, 8, loc.data());
  } catch (const afmm2d::Error& err) {
    std::printf("rejected: %d\n", (int)err.status);
  }
  return e < 1e-5 ? 0 : 1;
}
"""


def build_driver(tmp_path):
    src = tmp_path / "driver.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "driver"
    lib = os.path.join(ROOT, "afmm2d_b200")
    subprocess.run(["g++", "-std=c++17", "-O1", "-DAFMM2D_COMPAT_NO_EIGEN", "-I", os.path.join(ROOT, "include"),
                    str(src), "-L", lib, "-lafmm2d", f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    return exe


def test_compat_header_builds(tmp_path):
    assert build_driver(tmp_path).exists()


@pytest.mark.gpu
def test_compat_driver_runs(tmp_path):
    out = subprocess.run([str(build_driver(tmp_path))], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "nLevels 3" in out.stdout and "rejected: 1" in out.stdout
    assert "reload identical: 1" in out.stdout and "tuned identical: 1" in out.stdout
