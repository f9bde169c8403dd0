"""The register-window band sweeps (band_solve_window, used by the rotation
channels' drift) against the memory-chained dgbtrs-order sweeps
(band_solve_strided) they replace: both helpers compiled for the host from
fastearth3d_b200/csrc/vg_device.cuh and run on seeded random band records
(kl = 6, kv = 12, the degree-2 operator's bandwidths; interchange offsets
anywhere in 0 .. kl; sizes from 1 to past the configuration-2 operator's 403
dofs, including the sizes where the windows run off either end). The
solutions must agree bit for bit: the window only changes where the operands
live, not an operation or its order."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

PROGRAM = r"""
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>
#include "vg_device.cuh"

int main() {
  const int KL = 6, KV = 12, LDAB = 21;
  std::mt19937_64 rng(2024);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  const int sizes[] = {1, 2, 3, 7, 8, 12, 13, 14, 19, 20, 64, 403, 611};
  int bad = 0, cases = 0;
  for (int n : sizes) {
    for (int rep = 0; rep < 20; ++rep) {
      std::vector<double> ab((size_t)LDAB * n), x1(n), x2(n);
      std::vector<int> ipiv(n);
      for (double& v : ab) v = u(rng);
      for (int k = 0; k < n; ++k) {
        ab[(size_t)k * LDAB + KV] = (u(rng) < 0.0 ? -1.0 : 1.0) * (0.5 + std::fabs(u(rng)));
        const int room = std::min(KL, n - 1 - k);
        ipiv[k] = k + (int)(rng() % (unsigned long long)(room + 1));
        x1[k] = x2[k] = 1e3 * u(rng);
      }
      vg::band_solve_strided(ab.data(), LDAB, n, KL, KV, ipiv.data(), x1.data(), 1);
      vg::band_solve_window<6, 12>(ab.data(), LDAB, n, ipiv.data(), x2.data());
      ++cases;
      if (std::memcmp(x1.data(), x2.data(), sizeof(double) * n) != 0) {
        ++bad;
        std::printf("n %d rep %d differs\n", n, rep);
      }
    }
  }
  std::printf("%d cases, %d differ\n", cases, bad);
  return bad ? 1 : 0;
}
"""


def test_window_sweeps_equal_dgbtrs_order(tmp_path):
    if not os.path.exists(NVCC) and shutil.which("nvcc") is None:
        pytest.skip("nvcc not available")
    nvcc = NVCC if os.path.exists(NVCC) else shutil.which("nvcc")
    src = tmp_path / "band_window.cu"
    src.write_text(PROGRAM)
    exe = tmp_path / "band_window"
    cmd = [nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "fastearth3d_b200", "csrc"), str(src), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    print(run.stdout)
    assert run.returncode == 0, run.stdout
    assert "260 cases, 0 differ" in run.stdout
