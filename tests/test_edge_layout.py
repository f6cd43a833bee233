"""Layout of the exact adjoint's edge-band coefficients (seis_b200/csrc/
fd_internal.h edge_cells / edge_index, decoded by edge_coef_kernel in
fd_adjoint.cuh): every cell of the four 5-cell edge bands of a padded grid,
as the pad tiles address it, maps to an index inside the array, the index of
band b's cell decodes back to that cell, and no two cells of one band share
an index.  Compiled on the host with g++ (the two functions are host and
device inline code)."""
import os
import shutil
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "seis_b200", "csrc")
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")

PROG = r"""
#include <cstdio>
#include <set>
#include "fd_internal.h"
using namespace seis;
// the decode of edge_coef_kernel: index -> (band, column, row)
static void decode(int NX, int NZ, int i, int &b, int &cx, int &cz) {
  if (i < 5 * NX) { b = 0; cx = i / 5; cz = i % 5; }
  else if (i < 10 * NX) { b = 1; cx = (i - 5 * NX) / 5; cz = NZ - 5 + (i - 5 * NX) % 5; }
  else if (i < 10 * NX + 5 * NZ) { b = 2; cx = (i - 10 * NX) / NZ; cz = (i - 10 * NX) % NZ; }
  else { b = 3; cx = NX - 5 + (i - 10 * NX - 5 * NZ) / NZ; cz = (i - 10 * NX - 5 * NZ) % NZ; }
}
int main() {
  const int sizes[][2] = {{5, 5}, {7, 9}, {96, 64}, {2135, 1080}, {40, 6}};
  for (auto &sz : sizes) {
    const int NX = sz[0], NZ = sz[1], n = edge_cells(NX, NZ);
    for (int b = 0; b < 4; b++) {
      // the cells the pad tiles read in band b (clipped to the grid)
      const int xa = b == 3 ? (NX - 5 > 0 ? NX - 5 : 0) : 0, xb = b == 2 ? (NX < 5 ? NX : 5) : NX;
      const int za = b == 1 ? (NZ - 5 > 0 ? NZ - 5 : 0) : 0, zb = b == 0 ? (NZ < 5 ? NZ : 5) : NZ;
      std::set<int> seen;
      for (int cx = xa; cx < xb; cx++)
        for (int cz = za; cz < zb; cz++) {
          const int i = edge_index(b, NX, NZ, cx, cz);
          int bb, x, z;
          if (i < 0 || i >= n) { std::printf("out %d %d %d %d %d\n", NX, NZ, b, cx, cz); return 1; }
          decode(NX, NZ, i, bb, x, z);
          if (bb != b || x != cx || z != cz) { std::printf("decode %d %d %d %d %d\n", NX, NZ, b, cx, cz); return 1; }
          if (!seen.insert(i).second) { std::printf("dup %d %d %d\n", NX, NZ, b); return 1; }
        }
    }
  }
  std::printf("ok\n");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(CUDA_INC),
                    reason="needs g++ and the CUDA headers")
def test_edge_band_indices_cover_and_decode():
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "t.cpp"), os.path.join(d, "t")
        open(src, "w").write(PROG)
        subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC, "-I", CUDA_INC, src, "-o", exe],
                       check=True, capture_output=True)
        r = subprocess.run([exe], capture_output=True, text=True)
        assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout
