"""Host logic of the step kernels' tile grids (TileGrid in
ouc_b200/csrc/ouc_internal.h), compiled and run on the CPU: for many grid
sizes and absorbing widths,
* the full-step tiles cover the padded grid and the reconstruction's tiles,
  which start at (L, L rounded down to 4), cover the interior
  [L, X-L) x [L, Z-L);
* every tile's U box (the tensor-copy box: rows x0-SHX-N .. x0+TX+SHX+N,
  columns z0-HU .. z0+TZ+HU, for N = 2, 5, 6) lies inside the field
  allocation (Xc rows and Zc columns plus 16 guard rows and columns on each
  side), and the box's first column is a multiple of 4 (16-byte rule of the
  tensor copies)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cstdio>
#include "ouc_internal.h"
using namespace ouc;
int main() {
    int bad = 0, checked = 0;
    for (int X = 40; X < 700; X += 7)
        for (int Z = 40; Z < 400; Z += 11)
            for (int L : {4, 10, 12, 20, 30, 31, 33, 40}) {
                if (X <= 2 * L + 8 || Z <= 2 * L + 8) continue;
                const TileGrid g = tile_grid(X, Z, L);
                if (g.tiles_x * 32 < X || g.tiles_z * 64 < Z) ++bad;
                if (g.rec_x0 > L || g.rec_x0 + 32 * g.rec_tiles_x < X - L) ++bad;
                if (g.rec_z0 > L || g.rec_z0 % 4 || g.rec_z0 + 64 * g.rec_tiles_z < Z - L) ++bad;
                if (g.rec_tiles_x != rec_tiles_for(X, L)) ++bad;
                for (int N : {2, 5, 6}) {
                    const int SHX = (N + 1) & ~1, HS = (N + 3) & ~3, HU = (HS + N + 3) & ~3;
                    auto box_ok = [&](int x0, int z0) {
                        return x0 - SHX - N >= -kGX && x0 + 32 + SHX + N <= g.Xc + kGX && z0 - HU >= -kZOFF &&
                               z0 + 64 + HU <= g.Zc + kZOFF && (z0 - HU + kZOFF) % 4 == 0;
                    };
                    for (int tx = 0; tx < g.tiles_x; ++tx)
                        for (int tz = 0; tz < g.tiles_z; ++tz) bad += !box_ok(32 * tx, 64 * tz);
                    for (int tx = 0; tx < g.rec_tiles_x; ++tx)
                        for (int tz = 0; tz < g.rec_tiles_z; ++tz)
                            bad += !box_ok(g.rec_x0 + 32 * tx, g.rec_z0 + 64 * tz);
                    ++checked;
                }
            }
    std::printf("%d %d\n", checked, bad);
    return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_tile_grids_cover_and_stay_inside(tmp_path):
    src = tmp_path / "tg.cpp"
    src.write_text(SRC)
    exe = tmp_path / "tg"
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "ouc_b200", "csrc"), "-I", cuda_inc,
                    str(src), "-o", str(exe)], check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    checked, bad = map(int, r.stdout.split())
    assert checked > 1000 and bad == 0 and r.returncode == 0, r.stdout
