"""CPU check of the device storage order: the product's own index arithmetic (ewg_internal.cuh,
compiled for the host with nvcc) is a bijection, keeps colours split, and its neighbour lookup
agrees with the natural-order grid for 2D and 3D grids with even nx."""
import os
import subprocess

import pytest

from conftest import ROOT

SRC = r'''
#include <cstdio>
#include <vector>
#include "ewg_internal.cuh"
using namespace ewg;
int check(int dim, int nx, int ny, int nz) {
    Phys P{}; P.dim = dim; P.nx = nx; P.ny = ny; P.nz = dim == 3 ? nz : 1;
    set_index_constants(P);
    std::vector<int> seen(P.N, 0);
    int bad = 0;
    for (int col = 0; col < 2; ++col)
        for (int64_t h = 0; h < P.Nh; ++h) {
            CellIdx c = cell_of(P, col, h);
            if (c.c < 0 || c.c >= P.N) { ++bad; continue; }
            seen[c.c]++;
            if (((c.i + c.j + c.k) & 1) != col) ++bad;
            if (split_of(P, c.c) != col * P.Nh + h) ++bad;
            const int n[3] = {nx, ny, P.nz};
            const int id[3] = {c.i, c.j, c.k};
            const int64_t stride[3] = {1, nx, (int64_t)nx * ny};
            for (int a = 0; a < dim; ++a)
                for (int s = 0; s < 2; ++s) {
                    int64_t q = neighbour_split(P, col, h, c, a, s);
                    bool has = s == 0 ? id[a] > 0 : id[a] < n[a] - 1;
                    if (!has) { if (q != -1) ++bad; continue; }
                    int64_t nb = c.c + (s ? stride[a] : -stride[a]);
                    if (q != split_of(P, nb)) ++bad;
                    if (opposite_band(opposite_band(band_of(a, s))) != band_of(a, s)) ++bad;
                    if (opposite_band(band_of(a, s)) != band_of(a, 1 - s)) ++bad;
                }
        }
    for (int64_t c = 0; c < P.N; ++c) if (seen[c] != 1) ++bad;
    return bad;
}
int main() {
    int bad = 0;
    bad += check(2, 48, 32, 1); bad += check(2, 2, 1, 1); bad += check(2, 6, 5, 1);
    bad += check(3, 4, 3, 3); bad += check(3, 8, 6, 4); bad += check(3, 2, 1, 5); bad += check(3, 16, 7, 9);
    bad += check(3, 34, 18, 6); bad += check(3, 256, 12, 3); bad += check(3, 98, 97, 5);
    // the division by invariant integers used by cell_of, against plain division
    for (uint32_t d = 1; d < 3000; ++d) {
        FastDiv f = make_fastdiv(d);
        for (uint32_t n = 0; n < 20000; n += 7) if (fastdiv(f, n) != n / d) ++bad;
        for (uint32_t n = 0x7fffffffu; n > 0x7fff0000u; n -= 977) if (fastdiv(f, n) != n / d) ++bad;
    }
    printf("%d\n", bad);
    return bad != 0;
}
'''


def test_split_order_index_arithmetic(tmp_path):
    src = tmp_path / "layout.cu"
    src.write_text(SRC)
    exe = tmp_path / "layout"
    subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-I",
                           os.path.join(ROOT, "ewoms-numerics_b200", "csrc"), str(src), "-o", str(exe)])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "0"
