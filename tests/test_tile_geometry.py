"""The shared-memory tiles of the momentum sweeps (csrc/sweep_tile.cuh: TileGeom), on the CPU.

A small host program built with nvcc from the library's headers prints each tile's row pitches and dynamic
shared memory.  The packed FP32 kernel's warps read two box rows at once, each half warp every other word of its
row, so all its row pitches must be odd (with an even pitch both halves share 16 banks and each load takes two
wavefronts); the one-cell kernels keep the boxes' own widths.  Two CTAs of each kernel must fit on an SM, which
is why the FP64 tile is not padded: with odd pitches its two CTAs would need more than the SM's 228 KB.
"""
import os
import subprocess

import pytest

from les_impulse3d_64_b200 import _build

HARNESS = r'''
#include <cstdio>
#include "sweep_pair.cuh"
using namespace cavity;
template <class G, class T> void show(const char* name) {
    printf("%s %d %d %d %d %zu\n", name, G::UW, G::VW, G::WW, G::MW, G::template smem_bytes<T>());
}
int main() {
    show<TileGeom<4, 4, 256>, double>("fp64_tile");
    show<TileGeom<8, 4, 512>, float>("fp32_tile");
    show<TileGeom<8, 4, 256, true>, float>("fp32_pair");
    show<TileGeom<4, 4, 256, true>, double>("fp64_tile_odd");
    return 0;
}
'''
SM_SHARED = 228 * 1024          # shared memory of an sm_100 SM
CTA_RESERVED = 1024             # reserved by the system per resident CTA
# static shared memory of the kernels besides the tile (the box row offsets, a batch's argument record), as
# ptxas reports it: 2048 bytes for the FP64 tile kernel, 3072 for the packed one
STATIC = {'fp64_tile': 2048, 'fp64_tile_odd': 2048, 'fp32_pair': 3072}


@pytest.fixture(scope='module')
def tiles(tmp_path_factory):
    nvcc = _build.nvcc()
    if not os.path.exists(nvcc):
        pytest.skip('nvcc not found')
    d = tmp_path_factory.mktemp('tile_geometry')
    (d / 'geometry.cu').write_text(HARNESS)
    subprocess.run([nvcc, *_build.ARCH, '-std=c++17', f'-I{_build.ROOT / "include"}', f'-I{_build.CSRC}',
                    str(d / 'geometry.cu'), '-o', str(d / 'geometry')], check=True, capture_output=True)
    out = subprocess.run([str(d / 'geometry')], check=True, capture_output=True, text=True).stdout
    return {f[0]: tuple(int(v) for v in f[1:]) for f in (line.split() for line in out.splitlines())}


def test_packed_kernel_pitches_are_odd(tiles):
    assert all(p % 2 == 1 for p in tiles['fp32_pair'][:4])


def test_one_cell_kernels_keep_the_box_widths(tiles):
    # u box 32 + 3 x-faces, v and w boxes 32 + 6 cells, impulse boxes 32 + 2
    assert tiles['fp64_tile'][:4] == (35, 38, 38, 34)
    assert tiles['fp32_tile'][:4] == (35, 38, 38, 34)


def test_two_ctas_per_sm(tiles):
    def two_fit(name):
        return 2 * (tiles[name][4] + STATIC[name] + CTA_RESERVED) <= SM_SHARED
    assert two_fit('fp64_tile')
    assert two_fit('fp32_pair')
    assert not two_fit('fp64_tile_odd')
