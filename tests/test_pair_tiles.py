"""The launch shape of the paired FP64 pressure pass (csrc/fdm.cuh: pair_grid, pair_per), on the CPU.

A CTA of a paired launch takes `per` consecutive tiles (z-planes of a column or row block, or plane-column
blocks): one for a single cavity, up to 8 in a large batch.  A small host program built with nvcc from the
library's own header evaluates the rule; no GPU is needed (without one the SM count falls back to 148).  Checked:
the documented choices, and that every grid covers each tile of its axis exactly once with at most 8 per CTA.
"""
import os
import subprocess

import pytest

from les_impulse3d_64_b200 import _build

HARNESS = r'''
#include <cstdio>
#include <cstdlib>
#include "fdm.cuh"
using namespace cavity;
int main(int argc, char** argv) {
    if (argc != 7) return 2;
    const int ph = atoi(argv[1]), w = atoi(argv[2]), nx = atoi(argv[3]), ny = atoi(argv[4]), nz = atoi(argv[5]);
    g_launch_batch = atoi(argv[6]);
    const int per = pair_per(ph, w, nx, ny, nz);
    const dim3 g = pair_grid(ph, w, nx, ny, nz, per);
    printf("%d %u %u\n", per, g.x, g.y);
    return 0;
}
'''
XY, Z, YX = 0, 1, 2


@pytest.fixture(scope='module')
def rule(tmp_path_factory):
    nvcc = _build.nvcc()
    if not os.path.exists(nvcc):
        pytest.skip('nvcc not found')
    d = tmp_path_factory.mktemp('pair_rule')
    (d / 'rule.cu').write_text(HARNESS)
    subprocess.run([nvcc, *_build.ARCH, '-std=c++17', f'-I{_build.ROOT / "include"}', f'-I{_build.CSRC}',
                    str(d / 'rule.cu'), '-o', str(d / 'rule')], check=True, capture_output=True)

    def run(phase, w, nx, ny, nz, batch, forced=None):
        env = {k: v for k, v in os.environ.items() if k != 'CAVITY_PAIR_PER'}
        if forced is not None:
            env['CAVITY_PAIR_PER'] = str(forced)
        out = subprocess.run([str(d / 'rule'), *map(str, (phase, w, nx, ny, nz, batch))], env=env, check=True,
                             capture_output=True, text=True).stdout.split()
        return tuple(int(v) for v in out)
    return run


def tiles_along(phase, w, nx, ny, nz):
    return (nx * ny + w - 1) // w if phase == Z else nz


def test_single_cavity_takes_one_tile_per_cta(rule):
    for phase in (XY, Z, YX):
        for w, dims in ((16, (64, 64, 64)), (32, (64, 64, 64)), (32, (40, 40, 33)), (16, (7, 9, 11))):
            per, gx, gy = rule(phase, w, *dims, 1)
            assert per == 1, (phase, w, dims)
            nx, ny, nz = dims
            if phase == Z:
                assert (gx, gy) == ((nx * ny + w - 1) // w, 1)
            else:
                assert (gx, gy) == (((nx if phase == XY else ny) + w - 1) // w, nz)


def test_batch_of_64_cavities_of_64_cube_takes_eight(rule):
    """The measured best for 64 cavities of 64^3 (first passes 2.15 ms per step against 2.51 with one tile)."""
    assert rule(XY, 32, 64, 64, 64, 64) == (8, 2, 8)
    assert rule(YX, 32, 64, 64, 64, 64) == (8, 2, 8)
    assert rule(Z, 32, 64, 64, 64, 64) == (8, 16, 1)


@pytest.mark.parametrize('dims, batch', [((64, 64, 64), 256), ((24, 24, 24), 256), ((48, 48, 48), 256),
                                         ((40, 40, 33), 48), ((16, 24, 40), 128), ((64, 48, 7), 96)])
def test_every_tile_once_and_at_most_eight_per_cta(rule, dims, batch):
    for phase in (XY, Z, YX):
        per, gx, gy = rule(phase, 32, *dims, batch)
        n = tiles_along(phase, 32, *dims)
        ctas = gx if phase == Z else gy
        assert 1 <= per <= 8
        assert (ctas - 1) * per < n <= ctas * per, (phase, per, ctas, n)
        # evened out: the last CTA of the axis takes at least as many tiles as the others' shortfall allows
        assert n - (ctas - 1) * per > per - ctas or ctas == 1


def test_forced_tiles_per_cta(rule):
    """CAVITY_PAIR_PER forces the count, capped by the tiles of the axis (the tests' bit-for-bit comparisons)."""
    assert rule(XY, 16, 64, 64, 64, 1, forced=3) == (3, 4, 22)
    assert rule(Z, 16, 7, 9, 11, 1, forced=64)[0] == 4          # 63 plane columns: 4 blocks of 16
    assert rule(YX, 32, 40, 40, 33, 1, forced=64) == (33, 2, 1)
