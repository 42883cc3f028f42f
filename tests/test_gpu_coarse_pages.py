"""Coarse pages (regions whose header carries a stride of 2 or 4, solid or
air in aligned blocks of it): the far tier's block-area measure and the
presentation's block corners read the stride (voxel_stride). GPU against
the oracle word for word on the terrain with every third region coarse."""
import numpy as np
import pytest

import oracle_lib as O
import vgi
from test_gpu_far import clear_view, far_pair, unit
from test_gpu_parity import assert_words_equal, terrain_case
from test_gpu_reconstruction import reconstruct_pair

pytestmark = pytest.mark.gpu


def coarse_terrain(**kw):
    case = terrain_case(**kw)
    n = len(case.coords)
    strides = np.zeros(n, np.uint8)
    strides[0::3] = 1
    strides[1::6] = 2
    vox = case.vox.copy()
    for r in np.nonzero(strides)[0]:
        s = 1 << int(strides[r])
        page = vox[r * 4096:(r + 1) * 4096].reshape(16, 16, 16)  # z, y, x
        corner = page[::s, ::s, ::s]
        page[:] = np.repeat(np.repeat(np.repeat(corner, s, 0), s, 1), s, 2)
    coarse = terrain_case(**kw)
    coarse.vox = vox
    coarse.emitters, coarse.n_emit, coarse.total = vgi.host_emitters(coarse.coords, vox, coarse.materials)
    coarse.faces = vgi.exposed_faces(coarse.coords, vox)[::3].copy()
    coarse.strides = strides
    return coarse


@pytest.mark.parametrize("measure,threshold", [(2, 40.0), (1, 16.0)])
def test_far_tier_reads_block_strides_like_the_oracle(gpu, measure, threshold):
    case = coarse_terrain(bounces=2)
    case.load(gpu, with_faces=False)
    clear_view(gpu)
    f = unit((0.2, -1.0, 0.3))
    cams = [((48.5 + 1.5 * k, 80.25, 47.75 - k), f, (0.0, 0.0, 1.0), 0.45, 80, 64) for k in range(5)]
    stats = far_pair(gpu, case, cams, vgi.FarTierSettings(voxel_pixels=threshold, measure=measure, cell=2, rate=3, steps=96))
    assert stats[0] > 500 and stats[3] > 0


def test_presentation_of_coarse_pages_matches_oracle(gpu):
    case = coarse_terrain(bounces=2)
    cam = ((48.5, 80.25, 47.75), unit((0.2, -1.0, 0.3)), (0.0, 0.0, 1.0), 0.45, 96, 72)
    case.load(gpu, with_faces=False)
    pixels, faces = gpu.discover_faces(*cam)
    gpu.view_set_receivers(faces)
    for k in range(2):
        gpu.view_frame(clock_ms=10 * k)
    gx, gy = 24, 18
    tiles = vgi.witness_tiles(pixels, faces, gx, gy)
    gpu.view_set_tiles(tiles, 12, 9)
    _, published = reconstruct_pair(gpu, case, tiles, 12, 9, (0.031, 1.0, 1.0))
    geometry = gpu.geometry()
    params = case.params_fn(geometry)(1, 1)
    image = gpu.view_present(*cam, corners=True)
    want = O.present(geometry, params, published, *cam, corners=True)
    assert_words_equal(image.view(np.uint32), want.view(np.uint32), "presented image over coarse pages")
    clear_view(gpu)
