# SPDX-License-Identifier: GPL-3.0-or-later
"""The decomposition's patches (cw_decomp_patch, no device needed): CPPWRF's rule tile::set_domain
(src/core/tiles.hpp:70-74) -- patch t = tx + px ty owns [tx nx / px, (tx + 1) nx / px) x [ty ny / py, (ty + 1) ny / py)
-- so the patches cover the domain's mass points once each; and the refusals (a periodic direction split, a split
along y of a 2-D domain, patches under 6 points)."""
import ctypes as C

import numpy as np
import pytest

from cppwrf_b200 import capi


def patch(g, px, py, t):
    box = (C.c_int * 4)()
    assert capi.load().cw_decomp_patch(C.byref(g), px, py, t, box) == 0
    return tuple(box)


@pytest.mark.parametrize("nx,ny,px,py", [(119, 89, 3, 2), (40, 34, 2, 2), (64, 60, 5, 7), (37, 1, 3, 1)])
def test_patches_cover_the_domain_once(nx, ny, px, py):
    g = capi.grid(nx, ny, 10, 1000.0, 5.0, 5000.0, bc_x=capi.SPECIFIED, bc_y=capi.SPECIFIED if ny > 1 else capi.PERIODIC)
    owner = np.full((ny, nx), -1)
    for t in range(px * py):
        i0, i1, j0, j1 = patch(g, px, py, t)
        assert i1 - i0 >= 6 and (ny == 1 or j1 - j0 >= 6)
        assert np.all(owner[j0:j1, i0:i1] == -1)
        owner[j0:j1, i0:i1] = t
        tx, ty = t % px, t // px
        assert (i0, i1) == (tx * nx // px, (tx + 1) * nx // px)
        assert (j0, j1) == (ty * ny // py, (ty + 1) * ny // py)
    assert np.all(owner >= 0)


def test_refused_decompositions():
    lib = capi.load()
    box = (C.c_int * 4)()
    g = capi.grid(40, 30, 10, 1000.0, 5.0, 5000.0, bc_x=capi.PERIODIC, bc_y=capi.SYMMETRIC)
    assert lib.cw_decomp_patch(C.byref(g), 2, 1, 0, box) != 0  # a periodic direction is not split
    assert lib.cw_decomp_patch(C.byref(g), 1, 2, 1, box) == 0 and list(box) == [0, 40, 15, 30]
    assert lib.cw_decomp_patch(C.byref(g), 1, 6, 0, box) != 0  # patches under 6 points
    g2 = capi.grid(64, 1, 10, 100.0, 1.0, 1000.0, bc_x=capi.SYMMETRIC)
    assert lib.cw_decomp_patch(C.byref(g2), 1, 2, 0, box) != 0  # a 2-D domain splits along x only
    assert lib.cw_decomp_patch(C.byref(g2), 4, 1, 3, box) == 0 and list(box) == [48, 64, 0, 1]
