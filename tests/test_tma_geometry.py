"""Host-side check of the TMA-staged stencils' tile geometry
(maccpic_b200/csrc/tma_stencil.cuh), run before any GPU sees it.

The field block's rows are (nx+3) elements long, which a tensor map cannot
stride over (its row stride must be a multiple of 16 bytes), so the map's
rows are M = 16/sizeof(T) field rows each and a tile is assembled from M
boxes.  This restates the kernel's box coordinates and shared-memory
lookups in numpy, fills each box the way a tiled tensor copy does (elements
outside the map read as zero), and checks, for every tile of several grids
(every residue of nx+3 mod 4) and every staged array:

* every box starts on a 16-byte column and inside the map's rows;
* the map lies inside the allocation (13 arrays plus the tail of M rows);
* every element a cell's stencil reads (the cell and its 8 neighbours) is
  found in its box, at the field value of that position.
"""
import numpy as np
import pytest


def geo(elem):
    M = 16 // elem
    TXO = 64 if elem == 4 else 32
    TYO = 16
    HR = TYO + 2
    BH = (HR + M - 1) // M
    BW = (TXO + 2 + M - 1 + M - 1) // M * M
    return dict(M=M, TXO=TXO, TYO=TYO, BH=BH, BW=BW)


def check_grid(nx, ny, elem, nfield=13):
    G = geo(elem)
    M, TXO, TYO, BH, BW = G["M"], G["TXO"], G["TYO"], G["BH"], G["BW"]
    nxg = nx + 3
    w = nxg * (ny + 3)
    tail = M * nxg
    alloc = nfield * w + tail
    block = np.arange(alloc, dtype=np.int64) + 1  # unique non-zero values
    dim0 = M * nxg
    dim1 = (nfield * (ny + 3) + M - 1) // M
    assert dim1 * dim0 <= alloc, "the map reaches past the allocation"
    assert (dim0 * elem) % 16 == 0 and (BW * elem) % 16 == 0
    lines = np.zeros((dim1 + BH, dim0 + BW), dtype=np.int64)  # zero = out of the map
    lines[:dim1, :dim0] = block[: dim1 * dim0].reshape(dim1, dim0)
    ntx = (nx + 1 + TXO - 1) // TXO
    nty = (ny + 1 + TYO - 1) // TYO
    arrays = list(range(nfield))
    for t in range(ntx * nty):
        ix0 = 1 + (t % ntx) * TXO
        iy0 = 1 + (t // ntx) * TYO
        assert (ix0 - 1) % M == 0
        for k in arrays:
            row0 = k * (ny + 3)
            boxes = []
            for j in range(M):  # issue_tile
                R = row0 + iy0 - 1 + j
                line, r = R // M, R % M
                x = r * nxg + ix0 - 1
                x -= x % M
                assert x >= 0 and (x * elem) % 16 == 0
                assert 0 <= line < dim1
                boxes.append(lines[line:line + BH, x:x + BW])
            rb = (row0 + iy0 - 1) % M
            ix = np.arange(ix0, min(ix0 + TXO, nx + 2))  # cells <= nx+1
            iy = np.arange(iy0, min(iy0 + TYO, ny + 2))
            for ddy in (-1, 0, 1):
                for ddx in (-1, 0, 1):
                    dy = (iy - iy0 + 1) + ddy  # staged_row
                    dx = (ix - ix0 + 1) + ddx
                    assert dy.min() >= 0 and dy.max() <= TYO + 1
                    j = dy % M
                    tr = dy // M
                    r = (rb + j) % M
                    sh = (r * nxg) % M
                    assert tr.max() < BH
                    assert (sh.max() + dx.max()) < BW and dx.min() + sh.min() >= 0
                    got = np.stack([boxes[jj][trr, shh + dx] for jj, trr, shh in zip(j, tr, sh)])
                    want = block[k * w + (iy[:, None] + ddy) * nxg + (ix[None, :] + ddx)]
                    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("elem", [4, 8])
@pytest.mark.parametrize("nx,ny", [(4, 4), (5, 7), (6, 9), (7, 16), (64, 32), (65, 33),
                                   (126, 17), (128, 64), (200, 47), (257, 95), (300, 61)])
def test_tiles_read_what_the_stencils_need(nx, ny, elem):
    check_grid(nx, ny, elem)


def test_scratch_map_of_one_array():
    for elem in (4, 8):
        check_grid(61, 29, elem, nfield=1)
