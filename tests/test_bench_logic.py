"""bench.py's algorithmic bytes per launch (the roofline numerator) against a
cell-by-cell count of the compulsory traffic of one fused step: 16 B per
updated cell (p read, p1 read and p3 write, c2 read), 16 B more per C-PML
direction a cell lies in (phi in and out, chi read and write), and per
interior cell 4 B of snapshot (forward write, backward read) plus 8 B of
image read-modify-write (backward).  Rows above a free surface are never
updated."""
import numpy as np
import pytest


def _count(ny, nx, dpml, fs):
    dn = dpml + 6
    nyt, nxt = ny + 2 * dn, nx + 2 * dn
    z = np.arange(nyt)[None, :]
    x = np.arange(nxt)[:, None]
    live = np.ones((nxt, nyt), bool) & ~((z < dn) & bool(fs))
    xp = (x < dn) | (x >= dn + nx)
    zp = (z < dn) | (z >= dn + ny)
    interior = ~xp & ~zp
    base = 16 * live + 16 * (live & xp) + 16 * (live & zp)
    return int((base + 4 * interior).sum()), int((base + 12 * interior).sum())


@pytest.mark.parametrize("ny,nx,dpml,fs", [(36, 59, 8, 0), (40, 80, 8, 1), (200, 261, 40, 0), (1200, 1136, 50, 1)])
def test_algorithmic_bytes_match_cell_count(ny, nx, dpml, fs):
    import bench
    fwd, bwd, _ = bench.algorithmic_bytes(ny, nx, dpml, fs)
    assert (fwd, bwd) == _count(ny, nx, dpml, fs)


def test_config2_bytes_are_the_documented_ones():
    import bench
    fwd, bwd, g = bench.algorithmic_bytes(1200, 1136, 50, 1)
    assert (fwd, bwd) == (33901568, 44807168)
    assert g["n_pad"] == 1637376


def test_profiled_traffic_is_read_from_the_summary():
    import bench
    assert bench.profiled_traffic("fwd") == 21037824
    assert bench.profiled_traffic("bwd") == 31986176
