"""The tile plan of the two-step launches on the CPU (psdm::plan_pair,
psdm::pair_tile_rect, psdm::pair_rec_lists): every live cell of the padded
grid in exactly one tile and none above a free surface; clean interior tiles
aligned to float4 rows, within their size, with their bulk copies inside the
arrays and their 3-cell ring free of C-PML, free-surface and injection
cells; every read of a tile's second step inside the tile plus 3 cells and
every read of its first step inside the level-n cells it loads (the clamped
stencils and strip-local phi stencils included); each receiver in the tile
that owns its cell.  tests/pair_plan_check.cpp is compiled against the built
engine library and run here, without a GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def checker(engine_lib, tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("pplan") / "pair_plan_check")
    libdir = os.path.join(ROOT, "psdm_b200", "lib")
    cmd = [cxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "psdm_b200", "csrc"), os.path.join(ROOT, "tests", "pair_plan_check.cpp"), "-o", out,
           "-L", libdir, "-lpsdm_rtm", "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


@pytest.mark.parametrize("ny,nx,dPML,fs,nrec,rows", [
    (36, 59, 8, 0, 24, (2,)),
    (40, 80, 8, 1, 30, (0, 1)),
    (150, 317, 9, 0, 60, (4, 2)),
    (201, 263, 40, 0, 120, (0,)),        # config-1 sized window, ny not a multiple of 4
    (13, 9, 2, 1, 5, ()),                # smaller than one clean tile
    (7, 5, 3, 0, 3, ()),
    (100, 100, 17, 0, 10, (50,)),        # injection row in the middle of the interior
    (1200, 1136, 50, 1, 480, (0, 1)),    # config-2 window
    (1800, 1361, 50, 1, 120, (0, 1, 2, 3, 40)),
    (1200, 1136, 50, 0, 480, (1, 300, 301, 302, 700, 900, 1000)),  # many injection rows
    (3000, 2414, 50, 1, 960, (1,)),      # config-5 sized window
])
def test_pair_plan(checker, ny, nx, dPML, fs, nrec, rows):
    r = subprocess.run([checker, str(ny), str(nx), str(dPML), str(fs), str(nrec), *map(str, rows)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    n, nclean, cover, shape, clean, reach, rec = map(int, r.stdout.split())
    assert n > 0
    assert (cover, shape, clean, reach, rec) == (0, 0, 0, 0, 0)
    if ny >= 100 and nx >= 100:
        assert nclean > 0
