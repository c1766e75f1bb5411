"""The resident form's planner on the CPU: psdm::plan_resident cuts the live
padded grid into regions (on 4-row boundaries, 8 to 384 rows, at most
max_sw - 6 columns, no overlap), covers every live cell by exactly one warp
item of its region (none above a free surface), keeps interior float4 items
on interior rows without injection or the free surface and x-strip items on
the C-PML x-strips of the interior band, lists every region within the read
halo as a neighbour (symmetrically) and puts each receiver in the region
that owns its cell.  tests/res_plan_check.cpp is compiled against the built
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
    out = str(tmp_path_factory.mktemp("resplan") / "res_plan_check")
    libdir = os.path.join(ROOT, "psdm_b200", "lib")
    cmd = [cxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "psdm_b200", "csrc"), os.path.join(ROOT, "tests", "res_plan_check.cpp"), "-o", out,
           "-L", libdir, "-lpsdm_rtm", "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def _run(checker, ny, nx, dPML, fs, max_regions, max_sw, nrec, rows=()):
    r = subprocess.run([checker, str(ny), str(nx), str(dPML), str(fs), str(max_regions), str(max_sw), str(nrec),
                        *map(str, rows)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return [int(v) for v in r.stdout.split()]


# max_sw 72: the widest shared window of a B200 block (227 KB, two levels of 392 rows)
@pytest.mark.parametrize("ny,nx,dPML,fs,rows,nrec,max_regions", [
    (36, 59, 8, 0, (2,), 24, 148),
    (40, 80, 8, 1, (0, 1), 30, 148),
    (150, 317, 9, 0, (4, 2), 60, 148),
    (201, 263, 40, 0, (0,), 120, 148),        # config-1 sized window, ny not a multiple of 4
    (1200, 1136, 50, 1, (0, 1), 480, 148),    # config-2 window
    (1200, 1136, 50, 1, (0, 1), 480, 100),    # fewer regions than multiprocessors
    (203, 90, 11, 1, (3, 40), 12, 148),       # dn not a multiple of 4
])
def test_resident_plan_covers_grid_once(checker, ny, nx, dPML, fs, rows, nrec, max_regions):
    fits, nreg, cover, kind, shape, nbr, rec, lanes = _run(checker, ny, nx, dPML, fs, max_regions, 72, nrec, rows)
    assert fits == 1
    assert 1 <= nreg <= max_regions
    assert (cover, kind, shape, nbr, rec) == (0, 0, 0, 0, 0)
    assert 1 <= lanes <= 32


def test_resident_plan_config2_regions(checker):
    """The config-2 window is cut into about one region per multiprocessor."""
    fits, nreg, *_ = _run(checker, 1200, 1136, 50, 1, 148, 72, 480, (0, 1))
    assert fits == 1 and 120 <= nreg <= 148


def test_resident_plan_refuses_grids_that_do_not_fit(checker):
    """A config-5 window (3000 x 2620 cells) needs more than 148 regions of
    at most 384 x 66 cells."""
    fits, *_ = _run(checker, 3000, 2620, 50, 1, 148, 72, 0, (0, 1))
    assert fits == 0
