"""The tile planner on the CPU: psdm::plan_tiles / tile_rect cover every live
cell of the padded grid exactly once (and no cell above a free surface),
keep injection and free-surface rows out of the interior tiles, use the
interior and x-strip tile widths of the launch form and pass, and psdm::pass_lists gives
symmetric neighbour lists that hold every tile within the read halo and puts
each receiver in the tile that owns its cell.  tests/plan_check.cpp is
compiled against the built engine library and run here, without a GPU."""
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
    out = str(tmp_path_factory.mktemp("plan") / "plan_check")
    libdir = os.path.join(ROOT, "psdm_b200", "lib")
    cmd = [cxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(ROOT, "psdm_b200", "csrc"), os.path.join(ROOT, "tests", "plan_check.cpp"), "-o", out,
           "-L", libdir, "-lpsdm_rtm", "-Wl,-rpath," + libdir]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return out


def _run(checker, ny, nx, dPML, fs, form, nrec, rows=()):
    r = subprocess.run([checker, str(ny), str(nx), str(dPML), str(fs), str(int(form)), str(nrec),
                        *map(str, rows)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return [int(v) for v in r.stdout.split()]


@pytest.mark.parametrize("ny,nx,dPML,fs,rows,nrec", [
    (36, 59, 8, 0, (2,), 24),
    (40, 80, 8, 1, (0, 1), 30),
    (150, 317, 9, 0, (4, 2), 60),
    (201, 263, 40, 0, (0,), 120),        # config-1 sized window, ny not a multiple of 4
    (1200, 1136, 50, 1, (0, 1), 480),    # config-2 window
    (1800, 1361, 50, 1, (0, 1, 2, 3, 40), 120),
])
@pytest.mark.parametrize("form", [0, 1, 2])  # one-shot backward, batched, one-shot forward
def test_plan_covers_grid_once(checker, ny, nx, dPML, fs, rows, nrec, form):
    n, itx, ixb, cover, dead, typ, sym, rec = _run(checker, ny, nx, dPML, fs, form, nrec, rows)
    assert n > 0
    assert itx == {0: 28, 1: 32, 2: 24}[form]
    assert ixb == (8 if form == 2 else 16)
    assert (cover, dead, typ, sym, rec) == (0, 0, 0, 0, 0)


@pytest.mark.parametrize("form", [0, 2])
def test_config2_plan_fits_one_wave(checker, form):
    """The config-2 one-shot plans (backward and forward) have no more tiles
    than the 5 x 148 resident blocks of a step launch."""
    n, *_ = _run(checker, 1200, 1136, 50, 1, form, 0, (0, 1))
    assert 500 < n <= 740
