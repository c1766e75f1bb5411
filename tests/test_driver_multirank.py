"""Shot loop of psdm_b200.driver on two CPU ranks (gloo), against the same loop
evaluated serially.

The shot loop deals shots round-robin (calculate_PSDM_RTM.f90:164-166),
embeds each window image into the full grid, sums the ranks' images once per
round (MPI_ALLREDUCE, :493-494) and normalises by the fold
(auxiliar_PSDM.f90:1-20).  Window images here are seeded random arrays in
place of migrated shots, so the test needs no GPU; with two ranks the
per-round sum a + b is exact, so the comparison is exact.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from psdm_b200 import driver

NY, NX = 24, 80


def fake_shot(icount):
    """Deterministic window image of shot line `icount`; line 3 is skipped."""
    if icount == 3:
        return None
    rng = np.random.default_rng(1000 + icount)
    x_i = int(rng.integers(1, NX - 20))
    x_f = int(min(NX, x_i + rng.integers(5, 30)))
    img = rng.standard_normal((x_f - x_i + 1, NY)).astype(np.float32)
    return img, x_i, x_f


def serial_reference(line_i, line_f, world):
    """The loop evaluated in one process: per round, sum the ranks' embedded
    images in rank order, then add to the running sums."""
    nsamples = line_f - line_i + 1
    psdm = np.zeros((NX, NY), np.float32)
    cov = np.zeros((NX, NY), np.float32)
    for it in range(1, driver.n_rounds(nsamples, world) + 1):
        r_img = np.zeros((NX, NY), np.float32)
        r_cov = np.zeros((NX, NY), np.float32)
        for rank in range(world):
            ic = driver.shot_of(it, world, rank, line_i)
            res = fake_shot(ic) if line_i <= ic <= line_f else None
            if res is None:
                continue
            img, x_i, x_f = res
            t = np.zeros((NX, NY), np.float32)
            t[x_i - 1:x_f] = img
            r_img = r_img + t
            c = np.zeros((NX, NY), np.float32)
            c[x_i - 1:x_f] = 1.0
            r_cov = r_cov + c
        psdm = psdm + r_img
        cov = cov + r_cov
    return psdm, cov


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, line_i, line_f, out_dir):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        stack = driver.ImageStack(NY, NX)
        rounds = []

        def shot(ic):
            res = fake_shot(ic)
            if res is None:
                return None
            img, x_i, x_f = res
            return torch.from_numpy(img), x_i, x_f

        driver.migrate_lines(shot, line_i, line_f, stack, rank=rank, numtasks=world, on_round=rounds.append)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), psdm=stack.psdm_sum.numpy(), cov=stack.cov_sum.numpy(),
                 rounds=np.array(rounds))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("line_i,line_f", [(1, 8), (2, 6)])
def test_two_rank_stack_matches_serial(line_i, line_f):
    import torch.multiprocessing as tmp
    world = 2
    with tempfile.TemporaryDirectory() as d:
        tmp.start_processes(_worker, args=(world, _free_port(), line_i, line_f, d), nprocs=world, join=True,
                            start_method="spawn")
        r0 = np.load(os.path.join(d, "rank0.npz"))
        r1 = np.load(os.path.join(d, "rank1.npz"))
    want_psdm, want_cov = serial_reference(line_i, line_f, world)
    n = driver.n_rounds(line_f - line_i + 1, world)
    assert list(r0["rounds"]) == list(range(1, n + 1)) == list(r1["rounds"])
    # every rank holds the same sums after each all-reduce
    np.testing.assert_array_equal(r0["psdm"], r1["psdm"])
    np.testing.assert_array_equal(r0["cov"], r1["cov"])
    np.testing.assert_array_equal(r0["psdm"], want_psdm)
    np.testing.assert_array_equal(r0["cov"], want_cov)
    assert want_cov.max() >= 1


def test_round_robin_schedule():
    # ntimes (:151-159) and icount (:166) for a few shapes
    assert driver.n_rounds(10, 1) == 10
    assert driver.n_rounds(10, 4) == 3
    assert driver.n_rounds(3, 4) == 1
    assert driver.n_rounds(4, 4) == 1
    seen = sorted(driver.shot_of(it, 4, r, 5) for it in range(1, 4) for r in range(4))
    assert seen == list(range(5, 17))  # lines 5..14 are covered, 15..16 are past line_f=14


def test_single_process_stack_and_normalize(oracle):
    stack = driver.ImageStack(NY, NX)

    def shot(ic):
        import torch
        res = fake_shot(ic)
        if res is None:
            return None
        img, x_i, x_f = res
        return torch.from_numpy(img), x_i, x_f

    driver.migrate_lines(shot, 1, 6, stack)
    want_psdm, want_cov = serial_reference(1, 6, 1)
    np.testing.assert_array_equal(stack.psdm_sum.numpy(), want_psdm)
    np.testing.assert_array_equal(stack.cov_sum.numpy(), want_cov)
    np.testing.assert_array_equal(stack.normalized(), oracle.normalize_psdm(want_psdm, want_cov))


def test_float64_stack(oracle):
    """The cross-shot stack kept in float64: the running sums are the float64
    sums of the widened window images, and the image is the float64 quotient
    rounded once."""
    import torch
    stack = driver.ImageStack(NY, NX, dtype=torch.float64)

    def shot(ic):
        res = fake_shot(ic)
        if res is None:
            return None
        img, x_i, x_f = res
        return torch.from_numpy(img), x_i, x_f

    driver.migrate_lines(shot, 1, 6, stack)
    psdm = np.zeros((NX, NY), np.float64)
    cov = np.zeros((NX, NY), np.float64)
    for ic in range(1, 7):
        res = fake_shot(ic)
        if res is None:
            continue
        img, x_i, x_f = res
        psdm[x_i - 1:x_f] += img.astype(np.float64)
        cov[x_i - 1:x_f] += 1.0
    np.testing.assert_array_equal(stack.psdm_sum.numpy(), psdm)
    np.testing.assert_array_equal(stack.cov_sum.numpy(), cov)
    want = np.zeros_like(psdm)
    np.divide(psdm, cov, out=want, where=cov > 0)
    got = stack.normalized()
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, want.astype(np.float32))


def test_window_outside_model_is_rejected():
    stack = driver.ImageStack(NY, NX)
    with pytest.raises(ValueError):
        stack.add_round(np.zeros((10, NY), np.float32), NX - 3, NX + 6)
