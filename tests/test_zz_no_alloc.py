"""psdm_model_shot_noalloc: forward modelling that allocates no device memory.

The entry point is for callers that cannot allocate device memory when they
model a shot (applications whose device memory belongs to their own pool or
to a fixed budget, plugins that must not touch their host's device heap).
It keeps its scratch in one fixed static device array that every call
shares, so the tests below call it twice in a row on different shots and
check that the second call's traces do not depend on what the first one
left in the scratch.  Its traces must equal psdm_model_shot's bit for bit,
the tolerance of every parity test here (both run the same FP32 step
kernels).

This file is collected last on purpose, so that a run that stops at the
first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _prm(c):
    from psdm_b200.rtm import Params
    return Params(dPML=c["dPML"], fs=c["fs"], strategy=c["strategy"], precision=0)


def _noalloc(c):
    """One call through the C ABI with caller-owned device buffers."""
    import torch
    from psdm_b200 import _lib as L
    dev = torch.device("cuda", 0)
    src = torch.from_numpy(np.ascontiguousarray(c["src"], dtype=np.float32)).to(dev)
    vp = torch.from_numpy(np.ascontiguousarray(c["vp_w"], dtype=np.float32)).to(dev)
    nrec = int(c["nxRec"].size)
    # Filled with garbage: the entry point overwrites the whole output.
    out = torch.full((nrec, c["nt"]), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    rc = L.lib().psdm_model_shot_noalloc(
        C.byref(_prm(c).c()), nrec, int(c["nxSou"]), int(c["nySou"]),
        np.ascontiguousarray(c["nxRec"], dtype=np.int32), np.ascontiguousarray(c["nyRec"], dtype=np.int32),
        src.data_ptr(), c["dd"], c["dt"], c["ny"], c["nx"], c["nx_w"], vp.data_ptr(), c["added_space"], c["nt"],
        out.data_ptr(), stream.cuda_stream)
    L.check(rc)
    return out.cpu().numpy()


def _engine_traces(engine, c):
    return engine.model_shot(_prm(c), c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["dd"], c["dt"],
                             c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], c["nt"])


def _assert_same(got, want, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ (first at flat {bad[:1]})"


def test_noalloc_matches_model_shot_twice(engine):
    # Two different shots back to back: the second starts from the first's
    # leftovers in the shared scratch (larger grid first, then a smaller one
    # with a free surface and the other statement order).
    a = make_case(ny=150, nx_model=420, nt=90, dPML=11, fs=0, strategy=2, nrec=60, rec_step=3, sou_x=300,
                  sou_z=5, rec_z=3, added_space=150.0, seed=7)
    b = make_case(fs=1, nt=200, seed=4)
    got_a = _noalloc(a)
    got_b = _noalloc(b)
    _assert_same(got_a, _engine_traces(engine, a), "first call")
    _assert_same(got_b, _engine_traces(engine, b), "second call")


def test_noalloc_same_shot_twice(engine):
    c = make_case(fs=1, nt=150, dPML=8, seed=12)
    first = _noalloc(c)
    second = _noalloc(c)
    want = _engine_traces(engine, c)
    _assert_same(first, want, "first call")
    _assert_same(second, want, "second call")


def _noalloc_prepared(c):
    """Device buffers made first, so that the call itself is all that runs
    between two readings of the free device memory."""
    import torch
    from psdm_b200 import _lib as L
    dev = torch.device("cuda", 0)
    src = torch.from_numpy(np.ascontiguousarray(c["src"], dtype=np.float32)).to(dev)
    vp = torch.from_numpy(np.ascontiguousarray(c["vp_w"], dtype=np.float32)).to(dev)
    nrec = int(c["nxRec"].size)
    out = torch.zeros((nrec, c["nt"]), dtype=torch.float32, device=dev)
    nxr = np.ascontiguousarray(c["nxRec"], dtype=np.int32)
    nyr = np.ascontiguousarray(c["nyRec"], dtype=np.int32)
    prm = _prm(c).c()
    stream = torch.cuda.current_stream(dev)

    def call():
        L.check(L.lib().psdm_model_shot_noalloc(
            C.byref(prm), nrec, int(c["nxSou"]), int(c["nySou"]), nxr, nyr, src.data_ptr(), c["dd"], c["dt"],
            c["ny"], c["nx"], c["nx_w"], vp.data_ptr(), c["added_space"], c["nt"], out.data_ptr(),
            stream.cuda_stream))
    return call, out


def test_noalloc_allocates_nothing(engine):
    # After one call on a shot, a call on a different (larger) shot must not
    # change the device's free memory: the scratch is static.
    import torch
    a = make_case(fs=1, nt=120, seed=21)
    b = make_case(ny=150, nx_model=420, nt=90, dPML=11, fs=0, strategy=2, nrec=60, rec_step=3, sou_x=300,
                  sou_z=5, rec_z=3, added_space=150.0, seed=22)
    call_a, _ = _noalloc_prepared(a)
    call_b, out_b = _noalloc_prepared(b)
    call_a()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    call_b()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes across the call"
    _assert_same(out_b.cpu().numpy(), _engine_traces(engine, b), "traces")


def test_noalloc_rejects_oversized_shot(engine):
    from psdm_b200._lib import PsdmError
    # A 2000 x 242 window pads to 2048 x 270 cells, above the 2^19-cell scratch.
    c = make_case(ny=2000, nx_model=700, nt=20, nrec=50, rec_step=4, sou_x=650, added_space=200.0, seed=3)
    with pytest.raises(PsdmError, match="too large"):
        _noalloc(c)
