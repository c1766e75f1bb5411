"""Batched shots (psdm_rtm_batch / psdm_rtm_batch_device) against one shot at
a time (psdm_rtm_shot) and the oracle.

Shots of different window widths, record lengths and source positions run
together, fewer slots than shots so that slots are reused; every image must
equal the single-shot engine's (and so the oracle's) bit for bit.
"""
import numpy as np
import pytest

from tests.cases import make_case

pytestmark = pytest.mark.gpu


def _prm(dPML, fs, strategy):
    from psdm_b200.rtm import Params
    return Params(dPML=dPML, fs=fs, strategy=strategy, precision=0)


def _shots(dPML, fs, strategy, taper):
    kw = dict(ny=40, nx_model=160, dPML=dPML, fs=fs, strategy=strategy)
    if taper:
        kw.update(taper_option=1, N_taper=12, N_zeros=9)
    geo = [dict(nt=150, sou_x=52, nrec=24, rec_step=2, seed=1),
           dict(nt=210, sou_x=110, nrec=16, rec_step=3, seed=2, dir_boat=1),
           dict(nt=120, sou_x=80, nrec=30, rec_step=1, seed=3),
           dict(nt=180, sou_x=140, nrec=20, rec_step=2, seed=4)]
    cases = [make_case(**kw, **g) for g in geo]
    # one model grid, dd and dt for all shots; the source wavelet is shared
    longest = max(cases, key=lambda c: c["nt"])
    for c in cases:
        assert np.array_equal(c["src"], longest["src"][:c["nt"]])
    return cases, longest["src"]


def _single(engine, prm, c):
    return engine.rtm_shot(prm, c["nxSou"], c["nySou"], c["nxRec"], c["nyRec"], c["src"], c["tgt"], c["dd"],
                           c["dt"], c["ny"], c["nx"], c["nx_w"], c["vp_w"], c["added_space"], 1, c["nt_taper"],
                           c["nt_prop2"], c["nt_taper"], c["taper_option"], c["N_taper"], c["N_zeros"])


def _desc(c):
    return dict(nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"], nyRec=c["nyRec"], nx_w=c["nx_w"],
                nt_prop2=c["nt_prop2"], nt_taper=c["nt_taper"], Vp_w=c["vp_w"], Data_target=c["tgt"])


def _assert_same(got, want, what):
    assert got.shape == want.shape, (what, got.shape, want.shape)
    assert np.abs(want).max() > 0, what
    bad = np.flatnonzero(~(got == want))
    assert bad.size == 0, f"{what}: {bad.size} of {got.size} values differ"


@pytest.mark.parametrize("dPML,fs,strategy,taper,slots", [(8, 1, 1, 0, 2), (11, 0, 2, 1, 3), (10, 1, 2, 0, 16)])
def test_batch_host_matches_single_shots(engine, dPML, fs, strategy, taper, slots):
    cases, src = _shots(dPML, fs, strategy, taper)
    prm = _prm(dPML, fs, strategy)
    c0 = cases[0]
    imgs = engine.rtm_batch(prm, [_desc(c) for c in cases], src, c0["dd"], c0["dt"], c0["ny"], c0["nx"],
                            c0["added_space"], 1, c0["taper_option"], c0["N_taper"], c0["N_zeros"], max_slots=slots)
    assert engine.batch_slots() == min(slots, len(cases))
    for i, (c, img) in enumerate(zip(cases, imgs)):
        _assert_same(img, _single(engine, prm, c), f"shot {i}")


def test_batch_matches_oracle(engine, oracle):
    cases, src = _shots(8, 1, 1, 0)
    prm = _prm(8, 1, 1)
    c0 = cases[0]
    imgs = engine.rtm_batch(prm, [_desc(c) for c in cases[:2]], src, c0["dd"], c0["dt"], c0["ny"], c0["nx"],
                            c0["added_space"], max_slots=2)
    for c, img in zip(cases[:2], imgs):
        want = oracle.rtm_shot(dPML=8, fs=1, nxSou=c["nxSou"], nySou=c["nySou"], nxRec=c["nxRec"], nyRec=c["nyRec"],
                               Data_source=c["src"], Data_target=c["tgt"], dd=c["dd"], dt=c["dt"], nx=c["nx"],
                               vp_w=c["vp_w"], added_space=c["added_space"], store_snap=1, nt_snap=c["nt"],
                               nt_prop2=c["nt"], nt_taper=c["nt"], disk_mode=0)
        _assert_same(img, want, "batch vs oracle")


def test_batch_device_matches_single_shots(engine):
    import torch
    cases, src = _shots(9, 1, 1, 0)
    prm = _prm(9, 1, 1)
    dev = torch.device("cuda", 0)
    d_src = torch.from_numpy(src).to(dev)
    keep, descs, outs = [], [], []
    for c in cases:
        vp = torch.from_numpy(np.ascontiguousarray(c["vp_w"])).to(dev)
        tgt = torch.from_numpy(np.ascontiguousarray(c["tgt"])).to(dev)
        out = torch.full((c["nx_w"], c["ny"]), float("nan"), dtype=torch.float32, device=dev)
        keep += [vp, tgt]
        outs.append(out)
        d = _desc(c)
        d.update(d_Vp_w=vp.data_ptr(), d_Data_target=tgt.data_ptr(), d_PSDM_w=out.data_ptr())
        descs.append(d)
    torch.cuda.synchronize()
    c0 = cases[0]
    engine.rtm_batch_device(prm, descs, d_src.data_ptr(), c0["dd"], c0["dt"], c0["ny"], c0["nx"],
                            c0["added_space"], max_slots=3)
    for i, (c, out) in enumerate(zip(cases, outs)):
        _assert_same(out.cpu().numpy(), _single(engine, prm, c), f"shot {i}")


def test_batch_rejects_bad_shot(engine):
    from psdm_b200._lib import PsdmError
    cases, src = _shots(8, 1, 1, 0)
    d = _desc(cases[1])
    d["nx_w"] = d["nx_w"] + 1
    d["Vp_w"] = np.zeros((d["nx_w"], cases[1]["ny"]), np.float32)
    c0 = cases[0]
    with pytest.raises(PsdmError, match="nx_w"):
        engine.rtm_batch(_prm(8, 1, 1), [_desc(c0), d], src, c0["dd"], c0["dt"], c0["ny"], c0["nx"],
                         c0["added_space"], max_slots=2)
