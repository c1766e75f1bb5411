"""SU trace files written and read by the library (no SU tools), checked
field by field with numpy against the SEG-Y/SU trace header layout."""
import numpy as np
import pytest


def _header_dtype(big):
    e = ">" if big else "<"
    return np.dtype([("tracl", e + "i4"), ("tracr", e + "i4"), ("fldr", e + "i4"), ("tracf", e + "i4"),
                     ("ep", e + "i4"), ("cdp", e + "i4"), ("cdpt", e + "i4"), ("trid", e + "i2"),
                     ("pad1", "V84"), ("ns", e + "u2"), ("dt", e + "u2"), ("pad2", "V62"), ("d1", e + "f4"),
                     ("f1", e + "f4"), ("d2", e + "f4"), ("f2", e + "f4"), ("pad3", "V44")])


@pytest.mark.parametrize("big", [False, True])
def test_write_image_headers_and_samples(engine_lib, tmp_path, big):
    from psdm_b200 import rtm
    rng = np.random.default_rng(0)
    model = rng.standard_normal((7, 11)).astype(np.float32)  # ni = 7 traces of nj = 11 samples
    p = tmp_path / "img.su"
    rtm.su_write_image(p, model, di=12.5, dj=6.25, trid=200, big_endian=big)
    hd = _header_dtype(big)
    assert hd.itemsize == 240
    rec = np.dtype([("h", hd), ("d", (">" if big else "<") + "f4", (11,))])
    a = np.fromfile(p, dtype=rec)
    assert a.shape == (7,)
    assert list(a["h"]["tracl"]) == list(range(1, 8)) == list(a["h"]["tracr"])
    assert list(a["h"]["cdp"]) == [int(-12.5 + 12.5 * t) for t in range(1, 8)]
    assert set(a["h"]["ns"]) == {11} and set(a["h"]["trid"]) == {200}
    assert set(a["h"]["d1"]) == {6.25} and set(a["h"]["d2"]) == {12.5}
    assert not a["h"]["f1"].any() and not a["h"]["f2"].any()
    assert np.array_equal(a["d"].astype(np.float32), model)


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("delay", [0, 5, -3])
def test_read_shot_fixed_length_traces(engine_lib, tmp_path, big, delay):
    from psdm_b200 import rtm
    nrec, ns_max, nt = 9, 50, 40
    rng = np.random.default_rng(1)
    data = rng.standard_normal((nrec, ns_max)).astype(np.float32)
    hd = _header_dtype(big)
    rec = np.dtype([("h", hd), ("d", (">" if big else "<") + "f4", (ns_max,))])
    a = np.zeros(nrec, dtype=rec)
    a["d"] = data
    a["h"]["fldr"] = 4711                       # shot number at byte 9
    a["h"]["ep"] = -(100 + 25 * np.arange(nrec))  # an offset-like word at byte 17
    p = tmp_path / "shot.su"
    a.tofile(p)
    raw, delayed = rtm.su_read_shot(p, nrec, ns_max, nt, big_endian=big, delay_samples=delay)
    assert np.array_equal(raw, data[:, :nt])
    want = np.zeros_like(raw)
    if delay >= 0:
        want[:, delay:] = raw[:, :nt - delay]
    else:
        want[:, :nt + delay] = raw[:, -delay:]
    assert np.array_equal(delayed, want)
    assert set(rtm.su_read_header_i32(p, nrec, ns_max, 9, big_endian=big)) == {4711}
    assert np.array_equal(rtm.su_read_header_i32(p, nrec, ns_max, 17, big_endian=big), a["h"]["ep"])


def test_read_rejects_short_file(engine_lib, tmp_path):
    from psdm_b200 import rtm
    from psdm_b200._lib import PsdmError
    p = tmp_path / "short.su"
    np.zeros(100, np.float32).tofile(p)
    with pytest.raises(PsdmError, match="shorter"):
        rtm.su_read_shot(p, 3, 50, 40)
