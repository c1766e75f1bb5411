"""The HBM budget planner on the CPU (psdm_plan_memory, the engine's analogue
of rtm_strategy, optimization.f90:114-188): slots sized to a given budget,
shots whose snapshots do not fit (FP32 or 16-bit) switched to checkpoints
with a memory that fits, mixed-precision shots sized by their 16-bit
snapshots, and
PSDM_ERR_NOMEM with the sizes when nothing fits.  Budgets are given, so no
device is needed."""
import pytest

GB = 10 ** 9


def _prm(precision=0):
    from psdm_b200.rtm import Params
    return Params(dPML=50, fs=1, strategy=1, precision=precision)


def test_config2_fp32_fits_four(engine_lib):
    from psdm_b200 import rtm
    p = rtm.plan_memory(_prm(), 1200, 1136, 8000, 8000, 1, 480, 180 * GB)
    assert p["fits"] and p["checkpoint_interval"] == 0
    assert 43 * GB < p["bytes_per_slot"] < 44.5 * GB
    assert p["slots"] == 4  # 178.9 GB after the reserve, 43.7 GB per shot


def test_config2_fp16_many_slots(engine_lib):
    from psdm_b200 import rtm
    p = rtm.plan_memory(_prm(1), 1200, 1136, 8000, 8000, 4, 480, 180 * GB)
    assert p["fits"] and p["slots"] == 16  # capped by the engine's slot limit
    assert p["bytes_per_slot"] < 6 * GB
    p = rtm.plan_memory(_prm(1), 1200, 1136, 8000, 8000, 4, 480, 180 * GB, max_slots=4)
    assert p["slots"] == 4


def test_config5_fp32_checkpoints(engine_lib):
    from psdm_b200 import rtm
    # 3000 x 2620 window, nt 12000: 377 GB of FP32 snapshots
    p = rtm.plan_memory(_prm(), 3000, 2620, 12000, 12000, 1, 960, 180 * GB)
    assert p["fits"] and p["checkpoint_interval"] > 0
    assert 15 * GB < p["bytes_per_slot"] < 30 * GB  # about 21 GB at the memory-optimal interval
    assert p["slots"] == (180 * GB - 2 ** 30) // p["bytes_per_slot"]  # checkpointed shots in flight
    # a smaller budget still fits, one shot at a time
    p2 = rtm.plan_memory(_prm(), 3000, 2620, 12000, 12000, 1, 960, 30 * GB)
    assert p2["fits"] and p2["checkpoint_interval"] == p["checkpoint_interval"] and p2["slots"] == 1


def test_config5_mixed_checkpoints_when_snapshots_do_not_fit(engine_lib):
    from psdm_b200 import rtm
    # binary16 every 4 steps: 47 GB of snapshots, which a 40 GB budget cannot hold
    full = rtm.plan_memory(_prm(1), 3000, 2620, 12000, 12000, 4, 960, 180 * GB)
    assert full["fits"] and full["checkpoint_interval"] == 0 and 45 * GB < full["bytes_per_slot"] < 60 * GB
    p = rtm.plan_memory(_prm(1), 3000, 2620, 12000, 12000, 4, 960, 40 * GB)
    assert p["fits"] and p["checkpoint_interval"] >= 16 and p["slots"] >= 1
    assert p["bytes_per_slot"] < 40 * GB - 2 ** 30


def test_nothing_fits(engine_lib):
    from psdm_b200 import rtm
    from psdm_b200._lib import PsdmError
    with pytest.raises(PsdmError, match="GB"):
        rtm.plan_memory(_prm(), 3000, 2620, 12000, 12000, 1, 960, 2 * GB)
    with pytest.raises(PsdmError, match="GB"):
        rtm.plan_memory(_prm(1), 3000, 2620, 12000, 12000, 4, 960, 2 * GB)
