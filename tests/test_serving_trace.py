"""Host logic of the serving benchmark: the request trace generator (seeded,
bounded, both force models) and the offered-load arithmetic."""
import numpy as np

from parahpop_b200 import serving


def test_trace_is_seeded_and_bounded():
    a = serving.make_trace(**serving.PRESETS["fit"], seed=9)
    b = serving.make_trace(**serving.PRESETS["fit"], seed=9)
    assert [(r.arrival_s, r.kind, r.offset, r.n, r.duration_s) for r in a] == \
           [(r.arrival_s, r.kind, r.offset, r.n, r.duration_s) for r in b]
    cfg = serving.PRESETS["fit"]
    arr = np.array([r.arrival_s for r in a])
    assert np.all(np.diff(arr) > 0) and arr[-1] < cfg["seconds"]
    # Poisson rate within 10 % of the preset over a minute
    assert abs(len(a) / cfg["seconds"] - cfg["rate"]) < 0.1 * cfg["rate"]
    sizes = np.array([r.n for r in a])
    durs = np.array([r.duration_s for r in a])
    assert sizes.min() >= 1 and sizes.max() <= cfg["size_max"]
    assert durs.min() >= cfg["dur_min"] and durs.max() <= cfg["dur_max"]
    assert all(0 <= r.offset and r.offset + r.n <= 100000 for r in a)
    kinds = {r.kind for r in a}
    assert kinds == {"zonal", "full"}


def test_offered_load_counts_final_step_shortening():
    tr = [serving.TraceRequest(0.0, "full", 0, 10, 90.0), serving.TraceRequest(0.1, "zonal", 0, 3, 60.0)]
    off = serving.offered_object_steps(tr, step=60.0)
    assert off == {"full": 20, "zonal": 3}  # 90 s = one full and one shortened step


def test_full_preset_overloads_one_gpu():
    tr = serving.make_trace(**serving.PRESETS["full"], seed=4)
    off = serving.offered_object_steps(tr)
    # ~10^11 object-steps offered in one minute: two orders above one GPU
    assert sum(off.values()) > 5e10
