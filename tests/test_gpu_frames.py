"""Earth frame resolution (interface/naming/orientations Resolver.h):
with both high-precision Earth frames loaded the configuration must name
one, a named frame must have its data loaded, and IAU_EARTH can be chosen
explicitly beside a binary frame; each choice propagates to the same
results as the frame alone."""
import json

import numpy as np
import pytest

from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu


def _config(d, **kw):
    (d / "config.json").write_text(json.dumps(S.make_config(d, 600.0, 60.0, max_steps=1000, **kw)))
    return d / "config.json"


def test_two_earth_frames_need_a_choice(tmp_path):
    d = S.write_environment(tmp_path / "both", S.EnvSpec(earth_frame="both"))
    with pytest.raises(api.PhopError, match="more than one loaded high-precision orientation frame"):
        api.Propagator(_config(d))
    with pytest.raises(api.PhopError, match="needs its rotation data loaded"):
        api.Propagator(_config(d, earth_orientation="IAU_EARTH"))
    with pytest.raises(api.PhopError, match="Unknown Earth orientation"):
        api.Propagator(_config(d, earth_orientation="MARS_FIXED"))


def test_named_frame_matches_the_frame_alone(tmp_path):
    pop = S.population_leo(32, 33)
    tg = pop.targets_json()
    out = {}
    for name, frame, choice in (("itrf93", "itrf93", None), ("both_itrf93", "both", "ITRF93"),
                                ("iers", "iers", None), ("both_iers", "both", "ITRF_IERS2000")):
        d = S.write_environment(tmp_path / name, S.EnvSpec(earth_frame=frame))
        p = api.Propagator(_config(d, earth_orientation=choice), lanes=4)
        out[name] = p.propagate_targets(tg)[1]
        p.close()
    np.testing.assert_array_equal(out["both_itrf93"], out["itrf93"])
    np.testing.assert_array_equal(out["both_iers"], out["iers"])
    # the two frames differ (the synthetic ITRF93 angles are not the IERS model)
    assert np.abs(out["itrf93"] - out["iers"]).max() > 1e-9
