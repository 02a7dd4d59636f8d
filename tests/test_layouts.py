"""The oracle's readers of CBOR layout 1 and layout 2 (member-major metadata
arrays) give identical environments: the same synthetic ephemeris and
orientation units written both ways propagate to bit-identical states, for
each Earth frame kind (IERS2000 model unit, binary ITRF93 unit, IAU body
model with barycentric terms)."""
import json

import numpy as np
import pytest

from oracle import oracle as O
from parahpop_b200 import synthetic as S


@pytest.mark.parametrize("frame", ["iers", "itrf93", "iau"])
def test_layout2_reads_like_layout1(tmp_path, frame):
    pop = S.population_leo(6, 40)
    out = {}
    for layout in (1, 2):
        d = S.write_environment(tmp_path / f"l{layout}", S.EnvSpec(brie_layout=layout, earth_frame=frame))
        (d / "config.json").write_text(json.dumps(S.make_config(d, 600.0, 60.0, max_steps=1000)))
        _, _, out[layout] = O.propagate(O.load_environment(d / "config.json"), pop.targets_json())
    np.testing.assert_array_equal(out[1], out[2])
