"""Trajectory records (phop_propagate_trajectory): the states after every
k-th step of a uniform batch, written by the step kernel as it goes, are bit
for bit the final states of separate propagations to those epochs (same
kernel, lanes and epoch records), and the record count and epochs follow the
fixed-step grid, final-step shortening included."""
import json

import numpy as np
import pytest

from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prop(tmp_path_factory):
    d = S.write_environment(tmp_path_factory.mktemp("traj"))
    (d / "config.json").write_text(json.dumps(S.make_config(d, 600.0, 60.0, max_steps=100000)))
    p = api.Propagator(d / "config.json", lanes=4)
    yield p
    p.close()


def _args(pop):
    return (pop.mass, pop.drag_area, pop.srp_area, pop.cd, pop.cr)


def test_records_equal_separate_propagations(prop):
    pop = S.population_leo(96, 31)
    epoch = float(pop.epochs[0])
    ep, rec = prop.trajectory(epoch, pop.states, *_args(pop), 600.0, 60.0, every=1)
    assert rec.shape == (10, 96, 6)
    np.testing.assert_allclose(ep, epoch + 60.0 * np.arange(1, 11) / 86400.0, rtol=0, atol=1e-12)
    for k in (1, 4, 10):
        st = pop.states.copy()
        eps = np.full(len(pop), epoch)
        ep2, st2 = prop.propagate(eps, st, *_args(pop), np.full(len(pop), 60.0 * k), np.full(len(pop), 60.0))
        np.testing.assert_array_equal(rec[k - 1], st2)


def test_every_k_and_shortened_final_step(prop):
    pop = S.population_leo(40, 32)
    epoch = float(pop.epochs[0])
    ep, rec = prop.trajectory(epoch, pop.states, *_args(pop), 570.0, 60.0, every=5)
    assert len(rec) == 2  # 10 steps (the last one 30 s): records after steps 5 and 10
    assert abs(ep[-1] - (epoch + 570.0 / 86400.0)) < 1e-12
    _, fin = prop.propagate(np.full(len(pop), epoch), pop.states.copy(), *_args(pop), np.full(len(pop), 570.0),
                            np.full(len(pop), 60.0))
    np.testing.assert_array_equal(rec[-1], fin)
    with pytest.raises(api.PhopError, match="every"):
        prop.trajectory(epoch, pop.states, *_args(pop), 600.0, 60.0, every=0)
