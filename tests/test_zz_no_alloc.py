"""The allocation-free entry point, phop_propagate_device_noalloc.

It serves callers that cannot call cudaMalloc while they propagate: a
plug-in whose host application's pool allocator owns the GPU's memory, a
real-time loop that cannot take the device-wide synchronisation of a
cudaMalloc, or a service whose memory footprint is fixed at start-up.  It
takes its scratch from a device array built into the library, which every
call shares.

The tests call it through the C ABI and check its results against the
regular device-resident entry point (phop_propagate_device) on the same
inputs, with the parity tolerance the other GPU tests use: twice in a row on
one context, then on contexts with different gravity fields opened one after
the other (a closed context's tile must not be reused by the next one) and
with the precision switched on one context.  Each test creates its own
contexts, so the file runs the same alone in a fresh process and after the
rest of the suite.
"""
import ctypes as C
import json

import numpy as np
import pytest

from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu

POS_TOL_M = 1e-3
VEL_TOL_M_S = 1e-6
SPLIT_POS_TOL_M = 1e-2


def _noalloc(lib):
    f = lib.phop_propagate_device_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                  C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


class Batch:
    def __init__(self, pop):
        import torch
        self.pop = pop
        self.n = len(pop)
        self.soa0 = np.ascontiguousarray(pop.states.T).reshape(-1).copy()
        area = pop.drag_area * 1e-6
        crf = pop.cr * pop.srp_area / pop.drag_area
        self.d_bc = torch.from_numpy(pop.cd * area / pop.mass).cuda()
        self.d_ams = torch.from_numpy(crf * area / pop.mass).cuda()
        self.epoch = float(pop.epochs[0])

    def regular(self, prop):
        import torch
        st = torch.from_numpy(self.soa0.copy()).cuda()
        p = self.pop
        ep = prop.propagate_device(st.data_ptr(), self.n, self.epoch, p.mass, p.drag_area, p.srp_area, p.cd, p.cr,
                                   prop.duration, prop.step)
        return ep, st.cpu().numpy().reshape(6, self.n).T

    def noalloc(self, prop, duration=None, step=None):
        import torch
        st = torch.from_numpy(self.soa0.copy()).cuda()
        out_epoch = C.c_double()
        rc = _noalloc(api.library())(prop._h, self.n, C.c_void_p(st.data_ptr()), C.c_void_p(self.d_bc.data_ptr()),
                                     C.c_void_p(self.d_ams.data_ptr()), self.epoch,
                                     prop.duration if duration is None else duration,
                                     prop.step if step is None else step, C.byref(out_epoch))
        return rc, out_epoch.value, st.cpu().numpy().reshape(6, self.n).T


def _check(got, ref, pos_tol=POS_TOL_M):
    dpos = np.linalg.norm(got[:, :3] - ref[:, :3], axis=1).max() * 1e3
    dvel = np.linalg.norm(got[:, 3:] - ref[:, 3:], axis=1).max() * 1e3
    assert dpos <= pos_tol, dpos
    if pos_tol == POS_TOL_M:
        assert dvel <= VEL_TOL_M_S, dvel


def _context(tmp_path, degree, name):
    d = S.write_environment(tmp_path / name, S.EnvSpec(degree=degree))
    cfg = S.make_config(d, 1800.0, 60.0, max_steps=100000, degree=degree)
    (d / "config.json").write_text(json.dumps(cfg))
    return d / "config.json"


def test_noalloc_matches_device_entry_point(tmp_path):
    cfg = _context(tmp_path, 70, "d70")
    b = Batch(S.population_leo(257, seed=17))
    prop = api.Propagator(cfg)
    ref_epoch, ref = b.regular(prop)
    for _ in range(2):  # two calls in a row share the static scratch
        rc, ep, got = b.noalloc(prop)
        assert rc == 0, api.library().phop_last_error(prop._h).decode()
        _check(got, ref)
        assert abs(ep - ref_epoch) * 86400.0 <= 1e-4
    # requests beyond the static limit are refused with a clear error
    rc, _, _ = b.noalloc(prop, duration=300 * 60.0, step=60.0)
    assert rc == 1
    assert "at most 256 steps" in api.library().phop_last_error(prop._h).decode()
    prop.close()


def test_noalloc_contexts_in_sequence_and_precision_switch(tmp_path):
    """Degree 70, then degree 120 (opened after the first is closed), then
    degree 70 again, all at the same lane count: each call must use its own
    context's coefficient tile.  Then FP64 and split alternate on one
    context."""
    b = Batch(S.population_leo(96, seed=23))
    cfgs = {70: _context(tmp_path, 70, "a70"), 120: _context(tmp_path, 120, "b120")}
    for degree in (70, 120, 70):
        prop = api.Propagator(cfgs[degree], lanes=2)
        _, ref = b.regular(prop)
        rc, _, got = b.noalloc(prop)
        assert rc == 0, api.library().phop_last_error(prop._h).decode()
        _check(got, ref)
        prop.close()
    prop = api.Propagator(cfgs[120], lanes=2)
    _, ref64 = b.regular(prop)
    for split in (1, 0, 1):
        prop.set_option("split", split)
        rc, _, got = b.noalloc(prop)
        assert rc == 0, api.library().phop_last_error(prop._h).decode()
        if split:
            _check(got, ref64, SPLIT_POS_TOL_M)
        else:
            _check(got, ref64)
    # the FP64-below-a-height option needs a second tile: refused
    prop.set_option("split", 1)
    prop.set_option("split_floor_km", 600.0)
    rc, _, _ = b.noalloc(prop)
    assert rc == 1 and "split_floor_km" in api.library().phop_last_error(prop._h).decode()
    prop.close()
