"""The allocation-free entry point, phop_propagate_device_noalloc.

It serves callers that cannot call cudaMalloc while they propagate (for
example code inside a stream capture that must not allocate, or a plug-in
under a fixed memory budget): it takes its scratch from a device array built
into the library.  This test calls it through the C ABI twice in a row and
checks both results against the regular device-resident entry point
(phop_propagate_device) on the same inputs, with the parity tolerance the
other GPU tests use.  It creates its own context, so it runs the same alone
in a fresh process and after the rest of the suite.
"""
import ctypes as C
import json

import numpy as np
import pytest

from parahpop_b200 import api, synthetic as S

pytestmark = pytest.mark.gpu

POS_TOL_M = 1e-3
VEL_TOL_M_S = 1e-6


def _noalloc(lib):
    f = lib.phop_propagate_device_noalloc
    f.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                  C.POINTER(C.c_double)]
    f.restype = C.c_int
    return f


def test_noalloc_matches_device_entry_point(tmp_path):
    import torch
    d = S.write_environment(tmp_path)
    cfg = S.make_config(d, 1800.0, 60.0, max_steps=100000)
    (d / "config.json").write_text(json.dumps(cfg))
    pop = S.population_leo(257, seed=17)
    n = len(pop)
    prop = api.Propagator(d / "config.json")
    soa0 = np.ascontiguousarray(pop.states.T).reshape(-1).copy()
    area = pop.drag_area * 1e-6
    crf = pop.cr * pop.srp_area / pop.drag_area
    ams = crf * area / pop.mass
    bc = pop.cd * area / pop.mass
    epoch = float(pop.epochs[0])

    # regular entry point
    ref_state = torch.from_numpy(soa0.copy()).cuda()
    ref_epoch = prop.propagate_device(ref_state.data_ptr(), n, epoch, pop.mass, pop.drag_area, pop.srp_area,
                                      pop.cd, pop.cr, prop.duration, prop.step)
    ref = ref_state.cpu().numpy().reshape(6, n).T

    f = _noalloc(api.library())
    d_bc = torch.from_numpy(bc).cuda()
    d_ams = torch.from_numpy(ams).cuda()
    for _ in range(2):  # two calls in a row share the static scratch
        st = torch.from_numpy(soa0.copy()).cuda()
        out_epoch = C.c_double()
        rc = f(prop._h, n, C.c_void_p(st.data_ptr()), C.c_void_p(d_bc.data_ptr()), C.c_void_p(d_ams.data_ptr()),
               epoch, prop.duration, prop.step, C.byref(out_epoch))
        assert rc == 0, api.library().phop_last_error(prop._h).decode()
        got = st.cpu().numpy().reshape(6, n).T
        dpos = np.linalg.norm(got[:, :3] - ref[:, :3], axis=1).max() * 1e3
        dvel = np.linalg.norm(got[:, 3:] - ref[:, 3:], axis=1).max() * 1e3
        assert dpos <= POS_TOL_M and dvel <= VEL_TOL_M_S, (dpos, dvel)
        assert abs(out_epoch.value - ref_epoch) * 86400.0 <= 1e-4

    # requests beyond the static limit are refused with a clear error
    st = torch.from_numpy(soa0.copy()).cuda()
    rc = f(prop._h, n, C.c_void_p(st.data_ptr()), C.c_void_p(d_bc.data_ptr()), C.c_void_p(d_ams.data_ptr()),
           epoch, 300 * 60.0, 60.0, C.byref(C.c_double()))
    assert rc == 1
    assert "at most 256 steps" in api.library().phop_last_error(prop._h).decode()
    prop.close()
