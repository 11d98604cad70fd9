"""The reference's time loop around the step (kielflow.cpp:172-182, 277-340)
through the C ABI: the density's log/linear transforms against the oracle's
transforms (FP64: 1e-12 relative) and the slice / backup cadence of kf_run
against kf_rk4_steps + kf_get_output (bit for bit)."""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from oracle import bind

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def setup(name="fas128", n=32, **over):
    w = C.WORKLOADS[name]
    st, nd, mask, dt = C.make_inputs(w, n)
    ctx = kf.Context(C.config_for(w, n, **over))
    ctx.set_state(*st)
    ctx.set_sources(nd, mask)
    return ctx, st, dt


def test_set_state_linear_is_log_transform():
    ctx, st, dt = setup()
    with ctx:
        Fn = bind.r2c(np.exp(bind.c2r(st[3])))  # the file's linear density spectrum
        ctx.set_state_linear(st[0], st[1], st[2], Fn)
        got = ctx.get_state()
        assert rel(got[3], bind.r2c(np.log(bind.c2r(Fn)))) < TOL
        for q in range(3):
            assert np.array_equal(got[q], st[q])


def test_get_output_fields():
    ctx, st, dt = setup()
    with ctx:
        ctx.rk4(dt, 2)
        s = ctx.get_state()
        FUx, FUy, FUz, Fn, FPh = ctx.get_output()
        for a, b in zip((FUx, FUy, FUz), s[:3]):
            assert np.array_equal(a, b)
        assert rel(Fn, bind.r2c(np.exp(bind.c2r(s[3])))) < TOL
        assert rel(FPh, bind.r2c(ctx.get_phi())) < TOL


@pytest.mark.parametrize("name,over", [("fas128", {}), ("fp32bulk256", {}),
                                       ("jacobi32", {})])
def test_run_cadence_and_fields(name, over):
    ctx, st, dt = setup(name, 32, **over)
    outs = []
    with ctx:
        ctx.run(12, dt, t0=1.5, slice_every=3, backup_every=6,
                callback=lambda step, t, kind, f: outs.append((step, t, kind, f)))
    # counter.hpp semantics: outputs after loop steps 3, 6, 9; a backup at 6
    assert [(o[0], o[2]) for o in outs] == [(3, 1), (6, 3), (9, 1)]
    t = 1.5
    ts = []
    for step in range(12):
        ts.append(t)
        t += dt
    assert [o[1] for o in outs] == [ts[3], ts[6], ts[9]]
    # the fields at loop step s are those of s + 1 plain steps
    for step, _, _, fields in outs:
        ref, _, _ = setup(name, 32, **over)
        with ref:
            ref.rk4(dt, step + 1)
            want = ref.get_output()
        for a, b in zip(fields, want):
            assert np.array_equal(a, b)
