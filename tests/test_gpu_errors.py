"""Failure detection through the C ABI, made on the host or in the data (no
GPU fault): a Poisson solve that cannot reach its tolerance, NaN in the state,
invalid arguments -- each reported as its KF_ERR_* code, with the context
usable afterwards."""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C

pytestmark = pytest.mark.gpu


def make(n=32, name="fas128", **over):
    w = C.WORKLOADS[name]
    st, nd, mask, dt = C.make_inputs(w, n)
    ctx = kf.Context(C.config_for(w, n, **over))
    ctx.set_state(*st)
    ctx.set_sources(nd, mask)
    return ctx, st, dt


@pytest.mark.parametrize("host", [False, True])
def test_not_converged_is_reported_and_the_context_recovers(host):
    ctx, st, dt = make(res_tol=1e-15, max_cycles=2)
    with ctx:
        if host:
            ctx.profile(True)  # the host-driven step
        with pytest.raises(kf.KfError) as e:
            ctx.rk4(dt, 1)
        assert e.value.code == -4  # KF_ERR_NOT_CONVERGED
        assert ctx.diag().not_converged >= 1
        # the fields are finite and the context still answers
        assert np.isfinite(ctx.get_phi()).all()
        ctx.set_state(*st)
        assert all(np.isfinite(x).all() for x in ctx.get_state())


@pytest.mark.parametrize("host", [False, True])
def test_nan_in_the_state_is_reported(host):
    ctx, st, dt = make()
    with ctx:
        if host:
            ctx.profile(True)
        bad = [x.copy() for x in st]
        bad[3][3, 4, 5] = np.nan
        ctx.set_state(*bad)
        with pytest.raises(kf.KfError) as e:
            ctx.rk4(dt, 1)
        assert e.value.code == -3  # KF_ERR_NAN
        # a clean state runs again on the same context
        ctx.set_state(*st)
        ctx.set_phi(np.zeros((32, 32, 32)))
        ctx.rk4(dt, 1)
        assert np.isfinite(ctx.get_phi()).all()


def test_invalid_arguments():
    w = C.WORKLOADS["fas128"]
    with pytest.raises(kf.KfError) as e:
        kf.Context(C.config_for(w, 48))  # no radix plan for 48
    assert e.value.code == -1
    with pytest.raises(kf.KfError) as e:
        kf.Context(C.config_for(w, 32, pen_eta=1e-3))  # effect_penalization needs eta <= 0
    assert e.value.code == -1
    for om in (-0.5, 2.0):  # over-relaxation outside [0, 2)
        with pytest.raises(kf.KfError) as e:
            kf.Context(C.config_for(w, 32, mg_omega=om))
        assert e.value.code == -1
    ctx32, st, dt = make(precision=kf.KF_FP32_BULK)
    with ctx32:
        with pytest.raises(kf.KfError) as e:
            ctx32.adjoint(np.zeros((32, 32, 32)), 1, dt)  # the adjoint is FP64 only
        assert e.value.code == -1
        ctx32.rk4(dt, 1)  # still usable
    jac, _, dtj = make(name="jacobi32")
    with jac:
        with pytest.raises(kf.KfError) as e:
            kf.batch_rk4([jac], [dtj], 1)  # the Jacobi solver is host-driven: no captured step
        assert e.value.code == -1


def test_load_rejects_another_grid(tmp_path):
    a, _, dt = make(32)
    with a:
        a.save(str(tmp_path / "b.kfh"), kf.KF_FILE_BACKUP, 0.0)
    b, _, _ = make(64)
    with b:
        with pytest.raises(kf.KfError) as e:
            b.load(str(tmp_path / "b.kfh"))
        assert e.value.code == -1
        with pytest.raises(kf.KfError):
            b.load(str(tmp_path / "missing.kfh"))
