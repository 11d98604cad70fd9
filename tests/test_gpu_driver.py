"""The reference's time loop around the step (kielflow.cpp:172-182, 277-340)
through the C ABI: the density's log/linear transforms against the oracle's
transforms (FP64: 1e-12 relative) and the slice / backup cadence of kf_run
against kf_rk4_steps + kf_get_output (bit for bit)."""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import configs as C
from kielflow_b200 import inputs as I
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


def test_save_and_load_backup(tmp_path):
    ctx, st, dt = setup()
    p = str(tmp_path / "backup.kfh")
    with ctx:
        ctx.rk4(dt, 2)
        s = ctx.get_state()
        phi = ctx.get_phi()
        ctx.save(p, kf.KF_FILE_BACKUP, 0.75)
    f = kf.kfh.read(p)
    assert f["domain/N_x"] == 32 and f["time"] == 0.75 and f["domain/type_z"] == 1
    assert f["parameters/mach number M"] == C.WORKLOADS["fas128"]["M"]
    for q, name in enumerate(("Ux", "Uy", "Uz")):
        assert rel(f[f"data/{name}"], bind.c2r(s[q])) < TOL
    assert rel(f["data/ni"], np.exp(bind.c2r(s[3]))) < TOL
    assert np.array_equal(f["data/Ph"], phi)
    info = kf.file_info(p)
    assert info["kind"] == kf.KF_FILE_BACKUP and info["n"] == 32
    ctx2, _, _ = setup()
    with ctx2:
        assert ctx2.load(p) == 0.75
        s2 = ctx2.get_state()
        for q in range(3):
            assert rel(s2[q], bind.r2c(bind.c2r(s[q]))) < TOL
        assert rel(s2[3], bind.r2c(np.log(np.exp(bind.c2r(s[3]))))) < TOL
        assert np.array_equal(ctx2.get_phi(), phi)


def test_slice_is_the_z0_plane_of_the_backup(tmp_path):
    ctx, st, dt = setup()
    with ctx:
        ctx.rk4(dt, 1)
        ctx.save(str(tmp_path / "s.kfh"), kf.KF_FILE_SLICE, 0.0)
        ctx.save(str(tmp_path / "b.kfh"), kf.KF_FILE_BACKUP, 0.0)
    s = kf.kfh.read(str(tmp_path / "s.kfh"))
    b = kf.kfh.read(str(tmp_path / "b.kfh"))
    for name in ("Ux", "Uy", "Uz", "ni", "Ph"):
        assert s[f"data/{name}"].shape == (32, 32)
        assert np.array_equal(s[f"data/{name}"], b[f"data/{name}"][:, :, 16])  # index_at(0) = N/2


def test_run_writes_the_reference_files(tmp_path):
    ctx, st, dt = setup()
    with ctx:
        ctx.run(12, dt, t0=0.0, slice_every=3, backup_every=6, out_dir=str(tmp_path))
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["backup_at_6.kfh", "slice_0003.kfh", "slice_0006.kfh", "slice_0009.kfh"]
    ref, _, _ = setup()
    with ref:
        ref.rk4(dt, 7)
        ref.save(str(tmp_path / "ref.kfh"), kf.KF_FILE_BACKUP, 0.0)
    a = kf.kfh.read(str(tmp_path / "backup_at_6.kfh"))
    b = kf.kfh.read(str(tmp_path / "ref.kfh"))
    for name in ("Ux", "Uy", "Uz", "ni", "Ph"):
        assert np.array_equal(a[f"data/{name}"], b[f"data/{name}"])
    assert a["time"] == sum([dt] * 6)  # t_total accumulated over 6 loop steps


def oracle_for(cfg):
    return bind.Oracle(bind.KfoConfig(*[getattr(cfg, f) for f, _ in bind.KfoConfig._fields_]))


@pytest.mark.parametrize("mode", [kf.KF_PS_FAS, kf.KF_PS_CASCADIC])
def test_frontend_state_vs_oracle(mode):
    """frontend.cpp:255-330 restated with the oracle's Poisson solver and
    phi-filter table: phi from 0 with rho = 1 + n_d (a grain of charge -0.5
    in the uniform ion background), n = exp(-theta phi), both filtered,
    s^ = r2c(log n)."""
    w = C.WORKLOADS["fas128"]
    st, _, mask, dt = C.make_inputs(w, 32)
    nd = I.gauss_charge(32, C.L_BOX, -0.5, 0.5)
    cfg = C.config_for(w, 32, poisson_mode=mode)
    o = oracle_for(cfg)
    phi = o.poisson(np.zeros((32, 32, 32)), 1.0 + nd)
    _, _, PF = o.tables()
    n_f = bind.c2r(bind.r2c(np.exp(-cfg.theta * phi)) * PF)
    phi_f = bind.c2r(bind.r2c(phi) * PF)
    with kf.Context(cfg) as ctx:
        ctx.set_state(*st)
        ctx.set_sources(nd, mask)
        ctx.frontend_state(1.0)
        got = ctx.get_state()
        assert rel(ctx.get_phi(), phi_f) < TOL
        assert rel(got[3], bind.r2c(np.log(n_f))) < TOL
        for q in range(3):
            assert not np.any(got[q])
        ctx.rk4(dt, 1)  # the state is a valid start
        assert np.isfinite(ctx.get_phi()).all()
