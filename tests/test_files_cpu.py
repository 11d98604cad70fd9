"""The .kfh container (the reference's HDF5 layout, IO.cpp:60-505) on the CPU:
the Python writer/reader and the library's header reader agree."""
import numpy as np
import pytest

import kielflow_b200 as kf
from kielflow_b200 import kfh


def reference_layout(n=8, L=25.1, t=3.25, data_dims=3, axis_type=1, m=0.0):
    rng = np.random.default_rng(1)
    e = [("version", "test"), ("date", np.int64(1234567)), ("path", "/x")]
    for a in "xyz":
        e += [(f"domain/type_{a}", axis_type), (f"domain/m_{a}", m), (f"domain/l0_{a}", -0.5 * L),
              (f"domain/N_{a}", n), (f"domain/L_{a}", L)]
    e += [("time", t), ("parameters/mach number M", 1.2), ("parameters/damping ratio tau", 0.1),
          ("parameters/temperature ratio theta", 30.0), ("parameters/velocity diffusion mu", 1e-3),
          ("parameters/magnetization beta", 0.0)]
    shape = (n,) * data_dims
    for name in ("Ux", "Uy", "Uz", "ni", "Ph"):
        e.append((f"data/{name}", rng.standard_normal(shape)))
    return e


def test_roundtrip_python(tmp_path):
    e = reference_layout()
    p = str(tmp_path / "a.kfh")
    kfh.write(p, e)
    r = kfh.read(p)
    for name, v in e:
        if isinstance(v, np.ndarray):
            assert np.array_equal(r[name], v)
        else:
            assert r[name] == v


@pytest.mark.parametrize("dims,kind", [(3, kf.KF_FILE_BACKUP), (2, kf.KF_FILE_SLICE)])
def test_library_reads_header(tmp_path, dims, kind):
    p = str(tmp_path / "b.kfh")
    kfh.write(p, reference_layout(n=16, L=8.0, t=7.5, data_dims=dims))
    info = kf.file_info(p)
    assert info["n"] == 16 and info["L"] == 8.0 and info["l0"] == -4.0 and info["time"] == 7.5
    assert info["M"] == 1.2 and info["tau"] == 0.1 and info["theta"] == 30.0 and info["mu"] == 1e-3
    assert info["kind"] == kind
    assert info["type"] == 1 and info["m"] == 0.0


def test_library_reads_stretched_axes(tmp_path):
    """domain/type_ 3 and m_ of an axis_CoSiSt grid (IO.cpp:105 writes type_id)."""
    p = str(tmp_path / "s.kfh")
    kfh.write(p, reference_layout(n=16, L=8.0, axis_type=3, m=0.89))
    info = kf.file_info(p)
    assert info["type"] == 3 and info["m"] == 0.89 and info["n"] == 16


def test_library_rejects_bad_files(tmp_path):
    p = tmp_path / "c.kfh"
    p.write_bytes(b"HDF5 but not really")
    with pytest.raises(kf.KfError):
        kf.file_info(str(p))
    q = str(tmp_path / "d.kfh")
    kfh.write(q, [("time", 1.0)])
    with pytest.raises(kf.KfError):
        kf.file_info(q)
