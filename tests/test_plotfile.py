"""Plotfile output (vd_write_plotfile, the layout Vidyut::WritePlotFile produces
through amrex::WriteMultiLevelPlotfile, Source/Plot.cpp:29-39) read back with an
independent parser of that layout: header fields, the multi-fab header, the FAB
descriptor and every value bit for bit.  No GPU needed."""
import dataclasses

import numpy as np
import pytest

from vidyut_b200 import api, inputs
from vidyut_b200 import mechanism as mm


def read_plotfile(path):
    lines = (path / "Header").read_text().split("\n")
    assert lines[0] == "HyperCLaw-V1.1"
    nv = int(lines[1])
    names = lines[2:2 + nv]
    q = 2 + nv
    dim = int(lines[q])
    time = float(lines[q + 1])
    finest = int(lines[q + 2])
    prob_lo = [float(v) for v in lines[q + 3].split()]
    prob_hi = [float(v) for v in lines[q + 4].split()]
    assert lines[q + 5].strip() == ""          # no refinement ratios on one level
    domain = lines[q + 6].strip()
    step = int(lines[q + 7])
    dx = [float(v) for v in lines[q + 8].split()]
    coord, bwidth = int(lines[q + 9]), int(lines[q + 10])
    lev, ngrid, ltime = lines[q + 11].split()
    lstep = int(lines[q + 12])
    extents = [[float(v) for v in lines[q + 13 + d].split()] for d in range(dim)]
    assert lines[q + 13 + dim] == "Level_0/Cell"
    ch = (path / "Level_0" / "Cell_H").read_text().split("\n")
    assert ch[0] == "1" and ch[1] == "1" and int(ch[2]) == nv and ch[3] == "0"
    assert ch[4] == "(1 0" and ch[5] == domain and ch[6] == ")"
    assert ch[7] == "1" and ch[8] == "FabOnDisk: Cell_D_00000 0"
    assert ch[10] == f"1,{nv}"
    mins = [float(v) for v in ch[11].rstrip(",").split(",")]
    assert ch[13] == f"1,{nv}"
    maxs = [float(v) for v in ch[14].rstrip(",").split(",")]
    raw = (path / "Level_0" / "Cell_D_00000").read_bytes()
    eol = raw.index(b"\n")
    head = raw[:eol].decode()
    assert head.startswith("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))")
    assert head.endswith(f"{domain} {nv}")
    data = np.frombuffer(raw[eol + 1:], dtype="<f8")
    return dict(names=names, dim=dim, time=time, finest=finest, prob_lo=prob_lo, prob_hi=prob_hi,
                domain=domain, step=step, dx=dx, coord=coord, bwidth=bwidth, level=int(lev), ngrid=int(ngrid),
                ltime=float(ltime), lstep=lstep, extents=extents, mins=mins, maxs=maxs, data=data)


@pytest.mark.parametrize("dim,n", [(1, (40,)), (2, (24, 16)), (3, (8, 6, 5))])
def test_plotfile_round_trip(tmp_path, dim, n):
    m = mm.argon(10, 20261204)
    case = inputs.build_case(m, dim, n, (1e-5, 2e-5, 3e-5)[:dim], 41, density="blob")
    g = case.gvec
    valid = case.state[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1], g[0]:g[0] + case.n[0]]
    path = tmp_path / "plt00007"
    api.write_plotfile(path, case, valid, time=3.5e-9, step=7, prob_lo=(0.1, 0.2, 0.3))
    r = read_plotfile(path)
    nv = valid.shape[0]
    assert r["names"] == list(m.species) + list(api.PLASMA_VAR_NAMES)
    assert r["names"][nv - 1] == "ReducedEF" and len(r["names"]) == nv
    assert (r["dim"], r["time"], r["finest"], r["step"], r["level"], r["ngrid"], r["lstep"]) == (dim, 3.5e-9, 0, 7,
                                                                                              0, 1, 7)
    assert r["ltime"] == 3.5e-9 and r["coord"] == 0 and r["bwidth"] == 0
    hi = ",".join(str(v - 1) for v in case.n[:dim])
    zero = ",".join("0" * dim)
    assert r["domain"] == f"(({zero}) ({hi}) ({zero}))"
    for d in range(dim):
        assert r["dx"][d] == case.dx[d]
        assert r["prob_lo"][d] == (0.1, 0.2, 0.3)[d]
        assert r["prob_hi"][d] == pytest.approx((0.1, 0.2, 0.3)[d] + case.dx[d] * case.n[d], rel=1e-15)
        assert r["extents"][d][0] == r["prob_lo"][d]
    flat = np.ascontiguousarray(valid).reshape(nv, -1)
    assert np.array_equal(r["data"], flat.reshape(-1))
    assert r["mins"] == [float(v) for v in flat.min(axis=1)]
    assert r["maxs"] == [float(v) for v in flat.max(axis=1)]


def test_plotfile_refusals(tmp_path):
    m = mm.argon(10, 20261204)
    case = inputs.build_case(m, 2, (8, 8), (1e-5, 1e-5), 42, density="blob")
    g = case.gvec
    valid = case.state[:, g[2]:g[2] + 1, g[1]:g[1] + 8, g[0]:g[0] + 8]
    with pytest.raises(ValueError):
        api.write_plotfile(tmp_path / "p", case, valid, names=["a", "b"])
    from vidyut_b200 import _abi as abi
    with pytest.raises(abi.VidyutError):
        api.write_plotfile(tmp_path / "p", case, valid, names=["x"] * (valid.shape[0] - 1) + [""])


@pytest.mark.parametrize("dim,n", [(1, (30,)), (2, (12, 9)), (3, (6, 5, 4))])
def test_checkpoint_round_trip(tmp_path, dim, n):
    """Vidyut::WriteCheckpointFile's Header (title, finest level, istep / dt / t_new
    lines, box array) and the state read back bit for bit."""
    m = mm.argon(10, 20261204)
    case = inputs.build_case(m, dim, n, (1e-5,) * dim, 43, density="loguniform")
    g = case.gvec
    valid = np.ascontiguousarray(case.state[:, g[2]:g[2] + case.n[2], g[1]:g[1] + case.n[1],
                                            g[0]:g[0] + case.n[0]])
    path = tmp_path / "chk00042"
    api.write_checkpoint(path, case, valid, istep=42, dt=1.25e-12, time=5.25e-11)
    lines = (path / "Header").read_text().split("\n")
    assert lines[0] == "Checkpoint file for Vidyut" and lines[1] == "0"
    assert int(lines[2]) == 42 and float(lines[3]) == 1.25e-12 and float(lines[4]) == 5.25e-11
    assert lines[5] == "(1 0" and lines[7] == ")"
    st, lo, hi, d, istep, dt, time = api.read_checkpoint(path)
    assert (d, istep, dt, time) == (dim, 42, 1.25e-12, 5.25e-11)
    assert lo == (0, 0, 0) and hi == tuple(v - 1 for v in case.n)
    assert st.shape == valid.shape and np.array_equal(st, valid)
    assert (path / "Level_0" / "phi_H").exists()


def test_checkpoint_refusals(tmp_path):
    from vidyut_b200 import _abi as abi
    (tmp_path / "bad").mkdir()
    (tmp_path / "bad" / "Header").write_text("something else\n")
    with pytest.raises(abi.VidyutError):
        api.read_checkpoint(tmp_path / "bad")
    with pytest.raises(abi.VidyutError):
        api.read_checkpoint(tmp_path / "missing")


def test_restart_from_checkpoint_continues_the_run(tmp_path):
    """Two steps, a checkpoint, a restart from it and two more steps give the same
    state as four steps in one go (the C oracle steps the case; the restart refills
    the ghosts of species, EEN and ETEMP as the stepping does after each step)."""
    import oracle
    from vidyut_b200 import _abi as abi
    from vidyut_b200.inputs import MULTISTEP_PARAMS, fill_ghosts
    m = mm.synthetic(8, 40, 20261224)
    case = inputs.build_case(m, 2, (20, 14), (1e-5, 1e-5), 44, density="loguniform_smooth",
                             dens_range=(1e10, 1e18), te_range_ev=(0.3, 10.0), params=dict(MULTISTEP_PARAMS))
    prm = case.vd_params()
    port = oracle.Port(m)
    g = case.gvec
    valid = (slice(None), slice(g[2], g[2] + case.n[2]), slice(g[1], g[1] + case.n[1]),
             slice(g[0], g[0] + case.n[0]))
    four = oracle.run_steps(port, case, prm, 4)
    two = oracle.run_steps(port, case, prm, 2)
    api.write_checkpoint(tmp_path / "chk00002", case, two[valid], istep=2, dt=prm.dt, time=2 * prm.dt)
    st, _, _, _, istep, dt, time = api.read_checkpoint(tmp_path / "chk00002")
    assert (istep, dt, time) == (2, prm.dt, 2 * prm.dt)
    restored = case.state.copy()
    restored[valid] = st
    comps = list(range(m.ns)) + [abi.EEN(m.ns), abi.ETEMP(m.ns)]
    sub = np.ascontiguousarray(restored[comps])
    fill_ghosts(sub, case.dim, case.ghost, case.periodic)
    restored[comps] = sub
    assert np.array_equal(restored, two)
    again = oracle.run_steps(port, dataclasses.replace(case, state=restored), prm, 2)
    assert np.array_equal(again, four)
