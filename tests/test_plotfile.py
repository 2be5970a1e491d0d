"""Plotfile output (camr_write_plotfile, AMReX plotfile layout as
CAMR::writePlotFile writes it, Source/Utils/CAMR_io.cpp:408-565) and input.

* write -> read returns the state bit for bit, for several box chops;
* an independent parse of the files (this test's own reader of the AMReX
  layout: Header fields, the VisMF Cell_H box list / offsets / min / max,
  the FAB headers and the raw little-endian data) finds the same values;
* a level's state after GPU steps round-trips too (GPU).
"""
import re

import numpy as np
import pytest

from camr_b200 import hydro, native
from camr_b200 import problems as P

NAMES = ["density", "xmom", "ymom", "zmom", "rho_E", "rho_e", "Temp", "rho_F", "rho_A",
         "rho_P"]


def independent_read(path):
    """Parse a single-level plotfile without the library."""
    hdr = (path / "Header").read_text().split("\n")
    assert hdr[0] == "HyperCLaw-V1.1"
    nv = int(hdr[1])
    names = hdr[2:2 + nv]
    i = 2 + nv
    assert int(hdr[i]) == 3
    time = float(hdr[i + 1])
    assert int(hdr[i + 2]) == 0
    prob_lo = [float(x) for x in hdr[i + 3].split()]
    prob_hi = [float(x) for x in hdr[i + 4].split()]
    assert hdr[i + 5].strip() == ""
    dom = [int(x) for x in re.findall(r"-?\d+", hdr[i + 6])]
    step = int(hdr[i + 7].split()[0])
    dx = [float(x) for x in hdr[i + 8].split()]
    assert hdr[i + 9].strip() == "0" and hdr[i + 10].strip() == "0"
    lev, ngrid, t2 = hdr[i + 11].split()
    assert int(lev) == 0 and float(t2) == time
    ngrid = int(ngrid)
    assert int(hdr[i + 12]) == step
    ext = [[float(v) for v in hdr[i + 13 + g].split()] for g in range(3 * ngrid)]
    assert hdr[i + 13 + 3 * ngrid] == "Level_0/Cell"
    cell_h = (path / "Level_0" / "Cell_H").read_text().split("\n")
    assert cell_h[0] == "1" and cell_h[1] == "1" and int(cell_h[2]) == nv and cell_h[3] == "0"
    nb = int(cell_h[4].strip("(").split()[0])
    assert nb == ngrid
    boxes = [[int(x) for x in re.findall(r"-?\d+", cell_h[5 + b])] for b in range(nb)]
    assert cell_h[5 + nb] == ")" and int(cell_h[6 + nb]) == nb
    fabs = [cell_h[7 + nb + b].split() for b in range(nb)]
    data = (path / "Level_0" / "Cell_D_00000").read_bytes()
    n = [dom[3 + d] - dom[d] + 1 for d in range(3)]
    out = np.zeros((nv, n[2], n[1], n[0]))
    mins = [[float(v) for v in cell_h[9 + 2 * nb + b].rstrip(",").split(",")] for b in range(nb)]
    for b, (tag, fname, off) in enumerate(fabs):
        assert tag == "FabOnDisk:" and fname == "Cell_D_00000"
        off = int(off)
        end = data.index(b"\n", off)
        line = data[off:end].decode()
        assert line.startswith("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))")
        lo, hi = boxes[b][:3], boxes[b][3:6]
        assert line.endswith(f" {nv}")
        bn = [hi[d] - lo[d] + 1 for d in range(3)]
        cnt = bn[0] * bn[1] * bn[2]
        vals = np.frombuffer(data, dtype="<f8", count=cnt * nv, offset=end + 1)
        vals = vals.reshape(nv, bn[2], bn[1], bn[0])
        out[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = vals
        for c in range(nv):
            assert mins[b][c] == vals[c].min()
        # the extents in Header are the physical bounds of the box
        for d in range(3):
            elo, ehi = ext[3 * b + d]
            assert abs(elo - (prob_lo[d] + lo[d] * dx[d])) < 1e-12
            assert abs(ehi - (prob_lo[d] + (hi[d] + 1) * dx[d])) < 1e-12
    return {"names": names, "time": time, "step": step, "dom": dom, "dx": dx,
            "prob_hi": prob_hi, "state": out, "nboxes": nb}


@pytest.mark.parametrize("mgs", [(0, 0, 0), (8, 8, 8), (16, 8, 4)])
def test_plotfile_round_trip(tmp_path, native_lib, mgs):
    n = (24, 16, 16)
    dx = (1.0 / 24, 1.0 / 16, 1.0 / 16)
    s = P.random_smooth(n, seed=11)
    s[P.UTEMP] = np.linspace(300, 400, s[0].size).reshape(s[0].shape)
    geom = hydro.make_geom(n, dx=dx)
    path = tmp_path / "plt00007"
    hydro.write_plotfile(path, s, geom, (1.0, 1.0, 1.0), time=0.125, level_step=7,
                         max_grid_size=mgs)
    back, t, step = hydro.read_plotfile(path, geom)
    assert t == 0.125 and step == 7
    assert np.array_equal(back, s)
    ind = independent_read(path)
    assert ind["names"] == NAMES and ind["step"] == 7 and ind["time"] == 0.125
    assert ind["dom"][:6] == [0, 0, 0, 23, 15, 15]
    assert np.array_equal(ind["state"], s)
    assert ind["nboxes"] == len(hydro.level_boxes(n, mgs))


def test_plotfile_component_subset(tmp_path, native_lib):
    n = (8, 8, 8)
    s = P.random_smooth(n, seed=2)
    geom = hydro.make_geom(n)
    path = tmp_path / "plt_sub"
    hydro.write_plotfile(path, s, geom, (1.0, 1.0, 1.0), comps=[0, 6], names=["rho", "T"])
    ind = independent_read(path)
    assert ind["names"] == ["rho", "T"]
    assert np.array_equal(ind["state"][0], s[0]) and np.array_equal(ind["state"][1], s[6])
    back, _, _ = hydro.read_plotfile(path, geom, ncomp=2)
    assert np.array_equal(back[1], s[6])


def test_plotfile_rejects_bad_input(tmp_path, native_lib):
    geom = hydro.make_geom((8, 8, 8))
    with pytest.raises(native.CamrError):
        hydro.write_plotfile(tmp_path / "x", np.zeros((10, 8, 8, 8)), geom, (1, 1, 1),
                             comps=[12])
    with pytest.raises(native.CamrError):
        hydro.read_plotfile(tmp_path / "missing", geom)


def test_plotfile_readers_reject_more_components_than_nvar(tmp_path, native_lib):
    """A plotfile may repeat components (11 here); the readers fill NVAR-plane
    states, so they refuse ncomp > NVAR instead of writing past them."""
    n = (8, 8, 8)
    geom = hydro.make_geom(n)
    s = P.random_smooth(n, seed=3)
    comps = list(range(10)) + [0]
    path = tmp_path / "plt_11"
    hydro.write_plotfile(path, s, geom, (1, 1, 1), comps=comps,
                         names=NAMES + ["density_again"])
    assert independent_read(path)["names"][-1] == "density_again"
    for read in (lambda: hydro.read_plotfile(path, geom, ncomp=11),
                 lambda: hydro.read_plotfile_amr(path, geom, [((0, 0, 0), (3, 3, 3))], ncomp=11)):
        with pytest.raises(native.CamrError, match="ncomp exceeds NVAR"):
            read()


def test_plotfile_reader_rejects_damaged_box_count(tmp_path, native_lib):
    """A Cell_H whose box count is absurd (a damaged file) is refused with
    an error instead of sizing the box list from it."""
    n = (8, 8, 8)
    geom = hydro.make_geom(n)
    path = tmp_path / "plt_bad"
    hydro.write_plotfile(path, P.random_smooth(n, seed=4), geom, (1, 1, 1))
    cell_h = path / "Level_0" / "Cell_H"
    lines = cell_h.read_text().split("\n")
    assert lines[4].startswith("(")
    lines[4] = "(2147483647 0"
    cell_h.write_text("\n".join(lines))
    with pytest.raises(native.CamrError, match="bad box count"):
        hydro.read_plotfile(path, geom)


def read_level(path, lev, nv):
    """Boxes and per-box arrays of Level_<lev> (VisMF header + FAB data)."""
    cell_h = (path / f"Level_{lev}" / "Cell_H").read_text().split("\n")
    assert cell_h[0] == "1" and cell_h[1] == "1" and int(cell_h[2]) == nv and cell_h[3] == "0"
    nb = int(cell_h[4].strip("(").split()[0])
    boxes = [[int(x) for x in re.findall(r"-?\d+", cell_h[5 + b])] for b in range(nb)]
    fabs = [cell_h[7 + nb + b].split() for b in range(nb)]
    data = (path / f"Level_{lev}" / "Cell_D_00000").read_bytes()
    out = []
    for b, (tag, fname, off) in enumerate(fabs):
        assert tag == "FabOnDisk:" and fname == "Cell_D_00000"
        end = data.index(b"\n", int(off))
        assert data[int(off):end].decode().startswith("FAB ((8, (64 11 52 0 1 12 0 1023))")
        lo, hi = boxes[b][:3], boxes[b][3:6]
        bn = [hi[d] - lo[d] + 1 for d in range(3)]
        vals = np.frombuffer(data, dtype="<f8", count=nv * bn[0] * bn[1] * bn[2], offset=end + 1)
        out.append((lo, hi, vals.reshape(nv, bn[2], bn[1], bn[0])))
    return out


def test_two_level_plotfile(tmp_path, native_lib):
    """The AMR driver's two levels as one plotfile: the Header's finest
    level, refinement ratio, per-level domains, steps, cell sizes and grid
    extents, and both levels' data, parsed without the library."""
    n = (16, 16, 8)
    dx = (1.0 / 16, 1.0 / 16, 0.5 / 8)
    geom = hydro.make_geom(n, dx=dx, prob_hi=(1.0, 1.0, 0.5))
    s0 = P.random_smooth(n, seed=3)
    fine = [((4, 4, 2), (11, 19, 9)), ((20, 0, 0), (27, 7, 15))]
    rng = np.random.default_rng(9)
    parts = []
    for lo, hi in fine:
        bn = [hi[d] - lo[d] + 1 for d in range(3)]
        parts.append(rng.standard_normal((10, bn[2], bn[1], bn[0])))
    s1 = np.concatenate([p.ravel() for p in parts])
    path = tmp_path / "plt_amr"
    hydro.write_plotfile_amr(path, s0, s1, geom, (1.0, 1.0, 0.5), fine, time=0.25,
                             level_steps=(5, 10), max_grid_size=(8, 8, 8))
    hdr = (path / "Header").read_text().split("\n")
    assert hdr[0] == "HyperCLaw-V1.1" and int(hdr[1]) == 10 and hdr[2:12] == NAMES
    i = 12
    assert int(hdr[i]) == 3 and float(hdr[i + 1]) == 0.25 and int(hdr[i + 2]) == 1
    assert [float(x) for x in hdr[i + 4].split()] == [1.0, 1.0, 0.5]
    assert hdr[i + 5].split() == ["2"]
    doms = [[int(x) for x in m] for m in
            [re.findall(r"-?\d+", b) for b in re.findall(r"\(\([^)]*\) \([^)]*\) \([^)]*\)\)",
                                                        hdr[i + 6])]]
    assert doms[0][:6] == [0, 0, 0, 15, 15, 7] and doms[1][:6] == [0, 0, 0, 31, 31, 15]
    assert hdr[i + 7].split() == ["5", "10"]
    assert [float(x) for x in hdr[i + 8].split()] == list(dx)
    assert [float(x) for x in hdr[i + 9].split()] == [v / 2 for v in dx]
    assert hdr[i + 10] == "0" and hdr[i + 11] == "0"
    j = i + 12
    nb0 = len(hydro.level_boxes(n, (8, 8, 8)))
    assert hdr[j].split() == ["0", str(nb0), "0.25"] and hdr[j + 1] == "5"
    assert hdr[j + 2 + 3 * nb0] == "Level_0/Cell"
    j = j + 3 + 3 * nb0
    assert hdr[j].split() == ["1", "2", "0.25"] and hdr[j + 1] == "10"
    for b, (lo, hi) in enumerate(fine):
        for d in range(3):
            elo, ehi = (float(v) for v in hdr[j + 2 + 3 * b + d].split())
            assert abs(elo - lo[d] * dx[d] / 2) < 1e-15 and abs(ehi - (hi[d] + 1) * dx[d] / 2) < 1e-15
    assert hdr[j + 2 + 3 * len(fine)] == "Level_1/Cell"
    back0 = np.zeros_like(s0)
    for lo, hi, v in read_level(path, 0, 10):
        back0[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = v
    assert np.array_equal(back0, s0)
    lev1 = read_level(path, 1, 10)
    assert [(tuple(lo), tuple(hi)) for lo, hi, _ in lev1] == fine
    for (_, _, v), p in zip(lev1, parts):
        assert np.array_equal(v, p)


def test_two_level_plotfile_round_trip(tmp_path, native_lib):
    """write_plotfile_amr -> read_plotfile_amr returns both levels bit for
    bit; a hierarchy with other fine boxes is refused."""
    n = (8, 8, 8)
    geom = hydro.make_geom(n)
    s0 = P.random_smooth(n, seed=4)
    fine = [((0, 0, 0), (7, 5, 3)), ((10, 8, 6), (15, 15, 15))]
    rng = np.random.default_rng(5)
    cells = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in fine)
    s1 = rng.standard_normal(10 * cells)
    path = tmp_path / "plt_rt"
    hydro.write_plotfile_amr(path, s0, s1, geom, (1, 1, 1), fine, time=0.5, level_steps=(3, 6),
                             max_grid_size=(4, 4, 4))
    b0, b1, t, steps = hydro.read_plotfile_amr(path, geom, fine)
    assert np.array_equal(b0, s0) and np.array_equal(b1, s1)
    assert t == 0.5 and steps == (3, 6)
    with pytest.raises(native.CamrError):
        hydro.read_plotfile_amr(path, geom, [((0, 0, 0), (7, 5, 3))])
    with pytest.raises(native.CamrError):
        hydro.read_plotfile(path, geom)  # two levels: not a single-level plotfile
    # a single-level plotfile reads back through the two-level reader too
    hydro.write_plotfile(tmp_path / "plt_one", s0, geom, (1, 1, 1), time=0.25, level_step=2)
    c0, _, t1, st1 = hydro.read_plotfile_amr(tmp_path / "plt_one", geom, [])
    assert np.array_equal(c0, s0) and t1 == 0.25 and st1[0] == 2


def test_two_level_plotfile_rejects_fine_box_outside(tmp_path, native_lib):
    geom = hydro.make_geom((8, 8, 8))
    with pytest.raises(native.CamrError):
        hydro.write_plotfile_amr(tmp_path / "bad", np.zeros((10, 8, 8, 8)),
                                 np.zeros(10 * 8 ** 3), geom, (1, 1, 1),
                                 [((10, 10, 10), (17, 17, 17))])


@pytest.mark.gpu
def test_level_state_plotfile_restart(tmp_path):
    """A level's state written after GPU steps, read back and set into a new
    level, continues exactly as the original (restart from a plotfile that
    holds every state component)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    n = (32, 32, 32)
    s0 = P.blobs(n, tuple(1.0 / v for v in n), nblobs=3, seed=5)
    geom = hydro.make_geom(n)
    prm = native.default_params(ppm_type=1, cfl=0.7, fixed_dt=1e-3)
    a = hydro.Level(geom, prm)
    a.set_state(s0)
    a.init_finalize()
    a.advance(3)
    mid = a.get_state()
    hydro.write_plotfile(tmp_path / "chk", mid, geom, (1, 1, 1), time=3e-3, level_step=3)
    back, t, step = hydro.read_plotfile(tmp_path / "chk", geom)
    assert np.array_equal(back, mid) and step == 3
    a.advance(2)
    b = hydro.Level(geom, prm)
    b.set_state(back)
    b.advance(2)
    assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.gpu
def test_amr_hierarchy_two_level_plotfile(tmp_path):
    """Both levels of a GPU AMR run, written after a few coarse steps, parse
    back to exactly the states the hierarchy holds."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    n0 = (16, 16, 16)
    boxes = [((8, 8, 8), (23, 15, 15)), ((0, 16, 16), (7, 31, 23))]
    S0, S1 = P.amr_initial(n0, boxes, nblobs=3, r_min=0.1, r_max=0.2)
    geom = hydro.make_geom(n0)
    h = hydro.AmrHierarchy(geom, native.default_params(ppm_type=1, cfl=0.5), boxes)
    h.set_state(S0, S1)
    h.init_finalize()
    h.advance(2)
    c0, c1 = h.get_state()
    t0, t1 = h.clock()[:2]
    h.close()
    hydro.write_plotfile_amr(tmp_path / "plt_amr_gpu", c0, c1, geom, (1, 1, 1), boxes,
                             time=t0, level_steps=(2, 4))
    back0 = np.zeros_like(c0)
    for lo, hi, v in read_level(tmp_path / "plt_amr_gpu", 0, 10):
        back0[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = v
    assert np.array_equal(back0, c0)
    lev1 = read_level(tmp_path / "plt_amr_gpu", 1, 10)
    assert np.array_equal(np.concatenate([v.ravel() for _, _, v in lev1]), np.asarray(c1).ravel())
    assert t0 > 0 and abs(t0 - t1) <= 1e-12 * t0


def parse_checkpoint_header(path):
    """This test's own reading of the checkpoint Header layout."""
    L = (path / "Header").read_text().split("\n")
    assert L[0] == "CheckPointVersion_1.0" and int(L[1]) == 3
    out = {"time": float(L[2]), "max_level": int(L[3]), "finest": int(L[4]),
           "dt_level": [float(x) for x in L[7].split()],
           "n_cycle": [int(x) for x in L[9].split()],
           "level_steps": [int(x) for x in L[10].split()]}
    out["state_files"] = [x for x in L if x.startswith("Level_") and x.endswith("SD_0_New_MF")]
    return out


@pytest.mark.parametrize("levels", [1, 2])
def test_checkpoint_round_trip(tmp_path, native_lib, levels):
    """camr_write_checkpoint -> camr_read_checkpoint returns states, times,
    dts and level steps bit for bit; the Header and the VisMF data parse
    independently; CPUtime holds the CPU time."""
    n = (16, 8, 8)
    geom = hydro.make_geom(n)
    s0 = P.random_smooth(n, seed=8)
    fine = [((0, 0, 0), (7, 5, 3)), ((16, 8, 6), (23, 15, 15))] if levels == 2 else []
    rng = np.random.default_rng(1)
    cells = sum((h[0] - l[0] + 1) * (h[1] - l[1] + 1) * (h[2] - l[2] + 1) for l, h in fine)
    s1 = rng.standard_normal(10 * cells) if fine else None
    t = (0.25, 0.25) if levels == 2 else 0.25
    dt = (1e-3, 5e-4) if levels == 2 else 1e-3
    steps = (7, 14) if levels == 2 else 7
    path = tmp_path / "chk00007"
    hydro.write_checkpoint(path, geom, (1, 0.5, 0.5), s0, t, dt, steps, S1=s1, fine_boxes=fine,
                           max_grid_size=(8, 8, 8), cpu_time=12.5)
    b0, b1, tt, dd, ss = hydro.read_checkpoint(path, geom, fine)
    assert np.array_equal(b0, s0)
    if fine:
        assert np.array_equal(b1, s1)
    assert tt == (t if levels == 2 else (t,)) and dd == (dt if levels == 2 else (dt,))
    assert ss == (steps if levels == 2 else (steps,))
    h = parse_checkpoint_header(path)
    assert h["finest"] == levels - 1 and h["n_cycle"] == [1, 2][:levels]
    assert h["state_files"] == [f"Level_{l}/SD_0_New_MF" for l in range(levels)]
    assert float((path / "CPUtime").read_text()) == 12.5
    got = np.zeros_like(s0)
    for lo, hi, v in read_level_mf(path, 0, "SD_0_New_MF"):
        got[:, lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] = v
    assert np.array_equal(got, s0)
    with pytest.raises(native.CamrError):
        hydro.read_checkpoint(path, geom, [] if fine else [((0, 0, 0), (1, 1, 1))])


def read_level_mf(path, lev, mf):
    cell_h = (path / f"Level_{lev}" / f"{mf}_H").read_text().split("\n")
    nb = int(cell_h[4].strip("(").split()[0])
    boxes = [[int(x) for x in re.findall(r"-?\d+", cell_h[5 + b])] for b in range(nb)]
    fabs = [cell_h[7 + nb + b].split() for b in range(nb)]
    out = []
    for b, (tag, fname, off) in enumerate(fabs):
        assert tag == "FabOnDisk:" and fname == f"{mf}_D_00000"
        data = (path / f"Level_{lev}" / fname).read_bytes()
        end = data.index(b"\n", int(off))
        lo, hi = boxes[b][:3], boxes[b][3:6]
        bn = [hi[d] - lo[d] + 1 for d in range(3)]
        vals = np.frombuffer(data, dtype="<f8", count=10 * bn[0] * bn[1] * bn[2], offset=end + 1)
        out.append((lo, hi, vals.reshape(10, bn[2], bn[1], bn[0])))
    return out


@pytest.mark.gpu
def test_level_checkpoint_restart_continues_exactly(tmp_path):
    """Checkpoint after 4 steps (device dts), restart into a new level with
    camr_level_restart: the next steps (computeNewDt against the checkpoint's
    dt) give the same states and dts as the run that never stopped."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    n = (24, 24, 24)
    s0 = P.blobs(n, tuple(1.0 / v for v in n), nblobs=3, seed=5, r_min=0.1, r_max=0.2)
    geom = hydro.make_geom(n)
    prm = native.default_params(ppm_type=1, cfl=0.7)
    a = hydro.Level(geom, prm)
    a.set_state(s0)
    a.init_finalize()
    a.advance(4)
    mid = a.get_state()
    dt4 = a.last_dt()
    hydro.write_checkpoint(tmp_path / "chk4", geom, (1, 1, 1), mid, 0.0, dt4, 4)
    a.advance(3)
    want = a.get_state()
    want_dt = a.last_dt()
    a.close()
    back, _, _, dd, ss = hydro.read_checkpoint(tmp_path / "chk4", geom)
    b = hydro.Level(geom, prm)
    b.set_state(back)
    b.restart(dd[0], ss[0])
    b.advance(3)
    assert b.last_dt() == want_dt
    assert np.array_equal(b.get_state(), want)
    b.close()


@pytest.mark.gpu
def test_amr_checkpoint_restart_continues_exactly(tmp_path):
    """Two-level checkpoint after 3 coarse steps, restart into a new
    hierarchy with camr_amr_restart: the next coarse steps (CFL estimates
    of the restored states, computeNewDt against the checkpoint's dts) give
    the same states and clock as the run that never stopped."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    n0 = (16, 16, 16)
    boxes = [((8, 8, 8), (23, 15, 15)), ((0, 16, 16), (7, 31, 23))]
    S0, S1 = P.amr_initial(n0, boxes, nblobs=3, r_min=0.1, r_max=0.2)
    geom = hydro.make_geom(n0)
    prm = native.default_params(ppm_type=1, cfl=0.5)
    a = hydro.AmrHierarchy(geom, prm, boxes)
    a.set_state(S0, S1)
    a.init_finalize()
    a.advance(3)
    c0, c1 = a.get_state()
    t0, t1, d0, d1 = a.clock()
    hydro.write_checkpoint(tmp_path / "chk3", geom, (1, 1, 1), c0, (t0, t1), (d0, d1), (3, 6),
                           S1=c1, fine_boxes=boxes)
    a.advance(2)
    want0, want1 = a.get_state()
    want_clock = a.clock()
    a.close()
    b0, b1, tt, dd, ss = hydro.read_checkpoint(tmp_path / "chk3", geom, boxes)
    assert tt == (t0, t1) and dd == (d0, d1) and ss == (3, 6)
    b = hydro.AmrHierarchy(geom, prm, boxes)
    b.set_state(b0, b1)
    b.restart((tt[0], tt[1], dd[0], dd[1]), ss[0])
    b.advance(2)
    got0, got1 = b.get_state()
    assert b.clock() == want_clock
    assert np.array_equal(got0, want0)
    assert np.array_equal(np.asarray(got1).ravel(), np.asarray(want1).ravel())
    b.close()
