"""Reading a CAMR inputs file (camr_b200/inputs.py): ParmParse syntax, the
reference's parameter names and defaults, its boundary words and their
periodicity checks (Source/CAMR.cpp:80-157), the base geometry."""
import pytest

from camr_b200 import inputs, native

SOD_X = """
# Sod problem along x (written for this test)
max_step  = 200
stop_time = 0.2

geometry.is_periodic = 0 1 1
geometry.prob_lo     = 0.0 0.0 0.0
geometry.prob_hi     = 1.0 0.125 0.125
amr.n_cell           = 128 16 16
amr.max_grid_size    = 32

CAMR.lo_bc = Inflow   Interior Interior    # x: inflow, y and z periodic
CAMR.hi_bc = Outflow  Interior Interior
CAMR.do_mol   = 0
CAMR.ppm_type = 1
CAMR.cfl      = 0.5
CAMR.small_dens = 1.d-10
CAMR.cfl      = 0.6                        # the last definition wins
eos.gamma     = 1.67
CAMR.redistribution_type = "StateRedist"
"""


def test_sod_inputs(native_lib):
    t = inputs.parse(SOD_X, overrides=["max_step=3", "CAMR.ppm_type = 0"])
    assert t["max_step"] == ["3"] and t["stop_time"] == ["0.2"]
    p = inputs.hydro_params(t)
    assert p.do_mol == 0 and p.ppm_type == 0 and p.cfl == 0.6
    assert p.small_dens == 1e-10 and p.eos_gamma == 1.67
    d = native.default_params()
    # names the file leaves out keep the reference table's defaults
    for f in ("difmag", "small", "plm_iorder", "use_flattening", "change_max", "max_dt",
              "riemann_solver", "eb_weights_type"):
        assert getattr(p, f) == getattr(d, f), f
    g, mgs = inputs.geometry(t)
    assert mgs == (32, 32, 32)
    assert [g.dom_hi[k] for k in range(3)] == [127, 15, 15]
    assert [g.is_periodic[k] for k in range(3)] == [0, 1, 1]
    assert [g.bc_lo[k] for k in range(3)] == [1, 0, 0]
    assert [g.bc_hi[k] for k in range(3)] == [2, 0, 0]
    assert g.dx[0] == 1.0 / 128 and g.dx[1] == 0.125 / 16
    assert inputs.redistribution(t) == 2


def test_defaults_are_the_reference_table(native_lib):
    """With no CAMR names at all every field is camr_default_params', whose
    values are the reference's table (Source/Params/_cpp_parameters)."""
    p = inputs.hydro_params(inputs.parse(""))
    want = dict(do_mol=0, ppm_type=0, plm_iorder=4, use_pslope=0, use_flattening=1,
                transverse_reset_density=1, dual_energy_update_E_from_e=1,
                allow_negative_energy=0, allow_small_energy=1, add_grav_src=1,
                eb_weights_type=2, difmag=0.1, small=1.e-8, small_dens=1.e-7, small_temp=1.e2,
                small_pres=1.e-200, dual_energy_eta1=1.0, dual_energy_eta2=1.0e-4,
                const_grav=0.0, cfl=0.8, init_shrink=1.0, change_max=1.1, fixed_dt=-1.0,
                initial_dt=-1.0, max_dt=1.e200)
    for k, v in want.items():
        assert getattr(p, k) == v, k
    assert inputs.redistribution({}) == 1


@pytest.mark.parametrize("text,match", [
    ("CAMR.lo_bc = Wall Interior Interior\nCAMR.hi_bc = Outflow Interior Interior",
     "Wrong boundary condition word"),
    ("CAMR.lo_bc = Outflow Outflow Interior\nCAMR.hi_bc = Outflow Interior Interior",
     "periodic in direction 1"),
    ("CAMR.lo_bc = Interior Interior Interior\nCAMR.hi_bc = Outflow Interior Interior",
     "interior bc in direction 0"),
    ("CAMR.lo_bc = Outflow Interior\nCAMR.hi_bc = Outflow Interior Interior",
     "expected 3 words"),
])
def test_boundary_words_checked_as_the_reference_does(native_lib, text, match):
    base = "geometry.is_periodic = 0 1 1\ngeometry.prob_hi = 1 1 1\namr.n_cell = 8 8 8\n"
    with pytest.raises(ValueError, match=match):
        inputs.geometry(inputs.parse(base + text))


@pytest.mark.parametrize("text,match", [
    ("CAMR.do_mol = yes", "not an integer"),
    ("CAMR.cfl = fast", "not a real number"),
    ("CAMR.cfl = 0.5 0.6", "expected one value"),
    ("CAMR.cfl", "expected 'name = value'"),
    ("CAMR.cfl =", "has no value"),
])
def test_bad_values_are_refused(native_lib, text, match):
    with pytest.raises(ValueError, match=match):
        inputs.hydro_params(inputs.parse(text))


def test_geometry_needs_its_sizes(native_lib):
    with pytest.raises(ValueError, match="amr.n_cell is required"):
        inputs.geometry(inputs.parse("geometry.prob_hi = 1 1 1"))
    t = inputs.parse("amr.n_cell = 8 8 8\ngeometry.prob_hi = 1 1 1\ngeometry.is_periodic = 1 1 1\n"
                     "CAMR.lo_bc = Interior Interior Interior\n"
                     "CAMR.hi_bc = Interior Interior Interior\namr.max_grid_size = 4 8 8")
    g, mgs = inputs.geometry(t)
    assert mgs == (4, 8, 8) and g.dx[2] == 1.0 / 8
    t = inputs.parse("amr.n_cell = 8 8 8\ngeometry.prob_hi = 1 1 1\ngeometry.is_periodic = 1 1 1\n"
                     "CAMR.lo_bc = Interior Interior Interior\n"
                     "CAMR.hi_bc = Interior Interior Interior")
    assert inputs.geometry(t)[1] is None


def test_unused_names_are_listed():
    t = inputs.parse(SOD_X + "amr.max_level = 2\nCAMR.do_react = 0\namr.plot_int = 10\n")
    assert inputs.unused(t) == ["CAMR.do_react", "amr.max_level", "amr.plot_int",
                                "max_step", "stop_time"]
    assert "CAMR.cfl" not in inputs.unused(t) and "eos.gamma" not in inputs.unused(t)


def test_quotes_keep_blanks_and_hashes():
    t = inputs.parse('CAMR.job_name = "run #3 of 5"   # a comment\nx = a "b c" d')
    assert t["CAMR.job_name"] == ["run #3 of 5"]
    assert t["x"] == ["a", "b c", "d"]


def test_distributed_level_from_inputs(native_lib):
    """A box-distributed level built from an inputs file (constructed only:
    no device work)."""
    import torch

    from camr_b200 import distributed as D
    L = D.DistributedLevel.from_inputs(inputs.parse(SOD_X), device=torch.device("cpu"))
    assert L.n == (128, 16, 16) and len(L.boxes) == 4
    assert L.params.ppm_type == 1 and L.params.cfl == 0.6
    assert [L.geom.bc_lo[k] for k in range(3)] == [1, 0, 0]
    with pytest.raises(ValueError, match="max_grid_size"):
        D.DistributedLevel.from_inputs(inputs.parse(SOD_X.replace("amr.max_grid_size", "#")),
                                       device=torch.device("cpu"))
