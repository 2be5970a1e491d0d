"""A CAMR inputs file (AMReX ParmParse syntax) read into this library's
parameter and geometry structures, under the reference's own names.

Syntax, as ParmParse reads it: `prefix.name = value value ...`, `#` starts a
comment, values are separated by blanks, double quotes keep blanks inside a
string, and a name defined twice takes its last definition.  Command-line
style overrides (`max_step=3`) come after the file and win over it.

Names:

* `CAMR.<name>` for every field of camr_hydro_params that the reference's
  table holds (Source/Params/_cpp_parameters; read at Source/CAMR.cpp:66-79),
  with the table's defaults (those of camr_default_params) for names the
  file leaves out; `CAMR.riemann_solver` (0 = the reference's two-shock
  solver, 1 = HLLC) and `eos.gamma` (the reference's compile-time
  EOS::gamma, Source/EOS/GammaLaw/EOS.H:16) are the two names this library
  adds;
* `CAMR.lo_bc` / `CAMR.hi_bc`: the boundary words Interior, Inflow,
  Outflow, Symmetry, SlipWall, NoSlipWall, checked against the periodic
  directions as the reference checks them (Source/CAMR.cpp:80-157);
* `amr.n_cell`, `amr.max_grid_size` (one value or three),
  `geometry.prob_lo`, `geometry.prob_hi`, `geometry.is_periodic`;
* `CAMR.redistribution_type` (FluxRedist, StateRedist, NoRedist) as the
  `redist` argument of the EB calls.
"""
import shlex

from . import native

INT_FIELDS = ("do_mol", "ppm_type", "plm_iorder", "use_pslope", "use_flattening",
              "transverse_reset_density", "dual_energy_update_E_from_e",
              "allow_negative_energy", "allow_small_energy", "add_grav_src",
              "riemann_solver", "eb_weights_type")
REAL_FIELDS = ("difmag", "small", "small_dens", "small_temp", "small_pres",
               "dual_energy_eta1", "dual_energy_eta2", "const_grav", "cfl", "init_shrink",
               "change_max", "fixed_dt", "initial_dt", "max_dt")
REDIST = {"NoRedist": 0, "FluxRedist": 1, "StateRedist": 2}


def _strip_comment(line):
    """The line up to its first `#` outside double quotes."""
    quoted = False
    for k, ch in enumerate(line):
        if ch == '"':
            quoted = not quoted
        elif ch == "#" and not quoted:
            return line[:k]
    return line


def parse(text, overrides=()):
    """{name: [values]} from ParmParse text plus `name=value ...` overrides."""
    table = {}

    def take(line, where):
        line = _strip_comment(line).strip()
        if not line:
            return
        if "=" not in line:
            raise ValueError(f"{where}: expected 'name = value', got {line!r}")
        name, rest = line.split("=", 1)
        name = name.strip()
        if not name or any(c.isspace() for c in name):
            raise ValueError(f"{where}: bad name {name!r}")
        vals = shlex.split(rest, comments=False, posix=True)
        if not vals:
            raise ValueError(f"{where}: {name} has no value")
        table[name] = vals

    for k, line in enumerate(text.splitlines()):
        take(line, f"line {k + 1}")
    for o in overrides:
        take(o, f"override {o!r}")
    return table


def read(path, overrides=()):
    with open(path) as f:
        return parse(f.read(), overrides)


def _real(name, s):
    try:
        return float(s.replace("d", "e").replace("D", "e"))
    except ValueError:
        raise ValueError(f"{name}: {s!r} is not a real number") from None


def _int(name, s):
    try:
        return int(s)
    except ValueError:
        raise ValueError(f"{name}: {s!r} is not an integer") from None


def _one(table, name):
    v = table[name]
    if len(v) != 1:
        raise ValueError(f"{name}: expected one value, got {len(v)}")
    return v[0]


def _three(table, name, conv, default=None, allow_one=False):
    if name not in table:
        if default is None:
            raise ValueError(f"{name} is required")
        return tuple(default)
    v = table[name]
    if allow_one and len(v) == 1:
        v = v * 3
    if len(v) != 3:
        raise ValueError(f"{name}: expected 3 values, got {len(v)}")
    return tuple(conv(name, x) for x in v)


def hydro_params(table):
    """camr_hydro_params from CAMR.<name> (and eos.gamma), the table's
    defaults for the names left out."""
    p = native.default_params()
    for f in INT_FIELDS:
        if "CAMR." + f in table:
            setattr(p, f, _int("CAMR." + f, _one(table, "CAMR." + f)))
    for f in REAL_FIELDS:
        if "CAMR." + f in table:
            setattr(p, f, _real("CAMR." + f, _one(table, "CAMR." + f)))
    if "eos.gamma" in table:
        p.eos_gamma = _real("eos.gamma", _one(table, "eos.gamma"))
    return p


def boundary_words(table, periodic):
    """(bc_lo, bc_hi) as the library's BC numbers, checked as
    CAMR::read_params checks them: Interior exactly on periodic sides."""
    out = []
    for side in ("lo_bc", "hi_bc"):
        name = "CAMR." + side
        if name not in table:
            raise ValueError(f"{name} is required")
        words = table[name]
        if len(words) != 3:
            raise ValueError(f"{name}: expected 3 words, got {len(words)}")
        nums = []
        for d, w in enumerate(words):
            if w not in native.BC:
                raise ValueError(f"Wrong boundary condition word in {side}, please use: "
                                 "Interior, Inflow, Outflow, Symmetry, SlipWall, NoSlipWall")
            b = native.BC[w]
            if periodic[d] and b != 0:
                raise ValueError(f"periodic in direction {d} but {side} is not Interior")
            if not periodic[d] and b == 0:
                raise ValueError(f"interior bc in direction {d} but not periodic")
            nums.append(b)
        out.append(tuple(nums))
    return out[0], out[1]


def geometry(table):
    """(camr_geom, max_grid_size) of the base level; max_grid_size is None
    when the file leaves it out."""
    from . import hydro
    n = _three(table, "amr.n_cell", _int)
    if any(v <= 0 for v in n):
        raise ValueError("amr.n_cell: every extent must be positive")
    mgs = (_three(table, "amr.max_grid_size", _int, allow_one=True)
           if "amr.max_grid_size" in table else None)
    lo = _three(table, "geometry.prob_lo", _real, default=(0.0, 0.0, 0.0))
    hi = _three(table, "geometry.prob_hi", _real)
    if any(hi[d] <= lo[d] for d in range(3)):
        raise ValueError("geometry.prob_hi must exceed geometry.prob_lo")
    per = _three(table, "geometry.is_periodic", _int, default=(0, 0, 0))
    bc_lo, bc_hi = boundary_words(table, per)
    g = hydro.make_geom(n, is_periodic=per, bc_lo=bc_lo, bc_hi=bc_hi, prob_lo=lo, prob_hi=hi)
    return g, mgs


def redistribution(table):
    """The EB calls' `redist` argument from CAMR.redistribution_type
    (default FluxRedist, as in the reference's table)."""
    w = _one(table, "CAMR.redistribution_type") if "CAMR.redistribution_type" in table \
        else "FluxRedist"
    if w not in REDIST:
        raise ValueError(f"CAMR.redistribution_type: {w!r} is not one of {sorted(REDIST)}")
    return REDIST[w]


READ_NAMES = (tuple("CAMR." + f for f in INT_FIELDS + REAL_FIELDS)
              + ("eos.gamma", "CAMR.lo_bc", "CAMR.hi_bc", "CAMR.redistribution_type",
                 "amr.n_cell", "amr.max_grid_size", "geometry.prob_lo", "geometry.prob_hi",
                 "geometry.is_periodic"))


def unused(table):
    """The names of the file that none of this module's readers act on (run
    control, tagging, plotting, reactions ...), sorted: what a CAMR run of
    the same file would do that this library leaves to its caller."""
    return sorted(k for k in table if k not in READ_NAMES)
