"""CPU oracle for the hydro advance (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
package, and only as the checker.  It wraps two shared libraries with one C
interface (oracle_abi.h):

* ``restate``: the repo's CPU restatement (hydro_restate.cpp + level_driver.cpp)
* ``ref``: the reference's own per-box hydro sources compiled against the
  AMReX stand-in in amrex_shim/ (ref_glue.cpp + level_driver.cpp), built into
  oracle/_ref/ by ``make ref`` where the reference sources are available;
  ``make ref`` also builds the reference's EB hydro (with AMREX_USE_EB) with
  the EB per-box entry point and the EB level driver (ref_glue_eb.cpp).
"""
from .binding import (  # noqa: F401
    NVAR, QVAR, NGDNV, Params, Level, load, default_params, make_level,
    hydro_box, advance, advance_fixed_dt, est_dt, init_finalize,
    expand_state, clean_state, amr_run, build, lib_path, lib_path_eb, hydro_box_eb,
    eb_advance, eb_init_finalize, ref_ctoprim, ref_hydro_box_full,
    count_flops, lib_path_flops, fluxreg_reflux, avg_down, fine_fill_ghosts,
)
