// Forwarding header of the oracle's AMReX stand-in (EB build).
#pragma once
#include "AMReX_shim_core.H"
#include "AMReX_EBCellFlag.H"
