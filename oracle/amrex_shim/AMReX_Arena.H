// Forwarding header of the oracle's AMReX stand-in.
#pragma once
#include "AMReX_shim_core.H"
