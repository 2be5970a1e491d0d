// Stand-in for AMReX's EBCellFlag (test infrastructure of the oracle): the
// cell type and its connectivity to the 26 neighbours, in this encoding
// (shared with camr_b200's EB kernels, camr_b200/csrc/eb.cu):
//   bits 0-1  type: 0 regular, 1 single-valued (cut), 3 covered
//   bit 2 + (di+1) + 3 (dj+1) + 9 (dk+1)   connected to neighbour (di,dj,dk)
#pragma once
#include "AMReX_shim_core.H"

namespace amrex {

class EBCellFlag {
 public:
  EBCellFlag() = default;
  explicit EBCellFlag(unsigned int w) : w_(w) {}
  bool isRegular() const { return (w_ & 3u) == 0u; }
  bool isSingleValued() const { return (w_ & 3u) == 1u; }
  bool isMultiValued() const { return (w_ & 3u) == 2u; }
  bool isCovered() const { return (w_ & 3u) == 3u; }
  bool isConnected(int di, int dj, int dk) const {
    return (w_ >> (2 + (di + 1) + 3 * (dj + 1) + 9 * (dk + 1))) & 1u;
  }
  bool isConnected(const IntVect& iv) const { return isConnected(iv[0], iv[1], iv[2]); }
  unsigned int getValue() const { return w_; }

 private:
  unsigned int w_ = 0;
};

}  // namespace amrex
