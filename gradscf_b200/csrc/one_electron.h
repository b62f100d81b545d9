// One-electron integral launch interface (kernels in one_electron.cu).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace b200jk {

struct OneArgs {
  const int4* pair_info;  // (A, B, ...) work-shell pairs, l_A >= l_B
  const int* pairs;       // pair ids of this class
  int npairs;
  const int4* ws_info;    // (cart offset, l, mol, out offset)
  const double4* ws_xyz;
  const double2* prim;    // (exponent, normalised coefficient)
  const int* prim_off;    // per work shell, plus sentinel
  const double4* atoms;   // (x, y, z, charge) per global atm row
  const int* mol_atm_off;
  const int* mol_natm;
  const long long* mol_base;  // Cartesian block offsets
  const int* mol_n;
  const int* ws_atm;      // global atm row of each work shell's centre
  Tables tb;
  // integrals: raw Cartesian S, T, V blocks written to out_s/out_t/out_v
  double *out_s, *out_t, *out_v;
  // gradient: raw Cartesian densities and the (natm, 3) output
  const double *dm, *wm;
  double* grad;
};

// Launch the value (deriv = false: raw Cartesian S, T, V blocks) or gradient
// (deriv = true: D- and W-weighted centre derivatives) kernel of pair class pc.
void launch_one_electron(int pc, bool deriv, const OneArgs& a, cudaStream_t st);

}  // namespace b200jk
