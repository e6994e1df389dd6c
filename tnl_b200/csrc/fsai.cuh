// fsai.cuh -- the FSAI preconditioner data shared by fsai.cu and lfsai.cu.
#pragma once

#include "internal.cuh"

namespace tnlb {

// Lower-triangular pattern + values of G and its transpose, both as CSR
// segments the SpMV kernels run on; the CSR copy of A the values come from.
struct Fsai {
   int32_t n = 0;
   tnlb_real real = TNLB_F64;
   bool two_factor = false;      // g = G_L, gt = G_U (not G_L^T)
   tnlb_segments* g = nullptr;   // CSR of G
   tnlb_segments* gt = nullptr;  // CSR of G^T
   DeviceBuffer g_cols, g_vals, gt_cols, gt_vals, gt_src, tmp;
   DeviceBuffer a_rp, a_cols, a_vals;
   ~Fsai()
   {
      delete g;
      delete gt;
   }
};

}  // namespace tnlb
