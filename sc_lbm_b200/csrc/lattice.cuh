// lattice.cuh -- D2Q9 constants and small device helpers shared by all kernels.
//
// Lattice (include/lbm.h:118-128 and include/fluid.h:279-283 of the reference):
//   c_x = {0, 1, 0, -1, 0, 1, -1, -1, 1}, c_y = {0, 0, 1, 0, -1, 1, 1, -1, -1}
//   Shan-Chen weights  w_sc = {0, 1/9 x4, 1/36 x4}
//   equilibrium weights w = {4/9, 1/9 x4, 1/36 x4}
//   bounce-back partner bb(i) = {3,4,1,2,7,8,5,6} for i = 1..8 (the opposite
//   direction).
// Written as constexpr functions so fully unrolled loops fold them into
// immediates.
#pragma once
#include <cstddef>
#include <cstdint>

namespace sclbm {

__host__ __device__ constexpr int cx(int i)
{
    return (i == 1 || i == 5 || i == 8) ? 1 : ((i == 3 || i == 6 || i == 7) ? -1 : 0);
}
__host__ __device__ constexpr int cy(int i)
{
    return (i == 2 || i == 5 || i == 6) ? 1 : ((i == 4 || i == 7 || i == 8) ? -1 : 0);
}
// opposite direction (bb_rules, include/lbm.h:124)
__host__ __device__ constexpr int opp(int i)
{
    return i == 0 ? 0 : (i <= 4 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5);
}
// Shan-Chen weights as double constants (1.0/9, 1.0/36 exactly as the reference)
__host__ __device__ constexpr double w_sc(int i) { return i == 0 ? 0.0 : (i <= 4 ? 1.0 / 9 : 1.0 / 36); }
// equilibrium weights (wrt0, wrt1, wrt2 of include/fluid.h:282)
__host__ __device__ constexpr double w_eq(int i)
{
    return i == 0 ? 4.0 / 9.0 : (i <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
}

static_assert(opp(1) == 3 && opp(2) == 4 && opp(3) == 1 && opp(4) == 2, "bb axis");
static_assert(opp(5) == 7 && opp(6) == 8 && opp(7) == 5 && opp(8) == 6, "bb diagonal");

// periodic wrap for offsets in [-1, n]
__host__ __device__ inline int wrap1(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

} // namespace sclbm
