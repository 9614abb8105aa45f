// Host-only print-out of the ring kernel's shared-memory layout
// (sc_lbm_b200/csrc/fused_ring.cuh, RingLayout) for the forms the library
// launches; tests/test_ring_layout_cpu.py checks its alignments and budgets.
// Compiled by nvcc and run on the CPU: no kernel is launched.
#include <cstdio>

#include "fused_ring.cuh"

using namespace sclbm;

template <typename S, typename T, int R, int W, bool HB> static void row(const char *name)
{
    using L = RingLayout<S, T, R, W, HB>;
    std::printf("%s %d %d %d %d %zu %zu %zu %zu %zu %zu %zu %zu\n", name, R, W, HB ? 1 : 0, L::A, L::comp,
                L::halo, L::stage, L::pops, L::edge_at, L::edge, L::bars, L::bytes);
}

int main()
{
    // name R W HB A comp halo stage pops edge_at edge bars bytes
    row<double, double, 2, 128, true>("ring_fp64");
    row<float, float, 4, 128, true>("ring_fp32");
    row<float, float, 4, 128, false>("ring_fp32_edge");
    row<__half, float, 4, 128, true>("ring_fp16");
    row<double, double, 3, 128, true>("batch_fp64");
    row<float, float, 3, 128, true>("batch_fp32");
    row<float, float, 3, 64, true>("batch_fp32_w64");
    row<__half, float, 5, 128, true>("batch_fp16");
    return 0;
}
