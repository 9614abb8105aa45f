// fused_step.cuh -- the fused Shan-Chen time step (kernel b) and the density
// pass (kernel a), templated on storage type S, compute type T and the
// specialisation flags (volume force present, solid nodes present).
//
// One launch performs one complete time step of the reference driver sequence
//   compute_density x2            src/fluid.cpp:175-183
//   compute_fluid_repulsive_...   src/lbm.cpp:144-206
//   compute_equilibrium_velocities src/lbm.cpp:209-272
//   collide(f1, f2)               src/lbm.cpp:291-312 (+ src/fluid.cpp:246-278)
//   [add_volume_force]            src/lbm.cpp:315-340
//   stream(geom, f1, f2)          src/lbm.cpp:387-435
// reading the populations once and writing them once.
//
// Register-tile variant.  A CTA of TX threads owns W = TX-2 interior columns
// and tile_y rows.  Thread t handles column xb-1+t; threads 0 and TX-1 are
// halo columns that only produce a density.  The CTA marches up its rows: in
// iteration r it loads row r's populations into registers, reduces them to the
// density, puts density and mask into a 4-row shared-memory ring, synchronises
// once, then collides row r-1 using the 3x3 density stencil from the ring and
// pushes the post-collision populations to their destinations (half-way
// bounce-back at solid neighbours).  Rows yb-1 and yb+tile_y are halo rows
// (density only).  Every destination slot has exactly one writer, so the kernel
// is race free with separate input and output buffers.
//
// FP64 (EXACT) follows the reference's operation order term by term and is
// compiled with -fmad=false, so its populations are bit-identical to the
// serial reference.  The shifted forms (T = float) store d_i = f_i - w_i*rho_ref
// and evaluate the same physics in deviation form in FP32.
//
// Node indices are 32-bit (a lattice has fewer than 2^32 nodes); the per
// population base pointers fout[k] + i*N depend only on kernel arguments, so
// they are computed once per thread.
#pragma once
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>

#include "internal.h"
#include "lattice.cuh"

namespace sclbm {

// specialisation flags of the fused kernels
constexpr int KF_FORCE = 1; // a volume force is added to at least one component
constexpr int KF_SOLID = 2; // the lattice has solid nodes
// with KF_SOLID: solid lanes run the collision alongside the fluid ones (no
// branch around it) and store zeros into their own slots, so every lane of a
// warp issues the same instructions and every slot is written each step
constexpr int KF_UNIFORM = 4;

template <typename S> struct Store;
template <> struct Store<double> {
    static __device__ __forceinline__ double ld(const double *p) { return __ldg(p); }
    static __device__ __forceinline__ void st(double *p, double v) { *p = v; }
};
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float *p) { return __ldg(p); }
    static __device__ __forceinline__ void st(float *p, float v) { *p = v; }
};
template <> struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ void st(__half *p, float v) { *p = __float2half_rn(v); }
};

// Bulk prefetch of [p, p + bytes) into L2 (p and bytes multiples of 16): one
// instruction brings a whole row segment of a population array closer before
// the per-thread loads of a later row iteration ask for it.
__device__ __forceinline__ void prefetch_l2_bulk(const void *p, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// equal_floats(r, 0.0, 1e-16) of include/utils.h:145-150
template <typename T> __device__ __forceinline__ bool rho_is_zero(T r)
{
    T a = r < T(0) ? -r : r;
    T m = T(1);
    if (m < a) m = a;
    return a <= T(1e-16) * m;
}

// exact FP64 equilibrium, src/fluid.cpp:254-276 (operation order kept)
__device__ __forceinline__ void feq_exact(double r, double ux, double uy, double fe[9])
{
    const double rt0 = w_eq(0) * r, rt1 = w_eq(1) * r, rt2 = w_eq(5) * r;
    const double uxsq = ux * ux, uysq = uy * uy;
    const double u5 = ux + uy, u6 = -ux + uy, u7 = -ux - uy, u8 = ux - uy;
    const double usq = uxsq + uysq;
    fe[0] = rt0 * (1.0 - 1.5 * usq);
    fe[1] = rt1 * (1.0 + 3.0 * ux + 4.5 * uxsq - 1.5 * usq);
    fe[2] = rt1 * (1.0 + 3.0 * uy + 4.5 * uysq - 1.5 * usq);
    fe[3] = rt1 * (1.0 - 3.0 * ux + 4.5 * uxsq - 1.5 * usq);
    fe[4] = rt1 * (1.0 - 3.0 * uy + 4.5 * uysq - 1.5 * usq);
    fe[5] = rt2 * (1.0 + 3.0 * u5 + 4.5 * u5 * u5 - 1.5 * usq);
    fe[6] = rt2 * (1.0 + 3.0 * u6 + 4.5 * u6 * u6 - 1.5 * usq);
    fe[7] = rt2 * (1.0 + 3.0 * u7 + 4.5 * u7 * u7 - 1.5 * usq);
    fe[8] = rt2 * (1.0 + 3.0 * u8 + 4.5 * u8 * u8 - 1.5 * usq);
}

// A population as the lattice will hold it: FP16 storage rounds each value,
// and the rest population's remainder (mass_closing_rest) is taken from the
// rounded values (FP16 Laplace droplet, 150 steps: density error 1.6e-2
// against 3.9e-2 from the unrounded values, for 3 % of the FP16 step time).
template <typename S> __device__ __forceinline__ float stored_value(float v)
{
    if constexpr (sizeof(S) == 2) return __half2float(__float2half_rn(v));
    else return v;
}

// Rest population of a shifted-form node chosen so that the node's stored
// populations sum to what the collision conserves -- the incoming
// populations' sum plus the volume force's sum -- up to the rounding of this
// one value:  d*_0 = d_0 + sum_{i>=1} (d_i - d*_i) [+ sum_i F_i].  In exact
// arithmetic it equals the BGK rest population.  In float it closes two
// systematic leaks: the equilibrium weights rounded to float sum to
// 1 + 7.5e-9 (computing d*_0 like the others scaled every node's deviation by
// that each step, ~1e-4 of the mass over 20,000 steps), and the node density
// is a rounded nine-term sum whose error is the same at every node of a
// uniform bulk.  Near equilibrium d_i - d*_i is small and nearly exact, so
// the remainder is accurate.  d: incoming values; v[1..8]: the outgoing
// values as they will be stored.
template <typename Row>
__device__ __forceinline__ float mass_closing_rest(const Row &d, const float (&v)[9], float force_sum)
{
    const float a = (float(d[1]) - v[1]) + (float(d[3]) - v[3]);
    const float b = (float(d[2]) - v[2]) + (float(d[4]) - v[4]);
    const float c = (float(d[5]) - v[5]) + (float(d[7]) - v[7]);
    const float e = (float(d[6]) - v[6]) + (float(d[8]) - v[8]);
    return float(d[0]) + (((a + b) + (c + e)) + force_sum);
}

// shifted-form equilibrium deviation: w_i*(drho + rho*(3cu + 4.5cu^2 - 1.5u^2))
__device__ __forceinline__ float feq_dev(int i, float drho, float r, float ux, float uy, float usq15)
{
    const float cu = float(cx(i)) * ux + float(cy(i)) * uy;
    const float poly = fmaf(cu, fmaf(4.5f, cu, 3.0f), -usq15);
    return float(w_eq(i)) * fmaf(r, poly, drho);
}

// Packed FP32 pairs (sm_100 FFMA2 / FADD2 / FMUL2): in the float-arithmetic
// collision x holds component 0 and y component 1.  Each lane rounds exactly
// like the scalar operation (__fmaf_rn, __fadd_rn, __fmul_rn, a - b), so code
// written on pairs gives the scalar sequence's results bit for bit with half
// the arithmetic instructions.
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    unsigned long long pa, pb, pd;
    asm("mov.b64 %0, {%1, %2};" : "=l"(pa) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(pb) : "f"(b.x), "f"(b.y));
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(pd) : "l"(pa), "l"(pb));
    float2 d;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(d.x), "=f"(d.y) : "l"(pd));
    return d;
}
// one 64-bit read of a PairParams member
__device__ __forceinline__ float2 pair_of(const float (&p)[2])
{
    return *reinterpret_cast<const float2 *>(p);
}

// Both components' densities of one node, 0.0 + f_0 + ... + f_8 in that
// order (src/fluid.cpp:177-181); float arithmetic on packed pairs
template <typename T> __device__ __forceinline__ void node_density(const T (&f)[2][9], T &r0, T &r1)
{
    if constexpr (sizeof(T) == 4) {
        float2 s = f2(0.f);
#pragma unroll
        for (int i = 0; i < 9; ++i) s = add2(s, make_float2(f[0][i], f[1][i]));
        r0 = s.x;
        r1 = s.y;
    } else {
        T s0 = T(0), s1 = T(0);
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            s0 += f[0][i];
            s1 += f[1][i];
        }
        r0 = s0;
        r1 = s1;
    }
}

// The two components' densities of one node side by side, so a stencil read
// fetches both with one 8- (16-) byte shared-memory load.
template <typename T> struct Vec2;
template <> struct Vec2<float> {
    using type = float2;
    static __device__ __forceinline__ float2 make(float a, float b) { return make_float2(a, b); }
};
template <> struct Vec2<double> {
    using type = double2;
    static __device__ __forceinline__ double2 make(double a, double b) { return make_double2(a, b); }
};
template <typename T> using V2 = typename Vec2<T>::type;

// Density/mask stencil around one node: rows below (0), at (1) and above (2)
// the node, read at columns c-1, c, c+1; r[.][col] = (rho_0, rho_1).
template <typename T> struct Stencil {
    const V2<T> *r[3];
    const uint8_t *m[3];
    int c;
};

// 32-bit indices of a node (nb[0]) and of its periodic neighbours along c_i
struct Nbr {
    uint32_t nb[9];
};

__device__ __forceinline__ Nbr make_nbr(const int nx, const int x, const int xl, const int xr,
                                        const int yc, const int yd, const int yu)
{
    const uint32_t rc = (uint32_t)yc * (uint32_t)nx, rd = (uint32_t)yd * (uint32_t)nx,
                   ru = (uint32_t)yu * (uint32_t)nx;
    Nbr n;
#pragma unroll
    for (int i = 0; i < 9; ++i)
        n.nb[i] = (cy(i) == 0 ? rc : (cy(i) > 0 ? ru : rd)) +
                  (uint32_t)(cx(i) == 0 ? x : (cx(i) > 0 ? xr : xl));
    return n;
}

// Push one post-collision population: to the neighbour along c_i when it is a
// fluid node, else back into the opposite direction at the node itself.  The
// destination is selected, not branched on, so warps with both kinds of
// nodes issue one store per population.
// Element offsets i*N + node in 32 bits (one integer multiply-add per access)
// when the nine arrays of a component hold fewer than 2^32 elements; WIDE
// kernels, launched for larger lattices, compute them in 64 bits.
template <bool WIDE> using Off = std::conditional_t<WIDE, size_t, uint32_t>;
template <bool WIDE> __device__ __forceinline__ Off<WIDE> elem(int i, size_t N, uint32_t node)
{
    return (Off<WIDE>)i * (Off<WIDE>)N + (Off<WIDE>)node;
}
inline bool needs_wide_offsets(size_t N) { return 9 * (unsigned long long)N >= (1ull << 32); }

template <typename S, typename T, bool SOLID, bool WIDE = false>
__device__ __forceinline__ void push_one(const Fused2Args<S, T> &a, const int k, const int i,
                                         const T v, const uint32_t nf, const Nbr &n)
{
    if (i == 0 || !SOLID) {
        Store<S>::st(a.fout[k] + elem<WIDE>(i, a.N, n.nb[i]), v);
    } else {
        // nf is 0 or 1: the destination is masked in, which leaves the
        // compiler no select to turn into a divergent branch
        using O = Off<WIDE>;
        const O to = elem<WIDE>(i, a.N, n.nb[i]), back = elem<WIDE>(opp(i), a.N, n.nb[0]);
        Store<S>::st(a.fout[k] + (back ^ ((to ^ back) & (O(0) - O(nf)))), v);
    }
}

// The same push with the value already in the storage type (FP16: the
// rounded value the mass closure used, stored without converting again).
template <typename S, bool SOLID, bool WIDE = false, typename T>
__device__ __forceinline__ void push_one_raw(const Fused2Args<S, T> &a, const int k, const int i,
                                             const S v, const uint32_t nf, const Nbr &n)
{
    if (i == 0 || !SOLID) {
        a.fout[k][elem<WIDE>(i, a.N, n.nb[i])] = v;
    } else {
        using O = Off<WIDE>;
        const O to = elem<WIDE>(i, a.N, n.nb[i]), back = elem<WIDE>(opp(i), a.N, n.nb[0]);
        a.fout[k][back ^ ((to ^ back) & (O(0) - O(nf)))] = v;
    }
}

// Collide the node n.nb[0] from its populations f[k][i] (registers or shared
// memory) and the density stencil, then push the results: the reference
// sequence of src/lbm.cpp:177-204 (repulsive force), :250-269 (equilibrium
// velocity), src/fluid.cpp:254-276 + src/lbm.cpp:305-311 (equilibrium, BGK),
// :333-337 (volume force), :404-427 (stream with half-way bounce-back).
template <typename S, typename T, int FLAGS, bool WIDE = false, typename Pops>
__device__ __forceinline__ void collide_push(const Fused2Args<S, T> &a, const Pops &f,
                                             const Stencil<T> &st, const Nbr &n)
{
    constexpr bool EXACT = sizeof(T) == 8;
    constexpr bool FORCE = (FLAGS & KF_FORCE) != 0, SOLID = (FLAGS & KF_SOLID) != 0;
    constexpr bool UNIFORM = SOLID && (FLAGS & KF_UNIFORM) != 0;
    const uint32_t node = n.nb[0];
    // a solid lane of the uniform form treats every neighbour as solid: its
    // nine stores then land in its own slots, and carry zeros
    const bool self_fluid = !SOLID || st.m[1][st.c] != 0;
    if (SOLID && !UNIFORM && !self_fluid) {
        // solid node: the reference's stream leaves zeros (src/lbm.cpp:431-434);
        // on the domain path both buffers already hold them
        if (!a.solids_zero) {
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int i = 0; i < 9; ++i) Store<S>::st(a.fout[k] + elem<WIDE>(i, a.N, node), T(0));
        }
        return;
    }
    // nf[i] = 1 when the neighbour along c_i is a fluid node (mask bytes are 0 or 1)
    uint32_t nf[9];
    T p0[9], p1[9];
    const uint32_t self_u = SOLID ? (uint32_t)st.m[1][st.c] : 1u;
#pragma unroll
    for (int i = 1; i < 9; ++i) {
        const int sl = cy(i) + 1;
        const int col = st.c + cx(i);
        nf[i] = SOLID ? (uint32_t)st.m[sl][col] & (UNIFORM ? self_u : 1u) : 1u;
        const V2<T> v = st.r[sl][col];
        p0[i] = v.x;
        p1[i] = v.y;
    }
    nf[0] = 1u;
    const V2<T> self = st.r[1][st.c];
    const T psi0 = self.x, psi1 = self.y;
    if constexpr (EXACT) {
        // repulsive force, src/lbm.cpp:177-204
        // (selects, not branches: the sums take exactly the reference's terms)
        double F0x = 0.0, F0y = 0.0, F1x = 0.0, F1y = 0.0, Sx = 0.0, Sy = 0.0;
#pragma unroll
        for (int i = 1; i < 9; ++i) {
            const double wcx = w_sc(i) * cx(i), wcy = w_sc(i) * cy(i);
            const bool f = nf[i] != 0u;
            F0x = f ? F0x + wcx * p1[i] : F0x;
            F0y = f ? F0y + wcy * p1[i] : F0y;
            F1x = f ? F1x + wcx * p0[i] : F1x;
            F1y = f ? F1y + wcy * p0[i] : F1y;
            Sx = f ? Sx : Sx + wcx; // solid sums, src/lbm.cpp:131-134
            Sy = f ? Sy : Sy + wcy;
        }
        F0x *= a.c[0].gf * psi0;
        F0y *= a.c[0].gf * psi0;
        F1x *= a.c[1].gf * psi1;
        F1y *= a.c[1].gf * psi1;
        // momentum, src/lbm.cpp:250-255
        double j0x = 0.0, j0y = 0.0, j1x = 0.0, j1y = 0.0;
#pragma unroll
        for (int i = 0; i < 9; ++i) {
            j0x += f[0][i] * double(cx(i));
            j0y += f[0][i] * double(cy(i));
            j1x += f[1][i] * double(cx(i));
            j1y += f[1][i] * double(cy(i));
        }
        const double o0 = a.c[0].omega, o1 = a.c[1].omega;
        const double ucx = (j0x * o0 + j1x * o1) / (psi0 * o0 + psi1 * o1);
        const double ucy = (j0y * o0 + j1y * o1) / (psi0 * o0 + psi1 * o1);
        const double psi[2] = {psi0, psi1};
        const double Fx[2] = {F0x, F1x}, Fy[2] = {F0y, F1y};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            double ux, uy;
            if (!rho_is_zero(psi[k])) { // src/lbm.cpp:262-269
                double fsx, fsy;
                if (a.solid_from_mask) {
                    fsx = a.c[k].gs_neg * Sx;
                    fsy = a.c[k].gs_neg * Sy;
                } else {
                    fsx = a.fsx[k][node];
                    fsy = a.fsy[k][node];
                }
                const double io = a.c[k].inv_omega;
                ux = ucx + Fx[k] * io / psi[k] + fsx * io;
                uy = ucy + Fy[k] * io / psi[k] + fsy * io;
            } else {
                ux = a.uex_old[k] ? a.uex_old[k][node] : 0.0;
                uy = a.uey_old[k] ? a.uey_old[k][node] : 0.0;
            }
            double fe[9];
            feq_exact(psi[k], ux, uy, fe);
            const double om = a.c[k].omega, omm = a.c[k].one_m_omega;
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                double v = omm * f[k][i] + om * fe[i];
                if constexpr (FORCE) {
                    if (a.c[k].force_on) v += a.c[k].force[i];
                }
                if constexpr (UNIFORM) v = self_fluid ? v : 0.0;
                push_one<S, T, SOLID, WIDE>(a, k, i, v, nf[i], n);
            }
        }
    } else {
        // shifted form: the stencil holds rho - rho_ref, and 0 at solid nodes, so
        // the sums over fluid neighbours run over all neighbours without tests.
        // Both components advance side by side in packed pairs (x: component 0,
        // y: component 1); every lane takes the scalar operation sequence.
        const PairParams<T> &pc = a.pc;
        // Ps.x = sum_i w c_i drho_0(nbr), Ps.y = sum_i w c_i drho_1(nbr)
        float2 Psx = f2(0.f), Psy = f2(0.f);
        float Sx = 0.f, Sy = 0.f;
#pragma unroll
        for (int i = 1; i < 9; ++i) {
            const float wcx = float(w_sc(i) * cx(i)), wcy = float(w_sc(i) * cy(i));
            const float2 q = make_float2(p0[i], p1[i]);
            if (cx(i)) Psx = fma2(f2(wcx), q, Psx);
            if (cy(i)) Psy = fma2(f2(wcy), q, Psy);
            if constexpr (SOLID) {
                if (cx(i)) Sx += nf[i] ? 0.f : wcx;
                if (cy(i)) Sy += nf[i] ? 0.f : wcy;
            }
        }
        const float2 RR = pair_of(pc.rho_ref);
        const float2 DR = make_float2(psi0, psi1);
        const float2 R = add2(RR, DR); // rho = rho_ref + drho
        // each component feels the other's neighbours: sum over fluid
        // neighbours of w c psi_other = Ps_other - rho_ref_other * S
        float2 Ax = make_float2(Psx.y, Psx.x), Ay = make_float2(Psy.y, Psy.x);
        if constexpr (SOLID) {
            const float2 nRR = make_float2(-RR.y, -RR.x);
            Ax = fma2(nRR, f2(Sx), Ax);
            Ay = fma2(nRR, f2(Sy), Ay);
        }
        const float2 G = mul2(pair_of(pc.gf), R);
        const float2 Fx = mul2(G, Ax), Fy = mul2(G, Ay);
        // direction i of both components
        auto fp = [&](int i) { return make_float2(float(f[0][i]), float(f[1][i])); };
        const float2 Jx = add2(add2(sub2(fp(1), fp(3)), sub2(fp(5), fp(6))), sub2(fp(8), fp(7)));
        const float2 Jy = sub2(add2(sub2(fp(2), fp(4)), add2(fp(5), fp(6))), add2(fp(7), fp(8)));
        const float2 OM = pair_of(pc.omega);
        const float inv_den = __fdividef(1.0f, fmaf(R.x, OM.x, R.y * OM.y));
        const float ucx = fmaf(Jx.x, OM.x, Jx.y * OM.y) * inv_den;
        const float ucy = fmaf(Jy.x, OM.x, Jy.y * OM.y) * inv_den;
        const float2 IO = pair_of(pc.inv_omega);
        const float2 IR = mul2(IO, make_float2(__fdividef(1.0f, R.x), __fdividef(1.0f, R.y)));
        float2 Ux, Uy;
        if constexpr (SOLID) {
            const float2 GS = pair_of(pc.gs_neg);
            Ux = fma2(Fx, IR, fma2(mul2(GS, f2(Sx)), IO, f2(ucx)));
            Uy = fma2(Fy, IR, fma2(mul2(GS, f2(Sy)), IO, f2(ucy)));
        } else {
            Ux = fma2(Fx, IR, f2(ucx));
            Uy = fma2(Fy, IR, f2(ucy));
        }
        // a component of (numerically) zero density keeps the common velocity
        if (rho_is_zero(R.x)) {
            Ux.x = ucx;
            Uy.x = ucy;
        }
        if (rho_is_zero(R.y)) {
            Ux.y = ucx;
            Uy.y = ucy;
        }
        // BGK toward the shifted equilibrium w_i (drho + rho poly_i),
        // poly_i = 3 c.u + 4.5 (c.u)^2 - 1.5 u^2, written as
        // d*_i = (1 - omega) d_i + w_i (omega rho poly_i + omega drho); the
        // directions i and opp(i) share 4.5 (c.u)^2 - 1.5 u^2
        const float2 NUSQ = mul2(f2(-1.5f), fma2(Ux, Ux, mul2(Uy, Uy))); // -1.5 u^2
        const float2 OMM = pair_of(pc.one_m_omega);
        const float2 AM = mul2(OM, R), BM = mul2(OM, DR);
        const float2 Ux45 = mul2(f2(4.5f), Ux), Uy45 = mul2(f2(4.5f), Uy);
        // Store direction i's post-collision pair (volume force added) and
        // return d_i - d*_i as stored, the rest population's share
        auto emit = [&](int i, float2 V) -> float2 {
            if constexpr (FORCE) V = add2(V, pair_of(pc.force[i]));
            if constexpr (sizeof(S) == 2) {
                // FP16: round once, store the halves as they are, close the
                // mass with the rounded values
                const __half2 H = __float22half2_rn(V);
                __half h0 = __low2half(H), h1 = __high2half(H);
                if constexpr (UNIFORM) {
                    h0 = self_fluid ? h0 : __float2half_rn(0.f);
                    h1 = self_fluid ? h1 : __float2half_rn(0.f);
                }
                push_one_raw<S, SOLID, WIDE>(a, 0, i, h0, nf[i], n);
                push_one_raw<S, SOLID, WIDE>(a, 1, i, h1, nf[i], n);
                return sub2(fp(i), __half22float2(H));
            } else {
                float v0 = V.x, v1 = V.y;
                if constexpr (UNIFORM) {
                    v0 = self_fluid ? v0 : 0.f;
                    v1 = self_fluid ? v1 : 0.f;
                }
                push_one<S, T, SOLID, WIDE>(a, 0, i, v0, nf[i], n);
                push_one<S, T, SOLID, WIDE>(a, 1, i, v1, nf[i], n);
                return sub2(fp(i), V);
            }
        };
        // directions i and j = opp(i) along cu; returns (d_i - d*_i) + (d_j - d*_j)
        auto pair = [&](int i, int j, float2 CU, float2 CU45) -> float2 {
            const float2 SQ = fma2(CU45, CU, NUSQ);
            const float2 Vi = fma2(f2(float(w_eq(i))), fma2(AM, fma2(f2(3.f), CU, SQ), BM), mul2(OMM, fp(i)));
            const float2 Vj = fma2(f2(float(w_eq(j))), fma2(AM, fma2(f2(-3.f), CU, SQ), BM), mul2(OMM, fp(j)));
            const float2 Di = emit(i, Vi);
            return add2(Di, emit(j, Vj));
        };
        const float2 D13 = pair(1, 3, Ux, Ux45);                            // c = (+-1, 0)
        const float2 D24 = pair(2, 4, Uy, Uy45);                            // c = (0, +-1)
        const float2 D57 = pair(5, 7, add2(Ux, Uy), add2(Ux45, Uy45));     // c = +-(1, 1)
        const float2 D68 = pair(6, 8, sub2(Uy, Ux), sub2(Uy45, Ux45));     // c = +-(-1, 1)
        // the rest population closes the node's mass (sum_i d*_i = sum_i d_i + sum_i F_i):
        // d*_0 = d_0 + sum_{i>=1} (d_i - d*_i) [+ sum_i F_i]
        const float2 FS = FORCE ? pair_of(pc.force_sum) : f2(0.f);
        float2 V0 = add2(fp(0), add2(add2(add2(D13, D24), add2(D57, D68)), FS));
        if constexpr (sizeof(S) == 2) {
            const __half2 H = __float22half2_rn(V0);
            __half h0 = __low2half(H), h1 = __high2half(H);
            if constexpr (UNIFORM) {
                h0 = self_fluid ? h0 : __float2half_rn(0.f);
                h1 = self_fluid ? h1 : __float2half_rn(0.f);
            }
            push_one_raw<S, SOLID, WIDE>(a, 0, 0, h0, nf[0], n);
            push_one_raw<S, SOLID, WIDE>(a, 1, 0, h1, nf[0], n);
        } else {
            if constexpr (UNIFORM) {
                V0.x = self_fluid ? V0.x : 0.f;
                V0.y = self_fluid ? V0.y : 0.f;
            }
            push_one<S, T, SOLID, WIDE>(a, 0, 0, V0.x, nf[0], n);
            push_one<S, T, SOLID, WIDE>(a, 1, 0, V0.y, nf[0], n);
        }
    }
}

// shared-memory view of one node's populations in a ring: f[k][i]
template <typename S, typename T, int P> struct RingPops {
    const S *base; // stage base + column
    struct Row {
        const S *p;
        __device__ __forceinline__ T operator[](int i) const { return T(p[i * P]); }
    };
    __device__ __forceinline__ Row operator[](int k) const { return Row{base + k * 9 * P}; }
};

// ---------------------------------------------------------------------------
// kernel b, register-tile variant
// ---------------------------------------------------------------------------
// One tile: interior columns [xb, xb+W) and rows [yb, yb+tile_y) of domain a.
// PF: threads 0..17 prefetch, PF_DIST rows ahead, the row segments of the 18
// population arrays into L2 (cp.async.bulk.prefetch), so the row loads of the
// later iteration find them there.
constexpr int PF_DIST = 2;

// Loads one row ahead (single pass): iteration r issues the loads of row r+1
// into a third register buffer before it reduces row r (loaded during the
// previous iteration) and collides row r-1, so a row's load latency overlaps a
// whole iteration and each warp keeps two rows of loads in flight.  This is
// what keeps the memory pipe full when part of a warp's lanes sit on solid
// nodes and issue no loads.  Same arithmetic as fused2_tile, same results.
template <typename S, typename T, int TX, int FLAGS>
__device__ __forceinline__ void fused2_tile_ahead(const Fused2Args<S, T> &a, const int xb,
                                                  const int yb, V2<T> (&s_rho)[4][TX],
                                                  uint8_t (&s_m)[4][TX])
{
    constexpr bool SOLID = (FLAGS & KF_SOLID) != 0;
    constexpr int W = TX - 2;
    const int t = threadIdx.x;
    const int nx = a.nx, ny = a.ny;
    const int ncol = min(W, nx - xb);
    const int nrow = min(a.tile_y, (a.row_end > 0 ? a.row_end : ny) - yb);
    const bool active = t <= ncol + 1;
    const bool interior = t >= 1 && t <= ncol;
    const int x = wrap1(xb - 1 + t, nx);
    const int xl = wrap1(x - 1, nx), xr = wrap1(x + 1, nx);
    auto node_of = [&](int r) { return (uint32_t)wrap1(yb + r, ny) * (uint32_t)nx + (uint32_t)x; };

    // populations of row r into buf (solid nodes hold zeros on the domain path)
    auto load_row = [&](int r, uint8_t m, T(&buf)[2][9]) {
        if (active && (!SOLID || m || !a.solids_zero)) {
            const uint32_t node = node_of(r);
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    buf[k][i] = T(Store<S>::ld(a.fin[k] + elem<false>(i, a.N, node)));
        }
    };

    // masks of rows r (mr) and r+1 (mr1) at iteration r; row r+2's is loaded there
    uint8_t mr = 1, mr1 = 1;
    if (SOLID && active) {
        mr = a.mask[node_of(-1)];
        mr1 = a.mask[node_of(0)];
    }

    T A[2][9], B[2][9], C[2][9];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < 9; ++i) A[k][i] = B[k][i] = C[k][i] = T(0);
    load_row(-1, mr, B);

    // iteration r: load row r+1 into L, reduce row r (D), collide row r-1 (P)
    auto body = [&](const int r, T(&L)[2][9], const T(&D)[2][9], const T(&P)[2][9]) {
        uint8_t mr2 = 1;
        if (SOLID && active && r + 2 <= nrow) mr2 = a.mask[node_of(r + 2)];
        if (r + 1 <= nrow) load_row(r + 1, mr1, L);
        T rho[2] = {T(0), T(0)};
        uint8_t m = 0;
        if (active) {
            node_density(D, rho[0], rho[1]);
            m = SOLID ? mr : 1;
            if (SOLID && !m) rho[0] = rho[1] = T(0);
        }
        const int slot = (r + 1) & 3;
        s_rho[slot][t] = Vec2<T>::make(rho[0], rho[1]);
        s_m[slot][t] = m;
        __syncthreads();
        if (r >= 1 && interior) {
            const int sc = r & 3, sm = (r - 1) & 3, sp = (r + 1) & 3;
            const int yc = wrap1(yb + r - 1, ny);
            const Stencil<T> st{{s_rho[sm], s_rho[sc], s_rho[sp]},
                                {s_m[sm], s_m[sc], s_m[sp]}, t};
            const Nbr n = make_nbr(nx, x, xl, xr, yc, wrap1(yc - 1, ny), wrap1(yc + 1, ny));
            collide_push<S, T, FLAGS>(a, P, st, n);
        }
        mr = mr1;
        mr1 = mr2;
    };
    // three rows per trip: the buffers rotate roles (L, D, P) instead of copying
    for (int r = -1; r <= nrow; r += 3) {
        body(r, A, B, C);
        if (r + 1 <= nrow) body(r + 1, C, A, B);
        if (r + 2 <= nrow) body(r + 2, B, C, A);
    }
}

// Compacted fluid lanes (lattices with solid nodes).  Loading a row stays one
// column per thread, but the row's populations are also published in shared
// memory together with a per-warp ballot of its fluid interior columns; the
// collision of that row (next iteration) is then done by threads 0..F-1 for
// its F fluid nodes, thread j taking the j-th one.  Warps whose lanes would
// all sit on solid nodes skip the collision and the remaining warps run full,
// instead of every warp carrying its solid lanes idle through the collision.
// Three population slots: iteration q publishes row q while row q-1 is being
// collided, and row q+1 (written by a thread already in iteration q+1) never
// lands on row q-1's slot.  Same arithmetic per node, same single writes.
// bit index of the n-th (0-based) set bit of v; v has more than n bits set
__device__ __forceinline__ int nth_set_bit(uint32_t v, int n)
{
    int pos = 0;
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) {
        const uint32_t lo = v & ((1u << sh) - 1u);
        const int c = __popc(lo);
        if (n >= c) {
            n -= c;
            v >>= sh;
            pos += sh;
        } else {
            v = lo;
        }
    }
    return pos;
}

template <typename S, typename T, int TX> struct CompactSmem {
    T pop[3][18][TX];          // populations of the last rows, [k*9 + i][column]
    uint32_t ballot[3][TX / 32]; // fluid interior columns of those rows, per warp
};

template <typename S, typename T, int TX, int FLAGS>
__device__ __forceinline__ void fused2_tile_compact(const Fused2Args<S, T> &a, const int xb,
                                                    const int yb, V2<T> (&s_rho)[4][TX],
                                                    uint8_t (&s_m)[4][TX],
                                                    CompactSmem<S, T, TX> &cs, const bool down)
{
    static_assert((FLAGS & KF_SOLID) != 0, "compaction is for lattices with solid nodes");
    constexpr int W = TX - 2, NW = TX / 32;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nx = a.nx, ny = a.ny;
    const int ncol = min(W, nx - xb);
    const int nrow = min(a.tile_y, (a.row_end > 0 ? a.row_end : ny) - yb);
    const bool active = t <= ncol + 1;
    const bool interior = t >= 1 && t <= ncol;
    const int x = wrap1(xb - 1 + t, nx);
    auto phys = [&](int q) { return down ? nrow - 1 - q : q; };

    uint8_t m_ahead = 1;
    if (active) m_ahead = a.mask[(uint32_t)wrap1(yb + phys(-1), ny) * (uint32_t)nx + (uint32_t)x];

    T cur[2][9];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < 9; ++i) cur[k][i] = T(0);

    for (int q = -1; q <= nrow; ++q) {
        const int r = phys(q);
        const int y = wrap1(yb + r, ny);
        const int slot = (q + 1) & 3, ps = (q + 1) % 3;
        T rho[2] = {T(0), T(0)};
        uint8_t m = 0;
        if (active) {
            const uint32_t node = (uint32_t)y * (uint32_t)nx + (uint32_t)x;
            m = m_ahead;
            if (q < nrow)
                m_ahead = a.mask[(uint32_t)wrap1(yb + phys(q + 1), ny) * (uint32_t)nx + (uint32_t)x];
            if (m || !a.solids_zero) {
#pragma unroll
                for (int k = 0; k < 2; ++k)
#pragma unroll
                    for (int i = 0; i < 9; ++i)
                        cur[k][i] = T(Store<S>::ld(a.fin[k] + elem<false>(i, a.N, node)));
            }
            node_density(cur, rho[0], rho[1]);
            if (!m) rho[0] = rho[1] = T(0);
            if (!m && interior && !a.solids_zero && r >= 0 && r < nrow) {
                // caller-owned arrays: the reference's stream leaves zeros at solids
#pragma unroll
                for (int k = 0; k < 2; ++k)
#pragma unroll
                    for (int i = 0; i < 9; ++i) Store<S>::st(a.fout[k] + elem<false>(i, a.N, node), T(0));
            }
        }
        s_rho[slot][t] = Vec2<T>::make(rho[0], rho[1]);
        s_m[slot][t] = m;
        const bool work = interior && m && r >= 0 && r < nrow;
        if (work) {
#pragma unroll
            for (int k = 0; k < 2; ++k)
#pragma unroll
                for (int i = 0; i < 9; ++i) cs.pop[ps][k * 9 + i][t] = cur[k][i];
        }
        const uint32_t bal = __ballot_sync(0xffffffffu, work);
        if (lane == 0) cs.ballot[ps][warp] = bal;
        __syncthreads();

        if (q >= 1) {
            // the j-th fluid interior column of row phys(q-1), j = t
            const int pp = q % 3;
            int j = t, w = 0;
            uint32_t b = 0;
#pragma unroll
            for (int v = 0; v < NW; ++v) {
                const uint32_t bv = cs.ballot[pp][v];
                const int c = __popc(bv);
                if (w == v && j >= c) {
                    j -= c;
                    ++w;
                } else if (w == v) {
                    b = bv;
                }
            }
            if (w < NW) {
                const int col = w * 32 + nth_set_bit(b, j);
                const int xc = wrap1(xb - 1 + col, nx);
                const int s_old = (q - 1) & 3, sc = q & 3, s_new = (q + 1) & 3;
                const int sb = down ? s_new : s_old, sa = down ? s_old : s_new;
                const int yc = wrap1(yb + phys(q - 1), ny);
                const Stencil<T> st{{s_rho[sb], s_rho[sc], s_rho[sa]},
                                    {s_m[sb], s_m[sc], s_m[sa]}, col};
                const Nbr n = make_nbr(nx, xc, wrap1(xc - 1, nx), wrap1(xc + 1, nx), yc,
                                       wrap1(yc - 1, ny), wrap1(yc + 1, ny));
                const RingPops<T, T, TX> f{&cs.pop[pp][0][col]};
                collide_push<S, T, FLAGS>(a, f, st, n);
            }
        }
    }
}

// Tiles march up their rows (down = false) or down them (down = true).  The
// launches give vertically neighbouring tiles opposite directions, so the two
// rows a pair of tiles both read (each one's halo row is the other's edge row)
// are read by both near the same time -- at both tiles' starts or at both
// ends -- and the second read finds them in L2 instead of going to DRAM.
// Direction changes only the order of the rows; every node gets the same
// arithmetic and every destination slot the same single write.
// Barrier of the threads running one tile: the whole CTA (BAR = 0), or the TX
// threads of one part of a CTA that runs several tiles side by side (named
// barrier BAR = 1, 2, ...; TX a multiple of 32, each warp in one part).  The
// barrier number is an immediate: a register operand makes ptxas reserve all
// sixteen barriers of the CTA, which caps residency at four CTAs per SM.
// BAR = SYNC_WARP: the tile is one warp (TX = 32), which needs no barrier
// beyond the warp's own.
constexpr int SYNC_WARP = -1;
template <int TX, int BAR> __device__ __forceinline__ void tile_sync()
{
    if constexpr (BAR == SYNC_WARP) {
        static_assert(TX == 32, "warp tiles are 32 columns wide");
        __syncwarp();
    } else if constexpr (BAR == 0) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(TX) : "memory");
    }
}

template <typename S, typename T, int TX, bool TWO_PASS, int FLAGS, bool PF = false,
          bool AHEAD = false, bool WIDE = false, int BAR = 0>
__device__ __forceinline__ void fused2_tile(const Fused2Args<S, T> &a, const int xb, const int yb,
                                            V2<T> (&s_rho)[4][TX], uint8_t (&s_m)[4][TX],
                                            const bool down = false)
{
    if constexpr (AHEAD && !TWO_PASS) {
        fused2_tile_ahead<S, T, TX, FLAGS>(a, xb, yb, s_rho, s_m);
        return;
    }
    constexpr bool SOLID = (FLAGS & KF_SOLID) != 0;
    constexpr int W = TX - 2;
    static_assert((TX & (TX - 1)) == 0, "TX a power of two");
    const int t = threadIdx.x & (TX - 1); // column of this thread in its tile
    const int nx = a.nx, ny = a.ny;
    const int ncol = min(W, nx - xb);
    const int nrow = min(a.tile_y, (a.row_end > 0 ? a.row_end : ny) - yb);
    const bool active = t <= ncol + 1;
    const bool interior = t >= 1 && t <= ncol;
    const int x = wrap1(xb - 1 + t, nx);
    const int xl = wrap1(x - 1, nx), xr = wrap1(x + 1, nx);
    // row of the tile (-1 .. nrow, halos included) visited in iteration q
    auto phys = [&](int q) { return down ? nrow - 1 - q : q; };

    // the mask of the next row is loaded one iteration ahead, so the population
    // loads of a row never wait on its mask load
    uint8_t m_ahead = 1;
    if (SOLID && active)
        m_ahead = a.mask[(uint32_t)wrap1(yb + phys(-1), ny) * (uint32_t)nx + (uint32_t)x];

    // iteration q: load row phys(q) into cur, publish its density, collide row
    // phys(q-1) (prev) from the densities of rows phys(q-2), phys(q-1), phys(q)
    auto row = [&](const int q, T(&cur)[2][9], const T(&prev)[2][9]) {
        const int r = phys(q);
        const int y = wrap1(yb + r, ny);
        const int slot = (q + 1) & 3;
        if constexpr (PF) {
            const int qp = q + PF_DIST;
            if (t < 18 && qp <= nrow) {
                const int k = t >= 9 ? 1 : 0, i = t - 9 * k;
                const S *arr =
                    a.fin[k] + (size_t)i * a.N + (size_t)wrap1(yb + phys(qp), ny) * (size_t)nx;
                const uintptr_t lo = (uintptr_t)(arr + max(xb - 1, 0)) & ~uintptr_t(15);
                const uintptr_t end = (uintptr_t)(a.fin[k] + 9 * a.N) & ~uintptr_t(15);
                const uintptr_t up = ((uintptr_t)(arr + min(xb + ncol + 1, nx)) + 15) & ~uintptr_t(15);
                const uintptr_t hi = up < end ? up : end;
                if (hi > lo) prefetch_l2_bulk((const void *)lo, (uint32_t)(hi - lo));
            }
        }
        T rho[2] = {T(0), T(0)};
        uint8_t m = 1;
        if (active) {
            const uint32_t node = (uint32_t)y * (uint32_t)nx + (uint32_t)x;
            if (SOLID) {
                m = m_ahead;
                if (q < nrow)
                    m_ahead = a.mask[(uint32_t)wrap1(yb + phys(q + 1), ny) * (uint32_t)nx + (uint32_t)x];
            }
            // solid nodes hold zeros on the domain path: nothing to read there
            const bool need_pops = (!TWO_PASS || (interior && r >= 0 && r < nrow)) &&
                                   (!SOLID || m || !a.solids_zero);
            if (need_pops) {
#pragma unroll
                for (int k = 0; k < 2; ++k)
#pragma unroll
                    for (int i = 0; i < 9; ++i)
                        cur[k][i] = T(Store<S>::ld(a.fin[k] + elem<WIDE>(i, a.N, node)));
            }
            if (TWO_PASS) {
                rho[0] = a.rho_in[0][node];
                rho[1] = a.rho_in[1][node];
            } else {
                node_density(cur, rho[0], rho[1]);
            }
            if (SOLID && !m) rho[0] = rho[1] = T(0);
        } else {
            m = 0;
        }
        s_rho[slot][t] = Vec2<T>::make(rho[0], rho[1]);
        s_m[slot][t] = m;
        tile_sync<TX, BAR>();

        if (q >= 1 && interior) {
            // slots of the rows below (sb), at (sc) and above (sa) the node
            const int s_old = (q - 1) & 3, sc = q & 3, s_new = (q + 1) & 3;
            const int sb = down ? s_new : s_old, sa = down ? s_old : s_new;
            const int yc = wrap1(yb + phys(q - 1), ny);
            const Stencil<T> st{{s_rho[sb], s_rho[sc], s_rho[sa]},
                                {s_m[sb], s_m[sc], s_m[sa]}, t};
            const Nbr n = make_nbr(nx, x, xl, xr, yc, wrap1(yc - 1, ny), wrap1(yc + 1, ny));
            collide_push<S, T, FLAGS, WIDE>(a, prev, st, n);
        }
    };

    T A[2][9], B[2][9];
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int i = 0; i < 9; ++i) A[k][i] = B[k][i] = T(0);
    // two rows per trip so the buffers swap roles instead of being copied
    for (int q = -1; q <= nrow; q += 2) {
        row(q, A, B);
        if (q + 1 <= nrow) row(q + 1, B, A);
    }
}

// resident 128-thread CTAs per SM the register cap aims at: FP32 arithmetic
// fits 80 registers (six CTAs) with two row buffers and 102 (five) with the
// third buffer of the load-ahead form or the uniform solid form; FP64 fits
// 168 (three CTAs) without spills -- uncapped, its solid forms took 178 and
// ran two CTAs per SM -- and its all-fluid form 128 (four CTAs)
template <typename T, bool AHEAD, int FLAGS = 0, int TX = 128> constexpr int fused_min_ctas()
{
    // the same registers per thread for narrower tiles: proportionally more CTAs
    return (sizeof(T) == 8 ? (FLAGS == 0 && !AHEAD ? 4 : 3) : (AHEAD || (FLAGS & KF_UNIFORM) ? 5 : 6)) *
           (128 / TX);
}

template <typename S, typename T, int TX, bool TWO_PASS, int FLAGS, bool PF = false,
          bool AHEAD = false, bool COMPACT = false, bool WIDE = false>
__global__ void __launch_bounds__(TX, (fused_min_ctas<T, AHEAD, FLAGS, TX>()))
    k_fused2(const __grid_constant__ Fused2Args<S, T> a)
{
    __shared__ V2<T> s_rho[4][TX];
    __shared__ uint8_t s_m[4][TX];
    if constexpr (COMPACT && (FLAGS & KF_SOLID) != 0 && !TWO_PASS) {
        __shared__ CompactSmem<S, T, TX> cs;
        fused2_tile_compact<S, T, TX, FLAGS>(a, blockIdx.x * (TX - 2), a.row0 + blockIdx.y * a.tile_y,
                                             s_rho, s_m, cs, (blockIdx.y & 1) != 0);
    } else {
        fused2_tile<S, T, TX, TWO_PASS, FLAGS, PF, AHEAD, WIDE>(a, blockIdx.x * (TX - 2),
                                                                a.row0 + blockIdx.y * a.tile_y, s_rho,
                                                                s_m, (blockIdx.y & 1) != 0);
    }
}

// ---------------------------------------------------------------------------
// single-component fused step: collide(geom,f) + add_volume_force + stream
// (src/lbm.cpp:275-288, 315-325, 343-384; src/fluid.cpp:175-243)
// ---------------------------------------------------------------------------
template <typename S, typename T>
__global__ void __launch_bounds__(256) k_fused1(const Fused1Args<S, T> a)
{
    constexpr bool EXACT = sizeof(T) == 8;
    const size_t N = a.N;
    const int nx = a.nx, ny = a.ny;
    for (size_t node = blockIdx.x * (size_t)blockDim.x + threadIdx.x; node < N;
         node += (size_t)gridDim.x * blockDim.x) {
        const int x = int(node % nx), y = int(node / nx);
        const bool fl = a.mask[node] == 1;
        if (!fl) {
#pragma unroll
            for (int i = 0; i < 9; ++i) Store<S>::st(a.fout + i * N + node, T(0));
            continue;
        }
        T f[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) f[i] = T(Store<S>::ld(a.fin + i * N + node));
        T out[9];
        if constexpr (EXACT) {
            double r = 0.0, ux = 0.0, uy = 0.0;
#pragma unroll
            for (int i = 0; i < 9; ++i) r += f[i];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                ux += f[i] * double(cx(i));
                uy += f[i] * double(cy(i));
            }
            ux /= r;
            uy /= r;
            double fe[9];
            feq_exact(r, ux, uy, fe);
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                double v = a.c.one_m_omega * f[i] + a.c.omega * fe[i];
                if (a.c.force_on) v += a.c.force[i];
                out[i] = v;
            }
        } else {
            float dr = 0.f;
#pragma unroll
            for (int i = 0; i < 9; ++i) dr += f[i];
            const float r = a.c.rho_ref + dr;
            const float jx = (f[1] - f[3]) + (f[5] - f[6]) + (f[8] - f[7]);
            const float jy = (f[2] - f[4]) + (f[5] + f[6]) - (f[7] + f[8]);
            const float ir = 1.0f / r;
            const float ux = jx * ir, uy = jy * ir;
            const float usq15 = 1.5f * fmaf(ux, ux, uy * uy);
            float v[9];
#pragma unroll
            for (int i = 1; i < 9; ++i) {
                v[i] = fmaf(a.c.omega, feq_dev(i, dr, r, ux, uy, usq15) - f[i], f[i]);
                if (a.c.force_on) v[i] += a.c.force[i];
                v[i] = stored_value<S>(v[i]);
            }
            // the rest population closes the node's mass (see mass_closing_rest)
            v[0] = mass_closing_rest(f, v, a.c.force_on ? a.c.force_sum : 0.f);
#pragma unroll
            for (int i = 0; i < 9; ++i) out[i] = v[i];
        }
        const int xl = wrap1(x - 1, nx), xr = wrap1(x + 1, nx);
        const int yd = wrap1(y - 1, ny), yu = wrap1(y + 1, ny);
        Store<S>::st(a.fout + node, out[0]);
#pragma unroll
        for (int i = 1; i < 9; ++i) {
            const int xn = cx(i) == 0 ? x : (cx(i) > 0 ? xr : xl);
            const int yn = cy(i) == 0 ? y : (cy(i) > 0 ? yu : yd);
            const size_t nb = (size_t)yn * nx + xn;
            if (a.mask[nb] == 1)
                Store<S>::st(a.fout + i * N + nb, out[i]);
            else
                Store<S>::st(a.fout + opp(i) * N + node, out[i]);
        }
    }
}

// ---------------------------------------------------------------------------
// kernel a: density (shifted forms: deviation) of both components, 0 at solids
// ---------------------------------------------------------------------------
template <typename S, typename T>
__global__ void __launch_bounds__(256) k_density2(const uint8_t *__restrict__ mask,
                                                  const S *__restrict__ f0,
                                                  const S *__restrict__ f1, T *__restrict__ r0,
                                                  T *__restrict__ r1, size_t N)
{
    for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < N;
         n += (size_t)gridDim.x * blockDim.x) {
        T s0 = T(0), s1 = T(0);
        if (mask[n]) {
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                s0 += T(Store<S>::ld(f0 + i * N + n));
                s1 += T(Store<S>::ld(f1 + i * N + n));
            }
        }
        r0[n] = s0;
        r1[n] = s1;
    }
}

// specialisation flags of an argument block
template <typename S, typename T> inline int kernel_flags(const Fused2Args<S, T> &a)
{
    return (a.c[0].force_on || a.c[1].force_on ? KF_FORCE : 0) | (a.has_solid ? KF_SOLID : 0);
}

template <typename S, typename T, int TX, bool TWO, int FLAGS, bool PF = false, bool AHEAD = false,
          bool COMPACT = false, bool WIDE = false>
inline cudaError_t launch_fused2_f(const Fused2Args<S, T> &a, cudaStream_t s)
{
    constexpr int W = TX - 2;
    const int rows = (a.row_end > 0 ? a.row_end : a.ny) - a.row0;
    const dim3 grid((a.nx + W - 1) / W, (rows + a.tile_y - 1) / a.tile_y);
    k_fused2<S, T, TX, TWO, FLAGS, PF, AHEAD, COMPACT, WIDE><<<grid, TX, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename S, typename T, int TX, bool PF = false, bool AHEAD = false, bool COMPACT = false,
          int UNI = 0>
inline cudaError_t launch_fused2_tx(const Fused2Args<S, T> &a, bool two_pass, cudaStream_t s)
{
    if (two_pass) return launch_fused2_f<S, T, TX, true, KF_FORCE | KF_SOLID>(a, s);
    switch (kernel_flags(a)) {
    case 0: return launch_fused2_f<S, T, TX, false, 0, PF, AHEAD>(a, s);
    case KF_FORCE: return launch_fused2_f<S, T, TX, false, KF_FORCE, PF, AHEAD>(a, s);
    case KF_SOLID: return launch_fused2_f<S, T, TX, false, KF_SOLID | UNI, PF, AHEAD, COMPACT>(a, s);
    default:
        return launch_fused2_f<S, T, TX, false, KF_FORCE | KF_SOLID | UNI, PF, AHEAD, COMPACT>(a, s);
    }
}

// variant 1: two pass; 4: single pass with L2 row prefetch (128 threads);
// 5: single pass with loads one row ahead (128 threads); 6: single pass with
// the collision on compacted fluid lanes (lattices with solid nodes; 128
// threads); 8: the register tile with the uniform solid form (KF_UNIFORM);
// otherwise the single-pass register tile
template <typename S, typename T>
inline cudaError_t launch_fused2_any(const Fused2Args<S, T> &a, int variant, int tx,
                                     cudaStream_t s)
{
    if (a.tile_y < 1 || a.nx < 1 || a.ny < 1) return cudaErrorInvalidValue;
    // 64-bit offsets (lattices of 2^32/9 nodes and more; variant 7 asks for
    // them on any lattice): the general single-pass kernel
    if (needs_wide_offsets(a.N) || variant == 7)
        return launch_fused2_f<S, T, 128, false, KF_FORCE | KF_SOLID, false, false, false, true>(a, s);
    const bool two = variant == 1;
    if (tx == 64) return launch_fused2_tx<S, T, 64>(a, two, s);
    if (tx == 32) {
        // one-warp tiles (no CTA barrier); variant 8: with the uniform solid form
        if (variant == 8) return launch_fused2_tx<S, T, 32, false, false, false, KF_UNIFORM>(a, false, s);
        return launch_fused2_tx<S, T, 32>(a, two, s);
    }
    if (variant == 4) return launch_fused2_tx<S, T, 128, true>(a, false, s);
    if (variant == 5) return launch_fused2_tx<S, T, 128, false, true>(a, false, s);
    if (variant == 8) return launch_fused2_tx<S, T, 128, false, false, false, KF_UNIFORM>(a, false, s);
    if (variant == 6) {
        // FP64's three population rows would exceed the static shared memory
        if constexpr (sizeof(T) == 4) return launch_fused2_tx<S, T, 128, false, false, true>(a, false, s);
        else return launch_fused2_tx<S, T, 128>(a, false, s);
    }
    return launch_fused2_tx<S, T, 128>(a, two, s);
}

} // namespace sclbm
