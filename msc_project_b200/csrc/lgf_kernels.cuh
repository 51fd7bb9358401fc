// sm_100a kernels of the Wilson-flow engine.
//
//   k_rk3_stage<R,S>   one fused Luscher RK3 stage for every link: staple,
//                      projected force Z, su(3) accumulator update,
//                      Cayley-Hamilton exponential, link update (ping-pong).
//                      Replaces Wilson::calculate_FlowGradient
//                      (LGF/Action/Gauge/Wilson.cpp:55-71), SU3_field::staple
//                      (LGF/Field/SU3_field.cpp:519-530), HermTrLessExp
//                      (LGF/Math/SU3_mat.cpp:216-289) and the three update
//                      loops of GradientFlow::flow (GradientFlow.cpp:22-54).
//   k_measure<R>       clover F (E) and improved F (q) for every site and plane,
//                      per-site e(x), q(x), warp-shuffle block partials by
//                      x0 slice.  Replaces EnergyDensity::calculate and
//                      TopologicalCharge::calculate (Observables/*.cpp) and the
//                      loop averages of SU3_field.cpp:533-792.
//   k_reduce_slices / k_reduce_total
//                      fixed-order FP64 reductions (per x0 slice, then global)
//                      in place of MPI_Allreduce; deterministic run to run.
//   k_to_device / k_to_file    file-order float64 <-> device layout
//   k_generate_G       synthetic links exp(i s sum_a h_a T^a)
//   k_reunitarize      FP32-mixed: Gram-Schmidt rows 0,1; row 2 = conj(r0 x r1)
//   k_unitarity        max ||U^dag U - 1||_F and |det U - 1| per block
//   k_debug_*          per-function outputs for parity tests
#pragma once
#include "lgf_lattice.cuh"

// Launch bounds of the RK3 stage: (max threads per block, min resident
// blocks per SM), which cap the registers per thread at 65536 / 384 = 170,
// i.e. 168 once rounded to the allocation unit.  double: 384-thread blocks
// (12 warps per SM: 7% faster per stage than 8 warps at 250 registers on
// 24^3x48 and 48^4); float: 128-thread blocks, three per SM (at 170
// registers the rounding to 176 leaves room for only two: 15% slower).
#ifndef LGF_STAGE_MAXT_D
#define LGF_STAGE_MAXT_D 384
#endif
#ifndef LGF_STAGE_MAXT_F
#define LGF_STAGE_MAXT_F 384
#endif
#ifndef LGF_STAGE_MINB
#define LGF_STAGE_MINB 1
#endif
#ifndef LGF_MEAS_QSPLIT
#define LGF_MEAS_QSPLIT 2  // default measurement warps per plane (the four quadrants split between them)
#endif

namespace lgf {

// ----------------------------------------------------------------- staple
// Z = -1/2 [ (W - W^dag) - 1/3 Tr(W - W^dag) ],  W = U_mu(x) A,
// A = sum_{nu != mu} U_nu(x+mu) (U_nu(x) U_mu(x+nu))^dag
//                  + (U_mu(x-nu) U_nu(x-nu+mu))^dag U_nu(x-nu)
template <typename R>
__device__ __forceinline__ su3<R> staple_sum(const cplx<R>* __restrict__ U, const Geom& g, int s, const Coord& c, int mu) {
    const int V = g.V;
    const Dir dm = dir_of(g, c, mu);
    su3<R> S;
    su3_zero(S);
    const int xpm = fwd(s, dm);
#pragma unroll
    for (int nu = 0; nu < 4; ++nu) {
        if (nu == mu) continue;
        const int xpn = fwd(g, s, nu, c.x[nu]);
        const int xmn = bwd(g, s, nu, c.x[nu]);
        const int xmnpm = fwd(xmn, dm);  // the mu coordinate of x-nu is x_mu
        {
            su3<R> a2 = load_link(U, V, nu, s);
            su3<R> a3 = load_link(U, V, mu, xpn);
            su3<R> t = mul_nn_su3(a2, a3);
            su3<R> a1 = load_link(U, V, nu, xpm);
            acc_na(S, a1, t);
        }
        {
            su3<R> b1 = load_link(U, V, mu, xmn);
            su3<R> b2 = load_link(U, V, nu, xmnpm);
            su3<R> t = mul_nn_su3(b1, b2);
            su3<R> b3 = load_link(U, V, nu, xmn);
            acc_an(S, t, b3);
        }
    }
    return S;
}

#ifndef LGF_TA_ONLY
#define LGF_TA_ONLY 1  // the force's product forms only the entries its projection reads
#endif
// ta_part(A B, s) computing only what the projection reads: the imaginary
// parts of the diagonal and the three off-diagonal pairs (90 real
// operations instead of 108 for the full product)
template <typename R> __device__ __forceinline__ alg<R> ta_of_product(const su3<R>& A, const su3<R>& B, R s) {
    R d[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R im = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) im = fma(A.m[3 * i + k].re, B.m[3 * k + i].im, fma(A.m[3 * i + k].im, B.m[3 * k + i].re, im));
        d[i] = R(2) * im;
    }
    const R tr = (d[0] + d[1] + d[2]) * R(1.0 / 3.0);
    alg<R> z;
    z.v[0] = s * (d[0] - tr);
    z.v[1] = s * (d[1] - tr);
    const int I[3] = {0, 0, 1}, J[3] = {1, 2, 2};
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        const int i = I[o], j = J[o];
        cplx<R> wij = cmul(A.m[3 * i], B.m[j]);
        wij = cfma(A.m[3 * i + 1], B.m[3 + j], wij);
        wij = cfma(A.m[3 * i + 2], B.m[6 + j], wij);
        cplx<R> wji = cmul(A.m[3 * j], B.m[i]);
        wji = cfma(A.m[3 * j + 1], B.m[3 + i], wji);
        wji = cfma(A.m[3 * j + 2], B.m[6 + i], wji);
        z.v[2 + 2 * o] = s * (wij.re - wji.re);
        z.v[3 + 2 * o] = s * (wij.im + wji.im);
    }
    return z;
}

template <typename R>
__device__ __forceinline__ alg<R> flow_gradient(const cplx<R>* __restrict__ U, const Geom& g, int s, const Coord& c,
                                                int mu, su3<R>& u_out) {
    const su3<R> S = staple_sum<R>(U, g, s, c, mu);
    u_out = load_link(U, g.V, mu, s);
    return LGF_TA_ONLY ? ta_of_product(u_out, S, R(-0.5)) : ta_part(mul_nn(u_out, S), R(-0.5));
}

// Device descriptor of one resident lattice.  Every flow launch works on a
// table of these plus a work list of tiles, so one launch can cover one
// lattice or many lattices of uneven volumes (batch and serving forms).
template <typename R> struct LatDesc {
    Geom g;
    cplx<R>* U0;          // ring of link buffers: stage 1 U0->U1, 2 U1->U2, 3 U2->U0
    cplx<R>* U1;
    cplx<R>* U2;
    R* A;                 // su(3) RK3 accumulator, 8 coordinates per link
    double2* partial;     // [N0 * nchunk] block partials of the measurement
    double2* slice_sums;  // [N0]
    double* meas;         // [capacity * (2 + 2 N0)] measurement results
    int* slot;            // next measurement slot
    int nchunk;           // measurement blocks per x0 slice
    R eps;
};

// One RK3 stage (low-storage form of the reference's integrator):
//   S=1:  A = Z0;                    U1 = exp(eps/4 Z0) U0
//   S=2:  A = 8/9 Z1 - 17/36 A;      U2 = exp(eps A) U1
//   S=3:                             U3 = exp(eps (3/4 Z2 - A)) U2
// which equals GradientFlow.cpp:27-50 term by term.  Input and output are
// different buffers of the ring (every thread reads neighbours of the input).
// Persistent: blocks stride over one segment of the tile list (seg = first
// tile, count); tile = (lattice, first site).
// A tile of T threads (T a multiple of 128) covers T/4 consecutive sites with
// all four directions: warp w handles mu = w % 4 for the 32 sites of group
// w / 4, so the four link directions of a site range are read together and
// every load of a warp covers 32 consecutive sites.
template <typename R> struct StageMaxThreads { static constexpr int value = LGF_STAGE_MAXT_F; };
template <> struct StageMaxThreads<double> { static constexpr int value = LGF_STAGE_MAXT_D; };

template <typename R, int S>
__global__ void __launch_bounds__(StageMaxThreads<R>::value, LGF_STAGE_MINB) k_rk3_stage(const LatDesc<R>* __restrict__ descs, const int2* __restrict__ tiles,
                                                   const int2* __restrict__ seg) {
    const int2 r = *seg;  // this launch's tiles: tiles[r.x, r.x + r.y)
    for (int ti = r.x + blockIdx.x; ti < r.x + r.y; ti += gridDim.x) {
        const int2 tile = tiles[ti];
        const LatDesc<R>* d = descs + tile.x;
        const Geom g = d->g;
        const int mu = (threadIdx.x >> 5) & 3;
        const int s = tile.y + ((threadIdx.x >> 7) << 5) + (threadIdx.x & 31);
        if (s >= g.V) continue;
        const cplx<R>* Uin = S == 1 ? d->U0 : (S == 2 ? d->U1 : d->U2);
        cplx<R>* Uout = S == 1 ? d->U1 : (S == 2 ? d->U2 : d->U0);
        R* A = d->A;
        const R eps = d->eps;
        const Coord c = site_coord(g, s);
        su3<R> u;
        const alg<R> Z = flow_gradient<R>(Uin, g, s, c, mu, u);
        alg<R> X;
        if (S == 1) {
            store_alg(A, g.V, mu, s, Z);
            X = alg_scale(R(0.25) * eps, Z);
        } else if (S == 2) {
            const alg<R> a = load_alg(A, g.V, mu, s);
            const alg<R> an = alg_axpby(R(8.0 / 9.0), Z, R(-17.0 / 36.0), a);
            store_alg(A, g.V, mu, s, an);
            X = alg_scale(eps, an);
        } else {
            const alg<R> a = load_alg(A, g.V, mu, s);
            const alg<R> dd = alg_axpby(R(3.0 / 4.0), Z, R(-1.0), a);
            X = alg_scale(eps, dd);
        }
        const su3<R> E = expm_alg(X);
        // the stored link is the full product (rebuilding its third row from
        // the first two would let their rounding drift into it step after step)
        store_link(Uout, g.V, mu, s, mul_nn(E, u));
    }
}

// ---------------------------------------------------------- Wilson loops
// The clover-type averages of the reference (SU3_field.cpp:533-792) are sums
// of a x b rectangular loops through x, one per quadrant, in the orientation
//   q0: +nu^b +mu^a -nu^b -mu^a     q1: +mu^a -nu^b -mu^a +nu^b
//   q2: -mu^a +nu^b +mu^a -nu^b     q3: -nu^b -mu^a +nu^b +mu^a
// (a links along mu, b along nu).  With quadrant signs (sm, sn) = (+,+),
// (+,-), (-,+), (-,-), every leaf is  Pn Pm^dag  (q0, q3) or its adjoint
// (q1, q2), where Pn = (sn nu)^b (sm mu)^a and Pm = (sm mu)^a (sn nu)^b are
// the two L-shaped paths from x to the far corner.  The projection F[W] is
// linear and F[W^dag] = -F[W], so each quadrant adds sign * F[Pn Pm^dag]
// with sign = +1 for q0, q3 and -1 for q1, q2, weighted per shape:
//   F^ = 19/9 F[C11] + 1/36 F[C22] - 32/45 F[C12] + 1/15 F[C13]
//      C11 = 1/4 (1x1), C22 = 1/4 (2x2), C12 = 1/8 (1x2 + 2x1), C13 = 1/8 (1x3 + 3x1)
// (SU3_field.cpp:588-597), and the clover F = F[C11] for E.  The paths are
// built as shared chains (a path of a shape extends the path of the shape
// before it by one link) and from shared straight lines: 12 matrix products
// and 14 global link loads per quadrant (plane_fields_body) instead of 34 and
// 40 for separate loops.
struct PlanePos { int s, xm, xn; };

#ifndef LGF_MEAS_ROW3
#define LGF_MEAS_ROW3 1  // path products of the measurement rebuild their third row (mul_nn_su3)
#endif

template <typename R> struct Plane {
    const cplx<R>* __restrict__ U;
    int V, mu, nu;
    Dir dm, dn;  // .x unused: positions carry their own coordinates

    // the link of one step from p and the new position; adjoint for a backward step
    __device__ __forceinline__ su3<R> step(PlanePos& p, bool along_mu, int sign) const {
        const Dir& d = along_mu ? dm : dn;
        int& xc = along_mu ? p.xm : p.xn;
        const int dir = along_mu ? mu : nu;
        if (sign > 0) {
            su3<R> l = load_link(U, V, dir, p.s);
            p.s = (xc == d.n - 1) ? p.s - (d.n - 1) * d.stride : p.s + d.stride;
            xc = wrap_inc(xc, d.n);
            return l;
        }
        p.s = (xc == 0) ? p.s + (d.n - 1) * d.stride : p.s - d.stride;
        xc = wrap_dec(xc, d.n);
        su3<R> l = load_link(U, V, dir, p.s);
        su3<R> a;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) a.m[3 * r + c] = cmk<R>(l.m[3 * c + r].re, -l.m[3 * c + r].im);
        return a;
    }
    // move p by count steps without loading links
    __host__ __device__ __forceinline__ void advance(PlanePos& p, bool along_mu, int sign, int count) const {
        const Dir& d = along_mu ? dm : dn;
        int& xc = along_mu ? p.xm : p.xn;
        for (int i = 0; i < count; ++i) {
            if (sign > 0) {
                p.s = (xc == d.n - 1) ? p.s - (d.n - 1) * d.stride : p.s + d.stride;
                xc = wrap_inc(xc, d.n);
            } else {
                p.s = (xc == 0) ? p.s + (d.n - 1) * d.stride : p.s - d.stride;
                xc = wrap_dec(xc, d.n);
            }
        }
    }
    // P <- P * (link of one step from p)
    __device__ __forceinline__ void ext(su3<R>& P, PlanePos& p, bool along_mu, int sign) const {
        const Dir& d = along_mu ? dm : dn;
        int& xc = along_mu ? p.xm : p.xn;
        const int dir = along_mu ? mu : nu;
        if (sign > 0) {
            const su3<R> l = load_link(U, V, dir, p.s);
            p.s = (xc == d.n - 1) ? p.s - (d.n - 1) * d.stride : p.s + d.stride;
            xc = wrap_inc(xc, d.n);
            P = LGF_MEAS_ROW3 ? mul_nn_su3(P, l) : mul_nn(P, l);
        } else {
            p.s = (xc == 0) ? p.s + (d.n - 1) * d.stride : p.s - d.stride;
            xc = wrap_dec(xc, d.n);
            const su3<R> l = load_link(U, V, dir, p.s);
            P = LGF_MEAS_ROW3 ? mul_na_su3(P, l) : mul_na(P, l);
        }
    }
};

// Where a measurement thread keeps its two 8-coordinate sums: registers, or
// (double, LGF_MEAS_SMEM_ACC) its own column of shared memory.  The FP64
// kernel holds two path matrices, the incoming link and these sums at its
// peak; at 168 registers that spilled ~0.6 KB per thread, and with the sums in
// shared memory (48 KB per block) it spills ~50 B and runs 12-13% faster on
// 16^4 to 48^4.  Same operations, same order, either way (bit-identical).
template <typename R> struct RegAcc {
    alg<R>& a;
    __device__ __forceinline__ R get(int k) const { return a.v[k]; }
    __device__ __forceinline__ void set(int k, R x) { a.v[k] = x; }
};
template <typename R> struct SmemAcc {
    R* p;  // coordinate k at p[k * MEAS_ACC_STRIDE]
    __device__ __forceinline__ R get(int k) const;
    __device__ __forceinline__ void set(int k, R x);
};

// F += c * F[A B^dag] without forming the product: only the entries the
// projection reads (Im of the diagonal, both triangles) are computed.
template <typename R, typename Acc> __device__ __forceinline__ void leaf_acc(const su3<R>& A, const su3<R>& B, R c, Acc F) {
    // W_ij = sum_k A_ik conj(B_jk)
    R d[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        R im = R(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) im = fma(A.m[3 * i + k].im, B.m[3 * i + k].re, fma(-A.m[3 * i + k].re, B.m[3 * i + k].im, im));
        d[i] = im;
    }
    const R tr = (d[0] + d[1] + d[2]) * R(1.0 / 3.0);
    F.set(0, fma(c, d[0] - tr, F.get(0)));
    F.set(1, fma(c, d[1] - tr, F.get(1)));
    const int I[3] = {0, 0, 1}, J[3] = {1, 2, 2};
#pragma unroll
    for (int o = 0; o < 3; ++o) {
        const int i = I[o], j = J[o];
        cplx<R> wij = cmulc(A.m[3 * i], B.m[3 * j]);
        wij = cfmac(A.m[3 * i + 1], B.m[3 * j + 1], wij);
        wij = cfmac(A.m[3 * i + 2], B.m[3 * j + 2], wij);
        cplx<R> wji = cmulc(A.m[3 * j], B.m[3 * i]);
        wji = cfmac(A.m[3 * j + 1], B.m[3 * i + 1], wji);
        wji = cfmac(A.m[3 * j + 2], B.m[3 * i + 2], wji);
        // (-i/2)(a + ib) = (b/2, -a/2),  a + ib = W_ij - conj(W_ji)
        const R a = wij.re - wji.re, b = wij.im + wji.im;
        F.set(2 + 2 * o, fma(R(0.5) * c, b, F.get(2 + 2 * o)));
        F.set(3 + 2 * o, fma(R(-0.5) * c, a, F.get(3 + 2 * o)));
    }
}

template <typename R> __device__ __forceinline__ void store_alg_as_antiherm(double2* dst, const alg<R>& z) {
    const double v0 = z.v[0], v1 = z.v[1];
    dst[0] = make_double2(0.0, v0);
    dst[4] = make_double2(0.0, v1);
    dst[8] = make_double2(0.0, -(v0 + v1));
    dst[1] = make_double2(z.v[2], z.v[3]);
    dst[3] = make_double2(-(double)z.v[2], z.v[3]);
    dst[2] = make_double2(z.v[4], z.v[5]);
    dst[6] = make_double2(-(double)z.v[4], z.v[5]);
    dst[5] = make_double2(z.v[6], z.v[7]);
    dst[7] = make_double2(-(double)z.v[6], z.v[7]);
}
template <typename R> __device__ __forceinline__ void store_alg_as_herm(double2* dst, const alg<R>& f) {
    const double v0 = f.v[0], v1 = f.v[1];
    dst[0] = make_double2(v0, 0.0);
    dst[4] = make_double2(v1, 0.0);
    dst[8] = make_double2(-(v0 + v1), 0.0);
    dst[1] = make_double2(f.v[2], f.v[3]);
    dst[3] = make_double2(f.v[2], -(double)f.v[3]);
    dst[2] = make_double2(f.v[4], f.v[5]);
    dst[6] = make_double2(f.v[4], -(double)f.v[5]);
    dst[5] = make_double2(f.v[6], f.v[7]);
    dst[7] = make_double2(f.v[6], -(double)f.v[7]);
}

__device__ __constant__ int c_plane_mu[6] = {0, 0, 0, 1, 1, 2};
__device__ __constant__ int c_plane_nu[6] = {1, 2, 3, 2, 3, 3};

constexpr int MEAS_SITES = 32;  // sites per measurement block (x) ; planes in y

// Measurement tile geometry.  A tile's 32 sites are 32 consecutive sites of
// the slice (a strip), or, built with -DLGF_MEAS_PATCH=1, a patch of 4 x2 rows
// by 8 x3 positions at fixed (x0, x1) when N2 % 4 == 0 and N3 % 8 == 0.  The
// patch keeps the +-3 stencil of the six planes compact (a strip along x3
// touches ~5500 distinct sites per tile, a 4 x 8 patch ~3600) and each warp
// load still covers four whole 128-byte lines, but measured on one B200 it
// is 2-8% slower in FP64 (16^4 to 48^4), 4-6% faster in FP32 up to 32^4 and
// 13% slower on 48^4, so strips are the default.  Chunk c of a slice is patch
// (x1, b2, b3) = (c / (nb2 nb3), (c / nb3) % nb2, c % nb3); a slice has
// Vs / 32 chunks either way.  The geometry is a fixed function of the
// lattice shape, so the grouping of the partial sums (and every result bit)
// does not depend on tile shapes or batch partners.
#ifndef LGF_MEAS_PATCH
#define LGF_MEAS_PATCH 0
#endif
constexpr int MEAS_PATCH_ROWS = 4, MEAS_PATCH_COLS = 8;
__host__ __device__ __forceinline__ bool meas_patched(const Geom& g) {
    return LGF_MEAS_PATCH && g.n[2] % MEAS_PATCH_ROWS == 0 && g.n[3] % MEAS_PATCH_COLS == 0;
}
// offset within its x0 slice of lane l's site in measurement chunk c
__host__ __device__ __forceinline__ int meas_site_offset(const Geom& g, bool patched, int c, int l) {
    if (!patched) return c * MEAS_SITES + l;
    const int nb3 = g.n[3] / MEAS_PATCH_COLS, nb2 = g.n[2] / MEAS_PATCH_ROWS;
    const int x1 = c / (nb2 * nb3), r = c - x1 * (nb2 * nb3), b2 = r / nb3, b3 = r - b2 * nb3;
    return (x1 * g.n[2] + b2 * MEAS_PATCH_ROWS + l / MEAS_PATCH_COLS) * g.n[3] + b3 * MEAS_PATCH_COLS +
           l % MEAS_PATCH_COLS;
}
#ifndef LGF_MEAS_SMEM_ACC
#define LGF_MEAS_SMEM_ACC 1
#endif
constexpr int MEAS_ACC_STRIDE = MEAS_SITES * 12;  // one column per thread of a 12-warp block
template <typename R> __device__ __forceinline__ R SmemAcc<R>::get(int k) const { return p[k * MEAS_ACC_STRIDE]; }
template <typename R> __device__ __forceinline__ void SmemAcc<R>::set(int k, R x) { p[k * MEAS_ACC_STRIDE] = x; }
template <typename R> constexpr bool meas_smem_acc() { return LGF_MEAS_SMEM_ACC && sizeof(R) == sizeof(double); }

// A path matrix parked in the thread's own shared-memory column until it is
// extended by one more link.  Only its first two rows are kept when the
// extension rebuilds the third (mul_nn_su3 / mul_na_su3 read rows 0 and 1 of
// their left operand), so a parked path is exactly the one put there.
constexpr int MEAS_STASH_ENTRIES = LGF_MEAS_ROW3 ? 6 : 9;
template <typename R> struct PathStash {
    typename vec2_of<R>::type* p;  // entry k at p[k * MEAS_ACC_STRIDE]
    __device__ __forceinline__ void put(const su3<R>& P) const {
#pragma unroll
        for (int k = 0; k < MEAS_STASH_ENTRIES; ++k) {
            p[k * MEAS_ACC_STRIDE].x = P.m[k].re;
            p[k * MEAS_ACC_STRIDE].y = P.m[k].im;
        }
    }
    __device__ __forceinline__ su3<R> get() const {
        su3<R> P;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            if (k < MEAS_STASH_ENTRIES) {
                const typename vec2_of<R>::type v = p[k * MEAS_ACC_STRIDE];
                P.m[k] = cmk<R>(v.x, v.y);
            } else {
                P.m[k] = cmk<R>(R(0), R(0));  // never read: the next product rebuilds the row
            }
        }
        return P;
    }
};

constexpr int MEAS_QSPLIT = LGF_MEAS_QSPLIT;
constexpr int MEAS_WARPS = 6 * MEAS_QSPLIT;  // warp y: plane y % 6, quadrants of part y / 6
// resident measurement blocks per SM the launch bounds ask for (caps the
// registers): one block of 12 warps with the quadrants split, else two of 6
template <int QS> struct MeasMinBlocks { static constexpr int value = QS == 2 ? 1 : 2; };

// Shared memory of one measurement block: the straight lines of length 2 and
// 3 from each of its 32 sites in the 8 signed directions (every plane and
// quadrant of the site reuses them), then the per-plane results.
template <typename R, bool OUT> struct MeasSmem {
    union {
        R line[8][2][2 * MEAS_STASH_ENTRIES][MEAS_SITES];  // [2*dir + (sign<0)][length-2][real of entry][site]
        struct {                       // after the lines are dead: the second quadrant half's sums
            alg<R> G[6][MEAS_SITES];
            alg<R> Fh[6][MEAS_SITES];
        } part;
    };
    R acc[meas_smem_acc<R>() ? 16 : 1][meas_smem_acc<R>() ? MEAS_ACC_STRIDE : 1];  // G, Fhat columns (LGF_MEAS_SMEM_ACC)
    typename vec2_of<R>::type stash[2][MEAS_STASH_ENTRIES][MEAS_ACC_STRIDE];  // two paths per thread (PathStash)
    alg<R> F[6][MEAS_SITES];          // improved F per plane
    alg<R> C[OUT ? 6 : 1][MEAS_SITES];  // clover F per plane (single-lattice passes only)
    double E[6][MEAS_SITES];
};

// Optional per-site / per-(site, plane) outputs of a measurement pass (all
// null in the flow).  e, q: the densities of E and Q; e_imp, q_clov: the
// energy density with the improved F (ImprovedEnergyDensity.cpp:13-20) and
// the charge density with the clover F (UnImprovedTopologicalCharge.cpp:11-16);
// dbg_*: F and F^ as Hermitian 3x3 matrices per (site, plane).
struct MeasOut {
    double* e;
    double* q;
    double* e_imp;
    double* q_clov;
    double2* dbg_clover;
    double2* dbg_improved;
};

// A line is only ever extended (the left operand of a product that rebuilds
// the third row), so like a parked path it keeps its first two rows.
template <typename R, bool OUT>
__device__ __forceinline__ void store_line(MeasSmem<R, OUT>* sm, int sdir, int len, int lane, const su3<R>& L) {
#pragma unroll
    for (int k = 0; k < MEAS_STASH_ENTRIES; ++k) {
        sm->line[sdir][len - 2][2 * k][lane] = L.m[k].re;
        sm->line[sdir][len - 2][2 * k + 1][lane] = L.m[k].im;
    }
}
template <typename R, bool OUT>
__device__ __forceinline__ su3<R> load_line(const MeasSmem<R, OUT>* sm, int sdir, int len, int lane) {
    su3<R> L;
#pragma unroll
    for (int k = 0; k < 9; ++k)
        L.m[k] = k < MEAS_STASH_ENTRIES
                     ? cmk<R>(sm->line[sdir][len - 2][2 * k][lane], sm->line[sdir][len - 2][2 * k + 1][lane])
                     : cmk<R>(R(0), R(0));  // never read: the next product rebuilds the row
    return L;
}

#ifndef LGF_MEAS_REUSE
#define LGF_MEAS_REUSE 1  // paths extended from parked shorter paths: 12 products per quadrant instead of 15
#endif

// Quadrants [qa, qb) of plane (mu, nu) at the thread's site, using the
// block's shared lines: G = the sum of the 1x1 leaves' projections, Fhat =
// the weighted sum of the other shapes' (see the comment above Plane for the
// leaf decomposition).  The clover F is G/4 and the improved F is
// Fhat + 19/36 G.  With a b-fold path written as its steps (n = sn nu,
// m = sm mu), the twelve paths of a quadrant are
//   Pn(a,1) = n m^a        (a chain: each extends the one before by m)
//   Pm(1,b) = m n^b        (a chain along n)
//   Pm(a,1) = line_m(a) n,  Pn(1,b) = line_n(b) m   (from the shared lines)
//   Pn(2,2) = Pn(1,2) m,    Pm(2,2) = Pm(2,1) n
// 12 matrix products and 14 global link loads per quadrant; the paths that
// are extended after other work are parked in the thread's shared-memory
// column (PathStash: Pm(1,1), Pm(2,1), Pn(1,2)), and the leaves are added in
// the order (1,1) | (2,1), (3,1), (1,2), (1,3), (2,2), the order of the
// 15-product form (LGF_MEAS_REUSE=0), whose every product it repeats: both
// give the same bits.
template <typename R, bool OUT, typename Acc>
__device__ __forceinline__ void plane_fields_body(const cplx<R>* __restrict__ U, const Geom& g, int s, const Coord& c,
                                                  int mu, int nu, const MeasSmem<R, OUT>* sm, int lane, int qa, int qb,
                                                  Acc G, Acc Fhat, PathStash<R> sa, PathStash<R> sb) {
    Plane<R> P;
    P.U = U;
    P.V = g.V;
    P.mu = mu;
    P.nu = nu;
    P.dm = dir_of(g, c, mu);
    P.dn = dir_of(g, c, nu);
    const PlanePos x0 = {s, P.dm.x, P.dn.x};
    const R k12 = R(-4.0 / 45.0), k13 = R(1.0 / 120.0), k22 = R(1.0 / 144.0);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        G.set(k, R(0));
        Fhat.set(k, R(0));
    }
#pragma unroll 1
    for (int q = qa; q < qb; ++q) {
        const int sm_ = (q == 0 || q == 1) ? 1 : -1;
        const int sn = (q == 0 || q == 2) ? 1 : -1;
        const R sg = (q == 0 || q == 3) ? R(1) : R(-1);
        const int sdm = 2 * mu + (sm_ < 0 ? 1 : 0), sdn = 2 * nu + (sn < 0 ? 1 : 0);
        if (LGF_MEAS_REUSE) {
            // (1,1)
            PlanePos pn = x0;
            su3<R> Pn = P.step(pn, false, sn);
            P.ext(Pn, pn, true, sm_);  // Pn(1,1)
            PlanePos pm = x0;
            su3<R> Pm = P.step(pm, true, sm_);
            P.ext(Pm, pm, false, sn);  // Pm(1,1), pm at x + m + n
            leaf_acc(Pn, Pm, sg, G);
            sa.put(Pm);
            // (2,1)
            P.ext(Pn, pn, true, sm_);  // Pn(2,1)
            PlanePos p21 = x0;
            P.advance(p21, true, sm_, 2);
            Pm = load_line(sm, sdm, 2, lane);
            P.ext(Pm, p21, false, sn);  // Pm(2,1), p21 at x + 2m + n
            leaf_acc(Pn, Pm, sg * k12, Fhat);
            sb.put(Pm);
            // (3,1)
            P.ext(Pn, pn, true, sm_);  // Pn(3,1)
            PlanePos p31 = x0;
            P.advance(p31, true, sm_, 3);
            Pm = load_line(sm, sdm, 3, lane);
            P.ext(Pm, p31, false, sn);  // Pm(3,1)
            leaf_acc(Pn, Pm, sg * k13, Fhat);
            // (1,2)
            Pm = sa.get();
            P.ext(Pm, pm, false, sn);  // Pm(1,2)
            PlanePos p12 = x0;
            P.advance(p12, false, sn, 2);
            Pn = load_line(sm, sdn, 2, lane);
            P.ext(Pn, p12, true, sm_);  // Pn(1,2), p12 at x + 2n + m
            leaf_acc(Pn, Pm, sg * k12, Fhat);
            sa.put(Pn);
            // (1,3)
            P.ext(Pm, pm, false, sn);  // Pm(1,3)
            PlanePos p13 = x0;
            P.advance(p13, false, sn, 3);
            Pn = load_line(sm, sdn, 3, lane);
            P.ext(Pn, p13, true, sm_);  // Pn(1,3)
            leaf_acc(Pn, Pm, sg * k13, Fhat);
            // (2,2)
            Pn = sa.get();
            P.ext(Pn, p12, true, sm_);  // Pn(2,2)
            Pm = sb.get();
            P.ext(Pm, p21, false, sn);  // Pm(2,2)
            leaf_acc(Pn, Pm, sg * k22, Fhat);
            continue;
        }
        // row: (1,1), (2,1), (3,1)
        PlanePos pn = x0;
        su3<R> Rn = P.step(pn, false, sn);
        P.ext(Rn, pn, true, sm_);  // Pn(1,1)
        {
            PlanePos q2 = x0;
            su3<R> Pm = P.step(q2, true, sm_);
            P.ext(Pm, q2, false, sn);  // Pm(1,1)
            leaf_acc(Rn, Pm, sg, G);
        }
        P.ext(Rn, pn, true, sm_);  // Pn(2,1)
        {
            PlanePos q2 = x0;
            P.advance(q2, true, sm_, 2);
            su3<R> Pm = load_line(sm, sdm, 2, lane);
            P.ext(Pm, q2, false, sn);  // Pm(2,1)
            leaf_acc(Rn, Pm, sg * k12, Fhat);
        }
        P.ext(Rn, pn, true, sm_);  // Pn(3,1)
        {
            PlanePos q2 = x0;
            P.advance(q2, true, sm_, 3);
            su3<R> Pm = load_line(sm, sdm, 3, lane);
            P.ext(Pm, q2, false, sn);  // Pm(3,1)
            leaf_acc(Rn, Pm, sg * k13, Fhat);
        }
        // column: (1,2), (1,3)
        {
            PlanePos qm = x0;
            su3<R> Lm = P.step(qm, true, sm_);
            P.ext(Lm, qm, false, sn);
            P.ext(Lm, qm, false, sn);  // Pm(1,2)
            PlanePos q2 = x0;
            P.advance(q2, false, sn, 2);
            su3<R> Pn = load_line(sm, sdn, 2, lane);
            P.ext(Pn, q2, true, sm_);  // Pn(1,2)
            leaf_acc(Pn, Lm, sg * k12, Fhat);
            P.ext(Lm, qm, false, sn);  // Pm(1,3)
            PlanePos q3 = x0;
            P.advance(q3, false, sn, 3);
            Pn = load_line(sm, sdn, 3, lane);
            P.ext(Pn, q3, true, sm_);  // Pn(1,3)
            leaf_acc(Pn, Lm, sg * k13, Fhat);
        }
        // (2,2)
        {
            PlanePos q2 = x0;
            P.advance(q2, false, sn, 2);
            su3<R> Pn = load_line(sm, sdn, 2, lane);
            P.ext(Pn, q2, true, sm_);
            P.ext(Pn, q2, true, sm_);  // Pn(2,2)
            PlanePos qm = x0;
            P.advance(qm, true, sm_, 2);
            su3<R> Pm = load_line(sm, sdm, 2, lane);
            P.ext(Pm, qm, false, sn);
            P.ext(Pm, qm, false, sn);  // Pm(2,2)
            leaf_acc(Pn, Pm, sg * k22, Fhat);
        }
    }
}

template <typename R, bool OUT>
__device__ __forceinline__ void plane_fields_smem(const cplx<R>* __restrict__ U, const Geom& g, int s, const Coord& c,
                                                  int mu, int nu, MeasSmem<R, OUT>* sm, int lane, int qa, int qb,
                                                  alg<R>& Greg, alg<R>& Fhreg) {
    const int column = threadIdx.y * MEAS_SITES + lane;
    const PathStash<R> sa{&sm->stash[0][0][column]}, sb{&sm->stash[1][0][column]};
    if constexpr (meas_smem_acc<R>()) {
        R* col = &sm->acc[0][column];
        const SmemAcc<R> G{col}, Fhat{col + 8 * MEAS_ACC_STRIDE};
        plane_fields_body<R, OUT>(U, g, s, c, mu, nu, sm, lane, qa, qb, G, Fhat, sa, sb);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            Greg.v[k] = G.get(k);
            Fhreg.v[k] = Fhat.get(k);
        }
    } else {
        plane_fields_body<R, OUT>(U, g, s, c, mu, nu, sm, lane, qa, qb, RegAcc<R>{Greg}, RegAcc<R>{Fhreg}, sa, sb);
    }
}

// Measurement tile = (lattice, x0 slice, chunk of 32 consecutive sites of the
// slice); 6 x QS warps: warp y takes plane y % 6 and the quadrants of part
// y / 6 (QS = 1: all four; QS = 2: two each).  Phase 0: the block's lines
// (warp w builds the lines of signed direction w, w + 6 QS, ...) into shared
// memory.  Phase 1: the
// quadrant sums of every (site, plane); with two parts the second part's sums
// meet the first's in the (then dead) line storage, in a fixed order, for F
// and F^.  Phase 2: the six planes meet in shared
// memory for e(x) and q(x); the tile's sums go to the lattice's
// partial[slice * nchunk + chunk] (double2).  The optional outputs of
// MeasOut (single-lattice passes) receive per-site densities and per
// (site, plane) F and F^.
//   e(x) = sum_{mu<nu} ReTr(F F)                 (EnergyDensity.cpp:13-20)
//   q(x) = ReTr(F^32 F^01) + ReTr(F^31 F^20) + ReTr(F^30 F^12)
//        = -T(23,01) + T(13,02) - T(03,12),  T(a,b) = ReTr(F^a F^b)
//                                             (TopologicalCharge.cpp:11-16)
template <typename R, bool OUT = false, int QS = MEAS_QSPLIT>
__global__ void __launch_bounds__(MEAS_SITES * 6 * QS, MeasMinBlocks<QS>::value) k_measure(const LatDesc<R>* __restrict__ descs,
                                                                           const int4* __restrict__ mtiles,
                                                                           const int2* __restrict__ seg,
                                                                           MeasOut out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MeasSmem<R, OUT>* sm = reinterpret_cast<MeasSmem<R, OUT>*>(smem_raw);
    const int lane = threadIdx.x, w = threadIdx.y, p = w % 6, part = w / 6;
    constexpr int NW = 6 * QS;  // warps of the block
    const int qa = part * 2, qb = qa + 2;  // QS = 2: this warp's quadrant half
    const int2 r = *seg;  // this launch's tiles: mtiles[r.x, r.x + r.y)
    for (int ti = r.x + blockIdx.x; ti < r.x + r.y; ti += gridDim.x) {
        const int4 tile = mtiles[ti];
        const LatDesc<R>* d = descs + tile.x;
        const Geom g = d->g;
        const int slice = tile.y, chunk = tile.z;
        const int off = meas_site_offset(g, meas_patched(g), chunk, lane);
        const bool valid = off < g.Vs;
        const int s = slice * g.Vs + (valid ? off : 0);
        const Coord c = site_coord(g, s);
        const cplx<R>* __restrict__ U = d->U0;
        // phase 0: lines of length 2 and 3 in the 8 signed directions
        for (int sdir = w; sdir < 8; sdir += NW) {
            const int dir = sdir >> 1, sign = (sdir & 1) ? -1 : 1;
            Plane<R> L;
            L.U = U;
            L.V = g.V;
            L.mu = dir;
            L.nu = dir;
            L.dm = dir_of(g, c, dir);
            L.dn = L.dm;
            PlanePos y = {s, L.dm.x, L.dm.x};
            su3<R> acc = L.step(y, true, sign);
            L.ext(acc, y, true, sign);
            store_line(sm, sdir, 2, lane, acc);
            L.ext(acc, y, true, sign);
            store_line(sm, sdir, 3, lane, acc);
        }
        __syncthreads();
        // phase 1: this thread's plane and quadrants; with one warp per plane
        // the two quadrant halves are still summed apart and then added, the
        // order two warps per plane use, so both give the same bits
        alg<R> G, Fh;
        if (valid) {
            if (QS == 1) {
#pragma unroll 1
                for (int h = 0; h < 2; ++h) {
                    alg<R> G1, F1;
                    plane_fields_smem<R, OUT>(U, g, s, c, c_plane_mu[p], c_plane_nu[p], sm, lane, 2 * h, 2 * h + 2, G1, F1);
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        G.v[k] = h ? G.v[k] + G1.v[k] : G1.v[k];
                        Fh.v[k] = h ? Fh.v[k] + F1.v[k] : F1.v[k];
                    }
                }
            } else {
                plane_fields_smem<R, OUT>(U, g, s, c, c_plane_mu[p], c_plane_nu[p], sm, lane, qa, qb, G, Fh);
            }
        }
        if (QS == 2) {
            __syncthreads();  // every warp is done with the lines
            if (part == 1 && valid) {
                sm->part.G[p][lane] = G;
                sm->part.Fh[p][lane] = Fh;
            }
            __syncthreads();
            if (part == 0 && valid) {
                const alg<R> G1 = sm->part.G[p][lane], F1 = sm->part.Fh[p][lane];
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    G.v[k] += G1.v[k];
                    Fh.v[k] += F1.v[k];
                }
            }
        }
        if (part == 0 && valid) {
            alg<R> F11;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                F11.v[k] = R(0.25) * G.v[k];
                Fh.v[k] = fma(R(19.0 / 36.0), G.v[k], Fh.v[k]);
            }
            sm->F[p][lane] = Fh;
            sm->E[p][lane] = retr_hh(F11, F11);
            if (OUT) {
                sm->C[p][lane] = F11;
                if (out.dbg_clover) store_alg_as_herm(out.dbg_clover + ((size_t)s * 6 + p) * 9, F11);
                if (out.dbg_improved) store_alg_as_herm(out.dbg_improved + ((size_t)s * 6 + p) * 9, Fh);
            }
        }
        __syncthreads();
        // phase 2: the site's e(x), q(x) and the tile's sums
        if (w == 0) {
            double e = 0.0, q = 0.0;
            if (valid) {
                e = ((sm->E[0][lane] + sm->E[1][lane]) + (sm->E[2][lane] + sm->E[3][lane])) +
                    (sm->E[4][lane] + sm->E[5][lane]);
                q = -retr_hh(sm->F[5][lane], sm->F[0][lane]) + retr_hh(sm->F[4][lane], sm->F[1][lane]) -
                    retr_hh(sm->F[2][lane], sm->F[3][lane]);
                if (OUT && out.e) out.e[s] = e;
                if (OUT && out.q) out.q[s] = q;
                if (OUT && out.e_imp) {
                    double ei = 0.0;
#pragma unroll
                    for (int k = 0; k < 6; ++k) ei += retr_hh(sm->F[k][lane], sm->F[k][lane]);
                    out.e_imp[s] = ei;
                }
                if (OUT && out.q_clov)
                    out.q_clov[s] = -retr_hh(sm->C[5][lane], sm->C[0][lane]) + retr_hh(sm->C[4][lane], sm->C[1][lane]) -
                                    retr_hh(sm->C[2][lane], sm->C[3][lane]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                e += __shfl_xor_sync(0xffffffffu, e, o);
                q += __shfl_xor_sync(0xffffffffu, q, o);
            }
            if (lane == 0) d->partial[slice * d->nchunk + chunk] = make_double2(e, q);
        }
        __syncthreads();
    }
}

// Dynamic shared memory of k_measure<R> (above 48 KB for double: the
// attribute must be raised once per device before the first launch).
template <typename R, bool OUT = false> inline size_t measure_smem_bytes() { return sizeof(MeasSmem<R, OUT>); }
template <typename R, bool OUT = false, int QS = MEAS_QSPLIT> inline cudaError_t prepare_measure_kernel() {
    return cudaFuncSetAttribute(k_measure<R, OUT, QS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(MeasSmem<R, OUT>));
}

constexpr int RED_THREADS = 256;

// Slice sums in fixed order (deterministic run to run): thread i sums chunks
// i, i+256, ... sequentially, then a fixed binary tree.  One block per
// (lattice, slice) entry of rtiles.  Result slot layout per measurement:
// [E, Q, E_slice[N0], Q_slice[N0]] at meas + (*slot) * (2 + 2 N0).
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_slices(const LatDesc<R>* __restrict__ descs,
                                                               const int2* __restrict__ rtiles,
                                                               const int* __restrict__ nrtiles) {
    __shared__ double se[RED_THREADS], sq[RED_THREADS];
    const int n = *nrtiles;
    for (int ti = blockIdx.x; ti < n; ti += gridDim.x) {
        const int2 tile = rtiles[ti];
        const LatDesc<R>* d = descs + tile.x;
        const int t = tile.y;
        const int nchunk = d->nchunk;
        double e = 0.0, q = 0.0;
        for (int j = threadIdx.x; j < nchunk; j += RED_THREADS) {
            const double2 v = d->partial[t * nchunk + j];
            e += v.x;
            q += v.y;
        }
        se[threadIdx.x] = e;
        sq[threadIdx.x] = q;
        __syncthreads();
        for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                se[threadIdx.x] += se[threadIdx.x + w];
                sq[threadIdx.x] += sq[threadIdx.x + w];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const int N0 = d->g.n[0];
            const double inv4pi2 = 1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
            double* o = d->meas + (size_t)(*d->slot) * (2 + 2 * N0);
            o[2 + t] = se[0] / (double)d->g.Vs;
            o[2 + N0 + t] = sq[0] * inv4pi2;
            d->slice_sums[t] = make_double2(se[0], sq[0]);
        }
        __syncthreads();
    }
}

// Global sums over the slices (fixed tree), one block per lattice in jobs[].
template <typename R>
__global__ void __launch_bounds__(RED_THREADS) k_reduce_total(const LatDesc<R>* __restrict__ descs,
                                                              const int* __restrict__ jobs,
                                                              const int* __restrict__ njobs) {
    __shared__ double se[RED_THREADS], sq[RED_THREADS];
    const int n = *njobs;
    for (int ti = blockIdx.x; ti < n; ti += gridDim.x) {
        const LatDesc<R>* d = descs + jobs[ti];
        const int N0 = d->g.n[0];
        double e = 0.0, q = 0.0;
        for (int j = threadIdx.x; j < N0; j += RED_THREADS) {
            e += d->slice_sums[j].x;
            q += d->slice_sums[j].y;
        }
        se[threadIdx.x] = e;
        sq[threadIdx.x] = q;
        __syncthreads();
        for (int w = RED_THREADS / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) {
                se[threadIdx.x] += se[threadIdx.x + w];
                sq[threadIdx.x] += sq[threadIdx.x + w];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const double inv4pi2 = 1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
            double* o = d->meas + (size_t)(*d->slot) * (2 + 2 * N0);
            o[0] = se[0] * (1.0 / (double)d->g.V);  // EnergyDensity.cpp:26
            o[1] = sq[0] * inv4pi2;                 // TopologicalCharge.cpp:21
            *d->slot = *d->slot + 1;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- layouts
// File order (double, [s][mu][k][re,im]) <-> device layout in precision R.
// The 32 sites of one layout block occupy one contiguous run in both orders
// (file: 32 x 36 complex, site-major; device: 36 x 32 complex, entry-major),
// so a block of CONV_THREADS threads moves one layout block as a transpose
// through shared memory: both the global read and the global write are
// consecutive 16-byte (or 8-byte) words across the warp.  Sites past V in
// the last block are neither read nor written.
constexpr int CONV_THREADS = 256;
constexpr int CONV_PITCH = 37;  // 36 entries + 1: columns of the transpose hit distinct banks

template <typename R>
__global__ void __launch_bounds__(CONV_THREADS) k_to_device(const double2* __restrict__ file, cplx<R>* __restrict__ U,
                                                            int V) {
    __shared__ double2 t[LAYOUT_BLOCK * CONV_PITCH];
    const int b = blockIdx.x;
    const int s0 = b * LAYOUT_BLOCK;
    const int ns = min(LAYOUT_BLOCK, V - s0);
    const double2* src = file + (size_t)s0 * 36;
    for (int i = threadIdx.x; i < ns * 36; i += CONV_THREADS) t[(i / 36) * CONV_PITCH + i % 36] = src[i];
    __syncthreads();
    for (int j = threadIdx.x; j < 36 * LAYOUT_BLOCK; j += CONV_THREADS) {
        const int e = j / LAYOUT_BLOCK, site = j % LAYOUT_BLOCK;
        if (site < ns) {
            const double2 v = t[site * CONV_PITCH + e];
            stc(U + link_offset<R>(e / 9, e % 9, s0 + site), cmk<R>((R)v.x, (R)v.y));
        }
    }
}
template <typename R>
__global__ void __launch_bounds__(CONV_THREADS) k_to_file(const cplx<R>* __restrict__ U, double2* __restrict__ file,
                                                          int V) {
    __shared__ double2 t[LAYOUT_BLOCK * CONV_PITCH];
    const int b = blockIdx.x;
    const int s0 = b * LAYOUT_BLOCK;
    const int ns = min(LAYOUT_BLOCK, V - s0);
    for (int j = threadIdx.x; j < 36 * LAYOUT_BLOCK; j += CONV_THREADS) {
        const int e = j / LAYOUT_BLOCK, site = j % LAYOUT_BLOCK;
        if (site < ns) {
            const cplx<R> z = ldc(U + link_offset<R>(e / 9, e % 9, s0 + site));
            t[site * CONV_PITCH + e] = make_double2((double)z.re, (double)z.im);
        }
    }
    __syncthreads();
    double2* dst = file + (size_t)s0 * 36;
    for (int i = threadIdx.x; i < ns * 36; i += CONV_THREADS) dst[i] = t[(i / 36) * CONV_PITCH + i % 36];
}

// --------------------------------------------------------- generator G
// splitmix64 finaliser (Steele, Lea & Flood, OOPSLA 2014) as a counter hash;
// h_a ~ N(0,1) by Box-Muller; U = exp(i scale sum_a h_a lambda_a/2).
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double unit_open(unsigned long long seed, unsigned long long ctr) {
    const unsigned long long r = mix64(seed ^ mix64(ctr));
    return ((double)(r >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

template <typename R>
__global__ void k_generate_G(cplx<R>* __restrict__ U, int V, unsigned long long seed, double scale) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const int mu = t / V, s = t - mu * V;
    const unsigned long long l = (unsigned long long)s * 4ull + (unsigned long long)mu;  // file-order link index
    double h[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
        const unsigned long long c = l * 8ull + (unsigned long long)a;
        const double u1 = unit_open(seed, 2ull * c), u2 = unit_open(seed, 2ull * c + 1ull);
        h[a] = sqrt(-2.0 * log(u1)) * cos(6.28318530717958647692 * u2);
    }
    // X = i scale H,  H = sum_a h_a lambda_a / 2 ; coordinates of X:
    // X00 = i s (h2/2 + h7/(2 sqrt3)), X11 = i s (-h2/2 + h7/(2 sqrt3)),
    // X01 = i s (h0 - i h1)/2 = s (h1/2, h0/2), X02 = s (h4/2, h3/2), X12 = s (h6/2, h5/2)
    const double is3 = 0.57735026918962576451;
    alg<double> x;
    x.v[0] = scale * (0.5 * h[2] + 0.5 * is3 * h[7]);
    x.v[1] = scale * (-0.5 * h[2] + 0.5 * is3 * h[7]);
    x.v[2] = scale * 0.5 * h[1];
    x.v[3] = scale * 0.5 * h[0];
    x.v[4] = scale * 0.5 * h[4];
    x.v[5] = scale * 0.5 * h[3];
    x.v[6] = scale * 0.5 * h[6];
    x.v[7] = scale * 0.5 * h[5];
    const su3<double> e = expm_alg<double>(x);
    su3<R> o;
#pragma unroll
    for (int k = 0; k < 9; ++k) o.m[k] = cmk<R>((R)e.m[k].re, (R)e.m[k].im);
    store_link(U, V, mu, s, o);
}

// ------------------------------------------------------- reunitarisation
// FP32-mixed form only: rows r0, r1 by Gram-Schmidt in double, r2 = conj(r0 x r1).
template <typename R>
__global__ void k_reunitarize(cplx<R>* __restrict__ U, int V) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const int mu = t / V, s = t - mu * V;
    const su3<R> a = load_link(U, V, mu, s);
    cplx<double> r0[3], r1[3], r2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        r0[k] = cmk<double>(a.m[k].re, a.m[k].im);
        r1[k] = cmk<double>(a.m[3 + k].re, a.m[3 + k].im);
    }
    double n0 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) n0 += r0[k].re * r0[k].re + r0[k].im * r0[k].im;
    n0 = rsqrt(n0);
#pragma unroll
    for (int k = 0; k < 3; ++k) r0[k] = cmk<double>(r0[k].re * n0, r0[k].im * n0);
    cplx<double> d = cmk<double>(0.0, 0.0);  // <r0, r1> = sum conj(r0) r1
#pragma unroll
    for (int k = 0; k < 3; ++k) d = ccfma(r0[k], r1[k], d);
#pragma unroll
    for (int k = 0; k < 3; ++k) r1[k] = csub(r1[k], cmul(d, r0[k]));
    double n1 = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) n1 += r1[k].re * r1[k].re + r1[k].im * r1[k].im;
    n1 = rsqrt(n1);
#pragma unroll
    for (int k = 0; k < 3; ++k) r1[k] = cmk<double>(r1[k].re * n1, r1[k].im * n1);
    // r2 = conj(r0 x r1)
    r2[0] = csub(cmul(r0[1], r1[2]), cmul(r0[2], r1[1]));
    r2[1] = csub(cmul(r0[2], r1[0]), cmul(r0[0], r1[2]));
    r2[2] = csub(cmul(r0[0], r1[1]), cmul(r0[1], r1[0]));
    su3<R> o;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        o.m[k] = cmk<R>((R)r0[k].re, (R)r0[k].im);
        o.m[3 + k] = cmk<R>((R)r1[k].re, (R)r1[k].im);
        o.m[6 + k] = cmk<R>((R)r2[k].re, (R)(-r2[k].im));
    }
    store_link(U, V, mu, s, o);
}

// max over links of ||U^dag U - 1||_F (x) and |det U - 1| (y), per block
template <typename R>
__global__ void __launch_bounds__(256) k_unitarity(const cplx<R>* __restrict__ U, int V, double2* __restrict__ partial) {
    __shared__ double su[256], sd[256];
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double eu = 0.0, ed = 0.0;
    if (t < 4 * V) {
        const int mu = t / V, s = t - mu * V;
        const su3<R> a = load_link(U, V, mu, s);
        su3<double> b;
#pragma unroll
        for (int k = 0; k < 9; ++k) b.m[k] = cmk<double>(a.m[k].re, a.m[k].im);
        const su3<double> p = mul_an(b, b);
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const double re = p.m[k].re - ((k % 4) == 0 ? 1.0 : 0.0);
            acc += re * re + p.m[k].im * p.m[k].im;
        }
        eu = sqrt(acc);
        cplx<double> det = cmul(b.m[0], csub(cmul(b.m[4], b.m[8]), cmul(b.m[5], b.m[7])));
        det = csub(det, cmul(b.m[1], csub(cmul(b.m[3], b.m[8]), cmul(b.m[5], b.m[6]))));
        det = cadd(det, cmul(b.m[2], csub(cmul(b.m[3], b.m[7]), cmul(b.m[4], b.m[6]))));
        ed = hypot(det.re - 1.0, det.im);
    }
    su[threadIdx.x] = eu;
    sd[threadIdx.x] = ed;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            su[threadIdx.x] = fmax(su[threadIdx.x], su[threadIdx.x + w]);
            sd[threadIdx.x] = fmax(sd[threadIdx.x], sd[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(su[0], sd[0]);
}

// ---------------------------------------------------- per-function debug
// flow gradient Z(x, mu) for every link, file order [s][mu][9] (double2)
template <typename R>
__global__ void k_debug_gradient(const cplx<R>* __restrict__ U, Geom g, double2* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * g.V) return;
    const int mu = t / g.V, s = t - mu * g.V;
    const Coord c = site_coord(g, s);
    su3<R> u;
    const alg<R> Z = flow_gradient<R>(U, g, s, c, mu, u);
    store_alg_as_antiherm(out + ((size_t)s * 4 + mu) * 9, Z);
}

// exp(iP) for n anti-Hermitian traceless matrices given as full 3x3 (double2)
template <typename R>
__global__ void k_debug_exp(const double2* __restrict__ in, double2* __restrict__ out, int n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double2* m = in + (size_t)t * 9;
    alg<R> x;
    x.v[0] = (R)m[0].y;
    x.v[1] = (R)m[4].y;
    x.v[2] = (R)m[1].x;
    x.v[3] = (R)m[1].y;
    x.v[4] = (R)m[2].x;
    x.v[5] = (R)m[2].y;
    x.v[6] = (R)m[5].x;
    x.v[7] = (R)m[5].y;
    const su3<R> e = expm_alg(x);
#pragma unroll
    for (int k = 0; k < 9; ++k) out[(size_t)t * 9 + k] = make_double2(e.m[k].re, e.m[k].im);
}

}  // namespace lgf
