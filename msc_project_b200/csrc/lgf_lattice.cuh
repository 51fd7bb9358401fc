// Periodic 4-D lattice indexing and the device link layout.
//
// Replaces the reference's neighbour tables (LGF/Lattice/Lattice.cpp:190-230,
// LGF/Field/Field.h:49-62) with index arithmetic: global site index
// s = ((x0*N1 + x1)*N2 + x2)*N3 + x3 with x0 slowest (Lattice.cpp:423-436) and
// periodic wrap in every direction (the "torus" type, Lattice.cpp:447-459).
// One GPU holds the whole lattice, so there is no halo exchange.
//
// Device layout: blocks of 32 consecutive sites, each block holding every
// entry of its sites' four links (structure of arrays inside the block, see
// link_offset / alg_offset below for the exact placement):
//   links  36 complex entries per site and block row: double as 9 entry planes
//          per direction (a lane reads 16 B per entry), float as 4 planes of
//          entry pairs (16 B per lane) plus one plane of the 9th entry
//   su(3)  8 coordinates per link (lgf_su3.cuh), pairs (double) or quads
//          (float) per lane
// Every load of a warp of 32 consecutive sites is one contiguous run (512 B),
// and the links of a site range sit together (18 KB per block in double)
// instead of in 36 arrays of V entries each: a stencil over a large lattice
// touches a few pages per neighbour instead of dozens.  Buffers hold
// padded_sites(V) sites.
#pragma once
#include <stdint.h>
#include "lgf_su3.cuh"

// -DLGF_CHECKED: host-side uses of the index arithmetic assert that every
// coordinate, direction and site index stays in range (the CPU index check,
// lgf_check_index.cu); device code is unchanged.
#if defined(LGF_CHECKED) && !defined(__CUDA_ARCH__)
#include <cstdio>
#include <cstdlib>
#define LGF_INDEX_ASSERT(cond)                                                                      \
    do {                                                                                            \
        if (!(cond)) {                                                                              \
            std::fprintf(stderr, "LGF_CHECKED: index check failed: %s (%s:%d)\n", #cond, __FILE__, __LINE__); \
            std::abort();                                                                           \
        }                                                                                           \
    } while (0)
#else
#define LGF_INDEX_ASSERT(cond) ((void)0)
#endif

namespace lgf {

struct Geom {
    int n[4];          // extents N0..N3
    int stride[4];     // N1N2N3, N2N3, N3, 1
    int V;             // total sites
    int Vs;            // sites per x0 slice
};

inline Geom make_geom(const int shape[4]) {
    Geom g;
    for (int d = 0; d < 4; ++d) g.n[d] = shape[d];
    g.stride[3] = 1;
    g.stride[2] = shape[3];
    g.stride[1] = shape[3] * shape[2];
    g.stride[0] = shape[3] * shape[2] * shape[1];
    g.Vs = g.stride[0];
    g.V = g.stride[0] * shape[0];
    return g;
}

struct Coord { int x[4]; };

__host__ __device__ __forceinline__ Coord site_coord(const Geom& g, int s) {
    LGF_INDEX_ASSERT(s >= 0 && s < g.V);
    Coord c;
    unsigned r = (unsigned)s;
    c.x[3] = (int)(r % (unsigned)g.n[3]); r /= (unsigned)g.n[3];
    c.x[2] = (int)(r % (unsigned)g.n[2]); r /= (unsigned)g.n[2];
    c.x[1] = (int)(r % (unsigned)g.n[1]); r /= (unsigned)g.n[1];
    c.x[0] = (int)r;
    return c;
}

// index of the neighbour of s (whose d-coordinate is xd) one step forward / back in d
__host__ __device__ __forceinline__ int fwd(const Geom& g, int s, int d, int xd) {
    LGF_INDEX_ASSERT(d >= 0 && d < 4 && xd >= 0 && xd < g.n[d] && s >= 0 && s < g.V);
    const int r = (xd == g.n[d] - 1) ? s - (g.n[d] - 1) * g.stride[d] : s + g.stride[d];
    LGF_INDEX_ASSERT(r >= 0 && r < g.V);
    return r;
}
__host__ __device__ __forceinline__ int bwd(const Geom& g, int s, int d, int xd) {
    LGF_INDEX_ASSERT(d >= 0 && d < 4 && xd >= 0 && xd < g.n[d] && s >= 0 && s < g.V);
    const int r = (xd == 0) ? s + (g.n[d] - 1) * g.stride[d] : s - g.stride[d];
    LGF_INDEX_ASSERT(r >= 0 && r < g.V);
    return r;
}
__host__ __device__ __forceinline__ int wrap_inc(int x, int n) { return x == n - 1 ? 0 : x + 1; }
__host__ __device__ __forceinline__ int wrap_dec(int x, int n) { return x == 0 ? n - 1 : x - 1; }

// One lattice direction as plain scalars (extent, stride, and the thread's
// coordinate along it).  Selected without indexing a local array, so nothing
// spills to local memory when the direction is only known at run time.
struct Dir { int n, stride, x; };

__host__ __device__ __forceinline__ int sel4(int d, int a0, int a1, int a2, int a3) {
    return d == 0 ? a0 : (d == 1 ? a1 : (d == 2 ? a2 : a3));
}
__host__ __device__ __forceinline__ Dir dir_of(const Geom& g, const Coord& c, int d) {
    LGF_INDEX_ASSERT(d >= 0 && d < 4);
    Dir r;
    r.n = sel4(d, g.n[0], g.n[1], g.n[2], g.n[3]);
    r.stride = sel4(d, g.stride[0], g.stride[1], g.stride[2], g.stride[3]);
    r.x = sel4(d, c.x[0], c.x[1], c.x[2], c.x[3]);
    return r;
}
__host__ __device__ __forceinline__ int fwd(int s, const Dir& d) {
    LGF_INDEX_ASSERT(d.x >= 0 && d.x < d.n && s >= 0);
    return (d.x == d.n - 1) ? s - (d.n - 1) * d.stride : s + d.stride;
}
__host__ __device__ __forceinline__ int bwd(int s, const Dir& d) {
    LGF_INDEX_ASSERT(d.x >= 0 && d.x < d.n && s >= 0);
    return (d.x == 0) ? s + (d.n - 1) * d.stride : s - d.stride;
}

template <typename R> struct vec2_of;
template <> struct vec2_of<double> { typedef double2 type; };
template <> struct vec2_of<float> { typedef float2 type; };

template <typename R> __device__ __forceinline__ cplx<R> ldc(const cplx<R>* p) {
    typedef typename vec2_of<R>::type V2;
    V2 v = __ldg(reinterpret_cast<const V2*>(p));
    return cmk<R>(v.x, v.y);
}
template <typename R> __device__ __forceinline__ void stc(cplx<R>* p, cplx<R> z) {
    typedef typename vec2_of<R>::type V2;
    V2 v;
    v.x = z.re;
    v.y = z.im;
    *reinterpret_cast<V2*>(p) = v;
}

#ifndef LGF_LAYOUT_BLOCK
#define LGF_LAYOUT_BLOCK 32
#endif
constexpr int LAYOUT_BLOCK = LGF_LAYOUT_BLOCK;  // sites per layout block
__host__ __device__ __forceinline__ size_t padded_sites(size_t V) { return (V + LAYOUT_BLOCK - 1) / LAYOUT_BLOCK * LAYOUT_BLOCK; }
// Offset, in complex entries, of entry k (3*row + col) of link mu at site s.
//   double: per 32-site block and direction, 9 entry planes of 32 sites: a
//           lane's entry is one 16-byte double2 load, a warp's 512 B;
//   float:  entries 0..7 in pairs -- plane p holds entries 2p and 2p+1 of each
//           site side by side, one 16-byte float4 per lane -- and entry 8 in a
//           plane of float2: a link is four 128-bit loads and one 64-bit load.
// Both put the 36 entries of a block's four links in one contiguous run.
template <typename R> __host__ __device__ __forceinline__ size_t link_offset(int mu, int k, int s) {
    LGF_INDEX_ASSERT(mu >= 0 && mu < 4 && k >= 0 && k < 9 && s >= 0);
    const size_t base = (size_t)(s / LAYOUT_BLOCK) * 36 * LAYOUT_BLOCK + (size_t)mu * 9 * LAYOUT_BLOCK;
    const int l = s % LAYOUT_BLOCK;
    if constexpr (sizeof(R) == sizeof(double)) {
        return base + (size_t)k * LAYOUT_BLOCK + l;
    } else {
        return k < 8 ? base + (size_t)(k >> 1) * 2 * LAYOUT_BLOCK + 2 * l + (k & 1) : base + 8 * LAYOUT_BLOCK + l;
    }
}
// Offset, in reals, of coordinate c of the su(3) accumulator of link mu at
// site s: coordinates in pairs (double: one double2 per lane) or quads
// (float: one float4 per lane), planes of 32 sites per block and direction.
template <typename R> __host__ __device__ __forceinline__ size_t alg_offset(int mu, int c, int s) {
    LGF_INDEX_ASSERT(mu >= 0 && mu < 4 && c >= 0 && c < 8 && s >= 0);
    const size_t base = (size_t)(s / LAYOUT_BLOCK) * 32 * LAYOUT_BLOCK + (size_t)mu * 8 * LAYOUT_BLOCK;
    const int l = s % LAYOUT_BLOCK;
    if constexpr (sizeof(R) == sizeof(double))
        return base + (size_t)(c >> 1) * 2 * LAYOUT_BLOCK + 2 * l + (c & 1);
    else
        return base + (size_t)(c >> 2) * 4 * LAYOUT_BLOCK + 4 * l + (c & 3);
}

// (V is kept in the signatures: the lattice volume, no longer a stride)
template <typename R> __device__ __forceinline__ su3<R> load_link(const cplx<R>* __restrict__ U, int V, int mu, int s) {
    su3<R> a;
    if constexpr (sizeof(R) == sizeof(double)) {
        const cplx<R>* p = U + link_offset<R>(mu, 0, s);
#pragma unroll
        for (int k = 0; k < 9; ++k) a.m[k] = ldc(p + k * LAYOUT_BLOCK);
    } else {
        const float4* p = reinterpret_cast<const float4*>(U + link_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 v = __ldg(p + q * LAYOUT_BLOCK);
            a.m[2 * q] = cmk<R>(v.x, v.y);
            a.m[2 * q + 1] = cmk<R>(v.z, v.w);
        }
        a.m[8] = ldc(U + link_offset<R>(mu, 8, s));
    }
    return a;
}
template <typename R> __device__ __forceinline__ void store_link(cplx<R>* __restrict__ U, int V, int mu, int s, const su3<R>& a) {
    if constexpr (sizeof(R) == sizeof(double)) {
        cplx<R>* p = U + link_offset<R>(mu, 0, s);
#pragma unroll
        for (int k = 0; k < 9; ++k) stc(p + k * LAYOUT_BLOCK, a.m[k]);
    } else {
        float4* p = reinterpret_cast<float4*>(U + link_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 4; ++q)
            p[q * LAYOUT_BLOCK] = make_float4(a.m[2 * q].re, a.m[2 * q].im, a.m[2 * q + 1].re, a.m[2 * q + 1].im);
        stc(U + link_offset<R>(mu, 8, s), a.m[8]);
    }
}
template <typename R> __device__ __forceinline__ alg<R> load_alg(const R* __restrict__ A, int V, int mu, int s) {
    alg<R> z;
    if constexpr (sizeof(R) == sizeof(double)) {
        const double2* p = reinterpret_cast<const double2*>(A + alg_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const double2 v = __ldg(p + q * LAYOUT_BLOCK);
            z.v[2 * q] = v.x;
            z.v[2 * q + 1] = v.y;
        }
    } else {
        const float4* p = reinterpret_cast<const float4*>(A + alg_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const float4 v = __ldg(p + q * LAYOUT_BLOCK);
            z.v[4 * q] = v.x;
            z.v[4 * q + 1] = v.y;
            z.v[4 * q + 2] = v.z;
            z.v[4 * q + 3] = v.w;
        }
    }
    return z;
}
template <typename R> __device__ __forceinline__ void store_alg(R* __restrict__ A, int V, int mu, int s, const alg<R>& z) {
    if constexpr (sizeof(R) == sizeof(double)) {
        double2* p = reinterpret_cast<double2*>(A + alg_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 4; ++q) p[q * LAYOUT_BLOCK] = make_double2(z.v[2 * q], z.v[2 * q + 1]);
    } else {
        float4* p = reinterpret_cast<float4*>(A + alg_offset<R>(mu, 0, s));
#pragma unroll
        for (int q = 0; q < 2; ++q)
            p[q * LAYOUT_BLOCK] = make_float4(z.v[4 * q], z.v[4 * q + 1], z.v[4 * q + 2], z.v[4 * q + 3]);
    }
}

}  // namespace lgf
