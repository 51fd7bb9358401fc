// Register-resident SU(3) arithmetic for the Wilson-flow kernels.
//
// Replaces the reference's heap-allocated su3_mat / C_double
// (LGF/Math/SU3_mat.{h,cpp}, LGF/Math/C_double.h): a matrix is 9 complex
// entries held in registers, row-major m[3*r+c] like the reference.  R is the
// storage/arithmetic precision of links and matrix products (double for the
// plain FP64 form, float for the FP32-mixed form); the Cayley-Hamilton
// coefficient solve of the exponential always runs in double.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace lgf {

template <typename R> struct alignas(2 * sizeof(R)) cplx { R re, im; };

template <typename R> __host__ __device__ __forceinline__ cplx<R> cmk(R r, R i) { cplx<R> z; z.re = r; z.im = i; return z; }
template <typename R> __host__ __device__ __forceinline__ cplx<R> cadd(cplx<R> a, cplx<R> b) { return cmk<R>(a.re + b.re, a.im + b.im); }
template <typename R> __host__ __device__ __forceinline__ cplx<R> csub(cplx<R> a, cplx<R> b) { return cmk<R>(a.re - b.re, a.im - b.im); }
template <typename R> __host__ __device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
    return cmk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// a * conj(b)
template <typename R> __host__ __device__ __forceinline__ cplx<R> cmulc(cplx<R> a, cplx<R> b) {
    return cmk<R>(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im);
}
// conj(a) * b
template <typename R> __host__ __device__ __forceinline__ cplx<R> ccmul(cplx<R> a, cplx<R> b) {
    return cmk<R>(a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re);
}
// acc + a*b
template <typename R> __host__ __device__ __forceinline__ cplx<R> cfma(cplx<R> a, cplx<R> b, cplx<R> acc) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
    return acc;
}
// acc + a*conj(b)
template <typename R> __host__ __device__ __forceinline__ cplx<R> cfmac(cplx<R> a, cplx<R> b, cplx<R> acc) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(a.im, b.im, acc.re);
    acc.im = fma(a.im, b.re, acc.im);
    acc.im = fma(-a.re, b.im, acc.im);
    return acc;
}
// acc + conj(a)*b
template <typename R> __host__ __device__ __forceinline__ cplx<R> ccfma(cplx<R> a, cplx<R> b, cplx<R> acc) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(-a.im, b.re, acc.im);
    return acc;
}

template <typename R> struct su3 { cplx<R> m[9]; };

template <typename R> __host__ __device__ __forceinline__ void su3_zero(su3<R>& a) {
#pragma unroll
    for (int k = 0; k < 9; ++k) a.m[k] = cmk<R>(R(0), R(0));
}

// c = a * b
template <typename R> __device__ __forceinline__ su3<R> mul_nn(const su3<R>& a, const su3<R>& b) {
    su3<R> c;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = cmul(a.m[3 * r], b.m[col]);
            s = cfma(a.m[3 * r + 1], b.m[3 + col], s);
            s = cfma(a.m[3 * r + 2], b.m[6 + col], s);
            c.m[3 * r + col] = s;
        }
    return c;
}
// c = a * b^dag
template <typename R> __device__ __forceinline__ su3<R> mul_na(const su3<R>& a, const su3<R>& b) {
    su3<R> c;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = cmulc(a.m[3 * r], b.m[3 * col]);
            s = cfmac(a.m[3 * r + 1], b.m[3 * col + 1], s);
            s = cfmac(a.m[3 * r + 2], b.m[3 * col + 2], s);
            c.m[3 * r + col] = s;
        }
    return c;
}
// c = a^dag * b
template <typename R> __device__ __forceinline__ su3<R> mul_an(const su3<R>& a, const su3<R>& b) {
    su3<R> c;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = ccmul(a.m[r], b.m[col]);
            s = ccfma(a.m[3 + r], b.m[3 + col], s);
            s = ccfma(a.m[6 + r], b.m[6 + col], s);
            c.m[3 * r + col] = s;
        }
    return c;
}
// acc += a * b
template <typename R> __device__ __forceinline__ void acc_nn(su3<R>& acc, const su3<R>& a, const su3<R>& b) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = acc.m[3 * r + col];
            s = cfma(a.m[3 * r], b.m[col], s);
            s = cfma(a.m[3 * r + 1], b.m[3 + col], s);
            s = cfma(a.m[3 * r + 2], b.m[6 + col], s);
            acc.m[3 * r + col] = s;
        }
}
// acc += a * b^dag
template <typename R> __device__ __forceinline__ void acc_na(su3<R>& acc, const su3<R>& a, const su3<R>& b) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = acc.m[3 * r + col];
            s = cfmac(a.m[3 * r], b.m[3 * col], s);
            s = cfmac(a.m[3 * r + 1], b.m[3 * col + 1], s);
            s = cfmac(a.m[3 * r + 2], b.m[3 * col + 2], s);
            acc.m[3 * r + col] = s;
        }
}
// acc += a^dag * b
template <typename R> __device__ __forceinline__ void acc_an(su3<R>& acc, const su3<R>& a, const su3<R>& b) {
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = acc.m[3 * r + col];
            s = ccfma(a.m[r], b.m[col], s);
            s = ccfma(a.m[3 + r], b.m[3 + col], s);
            s = ccfma(a.m[6 + r], b.m[6 + col], s);
            acc.m[3 * r + col] = s;
        }
}

#ifndef LGF_SU3_ROW3
#define LGF_SU3_ROW3 1  // products of links that feed the force or a measurement: third row as conj(r0 x r1)
#endif
// c = a * b for a, b in SU(3): rows 0 and 1 as products, row 2 as
// conj(r0 x r1), which for a unitary product with det 1 is the same row
// (96 real operations instead of 108; equal to rounding on SU(3) inputs).
// Used for the staple's intermediate products, which only feed the force,
// and for the measurement's path products; a stored link is never built
// this way.
template <typename R> __device__ __forceinline__ su3<R> mul_nn_su3(const su3<R>& a, const su3<R>& b) {
    if (!LGF_SU3_ROW3) return mul_nn(a, b);
    su3<R> c;
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = cmul(a.m[3 * r], b.m[col]);
            s = cfma(a.m[3 * r + 1], b.m[3 + col], s);
            c.m[3 * r + col] = cfma(a.m[3 * r + 2], b.m[6 + col], s);
        }
    // conj(r0 x r1): (r0_1 r1_2 - r0_2 r1_1, r0_2 r1_0 - r0_0 r1_2, r0_0 r1_1 - r0_1 r1_0)*
    const cplx<R> x0 = csub(cmul(c.m[1], c.m[5]), cmul(c.m[2], c.m[4]));
    const cplx<R> x1 = csub(cmul(c.m[2], c.m[3]), cmul(c.m[0], c.m[5]));
    const cplx<R> x2 = csub(cmul(c.m[0], c.m[4]), cmul(c.m[1], c.m[3]));
    c.m[6] = cmk<R>(x0.re, -x0.im);
    c.m[7] = cmk<R>(x1.re, -x1.im);
    c.m[8] = cmk<R>(x2.re, -x2.im);
    return c;
}

// c = a * b^dag for a, b in SU(3), the third row rebuilt as in mul_nn_su3
template <typename R> __device__ __forceinline__ su3<R> mul_na_su3(const su3<R>& a, const su3<R>& b) {
    if (!LGF_SU3_ROW3) return mul_na(a, b);
    su3<R> c;
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int col = 0; col < 3; ++col) {
            cplx<R> s = cmulc(a.m[3 * r], b.m[3 * col]);
            s = cfmac(a.m[3 * r + 1], b.m[3 * col + 1], s);
            c.m[3 * r + col] = cfmac(a.m[3 * r + 2], b.m[3 * col + 2], s);
        }
    const cplx<R> x0 = csub(cmul(c.m[1], c.m[5]), cmul(c.m[2], c.m[4]));
    const cplx<R> x1 = csub(cmul(c.m[2], c.m[3]), cmul(c.m[0], c.m[5]));
    const cplx<R> x2 = csub(cmul(c.m[0], c.m[4]), cmul(c.m[1], c.m[3]));
    c.m[6] = cmk<R>(x0.re, -x0.im);
    c.m[7] = cmk<R>(x1.re, -x1.im);
    c.m[8] = cmk<R>(x2.re, -x2.im);
    return c;
}

template <typename R> __device__ __forceinline__ void su3_addto(su3<R>& a, const su3<R>& b) {
#pragma unroll
    for (int k = 0; k < 9; ++k) a.m[k] = cadd(a.m[k], b.m[k]);
}

// An element of su(3) stored as its 8 real coordinates.  For an
// anti-Hermitian traceless X:  v = (Im X00, Im X11, Re X01, Im X01,
// Re X02, Im X02, Re X12, Im X12), X22 = -i(v0+v1), X_ji = -conj(X_ij).
template <typename R> struct alg { R v[8]; };

// Traceless anti-Hermitian part  (W - W^dag) - 1/3 Tr(W - W^dag), scaled by s,
// as 8 coordinates.  Only the entries needed are read.
template <typename R> __device__ __forceinline__ alg<R> ta_part(const su3<R>& W, R s) {
    alg<R> z;
    R d0 = R(2) * W.m[0].im, d1 = R(2) * W.m[4].im, d2 = R(2) * W.m[8].im;
    R tr = (d0 + d1 + d2) * R(1.0 / 3.0);
    z.v[0] = s * (d0 - tr);
    z.v[1] = s * (d1 - tr);
    z.v[2] = s * (W.m[1].re - W.m[3].re);
    z.v[3] = s * (W.m[1].im + W.m[3].im);
    z.v[4] = s * (W.m[2].re - W.m[6].re);
    z.v[5] = s * (W.m[2].im + W.m[6].im);
    z.v[6] = s * (W.m[5].re - W.m[7].re);
    z.v[7] = s * (W.m[5].im + W.m[7].im);
    return z;
}

// Hermitian traceless Q = -i X from the 8 coordinates of X (double).
struct herm_d {
    double a0, a1, a2;            // real diagonal
    cplx<double> q01, q02, q12;   // upper triangle
};

template <typename R> __device__ __forceinline__ herm_d herm_from_alg(const alg<R>& x) {
    herm_d h;
    h.a0 = (double)x.v[0];
    h.a1 = (double)x.v[1];
    h.a2 = -(h.a0 + h.a1);
    // Q01 = -i X01 = (Im X01, -Re X01)
    h.q01 = cmk<double>((double)x.v[3], -(double)x.v[2]);
    h.q02 = cmk<double>((double)x.v[5], -(double)x.v[4]);
    h.q12 = cmk<double>((double)x.v[7], -(double)x.v[6]);
    return h;
}

// Cayley-Hamilton coefficients f0, f1, f2 with exp(iQ) = f0 + f1 Q + f2 Q^2
// for Hermitian traceless Q.  Below c1 = 0.25 the series form above; from
// there the closed form of Morningstar & Peardon (hep-lat/0311018, eqs.
// 14-34), with the reference's branch structure and thresholds
// (LGF/Math/SU3_mat.cpp:216-289): analytic form when c1 > 1e-4, otherwise the
// two-variable series; xi0 = sin(w)/w by series when |w| <= 0.05; the
// conjugation rule for c0 < 0.  c0 = ReTr(Q^3)/3 = det Q and
// c1 = ReTr(Q^2)/2 are taken as inputs.  The acos argument is clamped to
// [0, 1] (the reference clamps only in its _DEBUG build, SU3_mat.cpp:231-238;
// without the clamp a rounding excess above 1 would give NaN).
// Series form used below c1 = 0.25 (eigenvalues |lambda| <= 2 sqrt(c1/3) < 0.58):
// with Q^3 = c1 Q + c0 (Cayley-Hamilton), Q^n = a_n + b_n Q + d_n Q^2 where
// a_{n+1} = c0 d_n, b_{n+1} = a_n + c1 d_n, d_{n+1} = b_n, and
// f_j = sum_n i^n {a,b,d}_n / n!.  17 terms leave a remainder below 1e-19 for
// every c1 < 0.25; fewer suffice for smaller c1 (ch_series_terms), so it
// agrees with the closed form to rounding while needing no transcendental
// function (the flow's exponents are small: c1 is ~1e-5..1e-2 at eps = 0.01).
#ifndef LGF_CH_TERMS
#define LGF_CH_TERMS 1  // the series stops at the first term count whose tail bound is below 1e-17
#endif
// Terms the series needs for c1: the truncated series is the same polynomial
// in Q, so its error in operator norm is the exponential's tail,
// rho^(N+1)/(N+1)! * 2 with rho^2 = 4 c1 / 3 the largest |eigenvalue|^2;
// N terms keep it below 1e-17 for c1 below these bounds (compared through
// the high word of the non-negative double c1, an integer comparison: a
// smaller high word means a smaller value).
__device__ __forceinline__ int ch_series_terms(double c1) {
    if (!LGF_CH_TERMS) return 17;
    const int hi = __double2hiint(c1);
    return hi < 0x3ee818a5 ? 5    // c1 < 1.149e-5
         : hi < 0x3f1999da ? 6    // 9.766e-5
         : hi < 0x3f407746 ? 7    // 5.025e-4
         : hi < 0x3f5e3864 ? 8    // 1.8445e-3
         : hi < 0x3f75d5da ? 9    // 5.3309e-3
         : hi < 0x3f8a78af ? 10   // 1.29255e-2
         : hi < 0x3f9c1765 ? 11   // 2.7433e-2
         : hi < 0x3faae18a ? 12   // 5.2502e-2
         : hi < 0x3fb7b1af ? 13   // 9.2555e-2
         : hi < 0x3fc38b04 ? 14   // 0.15268
         : hi < 0x3fce877e ? 15   // 0.23851
                           : 17;
}

__device__ __forceinline__ void ch_series(double c0, double c1, cplx<double>& f0, cplx<double>& f1,
                                          cplx<double>& f2) {
    double a = 1.0, b = 0.0, d = 0.0, inv = 1.0;
    double r0 = 1.0, i0 = 0.0, r1 = 0.0, i1 = 0.0, r2 = 0.0, i2 = 0.0;
    const int nterms = ch_series_terms(c1);
#pragma unroll
    for (int n = 1; n <= 17; ++n) {
        if (n > nterms) break;
        const double an = c0 * d, bn = fma(c1, d, a);
        d = b;
        a = an;
        b = bn;
        inv *= 1.0 / (double)n;
        const double ta = a * inv, tb = b * inv, td = d * inv;
        switch (n & 3) {  // i^n
            case 0: r0 += ta; r1 += tb; r2 += td; break;
            case 1: i0 += ta; i1 += tb; i2 += td; break;
            case 2: r0 -= ta; r1 -= tb; r2 -= td; break;
            default: i0 -= ta; i1 -= tb; i2 -= td; break;
        }
    }
    f0 = cmk<double>(r0, i0);
    f1 = cmk<double>(r1, i1);
    f2 = cmk<double>(r2, i2);
}

__device__ __forceinline__ void ch_coefficients(double c0, double c1, cplx<double>& f0, cplx<double>& f1,
                                                cplx<double>& f2) {
    if (c1 < 0.25) {
        ch_series(c0, c1, f0, f1, f2);
        return;
    }
    if (c1 > 0.0001) {
        const double c1s = sqrt(c1);
        const double t = c1 * (1.0 / 3.0);
        double r = fabs(c0) / (2.0 * t * sqrt(t));
        r = fmin(r, 1.0);
        const double th3 = acos(r) * (1.0 / 3.0);
        double sth, cth;
        sincos(th3, &sth, &cth);
        const double u = 0.57735026918962576451 * c1s * cth;   // sqrt(1/3)
        const double w = c1s * sth;
        const double u2 = u * u, w2 = w * w;
        double us, uc, ws, wc;
        sincos(u, &us, &uc);
        sincos(w, &ws, &wc);
        const double xi0 = fabs(w) > 0.05 ? ws / w : 1.0 - w2 * (1.0 - w2 * (1.0 - w2 / 42.0) / 20.0) / 6.0;
        const double div = 1.0 / (9.0 * u2 - w2);
        const cplx<double> e2iu = cmk<double>(2.0 * uc * uc - 1.0, 2.0 * uc * us);
        const cplx<double> emiu = cmk<double>(uc, -us);
        cplx<double> h0 = cadd(cmk<double>(e2iu.re * (u2 - w2), e2iu.im * (u2 - w2)),
                               cmul(emiu, cmk<double>(8.0 * u2 * wc, 2.0 * u * (3.0 * u2 + w2) * xi0)));
        cplx<double> h1 = csub(cmk<double>(e2iu.re * 2.0 * u, e2iu.im * 2.0 * u),
                               cmul(emiu, cmk<double>(2.0 * u * wc, (w2 - 3.0 * u2) * xi0)));
        cplx<double> h2 = csub(e2iu, cmul(emiu, cmk<double>(wc, 3.0 * u * xi0)));
        f0 = cmk<double>(h0.re * div, h0.im * div);
        f1 = cmk<double>(h1.re * div, h1.im * div);
        f2 = cmk<double>(h2.re * div, h2.im * div);
        if (c0 < 0.0) {
            f0.im = -f0.im;
            f1.re = -f1.re;
            f2.im = -f2.im;
        }
    } else {
        const double c02 = c0 * c0;
        f0 = cmk<double>(1.0 - c02 / 720.0, -c0 * (1.0 - c1 * (1.0 - c1 / 42.0) / 20.0) / 6.0);
        f1 = cmk<double>(c0 * (1.0 - c1 * (1.0 - 3.0 * c1 / 112.0) / 15.0) / 24.0,
                         1.0 - c1 * (1.0 - c1 * (1.0 - c1 / 42.0) / 20.0) / 6.0 - c02 / 5040.0);
        f2 = cmk<double>((-1.0 + c1 * (1.0 - c1 * (1.0 - c1 / 56.0) / 30.0) / 12.0 + c02 / 20160.0) / 2.0,
                         (c0 * (1.0 - c1 * (1.0 - c1 / 48.0) / 21.0) / 60.0) / 2.0);
    }
}

#ifndef LGF_HERM_EXP
#define LGF_HERM_EXP 1  // exp(iQ) = f0 + f1 Q + f2 Q^2 assembled from Q's Hermitian structure
#endif

// f0 + f1 Q + f2 Q^2 for Hermitian traceless Q (diagonal a_i real, upper
// triangle q_ij, lower conj(q_ij)), using that structure: the diagonal of
// Q^2 is a sum of squares, Q^2_01 = -a2 q01 + q02 conj(q12),
// Q^2_02 = -a1 q02 + q01 q12, Q^2_12 = conj(q01) q02 - a0 q12 (a0+a1+a2 = 0),
// and real diagonals multiply the f's as reals: 33 + 60 real operations where
// the general complex products take 72 + 75.
template <typename R>
__device__ __forceinline__ su3<R> exp_assemble_herm(const herm_d& h, cplx<double> f0, cplx<double> f1, cplx<double> f2) {
    const R a0 = (R)h.a0, a1 = (R)h.a1, a2 = (R)h.a2;
    const cplx<R> q01 = cmk<R>((R)h.q01.re, (R)h.q01.im), q02 = cmk<R>((R)h.q02.re, (R)h.q02.im),
                  q12 = cmk<R>((R)h.q12.re, (R)h.q12.im);
    const R n01 = fma(q01.re, q01.re, q01.im * q01.im), n02 = fma(q02.re, q02.re, q02.im * q02.im),
            n12 = fma(q12.re, q12.re, q12.im * q12.im);
    const R d0 = fma(a0, a0, n01 + n02), d1 = fma(a1, a1, n01 + n12), d2 = fma(a2, a2, n02 + n12);
    // p01 = -a2 q01 + q02 conj(q12);  p02 = -a1 q02 + q01 q12;  p12 = conj(q01) q02 - a0 q12
    const cplx<R> t01 = cmulc(q02, q12), t02 = cmul(q01, q12), t12 = ccmul(q01, q02);
    const cplx<R> p01 = cmk<R>(fma(-a2, q01.re, t01.re), fma(-a2, q01.im, t01.im));
    const cplx<R> p02 = cmk<R>(fma(-a1, q02.re, t02.re), fma(-a1, q02.im, t02.im));
    const cplx<R> p12 = cmk<R>(fma(-a0, q12.re, t12.re), fma(-a0, q12.im, t12.im));
    const cplx<R> F0 = cmk<R>((R)f0.re, (R)f0.im), F1 = cmk<R>((R)f1.re, (R)f1.im), F2 = cmk<R>((R)f2.re, (R)f2.im);
    su3<R> E;
    // diagonal: f0 + f1 a_i + f2 d_i
    E.m[0] = cmk<R>(fma(F2.re, d0, fma(F1.re, a0, F0.re)), fma(F2.im, d0, fma(F1.im, a0, F0.im)));
    E.m[4] = cmk<R>(fma(F2.re, d1, fma(F1.re, a1, F0.re)), fma(F2.im, d1, fma(F1.im, a1, F0.im)));
    E.m[8] = cmk<R>(fma(F2.re, d2, fma(F1.re, a2, F0.re)), fma(F2.im, d2, fma(F1.im, a2, F0.im)));
    // upper: f1 q + f2 p;  lower: f1 conj(q) + f2 conj(p)
    E.m[1] = cfma(p01, F2, cmul(q01, F1));
    E.m[2] = cfma(p02, F2, cmul(q02, F1));
    E.m[5] = cfma(p12, F2, cmul(q12, F1));
    E.m[3] = cfma(F2, cmk<R>(p01.re, -p01.im), cmul(F1, cmk<R>(q01.re, -q01.im)));
    E.m[6] = cfma(F2, cmk<R>(p02.re, -p02.im), cmul(F1, cmk<R>(q02.re, -q02.im)));
    E.m[7] = cfma(F2, cmk<R>(p12.re, -p12.im), cmul(F1, cmk<R>(q12.re, -q12.im)));
    return E;
}

// exp(X) for X in su(3) given by 8 coordinates; the result in precision R.
// c0, c1 and the coefficients are computed in double from the (possibly
// float) coordinates; the matrix assembly f0 + f1 Q + f2 Q^2 runs in R.
template <typename R> __device__ __forceinline__ su3<R> expm_alg(const alg<R>& x) {
    const herm_d h = herm_from_alg(x);
    const double n01 = h.q01.re * h.q01.re + h.q01.im * h.q01.im;
    const double n02 = h.q02.re * h.q02.re + h.q02.im * h.q02.im;
    const double n12 = h.q12.re * h.q12.re + h.q12.im * h.q12.im;
    // c1 = ReTr(Q^2)/2 ;  c0 = ReTr(Q^3)/3 = det Q
    const double c1 = 0.5 * (h.a0 * h.a0 + h.a1 * h.a1 + h.a2 * h.a2) + (n01 + n02 + n12);
    const cplx<double> t = cmul(h.q01, h.q12);   // q01 q12 conj(q02)
    const double re3 = t.re * h.q02.re + t.im * h.q02.im;
    const double c0 = h.a0 * h.a1 * h.a2 + 2.0 * re3 - h.a0 * n12 - h.a1 * n02 - h.a2 * n01;
    cplx<double> f0, f1, f2;
    ch_coefficients(c0, c1, f0, f1, f2);

    if (LGF_HERM_EXP) return exp_assemble_herm<R>(h, f0, f1, f2);
    // Q and Q^2 in precision R (Q Hermitian traceless)
    su3<R> Q;
    Q.m[0] = cmk<R>((R)h.a0, R(0));
    Q.m[4] = cmk<R>((R)h.a1, R(0));
    Q.m[8] = cmk<R>((R)h.a2, R(0));
    Q.m[1] = cmk<R>((R)h.q01.re, (R)h.q01.im);
    Q.m[2] = cmk<R>((R)h.q02.re, (R)h.q02.im);
    Q.m[5] = cmk<R>((R)h.q12.re, (R)h.q12.im);
    Q.m[3] = cmk<R>(Q.m[1].re, -Q.m[1].im);
    Q.m[6] = cmk<R>(Q.m[2].re, -Q.m[2].im);
    Q.m[7] = cmk<R>(Q.m[5].re, -Q.m[5].im);
    // Q^2 is Hermitian: compute the diagonal and the upper triangle
    su3<R> Q2;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = r; c < 3; ++c) {
            cplx<R> s = cmul(Q.m[3 * r], Q.m[c]);
            s = cfma(Q.m[3 * r + 1], Q.m[3 + c], s);
            s = cfma(Q.m[3 * r + 2], Q.m[6 + c], s);
            Q2.m[3 * r + c] = s;
        }
    Q2.m[0].im = R(0);
    Q2.m[4].im = R(0);
    Q2.m[8].im = R(0);
    Q2.m[3] = cmk<R>(Q2.m[1].re, -Q2.m[1].im);
    Q2.m[6] = cmk<R>(Q2.m[2].re, -Q2.m[2].im);
    Q2.m[7] = cmk<R>(Q2.m[5].re, -Q2.m[5].im);

    const cplx<R> F0 = cmk<R>((R)f0.re, (R)f0.im);
    const cplx<R> F1 = cmk<R>((R)f1.re, (R)f1.im);
    const cplx<R> F2 = cmk<R>((R)f2.re, (R)f2.im);
    su3<R> E;
#pragma unroll
    for (int k = 0; k < 9; ++k) E.m[k] = cfma(Q2.m[k], F2, cmul(Q.m[k], F1));
    E.m[0] = cadd(E.m[0], F0);
    E.m[4] = cadd(E.m[4], F0);
    E.m[8] = cadd(E.m[8], F0);
    return E;
}

template <typename R> __device__ __forceinline__ alg<R> alg_axpby(R a, const alg<R>& x, R b, const alg<R>& y) {
    alg<R> z;
#pragma unroll
    for (int k = 0; k < 8; ++k) z.v[k] = a * x.v[k] + b * y.v[k];
    return z;
}
template <typename R> __device__ __forceinline__ alg<R> alg_scale(R a, const alg<R>& x) {
    alg<R> z;
#pragma unroll
    for (int k = 0; k < 8; ++k) z.v[k] = a * x.v[k];
    return z;
}

// Hermitian traceless field-strength components as 8 coordinates:
// (F00, F11, Re F01, Im F01, Re F02, Im F02, Re F12, Im F12), F22 = -(F00+F11).
// From a loop sum C:  F = -i/2 [ (C - C^dag) - 1/3 Tr(C - C^dag) ]
// (LGF/Field/SU3_field.cpp:575-579).
template <typename R> __device__ __forceinline__ alg<R> field_strength(const su3<R>& C, R scale) {
    // C - C^dag: diag 2i Im C_ii ; off (ij) = C_ij - conj(C_ji)
    // times -i/2:  diag Im C_ii ; off: (-i/2)(C_ij - conj C_ji)
    alg<R> f;
    R d0 = C.m[0].im, d1 = C.m[4].im, d2 = C.m[8].im;
    R tr = (d0 + d1 + d2) * R(1.0 / 3.0);
    f.v[0] = scale * (d0 - tr);
    f.v[1] = scale * (d1 - tr);
    // (-i/2)(a + ib) = (b/2, -a/2)
    R a, b;
    a = C.m[1].re - C.m[3].re; b = C.m[1].im + C.m[3].im;
    f.v[2] = scale * R(0.5) * b; f.v[3] = -scale * R(0.5) * a;
    a = C.m[2].re - C.m[6].re; b = C.m[2].im + C.m[6].im;
    f.v[4] = scale * R(0.5) * b; f.v[5] = -scale * R(0.5) * a;
    a = C.m[5].re - C.m[7].re; b = C.m[5].im + C.m[7].im;
    f.v[6] = scale * R(0.5) * b; f.v[7] = -scale * R(0.5) * a;
    return f;
}

// ReTr(A B) for Hermitian traceless A, B in field-strength coordinates.
template <typename R> __device__ __forceinline__ double retr_hh(const alg<R>& A, const alg<R>& B) {
    double a2 = -((double)A.v[0] + (double)A.v[1]);
    double b2 = -((double)B.v[0] + (double)B.v[1]);
    double s = (double)A.v[0] * B.v[0] + (double)A.v[1] * B.v[1] + a2 * b2;
    double o = (double)A.v[2] * B.v[2] + (double)A.v[3] * B.v[3] + (double)A.v[4] * B.v[4] +
               (double)A.v[5] * B.v[5] + (double)A.v[6] * B.v[6] + (double)A.v[7] * B.v[7];
    return s + 2.0 * o;
}

}  // namespace lgf
