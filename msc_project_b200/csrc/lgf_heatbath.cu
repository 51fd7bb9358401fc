// Gauge-configuration generation on the GPU: hot/cold start, Cabibbo-Marinari
// heatbath with overrelaxation, and the average plaquette.
//
// Follows SU3_Heatbath (LGF/SU3_Heatbath/SU3_Heatbath.cpp): update(n) =
// n x (one heatbath sweep + OR_per_HB overrelaxation sweeps) (:16-25); a sweep
// visits the links by site parity and direction (:68-70, :117-119) and updates
// the three SU(2) subgroups (m,n) = (0,1), (0,2), (1,2) of each link in turn
// (:71-75), recomputing W = U * staple after every subgroup.  The SU(2)
// heatbath samples x0 by the reference's rejection scheme (:199-205), the
// overrelaxation reflects the subgroup (:78-104).
//
// B200 mapping: one launch per (parity, direction) class updates all its links
// in place in parallel -- the staple of a link reads only other directions and
// opposite-parity links of its own direction, so the class has no internal
// dependencies.  Random numbers come from a counter hash of (seed, class epoch,
// subgroup, site, draw), so results do not depend on the launch shape.  The
// rejection loop is bounded (HB_MAX_ATTEMPTS); a subgroup whose draws all
// fail is left unchanged and counted.  The reference seeds from
// std::random_device, so runs are compared statistically (average plaquette),
// not bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "lgf_engine.cuh"

namespace lgf {
namespace {

constexpr int HB_MAX_ATTEMPTS = 128;
constexpr int HB_DRAW_BITS = 10;  // draws per (epoch, subgroup, site): <= 2 + 4 * HB_MAX_ATTEMPTS < 1024

__device__ __forceinline__ double hb_draw(unsigned long long seed, unsigned long long base, int k) {
    return unit_open(seed, base + (unsigned long long)k);
}

// site of parity p with index t among the V/2 sites of that parity
// (N3 is even: every x0,x1,x2 row holds N3/2 sites of each parity)
__device__ __forceinline__ int parity_site(const Geom& g, int p, int t) {
    const int half3 = g.n[3] >> 1;
    const int row = t / half3, k = t - row * half3;
    const int x2 = row % g.n[2];
    const int r1 = row / g.n[2];
    const int x1 = r1 % g.n[1];
    const int x0 = r1 / g.n[1];
    const int x3 = 2 * k + ((p + x0 + x1 + x2) & 1);
    return row * g.n[3] + x3;
}

template <typename R>
__global__ void __launch_bounds__(128) k_checkerboard(cplx<R>* __restrict__ U, Geom g, int mu, int parity, double beta,
                                                      unsigned long long seed, unsigned long long epoch, int overrelax,
                                                      unsigned int* __restrict__ failures) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (g.V >> 1)) return;
    const int s = parity_site(g, parity, t);
    const Coord c = site_coord(g, s);
    const su3<R> A = staple_sum<R>(U, g, s, c, mu);
    su3<R> u = load_link(U, g.V, mu, s);
#pragma unroll 1
    for (int sg = 0; sg < 3; ++sg) {
        const int m = sg == 2 ? 1 : 0, n = sg == 0 ? 1 : 2;  // (0,1), (0,2), (1,2)
        // the 2x2 block of W = u * A on rows/columns (m, n)
        cplx<double> w[2][2];
        const int rc[2] = {m, n};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int b = 0; b < 2; ++b) {
                cplx<double> acc = cmk<double>(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const cplx<R> x = u.m[3 * rc[a] + k], y = A.m[3 * k + rc[b]];
                    acc = cfma(cmk<double>(x.re, x.im), cmk<double>(y.re, y.im), acc);
                }
                w[a][b] = acc;
            }
        // O(4) coordinates of the subgroup block (GetSU2submatrix_O4_rep, SU3_mat.cpp:456-465)
        double r[4] = {w[0][0].re + w[1][1].re, w[0][1].im + w[1][0].im, w[0][1].re - w[1][0].re,
                       w[0][0].im - w[1][1].im};
        cplx<double> T[4];
        bool apply = true;
        if (overrelax) {  // SU3_Heatbath.cpp:78-99
            const double a = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
            double q[4] = {1.0, 0.0, 0.0, 0.0};
            if (a >= 0.00001) {
                const double ia = 1.0 / a;
                q[0] = ia * r[0];
                q[1] = -ia * r[1];
                q[2] = -ia * r[2];
                q[3] = -ia * r[3];
            }
            const double z0 = q[0] * q[0] - q[1] * q[1] - q[2] * q[2] - q[3] * q[3];
            const double z1 = 2.0 * q[0] * q[1], z2 = 2.0 * q[0] * q[2], z3 = 2.0 * q[0] * q[3];
            T[0] = cmk<double>(z0, z3);
            T[1] = cmk<double>(z2, z1);
            T[2] = cmk<double>(-z2, z1);
            T[3] = cmk<double>(z0, -z3);
        } else {  // SU3_Heatbath.cpp:169-223
            const double norm = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3]);
            const double alpha = norm * beta / 3.0;
            const double in = 1.0 / norm;
            const cplx<double> sub[4] = {cmk<double>(r[0] * in, -r[3] * in), cmk<double>(-r[2] * in, -r[1] * in),
                                         cmk<double>(r[2] * in, -r[1] * in), cmk<double>(r[0] * in, r[3] * in)};
            const unsigned long long base =
                ((((epoch * 3ull + (unsigned long long)sg) * (unsigned long long)g.V) + (unsigned long long)s)
                 << HB_DRAW_BITS);
            const double two_pi = 6.28318530717958647692;
            double delta = 0.0;
            bool ok = false;
            int k = 0;
            for (int it = 0; it < HB_MAX_ATTEMPTS && !ok; ++it) {
                const double X = -log(1.0 - hb_draw(seed, base, k++));
                const double Xp = -log(1.0 - hb_draw(seed, base, k++));
                const double cc = cos(two_pi * hb_draw(seed, base, k++));
                delta = (Xp + X * cc * cc) / alpha;
                const double u4 = hb_draw(seed, base, k++);
                ok = u4 * u4 <= 1.0 - 0.5 * delta;
            }
            if (!ok) {
                atomicAdd(failures, 1u);
                apply = false;
            } else {
                const double x0 = 1.0 - delta;
                const double ax = sqrt(fmax(0.0, 1.0 - x0 * x0));
                const double ct = 2.0 * hb_draw(seed, base, k++) - 1.0;
                const double phi = two_pi * hb_draw(seed, base, k++);
                const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
                double sp, cp;
                sincos(phi, &sp, &cp);
                const double x1 = ax * st * cp, x2 = ax * st * sp, x3 = ax * ct;
                const cplx<double> Vm[4] = {cmk<double>(x0, x3), cmk<double>(x2, x1), cmk<double>(-x2, x1),
                                            cmk<double>(x0, -x3)};
                T[0] = cadd(cmul(Vm[0], sub[0]), cmul(Vm[1], sub[2]));
                T[1] = cadd(cmul(Vm[0], sub[1]), cmul(Vm[1], sub[3]));
                T[2] = cadd(cmul(Vm[2], sub[0]), cmul(Vm[3], sub[2]));
                T[3] = cadd(cmul(Vm[2], sub[1]), cmul(Vm[3], sub[3]));
            }
        }
        if (apply) {  // rows m, n of u <- T * (rows m, n)   (SU3_Heatbath.cpp:100-104, 131-135)
#pragma unroll
            for (int col = 0; col < 3; ++col) {
                const cplx<double> um = cmk<double>(u.m[3 * m + col].re, u.m[3 * m + col].im);
                const cplx<double> un = cmk<double>(u.m[3 * n + col].re, u.m[3 * n + col].im);
                const cplx<double> nm = cadd(cmul(T[0], um), cmul(T[1], un));
                const cplx<double> nn = cadd(cmul(T[2], um), cmul(T[3], un));
                u.m[3 * m + col] = cmk<R>((R)nm.re, (R)nm.im);
                u.m[3 * n + col] = cmk<R>((R)nn.re, (R)nn.im);
            }
        }
    }
    store_link(U, g.V, mu, s, u);
}

// Random SU(3) per link as a product of three random SU(2) subgroup elements
// (Random::rnd_SU3_Group_elem, LGF/Math/Random.h:37-64): InitializeHotStart.
template <typename R>
__global__ void k_hot_start(cplx<R>* __restrict__ U, int V, unsigned long long seed) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const int mu = t / V, s = t - mu * V;
    const unsigned long long base = ((unsigned long long)s * 4ull + (unsigned long long)mu) * 16ull;
    const double PI = 3.14159265358979323846;
    su3<double> out;
    su3_zero(out);
    out.m[0] = out.m[4] = out.m[8] = cmk<double>(1.0, 0.0);
    int k = 0;
    const int I[3] = {0, 0, 1}, J[3] = {1, 2, 2};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const int i = I[q], j = J[q];
        const double alpha = PI * unit_open(seed, base + k++);
        const double phi = 2.0 * PI * unit_open(seed, base + k++);
        const double ct = 2.0 * unit_open(seed, base + k++) - 1.0;
        const double st = sqrt(1.0 - ct * ct);
        double sa, ca, sp, cp;
        sincos(alpha, &sa, &ca);
        sincos(phi, &sp, &cp);
        const double a0 = ca, a1 = sa * cp * st, a2 = sa * sp * st, a3 = sa * ct;
        su3<double> tmp;
        su3_zero(tmp);
        tmp.m[0] = tmp.m[4] = tmp.m[8] = cmk<double>(1.0, 0.0);
        tmp.m[3 * i + i] = cmk<double>(a0, a3);
        tmp.m[3 * i + j] = cmk<double>(a2, a1);
        tmp.m[3 * j + i] = cmk<double>(-a2, a1);
        tmp.m[3 * j + j] = cmk<double>(a0, -a3);
        out = mul_nn(tmp, out);
    }
    su3<R> o;
#pragma unroll
    for (int q = 0; q < 9; ++q) o.m[q] = cmk<R>((R)out.m[q].re, (R)out.m[q].im);
    store_link(U, V, mu, s, o);
}

template <typename R>
__global__ void k_cold_start(cplx<R>* __restrict__ U, int V) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 4 * V) return;
    const int mu = t / V, s = t - mu * V;
    su3<R> o;
    su3_zero(o);
    o.m[0] = o.m[4] = o.m[8] = cmk<R>(R(1), R(0));
    store_link(U, V, mu, s, o);
}

// per block: sum over its sites of sum_{mu<nu} ReTr P_mu_nu(x)
template <typename R>
__global__ void __launch_bounds__(256) k_plaquette(const cplx<R>* __restrict__ U, Geom g, double* __restrict__ partial) {
    __shared__ double sh[256];
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    double acc = 0.0;
    if (s < g.V) {
        const Coord c = site_coord(g, s);
#pragma unroll
        for (int mu = 0; mu < 4; ++mu)
#pragma unroll
            for (int nu = mu + 1; nu < 4; ++nu) {
                const su3<R> a = load_link(U, g.V, mu, s);
                const su3<R> b = load_link(U, g.V, nu, fwd(g, s, mu, c.x[mu]));
                const su3<R> cc = load_link(U, g.V, mu, fwd(g, s, nu, c.x[nu]));
                const su3<R> d = load_link(U, g.V, nu, s);
                const su3<R> ab = mul_nn(a, b);
                const su3<R> dc = mul_nn(d, cc);
                const su3<R> p = mul_na(ab, dc);  // U_mu(x) U_nu(x+mu) (U_nu(x) U_mu(x+nu))^dag
                acc += (double)p.m[0].re + (double)p.m[4].re + (double)p.m[8].re;
            }
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// n_iter x (heatbath sweep unless or_only, then or_per_hb overrelaxation sweeps)
template <typename R>
int heatbath_impl(lgf_ctx* ctx, lgf_lattice* lat, double beta, int n_iter, int or_per_hb, unsigned long long seed,
                  unsigned long long* rejected, bool or_only) {
    LatticeBuf& b = lat->buf;
    unsigned int* dfail = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&dfail, sizeof(unsigned int)));
    cudaMemsetAsync(dfail, 0, sizeof(unsigned int), ctx->stream);
    const int half = b.g.V / 2, th = 128, nb = (half + th - 1) / th;
    cudaError_t e = cudaSuccess;
    for (int it = 0; it < n_iter && e == cudaSuccess; ++it) {
        for (int sweep = or_only ? 1 : 0; sweep <= or_per_hb && e == cudaSuccess; ++sweep) {
            const int over = sweep > 0;
            for (int par = 0; par <= 1; ++par)
                for (int mu = 0; mu < 4; ++mu) {
                    const unsigned long long epoch = lat->hb_epoch++;
                    k_checkerboard<R><<<nb, th, 0, ctx->stream>>>((cplx<R>*)b.U[0], b.g, mu, par, beta, seed, epoch,
                                                                  over, dfail);
                }
            e = cudaGetLastError();
        }
    }
    unsigned int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, dfail, sizeof h, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dfail);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "heatbath failed: %s", cudaGetErrorString(e));
    if (rejected) *rejected = h;
    return LGF_OK;
}

}  // namespace
}  // namespace lgf

using namespace lgf;

extern "C" {

int lgf_heatbath(lgf_lattice* lat, double beta, int n_iter, int or_per_hb, uint64_t seed, uint64_t* rejected) {
    if (!lat || n_iter < 0 || or_per_hb < 0 || !(beta > 0.0)) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    if ((long long)lat->buf.g.V * 3 * (long long)(lat->hb_epoch + 8LL * n_iter * (or_per_hb + 1)) >=
        (1LL << (63 - HB_DRAW_BITS)))
        return set_error(ctx, LGF_EINVAL, "heatbath random-number counter space exhausted for this lattice");
    unsigned long long rej = 0;
    const int rc = lat->buf.prec == LGF_PREC_FP64
                       ? heatbath_impl<double>(ctx, lat, beta, n_iter, or_per_hb, seed, &rej, false)
                       : heatbath_impl<float>(ctx, lat, beta, n_iter, or_per_hb, seed, &rej, false);
    if (rejected) *rejected = rej;
    return rc;
}

int lgf_overrelax(lgf_lattice* lat, int n_sweeps) {
    if (!lat || n_sweeps < 0) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    return lat->buf.prec == LGF_PREC_FP64 ? heatbath_impl<double>(ctx, lat, 1.0, 1, n_sweeps, 0, nullptr, true)
                                          : heatbath_impl<float>(ctx, lat, 1.0, 1, n_sweeps, 0, nullptr, true);
}

int lgf_hot_start(lgf_lattice* lat, uint64_t seed) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    const int V = lat->buf.g.V, nb = (4 * V + 127) / 128;
    if (lat->buf.prec == LGF_PREC_FP64)
        k_hot_start<double><<<nb, 128, 0, ctx->stream>>>((cplx<double>*)lat->buf.U[0], V, seed);
    else
        k_hot_start<float><<<nb, 128, 0, ctx->stream>>>((cplx<float>*)lat->buf.U[0], V, seed);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    LGF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LGF_OK;
}

int lgf_cold_start(lgf_lattice* lat) {
    if (!lat) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    const int V = lat->buf.g.V, nb = (4 * V + 127) / 128;
    if (lat->buf.prec == LGF_PREC_FP64)
        k_cold_start<double><<<nb, 128, 0, ctx->stream>>>((cplx<double>*)lat->buf.U[0], V);
    else
        k_cold_start<float><<<nb, 128, 0, ctx->stream>>>((cplx<float>*)lat->buf.U[0], V);
    LGF_CUDA_TRY(ctx, cudaGetLastError());
    LGF_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
    return LGF_OK;
}

int lgf_plaquette(lgf_lattice* lat, double* avg) {
    if (!lat || !avg) return LGF_EINVAL;
    lgf_ctx* ctx = lat->ctx;
    cudaSetDevice(ctx->device);
    const Geom g = lat->buf.g;
    const int nb = (g.V + 255) / 256;
    double* dp = nullptr;
    LGF_CUDA_TRY(ctx, cudaMalloc(&dp, sizeof(double) * nb));
    if (lat->buf.prec == LGF_PREC_FP64)
        k_plaquette<double><<<nb, 256, 0, ctx->stream>>>((const cplx<double>*)lat->buf.U[0], g, dp);
    else
        k_plaquette<float><<<nb, 256, 0, ctx->stream>>>((const cplx<float>*)lat->buf.U[0], g, dp);
    std::vector<double> h(nb);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), dp, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(dp);
    if (e != cudaSuccess) return set_error(ctx, LGF_ECUDA, "plaquette failed: %s", cudaGetErrorString(e));
    double sum = 0.0;
    for (double v : h) sum += v;
    *avg = sum / (3.0 * 6.0 * (double)g.V);  // SU3_field::Avg_Plaquette (SU3_field.cpp:485-499)
    return LGF_OK;
}

}  // extern "C"
