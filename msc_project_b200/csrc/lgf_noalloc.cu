// E/Q measurement that allocates nothing.
//
// Some callers cannot allocate device memory: code that holds every byte of
// the GPU in its own pool (a framework's caching allocator, a serving process
// that reserves its memory at start-up and forbids allocation afterwards) or
// a real-time loop that must not enter the driver's allocator.  They already
// have the configuration in device memory and a place for the result, and
// only need the measurement.  lgf_measure_noalloc serves them: the per-block
// partial sums that lgf_measure keeps in memory it allocates live here in one
// file-scope device array of fixed size instead.
//
// The scratch array is a host-side symbol: host code must not pass its name
// to a kernel (that would hand the kernel a host address).  Its device address
// is looked up once per device with cudaGetSymbolAddress, with that device
// current.  CUDA loads modules lazily by default, so that lookup is also what
// places the array in the GPU's memory: lgf_ctx_create does it for its device
// (noalloc_preload), and otherwise the first call made on a device does it.
// Callers that reserve the rest of the GPU's memory must therefore create a
// context or make one call first, and the first call should come before any
// stream capture.  Once loaded, a GPU holds the array (4 MiB + 4 KiB) until
// the process exits.  All calls on one GPU share it and it keeps the last
// call's contents: two calls that can run at the same time on the same GPU
// (different streams, different host threads) race on it, so the caller must
// order them.  Nothing in it has to start at zero: each call writes every
// entry it later reads.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "lgf_engine.cuh"

namespace lgf {
namespace {

constexpr int NOALLOC_MAX_PARTIALS = 262144;  // (x0 slices) x (32-site chunks per slice)
constexpr int NOALLOC_MAX_SLICES = 256;       // x0 extent
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_MAX_PARTIALS + NOALLOC_MAX_SLICES];

std::mutex g_noalloc_mu;
double2* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

// one link in the caller's file order: double2 L[(s*4 + mu)*9 + k]
__device__ __forceinline__ su3<double> file_link(const double2* __restrict__ L, int s, int mu) {
    su3<double> a;
    const double2* p = L + ((size_t)s * 4 + mu) * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double2 v = __ldg(p + k);
        a.m[k] = cmk<double>(v.x, v.y);
    }
    return a;
}

// The a x b loops of the clover-type averages, walked over file-order links
// (same quadrants and orientation as the engine's measurement kernel).
template <int A, int B>
__device__ __forceinline__ void leaves_file(const double2* __restrict__ L, const Geom& g, int s, const Coord& c, int mu,
                                            int nu, su3<double>& sum) {
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        int y = s, ymu = c.x[mu], ynu = c.x[nu];
        bool first = true;
        su3<double> acc;
        auto step = [&](int dir, int sign) {
            int& yc = (dir == mu) ? ymu : ynu;
            if (sign > 0) {
                const su3<double> l = file_link(L, y, dir);
                y = fwd(g, y, dir, yc);
                yc = wrap_inc(yc, g.n[dir]);
                acc = first ? l : mul_nn(acc, l);
            } else {
                y = bwd(g, y, dir, yc);
                yc = wrap_dec(yc, g.n[dir]);
                const su3<double> l = file_link(L, y, dir);
                if (first) {
#pragma unroll
                    for (int r = 0; r < 3; ++r)
#pragma unroll
                        for (int cc = 0; cc < 3; ++cc) acc.m[3 * r + cc] = cmk<double>(l.m[3 * cc + r].re, -l.m[3 * cc + r].im);
                } else {
                    acc = mul_na(acc, l);
                }
            }
            first = false;
        };
        auto seg = [&](int dir, int sign, int len) {
            for (int i = 0; i < len; ++i) step(dir, sign);
        };
        if (q == 0) { seg(nu, +1, B); seg(mu, +1, A); seg(nu, -1, B); seg(mu, -1, A); }
        else if (q == 1) { seg(mu, +1, A); seg(nu, -1, B); seg(mu, -1, A); seg(nu, +1, B); }
        else if (q == 2) { seg(mu, -1, A); seg(nu, +1, B); seg(mu, +1, A); seg(nu, -1, B); }
        else { seg(nu, -1, B); seg(mu, -1, A); seg(nu, +1, B); seg(mu, +1, A); }
        su3_addto(sum, acc);
    }
}

__device__ __forceinline__ void plane_fields_file(const double2* __restrict__ L, const Geom& g, int s, const Coord& c,
                                                  int mu, int nu, alg<double>& F11, alg<double>& Fhat) {
    su3<double> C;
    su3_zero(C);
    leaves_file<1, 1>(L, g, s, c, mu, nu, C);
    F11 = field_strength(C, 0.25);
    Fhat = alg_scale(19.0 / 9.0, F11);
    su3_zero(C);
    leaves_file<2, 2>(L, g, s, c, mu, nu, C);
    Fhat = alg_axpby(1.0, Fhat, 1.0 / 36.0, field_strength(C, 0.25));
    su3_zero(C);
    leaves_file<1, 2>(L, g, s, c, mu, nu, C);
    leaves_file<2, 1>(L, g, s, c, mu, nu, C);
    Fhat = alg_axpby(1.0, Fhat, -32.0 / 45.0, field_strength(C, 1.0 / 8.0));
    su3_zero(C);
    leaves_file<1, 3>(L, g, s, c, mu, nu, C);
    leaves_file<3, 1>(L, g, s, c, mu, nu, C);
    Fhat = alg_axpby(1.0, Fhat, 1.0 / 15.0, field_strength(C, 1.0 / 8.0));
}

// grid (nchunk, N0), block (32 sites, 6 planes); partials[slice*nchunk + chunk]
__global__ void __launch_bounds__(MEAS_SITES * 6) k_noalloc_measure(const double2* __restrict__ L, Geom g,
                                                                    double2* __restrict__ partials) {
    __shared__ alg<double> sF[6][MEAS_SITES];
    __shared__ double sE[6][MEAS_SITES];
    const int lane = threadIdx.x, p = threadIdx.y;
    const int slice = blockIdx.y, chunk = blockIdx.x;
    const int off = chunk * MEAS_SITES + lane;
    const bool valid = off < g.Vs;
    const int s = slice * g.Vs + (valid ? off : 0);
    if (valid) {
        const Coord c = site_coord(g, s);
        alg<double> F11, Fh;
        plane_fields_file(L, g, s, c, c_plane_mu[p], c_plane_nu[p], F11, Fh);
        sF[p][lane] = Fh;
        sE[p][lane] = retr_hh(F11, F11);
    }
    __syncthreads();
    if (p == 0) {
        double e = 0.0, q = 0.0;
        if (valid) {
            e = ((sE[0][lane] + sE[1][lane]) + (sE[2][lane] + sE[3][lane])) + (sE[4][lane] + sE[5][lane]);
            q = -retr_hh(sF[5][lane], sF[0][lane]) + retr_hh(sF[4][lane], sF[1][lane]) -
                retr_hh(sF[2][lane], sF[3][lane]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            e += __shfl_xor_sync(0xffffffffu, e, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
        }
        if (lane == 0) partials[slice * gridDim.x + chunk] = make_double2(e, q);
    }
}

// one block per slice: fixed-order sums, then out = [E, Q, E_slice, Q_slice]
__global__ void __launch_bounds__(RED_THREADS) k_noalloc_slices(const double2* __restrict__ partials, int nchunk, Geom g,
                                                                double2* __restrict__ slice_sums, double* __restrict__ out) {
    __shared__ double se[RED_THREADS], sq[RED_THREADS];
    const int t = blockIdx.x;
    double e = 0.0, q = 0.0;
    for (int j = threadIdx.x; j < nchunk; j += RED_THREADS) {
        const double2 v = partials[t * nchunk + j];
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
        const double inv4pi2 = 1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846);
        out[2 + t] = se[0] / (double)g.Vs;
        out[2 + g.n[0] + t] = sq[0] * inv4pi2;
        slice_sums[t] = make_double2(se[0], sq[0]);
    }
}

__global__ void __launch_bounds__(RED_THREADS) k_noalloc_total(const double2* __restrict__ slice_sums, Geom g,
                                                               double* __restrict__ out) {
    __shared__ double se[RED_THREADS], sq[RED_THREADS];
    double e = 0.0, q = 0.0;
    for (int j = threadIdx.x; j < g.n[0]; j += RED_THREADS) {
        e += slice_sums[j].x;
        q += slice_sums[j].y;
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
        out[0] = se[0] * (1.0 / (double)g.V);
        out[1] = sq[0] * inv4pi2;
    }
}

// device address of the scratch array on the current device (looked up once)
int noalloc_scratch(int dev, double2** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            if (e != cudaSuccess) cudaGetLastError();  // this lookup's own error
            return LGF_ECUDA;
        }
        g_noalloc_addr[dev] = (double2*)p;
    }
    *out = g_noalloc_addr[dev];
    return LGF_OK;
}

}  // namespace

// Called by lgf_ctx_create with the context's device current: loads this
// file's module on that device (placing the scratch array) and caches its
// address, so the first measurement allocates nothing even under lazy loading.
int noalloc_preload(int dev) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return LGF_OK;  // such devices are served on first call
    double2* p = nullptr;
    return noalloc_scratch(dev, &p);
}

}  // namespace lgf

extern "C" int lgf_measure_noalloc(const double* links, const int shape[4], double* out, void* stream) {
    using namespace lgf;
    if (!links || !out || !valid_shape(shape)) return LGF_EINVAL;
    const Geom g = make_geom(shape);
    const int nchunk = (g.Vs + MEAS_SITES - 1) / MEAS_SITES;
    if (g.n[0] > NOALLOC_MAX_SLICES || (long long)nchunk * g.n[0] > NOALLOC_MAX_PARTIALS) return LGF_ETOOBIG;
    if (((uintptr_t)links % 16) != 0 || ((uintptr_t)out % 8) != 0) return LGF_EINVAL;
    // an error that earlier work left pending on this thread is the caller's:
    // report it without clearing it, and launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return LGF_ECUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return LGF_ECUDA;
    double2* scratch = nullptr;
    int rc = noalloc_scratch(dev, &scratch);
    if (rc != LGF_OK) return rc;
    double2* partials = scratch;
    double2* slice_sums = scratch + NOALLOC_MAX_PARTIALS;
    cudaStream_t st = (cudaStream_t)stream;
    k_noalloc_measure<<<dim3(nchunk, g.n[0]), dim3(MEAS_SITES, 6), 0, st>>>((const double2*)links, g, partials);
    k_noalloc_slices<<<g.n[0], RED_THREADS, 0, st>>>(partials, nchunk, g, slice_sums, out);
    k_noalloc_total<<<1, RED_THREADS, 0, st>>>(slice_sums, g, out);
    // nothing was pending at entry, so an error now comes from these launches
    if (cudaGetLastError() != cudaSuccess) return LGF_ECUDA;
    return LGF_OK;
}
