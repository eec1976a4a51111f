// Solver-side kernels: elementwise maps, TV regulariser, FP64 reductions.
//
// These carry the arithmetic of the reference's CuPy Solver
// (src/ptychotomo/solver.py:48-336) that is not an operator:
//   linear combinations of complex arrays (CG/ADMM updates), the TV
//   operator J and its adjoint (solver.py:128-146), the soft-threshold
//   regulariser step (solver.py:257-264), the exp/log maps (solver.py:48-64),
//   the linearisation of takexi (solver.py:149-168) and every norm / inner
//   product / likelihood sum, accumulated in FP64.
//
// Reductions are deterministic: fixed grid, per-block partials in a caller
// workspace, then one block sums the partials in order.
#include <cmath>
#include <cstdint>

#include "pt_common.cuh"

namespace {

constexpr int RB = 1184;    // reduction blocks (148 SMs x 8)
constexpr int RT = 256;     // reduction threads per block
constexpr int MAXK = 16;    // max outputs of one reduction

template <int K>
__device__ __forceinline__ void block_reduce_store(double (&acc)[K], double *work, int blk, int nblk)
{
    __shared__ double red[RT / 32][MAXK];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0;
        for (int w = 0; w < RT / 32; ++w) s += red[w][threadIdx.x];
        work[(size_t)threadIdx.x * nblk + blk] = s;
    }
}

// one block: out[k] = sum_b work[k * nblk + b] (fixed order per thread, then tree)
__global__ void k_finish(const double *__restrict__ work, double *__restrict__ out, int K, int nblk, int op_max,
                         const double *__restrict__ skip = nullptr)
{
    if (skip != nullptr && *skip != 0.0) return;   // a pass the caller's device-side decision made unnecessary
    __shared__ double red[RT];
    for (int k = 0; k < K; ++k) {
        double s = op_max ? -1.0 : 0.0;
        for (int b = threadIdx.x; b < nblk; b += RT) {
            const double v = work[(size_t)k * nblk + b];
            s = op_max ? fmax(s, v) : s + v;
        }
        red[threadIdx.x] = s;
        __syncthreads();
        for (int w = RT / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] = op_max ? fmax(red[threadIdx.x], red[threadIdx.x + w])
                                                           : red[threadIdx.x] + red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[k] = red[0];
        __syncthreads();
    }
}

// ---- generic reductions over complex64 arrays --------------------------------
// op 0: ||a||^2                         -> 1 value
// op 1: sum conj(a) b                   -> 2 values (re, im)
// op 2: ||a||^2, Re<a,b>, ||b||^2        -> 3 values
// op 3: max |a|                         -> 1 value
// op 4: sum angle(a) over columns [c0,c1) of rows of length ncol -> 1 value
// op 5: ||a - b||^2                     -> 1 value
// op 6: sum_i sqrt(|a_i|^2 + |a_{i+n}|^2 + |a_{i+2n}|^2) (a has 3n entries) -> 1 value
// op 7: max |angle(a)|                  -> 1 value
__global__ void __launch_bounds__(RT) k_reduce(int op, const float2 *__restrict__ a, const float2 *__restrict__ b,
                                               size_t n, int c0, int c1, int ncol, double *__restrict__ work)
{
    double acc[3] = {0, 0, 0};
    const bool is_max = (op == 3 || op == 7);
    if (is_max) acc[0] = -1.0;
    for (size_t i = (size_t)blockIdx.x * RT + threadIdx.x; i < n; i += (size_t)gridDim.x * RT) {
        const float2 x = a[i];
        if (op == 5) {
            const float2 y = b[i];
            const double dx = (double)x.x - y.x, dy = (double)x.y - y.y;
            acc[0] += dx * dx + dy * dy;
        } else if (op == 6) {
            const float2 y = a[i + n], z = a[i + 2 * n];
            acc[0] += (double)sqrtf(x.x * x.x + x.y * x.y + y.x * y.x + y.y * y.y + z.x * z.x + z.y * z.y);
        } else if (op == 7) {
            acc[0] = fmax(acc[0], (double)fabsf(atan2f(x.y, x.x)));
        } else if (op == 0) {
            acc[0] += (double)x.x * x.x + (double)x.y * x.y;
        } else if (op == 1) {
            const float2 y = b[i];
            acc[0] += (double)x.x * y.x + (double)x.y * y.y;
            acc[1] += (double)x.x * y.y - (double)x.y * y.x;
        } else if (op == 2) {
            const float2 y = b[i];
            acc[0] += (double)x.x * x.x + (double)x.y * x.y;
            acc[1] += (double)x.x * y.x + (double)x.y * y.y;
            acc[2] += (double)y.x * y.x + (double)y.y * y.y;
        } else if (op == 3) {
            acc[0] = fmax(acc[0], (double)hypotf(x.x, x.y));
        } else {
            const int col = (int)(i % ncol);
            if (col >= c0 && col < c1) acc[0] += (double)atan2f(x.y, x.x);
        }
    }
    if (is_max) {
        // max: reduce with max instead of sum
        __shared__ double red[RT];
        red[threadIdx.x] = acc[0];
        __syncthreads();
        for (int w = RT / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
            __syncthreads();
        }
        if (threadIdx.x == 0) work[blockIdx.x] = red[0];
        return;
    }
    block_reduce_store<3>(acc, work, blockIdx.x, gridDim.x);
}

// ---- ptycho data terms over detector frames (solver.py:208-214, :294-298) ---
// model 0 Poisson, 1 Gaussian.  With t(y) = |y|^2 - 2 D log(max(|y|, 1e-32))
// (Poisson) or (|y| - sqrt D)^2 (Gaussian), out[j] = sum t(f) - t(f + g_j d):
// the decrease of the data term for step g_j, formed per element in FP32
// without cancellation and summed in FP64: with a2 = |f|^2 and
//   delta = |f + g d|^2 - a2 = 2 g Re(conj(f) d) + g^2 |d|^2,
// Poisson:  t(f) - t(f + g d) = -delta + D log1p(delta / a2),
// Gaussian: t(f) - t(f + g d) = -delta / (|f| + |f + g d|) * (|f| + |f + g d| - 2 sqrt D);
// moduli below ~1e-15 (|f|^2 underflows in FP32) take the FP64 direct
// formula with mlog's 1e-32 clamp (out of line: rare, and its callers are unrolled).
__device__ __noinline__ double ls_decrease_f64(float2 f, float2 d, float g, float D, int model)
{
    const double a2 = (double)f.x * f.x + (double)f.y * f.y;
    const double fd = (double)f.x * d.x + (double)f.y * d.y;
    const double d2 = (double)d.x * d.x + (double)d.y * d.y;
    const double delta = 2.0 * g * fd + (double)g * g * d2;
    const double b2 = a2 + delta;
    if (model == 0) {
        const double lim = 1e-64;  // (1e-32)^2: mlog's clamp
        const double la = a2 >= lim ? 0.5 * log(a2) : -73.68272297580946;  // log 1e-32
        const double lb = b2 >= lim ? 0.5 * log(b2) : -73.68272297580946;
        return -delta - 2.0 * (double)D * (la - lb);
    }
    const double fa = sqrt(a2), fb = sqrt(fmax(b2, 0.0));
    const double sum = fa + fb;
    if (sum == 0.0) return 0.0;
    return -delta / sum * (sum - 2.0 * (double)sqrtf(D));
}

// Adds the decrease for each step gj[j], j < J, of one pixel to acc[j];
// MODEL 0 = Poisson, 1 = Gaussian.  1/|f|^2 (Poisson) or |f| and sqrt D
// (Gaussian) are formed once per pixel.
template <int JB, int MODEL>
__device__ __forceinline__ void ls_pixel(double (&acc)[JB], const float (&gj)[JB], int J, float2 x, float2 y, float D)
{
    const float a2 = x.x * x.x + x.y * x.y;
    const float fdot = x.x * y.x + x.y * y.y;
    const float d2 = y.x * y.x + y.y * y.y;
    const bool tiny = !(a2 >= 1e-30f);
    float ia2 = 0.f, fa = 0.f, sq = 0.f;
    if (MODEL == 0) {
        ia2 = tiny ? 0.f : 1.f / a2;
    } else {
        fa = sqrtf(a2);
        sq = sqrtf(D);
    }
#pragma unroll
    for (int j = 0; j < JB; ++j) {
        if (j < J) {
            const float g = gj[j];
            const float delta = g * (2.f * fdot + g * d2);
            const float b2 = a2 + delta;
            double dec;
            if (tiny || !(b2 >= 1e-30f)) {
                // d = 0 (a skipped scan's zero frame, say): no change for any step
                dec = d2 == 0.f ? 0.0 : ls_decrease_f64(x, y, g, D, MODEL);
            } else if (MODEL == 0) {
                dec = (double)(D * log1pf(delta * ia2) - delta);
            } else {
                const float s2 = fa + sqrtf(b2);  // >= 1e-15: __fdividef is within 2 ulp here
                dec = (double)(-__fdividef(delta, s2) * (s2 - 2.f * sq));
            }
            acc[j] += dec;
        }
    }
}

// JB = accumulator bucket (2, 8 or 16 step lengths); J <= JB are used.
// ADV: also store f + gam[0] d over f (the frames of the step gam[0], by
// linearity of F Q), in place: each pixel is read and written by one thread.
template <int JB, int MODEL, bool ADV = false>
__global__ void __launch_bounds__(RT) k_ls_frames(const float2 *__restrict__ f, const float2 *__restrict__ d,
                                                  const float *__restrict__ D, float dscale, size_t n,
                                                  const double *__restrict__ gam, int J, double *__restrict__ work,
                                                  float2 *fo = nullptr, const double *__restrict__ skip = nullptr)
{
    if (skip != nullptr && *skip != 0.0) return;   // the whole grid skips together
    double acc[JB];
#pragma unroll
    for (int j = 0; j < JB; ++j) acc[j] = 0;
    float gj[JB];
#pragma unroll
    for (int j = 0; j < JB; ++j) gj[j] = j < J ? (float)gam[j] : 0.f;
    // U pixels a stride apart per trip, loads first: 20 U bytes in flight per thread
    constexpr int U = JB <= 8 ? 4 : 1;
    const size_t stride = (size_t)gridDim.x * RT;
    size_t i = (size_t)blockIdx.x * RT + threadIdx.x;
    for (; i + (U - 1) * stride < n; i += U * stride) {
        float2 x[U], y[U];
        float dd[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            x[u] = f[i + u * stride];
            y[u] = d[i + u * stride];
            dd[u] = D[i + u * stride];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) ls_pixel<JB, MODEL>(acc, gj, J, x[u], y[u], dd[u] * dscale);
        if (ADV) {
#pragma unroll
            for (int u = 0; u < U; ++u)
                fo[i + u * stride] = make_float2(fmaf(gj[0], y[u].x, x[u].x), fmaf(gj[0], y[u].y, x[u].y));
        }
    }
    for (; i < n; i += stride) {
        const float2 x = f[i], y = d[i];
        ls_pixel<JB, MODEL>(acc, gj, J, x, y, D[i] * dscale);
        if (ADV) fo[i] = make_float2(fmaf(gj[0], y.x, x.x), fmaf(gj[0], y.y, x.y));
    }
    block_reduce_store<JB>(acc, work, blockIdx.x, gridDim.x);
}

// One wave of a k_ls_frames instance on the current device (at most RB
// blocks, the partials' capacity); fixed for a given device, so sums stay
// deterministic.
template <typename Kern>
int one_wave(Kern kern)
{
    int dev = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, RT, 0) != cudaSuccess)
        return -1;
    const int g = nsm * per_sm;
    return g < 1 ? 1 : (g > RB ? RB : g);
}

template <int JB, int MODEL, bool ADV = false>
int launch_ls_bucket(const float2 *f, const float2 *d, const float *data, float dscale, size_t n,
                     const double *gammas, int J, double *work, cudaStream_t st, int *nblk, float2 *fo = nullptr,
                     const double *skip = nullptr)
{
    const int grid = one_wave(k_ls_frames<JB, MODEL, ADV>);
    if (grid < 0) {
        pt::set_error("ls_frames: occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
        return PT_ERR_CUDA;
    }
    k_ls_frames<JB, MODEL, ADV><<<grid, RT, 0, st>>>(f, d, data, dscale, n, gammas, J, work, fo, skip);
    PT_LAUNCHED("k_ls_frames");
    *nblk = grid;
    return PT_OK;
}

// Launches k_ls_frames; *nblk receives the number of partials per step length.
// fo != nullptr: the advancing variant (fo = f + gammas[0] d, fo may be f).
int launch_ls_frames(const float2 *f, const float2 *d, const float *data, float dscale, size_t n, int model,
                     const double *gammas, int J, double *work, cudaStream_t st, int *nblk, float2 *fo = nullptr,
                     const double *skip = nullptr)
{
    if (fo != nullptr) {
        if (model == 0) {
            if (J <= 2) return launch_ls_bucket<2, 0, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
            if (J <= 8) return launch_ls_bucket<8, 0, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
            return launch_ls_bucket<16, 0, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
        }
        if (J <= 2) return launch_ls_bucket<2, 1, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
        if (J <= 8) return launch_ls_bucket<8, 1, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
        return launch_ls_bucket<16, 1, true>(f, d, data, dscale, n, gammas, J, work, st, nblk, fo);
    }
    if (model == 0) {
        if (J <= 2) return launch_ls_bucket<2, 0>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
        if (J <= 8) return launch_ls_bucket<8, 0>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
        return launch_ls_bucket<16, 0>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
    }
    if (J <= 2) return launch_ls_bucket<2, 1>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
    if (J <= 8) return launch_ls_bucket<8, 1>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
    return launch_ls_bucket<16, 1>(f, d, data, dscale, n, gammas, J, work, st, nblk, nullptr, skip);
}

// Lagrangian data term, solver.py:294-298.  Poisson also subtracts the
// minimum d - 2 d log(sqrt d) so the term is >= 0.
__global__ void __launch_bounds__(RT) k_lagr_frames(const float2 *__restrict__ f, const float *__restrict__ D,
                                                    float dscale, size_t n, int model, double *__restrict__ work)
{
    double acc[1] = {0};
    for (size_t i = (size_t)blockIdx.x * RT + threadIdx.x; i < n; i += (size_t)gridDim.x * RT) {
        const float2 x = f[i];
        const float dd = D[i] * dscale;
        const float a = sqrtf(x.x * x.x + x.y * x.y);
        if (model == 0) {
            const float sq = sqrtf(dd);
            acc[0] += (double)a * a - 2.0 * dd * (double)logf(fmaxf(a, 1e-32f)) -
                      ((double)dd - 2.0 * dd * (double)logf(fmaxf(sq, 1e-32f)));
        } else {
            const double t = (double)a - (double)sqrtf(dd);
            acc[0] += t * t;
        }
    }
    block_reduce_store<1>(acc, work, blockIdx.x, gridDim.x);
}

// ---- elementwise ----------------------------------------------------------
struct Lin4 {
    const float2 *x[4];
    float2 c[4];
};

// out = sum_{i<k} c_i x_i  (out may alias any x_i)
__global__ void k_lincomb(float2 *__restrict__ out, size_t n, int k, Lin4 p)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 acc = czero();
        for (int j = 0; j < k; ++j) acc = acc + cmul(p.c[j], p.x[j][i]);
        out[i] = acc;
    }
}

// mode 0: out = a * b;  mode 1: out = conj(a) * (b - c);  mode 2: out = conj(a) * b
__global__ void k_cmul(float2 *__restrict__ out, const float2 *__restrict__ a, const float2 *__restrict__ b,
                       const float2 *__restrict__ c, size_t n, int mode)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 x = a[i];
        float2 y = b[i];
        if (mode == 1) y = y - c[i];
        out[i] = mode == 0 ? cmul(x, y) : cmulc(x, y);
    }
}

// out = exp(i s x) * exp(i phi)   (exptomo, solver.py:59-60; h update, :322)
__global__ void k_expmap(float2 *__restrict__ out, const float2 *__restrict__ x, size_t n, float s, float phi)
{
    float cp, sp;
    sincosf(phi, &sp, &cp);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 v = x[i];
        const float mag = expf(-s * v.y);
        float sn, cs;
        sincosf(s * v.x, &sn, &cs);
        out[i] = cmul(make_float2(mag * cs, mag * sn), make_float2(cp, sp));
    }
}

// out = c * mlog(x),  mlog: |x| < 1e-32 -> 1e-32, then complex log (solver.py:48-52)
__global__ void k_logmap(float2 *__restrict__ out, const float2 *__restrict__ x, size_t n, float2 c)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 v = x[i];
        const float a = hypotf(v.x, v.y);
        if (a < 1e-32f) v = make_float2(1e-32f, 0.f);
        const float2 l = make_float2(logf(fmaxf(a, 1e-32f)), a < 1e-32f ? 0.f : atan2f(v.y, v.x));
        out[i] = cmul(c, l);
    }
}

// takexi second half (solver.py:163-166) with t given and tmax = max|t|:
//   K = i t / tmax;  xi0 = K * (-i mlog(t) / (voxel k)) * coeftomo
__global__ void k_takexi(float2 *__restrict__ K, float2 *__restrict__ xi0, const float2 *__restrict__ t, size_t n,
                         float inv_tmax, float cxi)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 v = t[i];
        const float kx = -v.y * inv_tmax, ky = v.x * inv_tmax;   // i t / tmax
        const float a = hypotf(v.x, v.y);
        if (a < 1e-32f) v = make_float2(1e-32f, 0.f);
        const float lr = logf(fmaxf(a, 1e-32f)), li = a < 1e-32f ? 0.f : atan2f(v.y, v.x);
        // -i * log(t) * cxi = (li - i lr) * cxi
        const float2 m = make_float2(li * cxi, -lr * cxi);
        K[i] = make_float2(kx, ky);
        xi0[i] = cmul(make_float2(kx, ky), m);
    }
}

// gradient residual of the ptycho data term (solver.py:220-224), D scaled by dscale:
//   Poisson  r = f - D f / (|f|^2 + 1e-32)
//   Gaussian r = f - sqrt(D) exp(i angle(f))
__global__ void k_residual(float2 *__restrict__ out, const float2 *__restrict__ f, const float *__restrict__ D,
                           float dscale, size_t n, int model)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 x = f[i];
        const float dd = D[i] * dscale;
        out[i] = model == 0 ? pt_residual_poisson(x, dd) : pt_residual_gaussian(x, dd);
    }
}

// out = |x|^2 * scale   (fwd_ptycho_batch intensities, solver.py:115)
__global__ void k_abs2(float *__restrict__ out, const float2 *__restrict__ x, size_t n, float scale)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 v = x[i];
        out[i] = (v.x * v.x + v.y * v.y) * scale;
    }
}

// ---- TV regulariser J, J* (solver.py:128-146) --------------------------------
// u [nz][ny][nx]; res [3][nz][ny][nx]: forward differences along x, y, z times s
__global__ void k_reg_fwd(float2 *__restrict__ res, const float2 *__restrict__ u, int nz, int ny, int nx, float s)
{
    const size_t vol = (size_t)nz * ny * nx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((size_t)nx * ny));
        const float2 c = u[i];
        res[i] = x < nx - 1 ? s * (u[i + 1] - c) : czero();
        res[vol + i] = y < ny - 1 ? s * (u[i + nx] - c) : czero();
        res[2 * vol + i] = z < nz - 1 ? s * (u[i + (size_t)nx * ny] - c) : czero();
    }
}

__global__ void k_reg_adj(float2 *__restrict__ res, const float2 *__restrict__ g, int nz, int ny, int nx, float s)
{
    const size_t vol = (size_t)nz * ny * nx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((size_t)nx * ny));
        const float2 *g0 = g, *g1 = g + vol, *g2 = g + 2 * vol;
        float2 r = x > 0 ? g0[i] - g0[i - 1] : g0[i];
        r = r + (y > 0 ? g1[i] - g1[i - nx] : g1[i]);
        r = r + (z > 0 ? g2[i] - g2[i - (size_t)nx * ny] : g2[i]);
        res[i] = s * r;
    }
}

// the entries of g [3][nz][ny][nx] outside the range of J: x = nx-1 of
// component 0, y = ny-1 of 1, z = nz-1 of 2
__global__ void k_reg_mask(float2 *__restrict__ g, int nz, int ny, int nx)
{
    const size_t vol = (size_t)nz * ny * nx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), z = (int)(i / ((size_t)nx * ny));
        if (x == nx - 1) g[i] = czero();
        if (y == ny - 1) g[vol + i] = czero();
        if (z == nz - 1) g[2 * vol + i] = czero();
    }
}

// solve_reg (solver.py:257-264): z = J u + mu/tau, isotropic soft threshold alpha/tau
__global__ void k_solve_reg(float2 *__restrict__ z, const float2 *__restrict__ u, const float2 *__restrict__ mu,
                            int nz, int ny, int nx, float s, float inv_tau, float thr)
{
    const size_t vol = (size_t)nz * ny * nx;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vol; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx), y = (int)((i / nx) % ny), zz = (int)(i / ((size_t)nx * ny));
        const float2 c = u[i];
        float2 v0 = x < nx - 1 ? s * (u[i + 1] - c) : czero();
        float2 v1 = y < ny - 1 ? s * (u[i + nx] - c) : czero();
        float2 v2 = zz < nz - 1 ? s * (u[i + (size_t)nx * ny] - c) : czero();
        v0 = v0 + inv_tau * mu[i];
        v1 = v1 + inv_tau * mu[vol + i];
        v2 = v2 + inv_tau * mu[2 * vol + i];
        const float za = sqrtf(v0.x * v0.x + v0.y * v0.y + v1.x * v1.x + v1.y * v1.y + v2.x * v2.x + v2.y * v2.y);
        if (za <= thr) {
            v0 = v1 = v2 = czero();
        } else {
            const float f = thr / za;
            v0 = v0 - f * v0;
            v1 = v1 - f * v1;
            v2 = v2 - f * v2;
        }
        z[i] = v0;
        z[vol + i] = v1;
        z[2 * vol + i] = v2;
    }
}

unsigned ew_blocks(size_t n)
{
    size_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 16 ? (b ? b : 1) : 148 * 16);
}

}  // namespace

extern "C" size_t pt_reduce_workspace_bytes(void) { return (size_t)RB * MAXK * sizeof(double); }

extern "C" int pt_reduce_c64(int op, const void *a, const void *b, size_t n, int c0, int c1, int ncol, void *work,
                             void *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(op >= 0 && op <= 7, "reduce: unknown op %d", op);
    PT_CHECK_ARG(a && work && out, "reduce: null pointer");
    PT_CHECK_ARG((op != 1 && op != 2 && op != 5) || b, "reduce: op %d needs two arrays", op);
    PT_CHECK_ARG(op != 4 || (ncol > 0 && c0 >= 0 && c1 <= ncol), "reduce: bad column band");
    cudaStream_t st = (cudaStream_t)stream;
    const int K = op == 1 ? 2 : (op == 2 ? 3 : 1);
    k_reduce<<<RB, RT, 0, st>>>(op, (const float2 *)a, (const float2 *)b, n, c0, c1, ncol, (double *)work);
    PT_LAUNCHED("k_reduce");
    k_finish<<<1, RT, 0, st>>>((const double *)work, (double *)out, K, RB, op == 3 || op == 7);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}

extern "C" int pt_ls_frames(const void *f, const void *d, const float *data, float dscale, size_t n, int model,
                            const double *gammas, int J, void *work, void *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(f && d && data && gammas && work && out, "ls_frames: null pointer");
    PT_CHECK_ARG(J >= 1 && J <= MAXK, "ls_frames: 1 <= J <= %d", MAXK);
    PT_CHECK_ARG(model == 0 || model == 1, "ls_frames: model 0 (poisson) or 1 (gaussian)");
    cudaStream_t st = (cudaStream_t)stream;
    int nblk = 0;
    const int rc = launch_ls_frames((const float2 *)f, (const float2 *)d, data, dscale, n, model, gammas, J,
                                    (double *)work, st, &nblk);
    if (rc != PT_OK) return rc;
    k_finish<<<1, RT, 0, st>>>((const double *)work, (double *)out, J, nblk, 0);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}

extern "C" int pt_ls_frames_advance(void *f, const void *d, const float *data, float dscale, size_t n, int model,
                                    const double *gammas, int J, void *work, void *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(f && d && data && gammas && work && out, "ls_frames_advance: null pointer");
    PT_CHECK_ARG(J >= 1 && J <= MAXK, "ls_frames_advance: 1 <= J <= %d", MAXK);
    PT_CHECK_ARG(model == 0 || model == 1, "ls_frames_advance: model 0 (poisson) or 1 (gaussian)");
    cudaStream_t st = (cudaStream_t)stream;
    int nblk = 0;
    const int rc = launch_ls_frames((const float2 *)f, (const float2 *)d, data, dscale, n, model, gammas, J,
                                    (double *)work, st, &nblk, (float2 *)f);
    if (rc != PT_OK) return rc;
    k_finish<<<1, RT, 0, st>>>((const double *)work, (double *)out, J, nblk, 0);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}

extern "C" int pt_ls_frames_dev(const void *f, const void *d, const float *data, float dscale, size_t n, int model,
                                const double *gammas, int J, void *work, void *out, const double *skip, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(f && d && data && gammas && work && out, "ls_frames_dev: null pointer");
    PT_CHECK_ARG(J >= 1 && J <= MAXK, "ls_frames_dev: 1 <= J <= %d", MAXK);
    PT_CHECK_ARG(model == 0 || model == 1, "ls_frames_dev: model 0 (poisson) or 1 (gaussian)");
    cudaStream_t st = (cudaStream_t)stream;
    int nblk = 0;
    const int rc = launch_ls_frames((const float2 *)f, (const float2 *)d, data, dscale, n, model, gammas, J,
                                    (double *)work, st, &nblk, nullptr, skip);
    if (rc != PT_OK) return rc;
    k_finish<<<1, RT, 0, st>>>((const double *)work, (double *)out, J, nblk, 0, skip);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}

extern "C" int pt_lagr_frames(const void *f, const float *data, float dscale, size_t n, int model, void *work,
                              void *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(f && data && work && out, "lagr_frames: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    k_lagr_frames<<<RB, RT, 0, st>>>((const float2 *)f, data, dscale, n, model, (double *)work);
    PT_LAUNCHED("k_lagr_frames");
    k_finish<<<1, RT, 0, st>>>((const double *)work, (double *)out, 1, RB, 0);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}

extern "C" int pt_lincomb_c64(void *out, size_t n, int k, const void *const *x, const float *coef, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x && coef && k >= 1 && k <= 4, "lincomb: 1..4 terms");
    Lin4 p;
    for (int j = 0; j < 4; ++j) {
        p.x[j] = j < k ? (const float2 *)x[j] : nullptr;
        p.c[j] = j < k ? make_float2(coef[2 * j], coef[2 * j + 1]) : czero();
        PT_CHECK_ARG(j >= k || p.x[j], "lincomb: null term %d", j);
    }
    k_lincomb<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, n, k, p);
    PT_LAUNCHED("k_lincomb");
    return PT_OK;
}

extern "C" int pt_cmul_c64(void *out, const void *a, const void *b, const void *c, size_t n, int mode, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && a && b && (mode != 1 || c) && mode >= 0 && mode <= 2, "cmul: bad arguments");
    k_cmul<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, (const float2 *)a, (const float2 *)b,
                                                           (const float2 *)c, n, mode);
    PT_LAUNCHED("k_cmul");
    return PT_OK;
}

extern "C" int pt_expmap_c64(void *out, const void *x, size_t n, float s, float phi, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x, "expmap: null pointer");
    k_expmap<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, (const float2 *)x, n, s, phi);
    PT_LAUNCHED("k_expmap");
    return PT_OK;
}

extern "C" int pt_logmap_c64(void *out, const void *x, size_t n, float cre, float cim, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x, "logmap: null pointer");
    k_logmap<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, (const float2 *)x, n,
                                                             make_float2(cre, cim));
    PT_LAUNCHED("k_logmap");
    return PT_OK;
}

extern "C" int pt_takexi_c64(void *K, void *xi0, const void *t, size_t n, float inv_tmax, float cxi, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(K && xi0 && t, "takexi: null pointer");
    k_takexi<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)K, (float2 *)xi0, (const float2 *)t, n,
                                                             inv_tmax, cxi);
    PT_LAUNCHED("k_takexi");
    return PT_OK;
}

extern "C" int pt_reg_fwd_c64(void *res, const void *u, int nz, int ny, int nx, float s, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(res && u && nz > 0 && ny > 0 && nx > 0, "reg_fwd: bad arguments");
    k_reg_fwd<<<ew_blocks((size_t)nz * ny * nx), 256, 0, (cudaStream_t)stream>>>((float2 *)res, (const float2 *)u,
                                                                                  nz, ny, nx, s);
    PT_LAUNCHED("k_reg_fwd");
    return PT_OK;
}

extern "C" int pt_reg_adj_c64(void *res, const void *g, int nz, int ny, int nx, float s, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(res && g && nz > 0 && ny > 0 && nx > 0, "reg_adj: bad arguments");
    k_reg_adj<<<ew_blocks((size_t)nz * ny * nx), 256, 0, (cudaStream_t)stream>>>((float2 *)res, (const float2 *)g,
                                                                                  nz, ny, nx, s);
    PT_LAUNCHED("k_reg_adj");
    return PT_OK;
}

extern "C" int pt_reg_mask_c64(void *g, int nz, int ny, int nx, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(g && nz > 0 && ny > 0 && nx > 0, "reg_mask: bad arguments");
    k_reg_mask<<<ew_blocks((size_t)nz * ny * nx), 256, 0, (cudaStream_t)stream>>>((float2 *)g, nz, ny, nx);
    PT_LAUNCHED("k_reg_mask");
    return PT_OK;
}

extern "C" int pt_solve_reg_c64(void *z, const void *u, const void *mu, int nz, int ny, int nx, float s,
                                float inv_tau, float thr, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(z && u && mu && nz > 0 && ny > 0 && nx > 0, "solve_reg: bad arguments");
    k_solve_reg<<<ew_blocks((size_t)nz * ny * nx), 256, 0, (cudaStream_t)stream>>>(
        (float2 *)z, (const float2 *)u, (const float2 *)mu, nz, ny, nx, s, inv_tau, thr);
    PT_LAUNCHED("k_solve_reg");
    return PT_OK;
}

extern "C" int pt_residual_c64(void *out, const void *f, const float *data, float dscale, size_t n, int model,
                               void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && f && data && (model == 0 || model == 1), "residual: bad arguments");
    k_residual<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, (const float2 *)f, data, dscale, n,
                                                               model);
    PT_LAUNCHED("k_residual");
    return PT_OK;
}

extern "C" int pt_abs2_c64(float *out, const void *x, size_t n, float scale, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x, "abs2: null pointer");
    k_abs2<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>(out, (const float2 *)x, n, scale);
    PT_LAUNCHED("k_abs2");
    return PT_OK;
}

// ---- pt_ls_frames without any allocation ------------------------------------
// Scratch of the reduction (one FP64 partial per block and step length) in a
// file-scope device array: 1184 blocks x 16 step lengths x 8 B = 148 KiB, held
// by every GPU that loads this library until the process exits.  Host code
// cannot use the array's name as a device address; cudaGetSymbolAddress gives
// the address in the calling thread's current context.  That address belongs
// to the context, not to the device: after cudaDeviceReset the module is
// loaded again (and may move), and a caller's own driver-API context on the
// same device holds a separate copy.  So the address is cached together with
// the unique id of the context it was looked up in (cuCtxGetId, reached
// through cudaGetDriverEntryPointByVersion so that the library needs no link
// to the driver), and looked up again whenever the current context differs.
// Devices past the cache, or a driver without context ids, look it up on
// every call.
#include <mutex>

namespace {
static __device__ __align__(256) double g_ls_scratch[RB * MAXK];

constexpr int MAX_CACHED_DEVICES = 64;
struct ScratchSlot {
    unsigned long long ctx_id;   // 0: nothing cached
    double *ptr;
};
ScratchSlot g_ls_scratch_slot[MAX_CACHED_DEVICES] = {};
std::mutex g_ls_scratch_mu;

typedef int (*ctx_get_current_fn)(void **ctx);
typedef int (*ctx_get_id_fn)(void *ctx, unsigned long long *id);

// Unique id of the calling thread's current CUDA context; 0 when there is
// none yet or the driver cannot report it.
unsigned long long current_context_id()
{
    static ctx_get_current_fn get_current = nullptr;
    static ctx_get_id_fn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *a = nullptr, *b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &a, 12000, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPointByVersion("cuCtxGetId", &b, 12000, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_current = (ctx_get_current_fn)a;
            get_id = (ctx_get_id_fn)b;
        }
        cudaGetLastError();   // a failed query leaves no sticky error behind
    });
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

int ls_scratch_for_current_context(double **ptr)
{
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    const bool cached = dev >= 0 && dev < MAX_CACHED_DEVICES;
    std::lock_guard<std::mutex> lock(g_ls_scratch_mu);
    unsigned long long id = current_context_id();
    if (cached && id != 0 && g_ls_scratch_slot[dev].ctx_id == id) {
        *ptr = g_ls_scratch_slot[dev].ptr;
        return PT_OK;
    }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ls_scratch);
    if (e != cudaSuccess || !p) {
        pt::set_error("ls_frames_noalloc: cudaGetSymbolAddress of the static scratch failed on device %d: %s", dev,
                      cudaGetErrorString(e));
        return PT_ERR_CUDA;
    }
    id = current_context_id();   // the look-up may have created the context
    if (cached) g_ls_scratch_slot[dev] = ScratchSlot{id, (double *)p};
    *ptr = (double *)p;
    return PT_OK;
}
}  // namespace

extern "C" int pt_ls_frames_noalloc(const void *f, const void *d, const float *data, float dscale, size_t n,
                                    int model, const double *gammas, int J, void *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(f && d && data && gammas && out, "ls_frames_noalloc: null pointer");
    PT_CHECK_ARG(J >= 1 && J <= MAXK,
                 "ls_frames_noalloc: J = %d step lengths exceeds the static scratch (1 <= J <= %d)", J, MAXK);
    PT_CHECK_ARG(model == 0 || model == 1, "ls_frames_noalloc: model 0 (poisson) or 1 (gaussian)");
    double *work = nullptr;
    const int rc = ls_scratch_for_current_context(&work);
    if (rc != PT_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // every partial that k_finish reads (J x nblk) is written by k_ls_frames in
    // this call, so nothing in the shared scratch needs clearing first
    int nblk = 0;
    const int rc2 =
        launch_ls_frames((const float2 *)f, (const float2 *)d, data, dscale, n, model, gammas, J, work, st, &nblk);
    if (rc2 != PT_OK) return rc2;
    k_finish<<<1, RT, 0, st>>>(work, (double *)out, J, nblk, 0);
    PT_LAUNCHED("k_finish");
    return PT_OK;
}
