// The learned Fourier preconditioner of the tomography CG (no counterpart in
// the reference, whose CG, src/ptychotomo/solver.py:180-203, is
// unpreconditioned).
//
// The tomography subproblem minimises rho ||K R u - xi0||^2 + tau ||J u - xi1||^2;
// its normal operator is A = rho R^T |K|^2 R + tau J^T J.  The preconditioner
//     P = D^-1/2  F2^-1 diag(p)  F2  D^-1/2        (per slice, 2-D DFT F2)
// is symmetric positive definite for p > 0, so a preconditioned CG keeps the
// subproblem's minimiser.  D is the diagonal of A with |K|^2 replaced by its
// mean kbar: D = rho kbar dR + tau dJ, dR[y][x] = ||R e_yx||^2 (exact, from
// one forward of a unit pixel per slice) and dJ the TV diagonal (4/3 times the
// number of forward differences that touch the voxel).  In the interior D is a
// constant dI, and there
//     p(w) = (rho kbar dI + tau dJI) / (rho kbar a(w) + tau j(w)),
// with j(w) = 4/3 (4 sin^2(pi kx/n) + 4 sin^2(pi ky/n) + jz) the TV symbol
// (jz: the mean of the z term over the slice frequencies) and a(w) the symbol
// of R^T R, learned: a = exp(MLP(features of w)).
//
// Kernels: the features of every frequency; the filter (rows, columns with
// p, inverse rows); the unit-pixel columns and per-slice norms for dR; and the
// per-frequency statistics of probe pairs (z, R^T R z) that give the network
// its training targets.
#include <cmath>
#include <vector>

#include "pt_common.cuh"
#include "pt_fft.cuh"

namespace {

constexpr int RPB = 8;   // rows (or columns) per block, one FFT of T threads each
constexpr int TF = 32;   // threads per FFT

// Feature window for the angular sampling density: +-3 degrees.
constexpr double DENS_HALF = 3.14159265358979323846 / 60.0;

// x[(ky n + kx) * 3 ..] for the 2-D DFT frequency (kx, ky) in FFT order:
//   0: |w| / (n/2)  (radial frequency, 0 .. sqrt 2)
//   1: angular sampling density at the direction of w: the number of
//      measured Fourier lines within +-3 degrees, over its value for ntheta
//      lines spread uniformly on [0, pi) (1 for a full uniform scan)
//   2: missing-wedge extent at the direction of w: the angle to the nearest
//      measured line over pi/2 (0 on a line, 1/3 in the middle of a 60-degree
//      wedge).
// The projection at angle theta samples the slice's DFT on the line through
// the origin with direction (cos theta, -sin theta) (the polar points of
// kernels.cuh:84-95), i.e. at the direction angle -theta modulo pi.
__global__ void k_features(const float *__restrict__ theta, int ntheta, int n, float *__restrict__ x)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * n) return;
    const int ix = i % n, iy = i / n;
    const int kx = ix < n / 2 ? ix : ix - n, ky = iy < n / 2 ? iy : iy - n;
    const double PI = 3.14159265358979323846;
    const double r = sqrt((double)kx * kx + (double)ky * ky) / (0.5 * n);
    double phi = (kx == 0 && ky == 0) ? 0.0 : atan2((double)ky, (double)kx);
    phi = fmod(phi + 2 * PI, PI);
    int count = 0;
    double gap = PI;
    for (int t = 0; t < ntheta; ++t) {
        double psi = fmod(-(double)theta[t], PI);
        if (psi < 0) psi += PI;
        double d = fabs(phi - psi);
        d = fmin(d, PI - d);
        gap = fmin(gap, d);
        count += d <= DENS_HALF;
    }
    const double uniform = 2 * DENS_HALF * ntheta / PI;
    x[3 * (size_t)i] = (float)r;
    x[3 * (size_t)i + 1] = (float)(count / uniform);
    x[3 * (size_t)i + 2] = (float)(gap / (0.5 * PI));
}

__device__ __forceinline__ float tv_count(int i, int len) { return (float)((i > 0) + (i < len - 1)); }

// D^-1/2 at voxel (z, y, x)
__device__ __forceinline__ float inv_sqrt_diag(const float *__restrict__ dR, int z, int y, int x, int n, int nz,
                                               float rk, float tau)
{
    const float dj = (4.f / 3.f) * (tv_count(x, n) + tv_count(y, n) + tv_count(z, nz));
    return rsqrtf(rk * __ldg(&dR[(size_t)y * n + x]) + tau * dj);
}

// rows of each slice: (optionally D^-1/2 *) in -> forward DFT along x -> tmp
// grid (nz * L / RPB); block RPB x TF
template <int L>
__global__ void __launch_bounds__(RPB *TF)
    k_pre_rows(const float2 *__restrict__ in, float2 *__restrict__ tmp, const float *__restrict__ dR, int nz,
               float rk, float tau, int scale_d, const float2 *__restrict__ tw, const double *__restrict__ rkt)
{
    constexpr int PITCH = L + 1;
    if (rkt) {   // rho * kbar and tau from device memory
        rk = (float)rkt[0];
        tau = (float)rkt[1];
    }
    __shared__ float2 sm[RPB * PITCH];
    const int row0 = blockIdx.x * RPB;
    const int f = threadIdx.x / TF, t = threadIdx.x % TF;
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int rr = e / L, x = e % L;
        const int row = row0 + rr;
        float2 v = in[(size_t)row * L + x];
        if (scale_d) v = inv_sqrt_diag(dR, row / L, row % L, x, L, nz, rk, tau) * v;
        sm[rr * PITCH + x] = v;
    }
    __syncthreads();
    ptfft::fft<L, -1, TF>(sm + f * PITCH, 1, t, tw);
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int rr = e / L, x = e % L;
        tmp[(size_t)(row0 + rr) * L + x] = sm[rr * PITCH + x];
    }
}

// columns of each slice, in place.  MODE 0: forward DFT along y; 1: forward,
// x p(kx, ky), inverse; 2: inverse only.  grid (L / RPB, nz); block RPB x TF
template <int L, int MODE>
__global__ void __launch_bounds__(RPB *TF)
    k_pre_cols(float2 *__restrict__ tmp, const float *__restrict__ a, float rk, float tau, float jz, float dI, float dJI,
               const float2 *__restrict__ tw, const double *__restrict__ rkt)
{
    constexpr int PITCH = L + 1;
    if (rkt) {
        rk = (float)rkt[0];
        tau = (float)rkt[1];
    }
    const float num = rk * dI + tau * dJI;
    __shared__ float2 sm[RPB * PITCH];
    const int kx0 = blockIdx.x * RPB, z = blockIdx.y;
    float2 *sl = tmp + (size_t)z * L * L;
    const int f = threadIdx.x / TF, t = threadIdx.x % TF;
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int y = e / RPB, c = e % RPB;
        sm[c * PITCH + y] = sl[(size_t)y * L + kx0 + c];
    }
    __syncthreads();
    if (MODE != 2) ptfft::fft<L, -1, TF>(sm + f * PITCH, 1, t, tw);
    if (MODE == 1) {
        for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
            const int c = e / L, ky = e % L;
            const int kx = kx0 + c;
            const float sx = sinpif((float)kx / L), sy = sinpif((float)ky / L);
            const float j = (4.f / 3.f) * (4.f * sx * sx + 4.f * sy * sy + jz);
            const float p = num / (rk * __ldg(&a[(size_t)ky * L + kx]) + tau * j);
            sm[c * PITCH + ky] = p * sm[c * PITCH + ky];
        }
        __syncthreads();
    }
    if (MODE != 0) ptfft::fft<L, +1, TF>(sm + f * PITCH, 1, t, tw);
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int y = e / RPB, c = e % RPB;
        sl[(size_t)y * L + kx0 + c] = sm[c * PITCH + y];
    }
}

// a random phase per element, keeping the modulus (floored): x <-
// sqrt(|x|^2 + floor^2) exp(2 pi i u),
// u from a counter-based hash of (seed, index) (C. Wellons' "lowbias32"
// integer hash, applied twice), so probes are reproducible
__device__ __forceinline__ unsigned mix32(unsigned x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}
__global__ void k_random_phase(float2 *__restrict__ x, size_t total, unsigned seed, float floor2)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const unsigned h = mix32(mix32((unsigned)i ^ mix32(seed)) + (unsigned)(i >> 32));
    const float u = (float)(h >> 8) * (1.f / 16777216.f);
    float sn, cs;
    sincospif(2.f * u, &sn, &cs);
    const float2 v = x[i];
    const float m = sqrtf(v.x * v.x + v.y * v.y + floor2);
    x[i] = make_float2(m * cs, m * sn);
}

// inverse DFT along x, x (D^-1/2 if scale_d) / L^2 -> out.  grid (nz * L / RPB)
template <int L>
__global__ void __launch_bounds__(RPB *TF)
    k_pre_rows_inv(const float2 *__restrict__ tmp, float2 *__restrict__ out, const float *__restrict__ dR, int nz,
                   float rk, float tau, int scale_d, const float2 *__restrict__ tw, const double *__restrict__ rkt)
{
    constexpr int PITCH = L + 1;
    if (rkt) {
        rk = (float)rkt[0];
        tau = (float)rkt[1];
    }
    __shared__ float2 sm[RPB * PITCH];
    const int row0 = blockIdx.x * RPB;
    const int f = threadIdx.x / TF, t = threadIdx.x % TF;
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int rr = e / L, x = e % L;
        sm[rr * PITCH + x] = tmp[(size_t)(row0 + rr) * L + x];
    }
    __syncthreads();
    ptfft::fft<L, +1, TF>(sm + f * PITCH, 1, t, tw);
    const float inv = 1.f / ((float)L * (float)L);
    for (int e = threadIdx.x; e < RPB * L; e += blockDim.x) {
        const int rr = e / L, x = e % L;
        const int row = row0 + rr;
        const float sc = scale_d ? inv * inv_sqrt_diag(dR, row / L, row % L, x, L, nz, rk, tau) : inv;
        out[(size_t)row * L + x] = sc * sm[rr * PITCH + x];
    }
}

// num[k] += sum_z Re(conj(Z_z[k]) AZ_z[k]), den[k] += sum_z |Z_z[k]|^2 (FP64, z in order)
__global__ void k_spectrum(const float2 *__restrict__ Z, const float2 *__restrict__ AZ, int nz, int nn,
                           double *__restrict__ num, double *__restrict__ den)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nn) return;
    double s = 0, d = 0;
    for (int z = 0; z < nz; ++z) {
        const float2 a = Z[(size_t)z * nn + k], b = AZ[(size_t)z * nn + k];
        s += (double)a.x * b.x + (double)a.y * b.y;
        d += (double)a.x * a.x + (double)a.y * a.y;
    }
    num[k] += s;
    den[k] += d;
}

// y = log(num / den) and w = 1 where the quotient is positive and den carries
// energy (den > rel * max den), else y = w = 0
__global__ void k_targets(const double *__restrict__ num, const double *__restrict__ den, int nn, double thr,
                          float *__restrict__ y, float *__restrict__ w)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nn) return;
    const double d = den[i], q = d > 0 ? num[i] / d : 0.0;
    const bool ok = d > thr && q > 0;
    y[i] = ok ? (float)log(q) : 0.f;
    w[i] = ok ? 1.f : 0.f;
}

// x[z][y][x] *= W(y, x): a radial window, 1 inside radius r0 (pixels, about
// the slice centre), falling linearly to 0 at r1; probes that vanish near
// the slice border see the interior operator (no edge replication)
__global__ void k_window(float2 *__restrict__ x, int nz, int n, float r0, float r1)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nz * n * n) return;
    const int c = (int)(i % n), r = (int)((i / n) % n);
    const float dx = c - 0.5f * (n - 1), dy = r - 0.5f * (n - 1);
    const float d = sqrtf(dx * dx + dy * dy);
    const float w = d <= r0 ? 1.f : (d >= r1 ? 0.f : (r1 - d) / (r1 - r0));
    x[i] = w * x[i];
}

__global__ void k_exp(const float *__restrict__ z, float *__restrict__ a, int nn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nn) a[i] = expf(z[i]);
}

// unit pixels: slice q of the batch holds pixel pix[q0 + q] (or nothing)
__global__ void k_unit_pixels(float2 *__restrict__ u, const int *__restrict__ pix, int q0, int npix, int nz, int nn)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nz * nn) return;
    const int q = (int)(i / nn), k = (int)(i % nn);
    u[i] = (q0 + q < npix && pix[q0 + q] == k) ? make_float2(1.f, 0.f) : czero();
}

// out[q] = ||g[:, q, :]||^2 for projections g [ntheta][nz][n] (one block per slice)
__global__ void k_slice_norm2(const float2 *__restrict__ g, int ntheta, int nz, int n, double *__restrict__ out)
{
    __shared__ double red[256];
    const int q = blockIdx.x;
    double s = 0;
    for (int e = threadIdx.x; e < ntheta * n; e += blockDim.x) {
        const int th = e / n, c = e % n;
        const float2 v = g[((size_t)th * nz + q) * n + c];
        s += (double)v.x * v.x + (double)v.y * v.y;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = red[0];
}

}  // namespace

// ============================================================================
struct pt_precond {
    int nz = 0, n = 0;
    float2 *tw = nullptr;
    float2 *tmp = nullptr, *tmp2 = nullptr;
    float *a = nullptr;    // [n][n] symbol of R^T R
    float *dR = nullptr;   // [n][n] diagonal of R^T R
    float dI = 0.f;        // its interior value
    bool have_a = false, have_d = false;
};

namespace {

void precond_free(pt_precond *h)
{
    void *bufs[] = {h->tw, h->tmp, h->tmp2, h->a, h->dR};
    for (void *p : bufs)
        if (p) cudaFree(p);
}

#define PT_PRECOND_SIZES(X) X(16) X(32) X(64) X(128) X(256) X(512)

bool size_supported(int n)
{
#define PT_CASE(L) \
    if (n == L) return true;
    PT_PRECOND_SIZES(PT_CASE)
#undef PT_CASE
    return false;
}

template <int L>
int run_filter(pt_precond *h, float2 *out, const float2 *in, float rk, float tau, cudaStream_t st,
               const double *rkt)
{
    const float jz = h->nz > 1 ? 2.f : 0.f;
    const float dJI = (4.f / 3.f) * (2.f + 2.f + (h->nz > 1 ? 2.f : 0.f));
    const unsigned rows = (unsigned)((size_t)h->nz * L / RPB);
    k_pre_rows<L><<<rows, RPB * TF, 0, st>>>(in, h->tmp, h->dR, h->nz, rk, tau, 1, h->tw, rkt);
    PT_LAUNCHED("k_pre_rows");
    k_pre_cols<L, 1><<<dim3(L / RPB, h->nz), RPB * TF, 0, st>>>(h->tmp, h->a, rk, tau, jz, h->dI, dJI, h->tw, rkt);
    PT_LAUNCHED("k_pre_cols");
    k_pre_rows_inv<L><<<rows, RPB * TF, 0, st>>>(h->tmp, out, h->dR, h->nz, rk, tau, 1, h->tw, rkt);
    PT_LAUNCHED("k_pre_rows_inv");
    return PT_OK;
}

template <int L>
int run_dft2(pt_precond *h, float2 *dst, const float2 *in, cudaStream_t st)
{
    const unsigned rows = (unsigned)((size_t)h->nz * L / RPB);
    k_pre_rows<L><<<rows, RPB * TF, 0, st>>>(in, dst, h->dR, h->nz, 0.f, 0.f, 0, h->tw, nullptr);
    PT_LAUNCHED("k_pre_rows");
    k_pre_cols<L, 0><<<dim3(L / RPB, h->nz), RPB * TF, 0, st>>>(dst, nullptr, 0.f, 0.f, 0.f, 0.f, 0.f, h->tw,
                                                                nullptr);
    PT_LAUNCHED("k_pre_cols");
    return PT_OK;
}

// dst = the same modulus spectrum as src with random phases, back in space:
// IDFT2(|DFT2(src)| exp(2 pi i u)) / L^2 (src and dst may alias)
template <int L>
int run_phase_probe(pt_precond *h, float2 *dst, const float2 *src, unsigned seed, float floor, cudaStream_t st)
{
    const size_t tot = (size_t)h->nz * L * L;
    if (src) {
        int rc = run_dft2<L>(h, h->tmp, src, st);
        if (rc != PT_OK) return rc;
    } else {   // white: unit modulus at every frequency
        PT_CUDA(cudaMemsetAsync(h->tmp, 0, tot * sizeof(float2), st));
        floor = 1.f;
    }
    k_random_phase<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(h->tmp, tot, seed, floor * floor);
    PT_LAUNCHED("k_random_phase");
    k_pre_cols<L, 2><<<dim3(L / RPB, h->nz), RPB * TF, 0, st>>>(h->tmp, nullptr, 0.f, 0.f, 0.f, 0.f, 0.f, h->tw,
                                                                nullptr);
    PT_LAUNCHED("k_pre_cols");
    const unsigned rows = (unsigned)((size_t)h->nz * L / RPB);
    k_pre_rows_inv<L><<<rows, RPB * TF, 0, st>>>(h->tmp, dst, h->dR, h->nz, 0.f, 0.f, 0, h->tw, nullptr);
    PT_LAUNCHED("k_pre_rows_inv");
    return PT_OK;
}

int dispatch_phase_probe(pt_precond *h, float2 *dst, const float2 *src, unsigned seed, float floor, cudaStream_t st)
{
#define PT_CASE(L) \
    if (h->n == L) return run_phase_probe<L>(h, dst, src, seed, floor, st);
    PT_PRECOND_SIZES(PT_CASE)
#undef PT_CASE
    return PT_ERR_UNSUPPORTED;
}

int dispatch_filter(pt_precond *h, float2 *out, const float2 *in, float rk, float tau, cudaStream_t st,
                    const double *rkt = nullptr)
{
#define PT_CASE(L) \
    if (h->n == L) return run_filter<L>(h, out, in, rk, tau, st, rkt);
    PT_PRECOND_SIZES(PT_CASE)
#undef PT_CASE
    return PT_ERR_UNSUPPORTED;
}

int dispatch_dft2(pt_precond *h, float2 *dst, const float2 *in, cudaStream_t st)
{
#define PT_CASE(L) \
    if (h->n == L) return run_dft2<L>(h, dst, in, st);
    PT_PRECOND_SIZES(PT_CASE)
#undef PT_CASE
    return PT_ERR_UNSUPPORTED;
}

}  // namespace

extern "C" int pt_precond_create(size_t nz, size_t n, pt_precond **out)
{
    pt::clear_error();
    PT_CHECK_ARG(out != nullptr, "precond: null handle slot");
    PT_CHECK_ARG(nz >= 1 && n >= 1, "precond: empty volume");
    if (!size_supported((int)n)) {
        pt::set_error("precond: slice width %zu not compiled (16..512, powers of two)", n);
        return PT_ERR_UNSUPPORTED;
    }
    pt_precond *h = new pt_precond();
    h->nz = (int)nz;
    h->n = (int)n;
    const size_t vol = nz * n * n;
    bool ok = cudaMalloc(&h->tw, n * sizeof(float2)) == cudaSuccess &&
              cudaMalloc(&h->tmp, vol * sizeof(float2)) == cudaSuccess &&
              cudaMalloc(&h->tmp2, vol * sizeof(float2)) == cudaSuccess &&
              cudaMalloc(&h->a, n * n * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&h->dR, n * n * sizeof(float)) == cudaSuccess;
    if (ok) {
        std::vector<float2> tw(n);
        pt_make_twiddles(tw.data(), (int)n);
        ok = cudaMemcpy(h->tw, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        precond_free(h);
        delete h;
        pt::set_error("precond: device allocation failed");
        return PT_ERR_ALLOC;
    }
    *out = h;
    return PT_OK;
}

extern "C" int pt_precond_destroy(pt_precond *h)
{
    if (!h) return PT_OK;
    precond_free(h);
    delete h;
    return PT_OK;
}

extern "C" int pt_precond_features(const float *theta, int ntheta, int n, float *x, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(theta && x && ntheta >= 1 && n >= 1, "precond_features: bad arguments");
    const int nn = n * n;
    k_features<<<(nn + 255) / 256, 256, 0, (cudaStream_t)stream>>>(theta, ntheta, n, x);
    PT_LAUNCHED("k_features");
    return PT_OK;
}

extern "C" int pt_precond_set_log_symbol(pt_precond *h, const float *log_a, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && log_a, "precond_set_log_symbol: null pointer");
    const int nn = h->n * h->n;
    k_exp<<<(nn + 255) / 256, 256, 0, (cudaStream_t)stream>>>(log_a, h->a, nn);
    PT_LAUNCHED("k_exp");
    h->have_a = true;
    return PT_OK;
}

extern "C" int pt_precond_get_symbol(const pt_precond *h, float *a, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && a, "precond_get_symbol: null pointer");
    if (!h->have_a) {
        pt::set_error("precond_get_symbol: no symbol set");
        return PT_ERR_STATE;
    }
    PT_CUDA(cudaMemcpyAsync(a, h->a, (size_t)h->n * h->n * sizeof(float), cudaMemcpyDefault, (cudaStream_t)stream));
    return PT_OK;
}

// diagonal of (scale R)^T (scale R): exact for the edge pixels (the only ones
// the forward's edge replication copies) and one interior pixel, whose value
// every other pixel takes (the transform is translation invariant inside)
extern "C" int pt_precond_set_diag(pt_precond *h, pt_radon *r, float scale, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && r, "precond_set_diag: null pointer");
    int N = 0, M = 0;
    float mu = 0;
    int rc = pt_radon_get_params(r, &N, &M, &mu);
    if (rc != PT_OK) return rc;
    const int n = h->n, nn = n * n;
    PT_CHECK_ARG(2 * N == 3 * n, "precond_set_diag: the radon operator's width differs from %d", n);
    // the radon operator's own slice count and angles
    int rnz = 0, rnt = 0;
    rc = pt::radon_dims(r, &rnz, &rnt);
    if (rc != PT_OK) return rc;
    std::vector<int> pix;
    for (int x = 0; x < n; ++x) pix.push_back(x);                       // row 0
    for (int x = 0; x < n; ++x) pix.push_back((n - 1) * n + x);         // row n-1
    for (int y = 1; y < n - 1; ++y) pix.push_back(y * n);               // column 0
    for (int y = 1; y < n - 1; ++y) pix.push_back(y * n + n - 1);       // column n-1
    pix.push_back((n / 2) * n + n / 2);                                  // interior
    const int npix = (int)pix.size();
    cudaStream_t st = (cudaStream_t)stream;
    int *dpix = nullptr;
    float2 *u = nullptr, *g = nullptr;
    double *norms = nullptr;
    std::vector<double> hn((size_t)rnz), val(npix);
    cudaError_t e = cudaMalloc(&dpix, npix * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&u, (size_t)rnz * nn * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&g, (size_t)rnt * rnz * n * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&norms, (size_t)rnz * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(dpix, pix.data(), npix * sizeof(int), cudaMemcpyHostToDevice);
    for (int q0 = 0; e == cudaSuccess && rc == PT_OK && q0 < npix; q0 += rnz) {
        const size_t tot = (size_t)rnz * nn;
        k_unit_pixels<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(u, dpix, q0, npix, rnz, nn);
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        rc = pt_radon_fwd_scaled(r, g, u, scale, st);
        if (rc != PT_OK) break;
        k_slice_norm2<<<rnz, 256, 0, st>>>(g, rnt, rnz, n, norms);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hn.data(), norms, rnz * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        for (int q = 0; e == cudaSuccess && q < rnz && q0 + q < npix; ++q) val[q0 + q] = hn[q];
    }
    if (e == cudaSuccess && rc == PT_OK) {
        std::vector<float> d(nn, (float)val[npix - 1]);
        for (int k = 0; k + 1 < npix; ++k) d[pix[k]] = (float)val[k];
        h->dI = (float)val[npix - 1];
        e = cudaMemcpy(h->dR, d.data(), nn * sizeof(float), cudaMemcpyHostToDevice);
    }
    cudaFree(dpix);
    cudaFree(u);
    cudaFree(g);
    cudaFree(norms);
    if (rc != PT_OK) return rc;
    if (e != cudaSuccess) {
        pt::set_error("precond_set_diag: %s", cudaGetErrorString(e));
        return PT_ERR_CUDA;
    }
    h->have_d = true;
    return PT_OK;
}

extern "C" int pt_precond_get_diag(const pt_precond *h, float *dR, float *dI, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h, "precond_get_diag: null handle");
    if (!h->have_d) {
        pt::set_error("precond_get_diag: set_diag has not been called");
        return PT_ERR_STATE;
    }
    if (dR) PT_CUDA(cudaMemcpyAsync(dR, h->dR, (size_t)h->n * h->n * sizeof(float), cudaMemcpyDefault,
                                    (cudaStream_t)stream));
    if (dI) *dI = h->dI;
    return PT_OK;
}

extern "C" int pt_precond_apply(pt_precond *h, void *out, const void *in, float rho_kbar, float tau, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && out && in, "precond_apply: null pointer");
    PT_CHECK_ARG(rho_kbar > 0.f && tau >= 0.f, "precond_apply: needs rho * kbar > 0 and tau >= 0");
    if (!h->have_a || !h->have_d) {
        pt::set_error("precond_apply: the symbol (set_symbol) and the diagonal (set_diag) must be set first");
        return PT_ERR_STATE;
    }
    return dispatch_filter(h, (float2 *)out, (const float2 *)in, rho_kbar, tau, (cudaStream_t)stream);
}

extern "C" int pt_precond_apply_dev(pt_precond *h, void *out, const void *in, const double *rk_tau, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && out && in && rk_tau, "precond_apply_dev: null pointer");
    if (!h->have_a || !h->have_d) {
        pt::set_error("precond_apply_dev: the symbol (set_log_symbol) and the diagonal (set_diag) must be set first");
        return PT_ERR_STATE;
    }
    return dispatch_filter(h, (float2 *)out, (const float2 *)in, 0.f, 0.f, (cudaStream_t)stream, rk_tau);
}

extern "C" int pt_precond_spectrum(pt_precond *h, double *num, double *den, const void *z, const void *az,
                                   void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && num && den && z && az, "precond_spectrum: null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = dispatch_dft2(h, h->tmp, (const float2 *)z, st);
    if (rc == PT_OK) rc = dispatch_dft2(h, h->tmp2, (const float2 *)az, st);
    if (rc != PT_OK) return rc;
    const int nn = h->n * h->n;
    k_spectrum<<<(nn + 255) / 256, 256, 0, st>>>(h->tmp, h->tmp2, h->nz, nn, num, den);
    PT_LAUNCHED("k_spectrum");
    return PT_OK;
}

extern "C" int pt_precond_dft2(pt_precond *h, void *dst, const void *src, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && dst && src, "precond_dft2: null pointer");
    return dispatch_dft2(h, (float2 *)dst, (const float2 *)src, (cudaStream_t)stream);
}

extern "C" int pt_precond_phase_probe(pt_precond *h, void *dst, const void *src, unsigned seed, float floor,
                                      void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && dst && floor >= 0.f, "precond_phase_probe: bad arguments");
    return dispatch_phase_probe(h, (float2 *)dst, (const float2 *)src, seed, floor, (cudaStream_t)stream);
}

extern "C" int pt_precond_targets(const double *num, const double *den, int nn, double den_max_rel, float *y, float *w,
                                  void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(num && den && y && w && nn > 0, "precond_targets: bad arguments");
    // the threshold needs max(den): one small reduction on the host side of the stream
    std::vector<double> hd(nn);
    PT_CUDA(cudaMemcpyAsync(hd.data(), den, nn * sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    PT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    double mx = 0;
    for (double v : hd) mx = v > mx ? v : mx;
    k_targets<<<(nn + 255) / 256, 256, 0, (cudaStream_t)stream>>>(num, den, nn, den_max_rel * mx, y, w);
    PT_LAUNCHED("k_targets");
    return PT_OK;
}

extern "C" int pt_precond_window(pt_precond *h, void *x, float r0, float r1, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && x && r0 >= 0.f && r1 > r0, "precond_window: bad arguments");
    const size_t tot = (size_t)h->nz * h->n * h->n;
    k_window<<<(unsigned)((tot + 255) / 256), 256, 0, (cudaStream_t)stream>>>((float2 *)x, h->nz, h->n, r0, r1);
    PT_LAUNCHED("k_window");
    return PT_OK;
}

