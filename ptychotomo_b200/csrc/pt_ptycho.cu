// Ptychography operator for sm_100a.
//
// Replaces class ptychofft of the reference (src/cuda/ptychofft.cu:1-93,
// kernels mul/mula/takeshifts/shifts/shiftsa in src/include/kernels.cuh).
//
//  forward  g = F Q psi   (ptychofft.cu:58-76): one block per frame
//    (angle, scan).  Each 1-D DFT of length det is a four-step factorisation
//    det = N1 x N2: N1 points per thread in registers, N2 threads per line,
//    one swizzled shared-memory exchange inside the group.  The probe-weighted
//    patch (detector row = object column, kernels.cuh:257-263) is loaded
//    straight into registers, transformed along the object row, transposed
//    once through shared memory, transformed along the other axis and written
//    with the per-scan phase (kernels.cuh:306-336) applied.
//  adjoint  psi = Q* F* g (ptychofft.cu:78-93): the same transform in reverse;
//    block (part, angle) walks scans s = part, part + parts, ... in order and
//    accumulates conj(probe) x frame into its own slab; with parts > 1 the
//    slabs are summed in a fixed order by a second kernel.  Deterministic,
//    no atomics.
//  Detector 128x128 (k_ptycho_fwd128, k_ptycho_adj128) splits the 2-D
//    transform 16 x 8 by 4 x 32 instead, so a frame passes through shared
//    memory twice rather than three times, with coalesced 256-byte warp
//    accesses on both sides; one 512-thread block per SM.  The adjoint also
//    serves the residual-on-load and probe adjoints.
//  Detector 8x8 uses a plain shared-memory Stockham path.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstdint>
#include <map>
#include <type_traits>
#include <vector>

#include "pt_common.cuh"
#include "pt_fft.cuh"

namespace {

constexpr double PI_REF = 3.1415926535;  // kernels.cuh:1

// Residual of the ptycho data term applied to a frame value x on load
// (solver.py:220-224, D = dscale * data): RESID 0 = none (plain adjoint),
// 1 = Poisson x - D x / (|x|^2 + 1e-32), 2 = Gaussian x - sqrt(D) exp(i angle x).
template <int RESID>
__device__ __forceinline__ float2 resid_of(float2 x, float D)
{
    if constexpr (RESID == 1)
        return pt_residual_poisson(x, D);
    else if constexpr (RESID == 2)
        return pt_residual_gaussian(x, D);
    else
        return x;
}
template <int RESID>
__device__ __forceinline__ float2 resid(float2 x, const float *__restrict__ data, size_t idx, float dscale)
{
    if constexpr (RESID == 0)
        return x;
    else
        return resid_of<RESID>(x, __ldg(&data[idx]) * dscale);
}

template <int DET>
constexpr int ptycho_fft_threads() { return (512 / DET) < 4 ? 4 : ((512 / DET) > 32 ? 32 : 512 / DET); }
template <int DET>
constexpr int ptycho_block() { return DET * ptycho_fft_threads<DET>(); }

// setobj tables: integer corners (kernels.cuh:255-256) and the per-scan
// phase shiftx*shifty (takeshifts, kernels.cuh:306-317, same expressions);
// frac: the offsets s - round(s) in [-1/2, 1/2] (the sub-pixel model's shifts).
__global__ void k_ptycho_tables(const float *__restrict__ scan, int *__restrict__ corner,
                                float2 *__restrict__ phase, float *__restrict__ frac, int nframes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nframes) return;
    const float sx = scan[i], sy = scan[nframes + i];
    corner[2 * i] = (int)roundf(sx);
    corner[2 * i + 1] = (int)roundf(sy);
    frac[2 * i] = sx - roundf(sx);
    frac[2 * i + 1] = sy - roundf(sy);
    float2 px, py;
    px.x = cosf(2 * PI_REF * (sx - roundf(sx)));
    px.y = sinf(2 * PI_REF * (sx - roundf(sx)));
    py.x = cosf(2 * PI_REF * (sy - roundf(sy)));
    py.y = sinf(2 * PI_REF * (sy - roundf(sy)));
    phase[i] = cmul(px, py);
}

template <int DET>
__global__ void __launch_bounds__(ptycho_block<DET>(), 1)
    k_ptycho_fwd_small(const float2 *__restrict__ psi, float2 *__restrict__ g, const int *__restrict__ corner,
                 const float2 *__restrict__ phase, const float2 *__restrict__ prb, int nz, int n, int nscan,
                 int P, float c, float scale, const float2 *__restrict__ tw)
{
    constexpr int T = ptycho_fft_threads<DET>(), NT = ptycho_block<DET>(), PITCH = DET + 1;
    extern __shared__ float2 fr[];
    const int s = blockIdx.x, th = blockIdx.y;
    const int fid = th * nscan + s;
    const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
    float2 *out = g + (size_t)fid * DET * DET;
    if (stx < 0 || sty < 0) {  // skipped scan: the reference leaves a zero frame
        for (int e = threadIdx.x; e < DET * DET; e += NT) out[e] = czero();
        return;
    }
    if (P < DET) {
        for (int e = threadIdx.x; e < DET * DET; e += NT) fr[(e / DET) * PITCH + e % DET] = czero();
        __syncthreads();
    }
    const int off = (DET - P) / 2;
    const float2 *src = psi + ((size_t)th * nz + sty) * n + stx;
    for (int e = threadIdx.x; e < P * P; e += NT) {
        const int iy = e / P, ix = e % P;
        const float2 v = src[(size_t)iy * n + ix];
        const float2 pr = prb[ix * P + iy];
        fr[(off + ix) * PITCH + off + iy] = c * cmul(pr, v);
    }
    __syncthreads();
    const int f = threadIdx.x / T, t = threadIdx.x % T;
    ptfft::fft<DET, -1, T>(fr + f * PITCH, 1, t, tw);  // along the detector row
    ptfft::fft<DET, -1, T>(fr + f, PITCH, t, tw);      // along the detector column
    const float2 ph = scale * phase[fid];
    for (int e = threadIdx.x; e < DET * DET; e += NT) out[e] = cmul(fr[(e / DET) * PITCH + e % DET], ph);
}

template <int DET, int RESID>
__global__ void __launch_bounds__(ptycho_block<DET>(), 1)
    k_ptycho_adj_small(const float2 *__restrict__ g, float2 *__restrict__ psi, const int *__restrict__ corner,
                 const float2 *__restrict__ phase, const float2 *__restrict__ prb, int nz, int n, int nscan,
                 int P, float c, float scale, const float2 *__restrict__ tw, const float *__restrict__ data,
                 float dscale)
{
    constexpr int T = ptycho_fft_threads<DET>(), NT = ptycho_block<DET>(), PITCH = DET + 1;
    extern __shared__ float2 fr[];
    const int th = blockIdx.x;
    float2 *slab = psi + (size_t)th * nz * n;
    for (int e = threadIdx.x; e < nz * n; e += NT) slab[e] = czero();
    __syncthreads();
    const int off = (DET - P) / 2;
    const int f = threadIdx.x / T, t = threadIdx.x % T;
    const float cs = c * scale;
    for (int s = 0; s < nscan; ++s) {
        const int fid = th * nscan + s;
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        if (stx < 0 || sty < 0) continue;
        const float2 ph = phase[fid];
        const float2 *in = g + (size_t)fid * DET * DET;
        for (int e = threadIdx.x; e < DET * DET; e += NT)
            fr[(e / DET) * PITCH + e % DET] = cmulc(ph, resid<RESID>(in[e], data, (size_t)fid * DET * DET + e, dscale));
        __syncthreads();
        ptfft::fft<DET, +1, T>(fr + f * PITCH, 1, t, tw);
        ptfft::fft<DET, +1, T>(fr + f, PITCH, t, tw);
        float2 *dst = slab + (size_t)sty * n + stx;
        for (int e = threadIdx.x; e < P * P; e += NT) {
            const int iy = e / P, ix = e % P;
            const float2 v = cs * cmulc(prb[ix * P + iy], fr[(off + ix) * PITCH + off + iy]);
            float2 *d = dst + (size_t)iy * n + ix;
            *d = *d + v;
        }
        __syncthreads();
    }
}


// ---- register four-step transforms (det >= 16) -----------------------------
template <int DET>
struct PF {
    static constexpr int N2 = DET >= 64 ? 8 : 4;           // threads per line
    static constexpr int N1 = DET / N2;                    // points per thread
    static constexpr int KPT = N1 / N2;                    // k1 values per thread after the exchange
    static constexpr int NT = DET * N2 < 512 ? DET * N2 : 512;  // threads per block
    static constexpr int NG = NT / N2;                     // thread groups
    static constexpr int CPG = DET / NG;                   // lines per group
    static constexpr int P = DET + 8;                      // frame pitch (P = 8 mod 16)
    static constexpr size_t SMEM = (size_t)(DET * P + DET) * sizeof(float2);
};

// frame swizzle: row r, column c live at r * P + (c ^ fswz(r))
template <int DET>
__device__ __forceinline__ int fswz(int r)
{
    return ((r / PF<DET>::KPT) % PF<DET>::N2) * 2;
}

// DFT of one line held as v[m] = x[t + N2 m] by the N2 threads t of a group.
// On return v[j N2 + k2] = X[t KPT + j + N1 k2].  `sc` is the group's
// scratch (DET + 1 complex), `tws` the table exp(-2 pi i m / DET).
template <int DET, int DIR>
__device__ __forceinline__ void line_dft(float2 (&v)[PF<DET>::N1], int t, float2 *sc, const float2 *tws)
{
    using F = PF<DET>;
    ptfft::Dft<F::N1, DIR>::run(v);
#pragma unroll
    for (int k1 = 1; k1 < F::N1; ++k1) {
        float2 w = tws[t * k1];
        if (DIR > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < F::N1; ++k1) sc[t * F::N1 + ((k1 + t * F::KPT) % F::N1)] = v[k1];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < F::KPT; ++j) {
        float2 u[F::N2];
        const int k1 = t * F::KPT + j;
#pragma unroll
        for (int n2 = 0; n2 < F::N2; ++n2) u[n2] = sc[n2 * F::N1 + ((k1 + n2 * F::KPT) % F::N1)];
        ptfft::Dft<F::N2, DIR>::run(u);
#pragma unroll
        for (int k2 = 0; k2 < F::N2; ++k2) v[j * F::N2 + k2] = u[k2];
    }
}

template <int DET, bool SUB = false>
__global__ void __launch_bounds__(PF<DET>::NT, 1)
    k_ptycho_fwd(const float2 *__restrict__ psi, float2 *__restrict__ g, const int *__restrict__ corner,
                 const float2 *__restrict__ phase, const float2 *__restrict__ prbT, int nz, int n, int nscan,
                 int nframes, int P, float scale, const float2 *__restrict__ tw, const int *__restrict__ sid = nullptr)
{
    using F = PF<DET>;
    extern __shared__ float2 sm[];
    float2 *fr = sm;
    float2 *tws = sm + DET * F::P;
    for (int i = threadIdx.x; i < DET; i += F::NT) tws[i] = tw[i];
    const int t = threadIdx.x % F::N2, grp = threadIdx.x / F::N2;
    float2 *sc = fr + grp * (DET + 1);
    const int off = (DET - P) / 2;
    __syncthreads();
    for (int fid = blockIdx.x; fid < nframes; fid += gridDim.x) {
        const int th = fid / nscan;
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        float2 *out = g + (size_t)fid * DET * DET;
        if (stx < 0 || sty < 0) {  // skipped scan: the reference leaves a zero frame
            for (int e = threadIdx.x; e < DET * DET; e += F::NT) out[e] = czero();
            continue;
        }
        const float2 *src = psi + ((size_t)th * nz + sty) * n + stx;
        const float2 *pr = SUB ? prbT + (size_t)sid[fid] * P * P : prbT;  // sub-pixel: the frame's shifted probe
        float2 v[F::CPG][F::N1];
        // along the object row: line = detector column iy, points ix = t + N2 m
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int py = grp + F::NG * c - off;
#pragma unroll
            for (int m = 0; m < F::N1; ++m) {
                const int px = t + F::N2 * m - off;
                float2 val = czero();
                if (py >= 0 && py < P && px >= 0 && px < P)
                    val = cmul(__ldg(&pr[py * P + px]), __ldg(&src[(size_t)py * n + px]));
                v[c][m] = val;
            }
            line_dft<DET, -1>(v[c], t, sc, tws);
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int iy = grp + F::NG * c;
#pragma unroll
            for (int j = 0; j < F::KPT; ++j)
#pragma unroll
                for (int k2 = 0; k2 < F::N2; ++k2) {
                    const int kx = t * F::KPT + j + F::N1 * k2;
                    fr[kx * F::P + (iy ^ fswz<DET>(kx))] = v[c][j * F::N2 + k2];
                }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int kx = grp + F::NG * c;
            const int sw = fswz<DET>(kx);
#pragma unroll
            for (int m = 0; m < F::N1; ++m) v[c][m] = fr[kx * F::P + ((t + F::N2 * m) ^ sw)];
        }
        __syncthreads();
        const float2 ph = scale * phase[fid];
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            line_dft<DET, -1>(v[c], t, sc, tws);
            const int kx = grp + F::NG * c;
#pragma unroll
            for (int k2 = 0; k2 < F::N2; ++k2)
#pragma unroll
                for (int j = 0; j < F::KPT; ++j)
                    out[kx * DET + t * F::KPT + j + F::N1 * k2] = cmul(v[c][j * F::N2 + k2], ph);
        }
        __syncthreads();
    }
}

// grid (parts, ntheta): block (part, angle) owns slab dst[angle][part]
template <int DET, int RESID, bool SUB = false>
__global__ void __launch_bounds__(PF<DET>::NT, 1)
    k_ptycho_adj(const float2 *__restrict__ g, float2 *__restrict__ dst, const int *__restrict__ corner,
                 const float2 *__restrict__ phase, const float2 *__restrict__ prbT, int nz, int n, int nscan,
                 int P, float scale, const float2 *__restrict__ tw, const float *__restrict__ data, float dscale,
                 const int *__restrict__ sid = nullptr)
{
    using F = PF<DET>;
    extern __shared__ float2 sm[];
    float2 *fr = sm;
    float2 *tws = sm + DET * F::P;
    const int part = blockIdx.x, parts = gridDim.x, th = blockIdx.y;
    float2 *slab = dst + ((size_t)th * parts + part) * nz * n;
    for (int i = threadIdx.x; i < DET; i += F::NT) tws[i] = tw[i];
    for (int e = threadIdx.x; e < nz * n; e += F::NT) slab[e] = czero();
    const int t = threadIdx.x % F::N2, grp = threadIdx.x / F::N2;
    float2 *sc = fr + grp * (DET + 1);
    const int off = (DET - P) / 2;
    __syncthreads();
    for (int s = part; s < nscan; s += parts) {
        const int fid = th * nscan + s;
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        if (stx < 0 || sty < 0) continue;
        const float2 ph = phase[fid];
        const float2 *pr = SUB ? prbT + (size_t)sid[fid] * P * P : prbT;
        const float2 *in = g + (size_t)fid * DET * DET;
        float2 v[F::CPG][F::N1];
        // along the detector row: line = kx, points ky = t + N2 m (contiguous)
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int kx = grp + F::NG * c;
#pragma unroll
            for (int m = 0; m < F::N1; ++m) {
                const int e = kx * DET + t + F::N2 * m;
                v[c][m] = scale * cmulc(ph, resid<RESID>(__ldg(&in[e]), data, (size_t)fid * DET * DET + e, dscale));
            }
            line_dft<DET, +1>(v[c], t, sc, tws);
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int kx = grp + F::NG * c;
#pragma unroll
            for (int j = 0; j < F::KPT; ++j)
#pragma unroll
                for (int k2 = 0; k2 < F::N2; ++k2) {
                    const int iy = t * F::KPT + j + F::N1 * k2;
                    fr[iy * F::P + (kx ^ fswz<DET>(iy))] = v[c][j * F::N2 + k2];
                }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int iy = grp + F::NG * c;
            const int sw = fswz<DET>(iy);
#pragma unroll
            for (int m = 0; m < F::N1; ++m) v[c][m] = fr[iy * F::P + ((t + F::N2 * m) ^ sw)];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            line_dft<DET, +1>(v[c], t, sc, tws);
            const int py = grp + F::NG * c - off;
            if (py < 0 || py >= P) continue;
            float2 *row = slab + (size_t)(sty + py) * n + stx;
            float2 cur[F::N1];
#pragma unroll
            for (int k2 = 0; k2 < F::N2; ++k2)
#pragma unroll
                for (int j = 0; j < F::KPT; ++j) {
                    const int px = t * F::KPT + j + F::N1 * k2 - off;
                    cur[j * F::N2 + k2] = (px >= 0 && px < P) ? row[px] : czero();
                }
#pragma unroll
            for (int k2 = 0; k2 < F::N2; ++k2)
#pragma unroll
                for (int j = 0; j < F::KPT; ++j) {
                    const int px = t * F::KPT + j + F::N1 * k2 - off;
                    if (px >= 0 && px < P)
                        row[px] = cur[j * F::N2 + k2] + cmulc(__ldg(&pr[py * P + px]), v[c][j * F::N2 + k2]);
                }
        }
        __syncthreads();
    }
}

// ---- det = 128 ---------------------------------------------------------
// shared memory: the 128 KB exchange buffer alone.  The remaining ~100 KB of
// L1 keeps most of the 128 KB probe table, reread for every frame, resident.
constexpr int P128_SMEM = 128 * 128 * 8;

// The det-128 twiddles a thread needs, w(t k1) for k1 = 0..15, in pairs:
// entry q * 8 + t of the 64-entry float4 table holds w(2q t) and w((2q+1) t)
// (w = exp(-2 pi i / 128); DIR > 0 takes the conjugates).
template <int DIR>
__device__ __forceinline__ void twiddle16(float2 (&v)[16], float4 w, int q)
{
    float2 w0 = make_float2(w.x, w.y), w1 = make_float2(w.z, w.w);
    if (DIR > 0) {
        w0.y = -w0.y;
        w1.y = -w1.y;
    }
    if (q > 0) v[2 * q] = cmul(v[2 * q], w0);
    v[2 * q + 1] = cmul(v[2 * q + 1], w1);
}

// ---- det-128 frames with two shared-memory exchanges --------------------
// B[u][v] = f sum_{r,q} A[r][q] w128^(DIR (u r + v q)) for a 128 x 128 array
// A whose q runs along memory, in three register rounds:
//   R1  thread (q = tid & 127, rt = (tid >> 7) + 4 c, c = 0, 1): 16-point
//       DFTs over m of r = rt + 8 m, times w128^(rt k1)   -> (k1, q, rt)
//   R2  thread (k1 = warp, qb = lane): the 8-point DFT over rt gives
//       u = k1 + 16 k2; the 4-point DFT over qa of q = qb + 32 qa gives v1;
//       times w128^(qb v1) and the frame factor f        -> (v1, u, qb)
//   R3  thread (u = tid & 127, v1 = tid >> 7): the 32-point DFT over qb
//       gives v = v1 + 4 v2.
// R1's lanes load 32 consecutive q (256 B of one row) and R3's lanes hold 32
// consecutive u.  The forward takes A = probe x patch [y][x] and stores
// frame[kx = v][ky = u]; the adjoint takes A = frame[kx][ky] and adds
// pixel [y = v][x = u] into the slab, so both touch 256 consecutive bytes per
// warp access.  Between the rounds the frame goes once through the 128 KB
// buffer ex, as E1[k1][qa][rt][qb] and E2[v1][u][qb]; E2's rows of 32 values
// (256 B) have their 16-byte slots permuted by an XOR with u & 7, so that
// every exchange access of a warp takes the minimum number of shared
// wavefronts (two for 8-byte, four for 16-byte accesses).
__device__ __forceinline__ int e1_at(int k1, int qa, int rt, int qb) { return ((k1 * 4 + qa) * 8 + rt) * 32 + qb; }
__device__ __forceinline__ int e2_at(int v1, int u, int qb)
{
    return (v1 * 128 + u) * 32 + 2 * ((qb >> 1) ^ (u & 7)) + (qb & 1);
}

// R1 of one frame: v[c][m] holds A[rt + 8 m][q], rt = (tid >> 7) + 4 c;
// transformed and written to E1.  The caller synchronises before and after.
// tw4 is twiddle16's pair table; rt is the same across a warp, so its
// loads are broadcasts.
template <int DIR>
__device__ __forceinline__ void frame_r1(float2 (&v)[2][16], float2 *ex, const float4 *__restrict__ tw4)
{
    const int q = threadIdx.x & 127;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        const int rt = (threadIdx.x >> 7) + 4 * c;
        ptfft::Dft<16, DIR>::run(v[c]);
#pragma unroll
        for (int k = 0; k < 8; ++k) twiddle16<DIR>(v[c], __ldg(&tw4[k * 8 + rt]), k);
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) ex[e1_at(k1, q >> 5, rt, q & 31)] = v[c][k1];
    }
}

// R2 of one frame for thread (k1 = warp, qb = lane): reads E1, synchronises
// (E1 fully read), transforms, and writes E2.  The twiddles w128^(qb j)
// (j = 1..3, in direction DIR; w128[m] = exp(-2 pi i m / 128)) times the
// frame factor f, and f itself for j = 0: the factor rides on the twiddles.
template <int DIR>
__device__ __forceinline__ void frame_r2(float2 *ex, float2 f, const float2 *__restrict__ w128)
{
    const int k1 = threadIdx.x >> 5, qb = threadIdx.x & 31;
    float2 rw1 = __ldg(&w128[qb]), rw2 = __ldg(&w128[2 * qb]), rw3 = __ldg(&w128[3 * qb]);
    if (DIR > 0) {
        rw1.y = -rw1.y;
        rw2.y = -rw2.y;
        rw3.y = -rw3.y;
    }
    float2 a[4][8];
#pragma unroll
    for (int qa = 0; qa < 4; ++qa)
#pragma unroll
        for (int rt = 0; rt < 8; ++rt) a[qa][rt] = ex[e1_at(k1, qa, rt, qb)];
    __syncthreads();
#pragma unroll
    for (int qa = 0; qa < 4; ++qa) ptfft::Dft<8, DIR>::run(a[qa]);
    const float2 r1 = cmul(rw1, f), r2 = cmul(rw2, f), r3 = cmul(rw3, f);
#pragma unroll
    for (int k2 = 0; k2 < 8; ++k2) {
        ptfft::dft4<DIR>(a[0][k2], a[1][k2], a[2][k2], a[3][k2]);
        const int u = k1 + 16 * k2;
        ex[e2_at(0, u, qb)] = cmul(a[0][k2], f);
        ex[e2_at(1, u, qb)] = cmul(a[1][k2], r1);
        ex[e2_at(2, u, qb)] = cmul(a[2][k2], r2);
        ex[e2_at(3, u, qb)] = cmul(a[3][k2], r3);
    }
}

// R3's read of E2 for thread (u = tid & 127, v1 = tid >> 7): w[qb], qb = 0..31.
__device__ __forceinline__ void frame_r3_read(float2 (&w)[32], const float2 *ex)
{
    const int u = threadIdx.x & 127, v1 = threadIdx.x >> 7;
    const float4 *e4 = reinterpret_cast<const float4 *>(ex) + (v1 * 128 + u) * 16;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const float4 q = e4[s ^ (u & 7)];
        w[2 * s] = make_float2(q.x, q.y);
        w[2 * s + 1] = make_float2(q.z, q.w);
    }
}

// The forward with two exchanges (see above); grid-stride over frames, one
// resident block per SM.  w128[m] = exp(-2 pi i m / 128).
template <bool FULL, bool SUB = false>
__global__ void __launch_bounds__(512, 1)
    k_ptycho_fwd128(const float2 *__restrict__ psi, float2 *__restrict__ g, const int *__restrict__ corner,
                    const float2 *__restrict__ phase, const float2 *__restrict__ prbT, int nz, int n, int nscan,
                    int nframes, int P, float scale, const float4 *__restrict__ tw4,
                    const float2 *__restrict__ w128, const int *__restrict__ sid = nullptr)
{
    extern __shared__ float4 sm4[];
    float2 *ex = reinterpret_cast<float2 *>(sm4);
    const int q = threadIdx.x & 127, r0 = threadIdx.x >> 7;  // R1: x = q, y = r0 + 4 c + 8 m; R3: ky = q
    const int off = FULL ? 0 : (128 - P) / 2;
    for (int fid = blockIdx.x; fid < nframes; fid += gridDim.x) {
        const int th = fid / nscan;
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        float2 *out = g + (size_t)fid * 128 * 128;
        if (stx < 0 || sty < 0) {
            for (int e = threadIdx.x; e < 128 * 128 / 2; e += 512) reinterpret_cast<float4 *>(out)[e] = make_float4(0, 0, 0, 0);
            continue;
        }
        const float2 *src = psi + ((size_t)th * nz + sty) * n + stx;
        const float2 *pr = SUB ? prbT + (size_t)sid[fid] * P * P : prbT;  // sub-pixel: the frame's shifted probe
        // an opaque per-frame copy of the probe pointer and window offset: the
        // 32 probe addresses and window tests are formed here, not hoisted out
        // of the frame loop into registers
        int offf = off;
        asm volatile("mov.b64 %0, %0;" : "+l"(pr));
        asm volatile("mov.b32 %0, %0;" : "+r"(offf));
        const int PS = FULL ? 128 : P;  // a constant row stride: the probe rows are immediate offsets
        {
            float2 v[2][16];
            const int px = q - offf;
#pragma unroll
            for (int c = 0; c < 2; ++c) {
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int py = r0 + 4 * c + 8 * m - offf;
                    if (FULL) {
                        v[c][m] = cmul(__ldg(&pr[py * PS + px]), __ldg(&src[(size_t)py * n + px]));
                    } else {
                        float2 val = czero();
                        if (py >= 0 && py < P && px >= 0 && px < P)
                            val = cmul(__ldg(&pr[py * PS + px]), __ldg(&src[(size_t)py * n + px]));
                        v[c][m] = val;
                    }
                }
            }
            frame_r1<-1>(v, ex, tw4);
        }
        __syncthreads();
        frame_r2<-1>(ex, scale * phase[fid], w128);
        __syncthreads();
        float2 w[32];
        frame_r3_read(w, ex);
        __syncthreads();  // E2 fully read: the next frame's R1 may write
        ptfft::Dft<32, -1>::run(w);
#pragma unroll
        for (int v2 = 0; v2 < 32; ++v2) __stcs(&out[(r0 + 4 * v2) * 128 + q], w[v2]);  // frame[kx = r0 + 4 v2][ky = q]
    }
}

// Loads of data read once (frames, counts) that do not allocate in L1, so
// that the probe table, reread for every frame, keeps its L1 lines (at
// 256^3 / 384 angles: plain adjoint 4.39 -> 4.24 ms, Poisson residual 5.85
// -> 5.52 ms, Gaussian 6.32 -> 5.99 ms).
__device__ __forceinline__ float2 ld_once(const float2 *p)
{
    float2 r;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];\n" : "=f"(r.x), "=f"(r.y) : "l"(p));
    return r;
}
__device__ __forceinline__ float ld_once(const float *p)
{
    float r;
    asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];\n" : "=f"(r) : "l"(p));
    return r;
}

// Asks for `bytes` (a multiple of 16) at the 16-byte aligned p to be brought
// into L2; no data moves to the SM.
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// The adjoints with two exchanges (see k_ptycho_fwd128).  Object adjoint:
// grid (parts, ntheta), block (part, angle) owns slab dst[angle][part] and
// walks that angle's scans part, part + parts, ...  PROBE (the adjoint with
// respect to the probe, as k_ptycho_adj_probe): grid (blocks, 1), block b
// walks frames b, b + gridDim.x, ... < nframes and accumulates
// conj(psi patch) x frame into its P x P partial dst[b].  RESID forms the
// Poisson / Gaussian residual of each frame value on load.  R3's thread adds
// pixel column x = u, rows y = v1 + 4 v2, so the 32 lanes of a warp touch
// 256 consecutive bytes of one slab (or partial) row whatever the frame's
// column parity.  w128[m] = exp(-2 pi i m / 128).
template <bool FULL, int RESID, bool SUB = false, bool PROBE = false>
__global__ void __launch_bounds__(512, 1)
    k_ptycho_adj128(const float2 *__restrict__ g, float2 *dst, const int *__restrict__ corner,
                    const float2 *__restrict__ phase, const float2 *prbT, int nz, int n, int nscan,
                    int P, float scale, const float4 *__restrict__ tw4, const float2 *__restrict__ w128,
                    const float *__restrict__ data, float dscale, const int *__restrict__ sid = nullptr,
                    const float2 *psi = nullptr, int nframes = 0)
{
    extern __shared__ float4 sm4[];
    float2 *ex = reinterpret_cast<float2 *>(sm4);
    const int part = blockIdx.x, parts = gridDim.x, th0 = blockIdx.y;
    float2 *slab = PROBE ? dst + (size_t)part * P * P : dst + ((size_t)th0 * parts + part) * nz * n;
    for (int e = threadIdx.x; e < (PROBE ? P * P : nz * n); e += 512) slab[e] = czero();
    const int q = threadIdx.x & 127, r0 = threadIdx.x >> 7;  // R1: ky = q, kx = r0 + 4 c + 8 m; R3: x = q
    const int off = FULL ? 0 : (128 - P) / 2;
    const int count = PROBE ? nframes : nscan;
    for (int s = part; s < count; s += parts) {
        const int fid = PROBE ? s : th0 * nscan + s;
        const int th = PROBE ? fid / nscan : th0;
        // the block's next frame (and its counts) into L2 one frame ahead, in
        // 16 KB pieces: its loads then wait on L2 rather than on HBM.  At
        // 256^3 / 384 angles: plain 4.64 -> 4.42 ms, probe adjoint 5.04 ->
        // 4.95 ms; the object adjoint with the residual went 5.89 -> 5.99 ms
        // (Poisson), so it goes without.
        constexpr bool PREFETCH = RESID == 0 || PROBE;
        if (PREFETCH && threadIdx.x < 8 && s + parts < count) {
            const size_t nf = (size_t)fid + parts;
            prefetch_l2(g + (nf * 128 * 128 + threadIdx.x * 2048), 16384);
            if (RESID != 0 && threadIdx.x < 4) prefetch_l2(data + (nf * 128 * 128 + threadIdx.x * 4096), 16384);
        }
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        if (stx < 0 || sty < 0) continue;
        {
            const float2 *in = g + (size_t)fid * 128 * 128;
            const float *din = RESID ? data + (size_t)fid * 128 * 128 : nullptr;
            // all 32 frame values (and counts) are loaded before the first
            // residual: its branches would otherwise hold each later load back
            float2 v[2][16];
            float d[2][16];
#pragma unroll
            for (int c = 0; c < 2; ++c)
#pragma unroll
                for (int m = 0; m < 16; ++m) {
                    const int e = (r0 + 4 * c + 8 * m) * 128 + q;
                    v[c][m] = ld_once(&in[e]);
                    if constexpr (RESID != 0) d[c][m] = ld_once(&din[e]);
                }
            if constexpr (RESID != 0) {
#pragma unroll
                for (int c = 0; c < 2; ++c)
#pragma unroll
                    for (int m = 0; m < 16; ++m) v[c][m] = resid_of<RESID>(v[c][m], d[c][m] * dscale);
            }
            frame_r1<+1>(v, ex, tw4);
        }
        __syncthreads();
        const float2 ph = phase[fid];
        frame_r2<+1>(ex, make_float2(scale * ph.x, -scale * ph.y), w128);
        __syncthreads();
        float2 w[32];
        frame_r3_read(w, ex);
        __syncthreads();  // E2 fully read: the next frame's R1 may write
        ptfft::Dft<32, +1>::run(w);
        // object: slab += conj(probe) x value; probe: partial += conj(psi) x value
        const float2 *mul = PROBE ? psi + ((size_t)th * nz + sty) * n + stx
                                  : (SUB ? prbT + (size_t)sid[fid] * P * P : prbT);  // sub-pixel: the frame's shifted probe
        // an opaque per-frame copy of the multiplier pointer: the 32 row
        // addresses are formed here, not hoisted out of the frame loop into
        // registers; likewise the row window's offset and its 32 tests
        int offf = off;
        asm volatile("mov.b64 %0, %0;" : "+l"(mul));
        asm volatile("mov.b32 %0, %0;" : "+r"(offf));
        const int px = q - offf;
        if (!FULL && (px < 0 || px >= P)) continue;
        float2 *col = PROBE ? slab + px : slab + (size_t)sty * n + stx + px;
        const size_t cs = PROBE ? P : n;                // row stride of col
        const int ms = PROBE ? n : (FULL ? 128 : P);  // row stride of mul (a constant for the probe table)
        // RB rows at a time: their multiplier and slab loads are issued
        // before the first store
        constexpr int RB = 8;
#pragma unroll
        for (int h = 0; h < 32; h += RB) {
            float2 cur[RB], pv[RB];
#pragma unroll
            for (int j = 0; j < RB; ++j) {
                const int py = r0 + 4 * (h + j) - offf;
                const bool ok = FULL || (py >= 0 && py < P);
                pv[j] = ok ? mul[(size_t)py * ms + px] : czero();
                cur[j] = ok ? col[py * cs] : czero();
            }
#pragma unroll
            for (int j = 0; j < RB; ++j) {
                const int py = r0 + 4 * (h + j) - offf;
                if (FULL || (py >= 0 && py < P)) col[py * cs] = cur[j] + cmulc(pv[j], w[h + j]);
            }
        }
    }
}

// out[angle] = sum over parts of dst[angle][part], fixed order
__global__ void k_ptycho_reduce(const float2 *__restrict__ part, float2 *__restrict__ out, size_t slab,
                                int parts, size_t total)
{
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t th = e / slab, i = e % slab;
        const float2 *p = part + th * parts * slab + i;
        float2 acc = p[0];
        for (int k = 1; k < parts; ++k) acc = acc + p[k * slab];
        out[e] = acc;
    }
}

// prbT[iy][ix] = c * prb[ix][iy] (the reference's mul/mula index prb[iy + ix*Nprb])
__global__ void k_probe_t(const float2 *__restrict__ prb, float2 *__restrict__ prbT, int P, float c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * P) return;
    const int iy = i / P, ix = i % P;
    prbT[i] = c * prb[ix * P + iy];
}

// ---- adjoint with respect to the probe (no counterpart in the reference) ----
// The forward is linear in the probe too: with c prbT[py][px] = c prb[px P + py]
// multiplying psi[th][sty + py][stx + px] (ptychofft.cu:58-76, kernels.cuh:
// 243-265), the adjoint maps frames g to
//   gprb[px P + py] = c sum_frames conj(psi[th][sty + py][stx + px]) G[py][px],
// G = scale x inverse DFT of conj(phase) g (the same transform as the object
// adjoint).  Block b walks frames b, b + gridDim.x, ... and accumulates into
// its own P x P partial part[b] (prbT layout); every (py, px) of the window
// belongs to one thread, so no atomics; k_probe_reduce sums the partials in
// block order.  RESID: the frames are the data-term residual of g (as
// k_ptycho_adj).
template <int DET, int RESID>
__global__ void __launch_bounds__(PF<DET>::NT, 1)
    k_ptycho_adj_probe(const float2 *__restrict__ g, float2 *__restrict__ part, const float2 *__restrict__ psi,
                       const int *__restrict__ corner, const float2 *__restrict__ phase, int nz, int n, int nscan,
                       int nframes, int P, float scale, const float2 *__restrict__ tw, const float *__restrict__ data,
                       float dscale)
{
    using F = PF<DET>;
    extern __shared__ float2 sm[];
    float2 *fr = sm;
    float2 *tws = sm + DET * F::P;
    float2 *acc = part + (size_t)blockIdx.x * P * P;
    for (int i = threadIdx.x; i < DET; i += F::NT) tws[i] = tw[i];
    for (int e = threadIdx.x; e < P * P; e += F::NT) acc[e] = czero();
    const int t = threadIdx.x % F::N2, grp = threadIdx.x / F::N2;
    float2 *sc = fr + grp * (DET + 1);
    const int off = (DET - P) / 2;
    __syncthreads();
    for (int fid = blockIdx.x; fid < nframes; fid += gridDim.x) {
        const int th = fid / nscan;
        const int stx = corner[2 * fid], sty = corner[2 * fid + 1];
        if (stx < 0 || sty < 0) continue;
        const float2 ph = phase[fid];
        const float2 *in = g + (size_t)fid * DET * DET;
        float2 v[F::CPG][F::N1];
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int kx = grp + F::NG * c;
#pragma unroll
            for (int m = 0; m < F::N1; ++m) {
                const int e = kx * DET + t + F::N2 * m;
                v[c][m] = scale * cmulc(ph, resid<RESID>(__ldg(&in[e]), data, (size_t)fid * DET * DET + e, dscale));
            }
            line_dft<DET, +1>(v[c], t, sc, tws);
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int kx = grp + F::NG * c;
#pragma unroll
            for (int j = 0; j < F::KPT; ++j)
#pragma unroll
                for (int k2 = 0; k2 < F::N2; ++k2) {
                    const int iy = t * F::KPT + j + F::N1 * k2;
                    fr[iy * F::P + (kx ^ fswz<DET>(iy))] = v[c][j * F::N2 + k2];
                }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            const int iy = grp + F::NG * c;
            const int sw = fswz<DET>(iy);
#pragma unroll
            for (int m = 0; m < F::N1; ++m) v[c][m] = fr[iy * F::P + ((t + F::N2 * m) ^ sw)];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < F::CPG; ++c) {
            line_dft<DET, +1>(v[c], t, sc, tws);
            const int py = grp + F::NG * c - off;
            if (py < 0 || py >= P) continue;
            const float2 *orow = psi + ((size_t)th * nz + sty + py) * n + stx;
            float2 *arow = acc + (size_t)py * P;
#pragma unroll
            for (int k2 = 0; k2 < F::N2; ++k2)
#pragma unroll
                for (int j = 0; j < F::KPT; ++j) {
                    const int px = t * F::KPT + j + F::N1 * k2 - off;
                    if (px >= 0 && px < P) arow[px] = arow[px] + cmulc(__ldg(&orow[px]), v[c][j * F::N2 + k2]);
                }
        }
    }
}

// gprb[px P + py] = c sum_b part[b][py P + px], blocks in order
__global__ void k_probe_reduce(const float2 *__restrict__ part, float2 *__restrict__ gprb, int nblk, int P, float c)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P * P) return;
    float2 s = part[i];
    for (int b = 1; b < nblk; ++b) s = s + part[(size_t)b * P * P + i];
    const int py = i / P, px = i % P;
    gprb[px * P + py] = c * s;
}

}  // namespace

// ---- sub-pixel scan model (no counterpart in the reference) -----------------
// The reference rounds each scan position s to the object grid and multiplies
// the frame by a constant phase (kernels.cuh:306-336), which leaves the
// intensities unchanged.  The sub-pixel model keeps the object on its grid and
// evaluates the probe at the scan's offset instead: the exit wave is
// P(r - d) psi(c + r), c = round(s), d = s - c in [-1/2, 1/2]^2, r the patch
// pixel, with P(r - d) the band-limited (trigonometric) interpolation of the
// probe's samples, separable in x and y:
//   P_d[y][x] = sum_{i,j} D(y - dy - i) P[i][j] D(x - dx - j),
//   D(t) = sin(pi t) / (P tan(pi t / P))  (even P;  P sin(pi t / P) for odd P),
// the Dirichlet kernel whose spectrum is 1 below Nyquist and cos(pi d) at it.
// Offsets are quantised to multiples of 1/quant pixel; one shifted table is
// kept per distinct offset pair and each frame indexes its own.

// tmp[s][i][x] = sum_j prbT[i][j] MxT[kx_s][j][x]   (one thread per (s, i, x))
__global__ void k_probe_shift_x(const float2 *__restrict__ prbT, const float *__restrict__ mxT,
                                const int2 *__restrict__ pairs, float2 *__restrict__ tmp, int P, int npairs)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)npairs * P * P) return;
    const int x = (int)(e % P), i = (int)((e / P) % P), sidx = (int)(e / ((size_t)P * P));
    const float *m = mxT + (size_t)pairs[sidx].x * P * P;
    double re = 0, im = 0;
    for (int j = 0; j < P; ++j) {
        const float2 v = prbT[(size_t)i * P + j];
        const double w = m[(size_t)j * P + x];
        re += w * v.x;
        im += w * v.y;
    }
    tmp[e] = make_float2((float)re, (float)im);
}

// out[s][y][x] = sum_i My[ky_s][y][i] tmp[s][i][x]
__global__ void k_probe_shift_y(const float2 *__restrict__ tmp, const float *__restrict__ my,
                                const int2 *__restrict__ pairs, float2 *__restrict__ out, int P, int npairs)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)npairs * P * P) return;
    const int x = (int)(e % P), y = (int)((e / P) % P), sidx = (int)(e / ((size_t)P * P));
    const float *m = my + (size_t)pairs[sidx].y * P * P + (size_t)y * P;
    const float2 *src = tmp + (size_t)sidx * P * P + x;
    double re = 0, im = 0;
    for (int i = 0; i < P; ++i) {
        const float2 v = src[(size_t)i * P];
        const double w = m[i];
        re += w * v.x;
        im += w * v.y;
    }
    out[e] = make_float2((float)re, (float)im);
}

__global__ void k_fill_one(float2 *__restrict__ a, size_t n)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] = make_float2(1.f, 0.f);
}

struct pt_ptycho {
    int ntheta = 0, nz = 0, n = 0, nscan = 0, det = 0, P = 0, parts = 1;
    int device = -1, nsm = 148;
    bool ready = false;
    float c = 0.f;
    float2 *tw = nullptr, *prb = nullptr, *prbT = nullptr, *phase = nullptr, *partial = nullptr;
    float4 *tw128 = nullptr;  // det = 128: the twiddles in twiddle16's pair layout
    int *corner = nullptr;
    // probe retrieval: a second transposed probe table (forward with a given
    // probe) and one P x P partial per block of the probe adjoint
    float2 *prbT2 = nullptr, *prb_part = nullptr;
    int prb_blocks = 0;
    // sub-pixel scan model (quant > 0): frac = per-frame offsets s - round(s);
    // prbS = one shifted probe table per distinct quantised offset pair (prbT
    // layout), sid = each frame's table, ones = the unit phase the model uses
    float *frac = nullptr;
    float2 *prbS = nullptr, *ones = nullptr;
    int *sid = nullptr;
    int quant = 0, nshift = 0;
    // the tables the kernels take
    const float2 *probe_tab() const { return quant ? prbS : prbT; }
    const float2 *phase_tab() const { return quant ? ones : phase; }
    const int *shift_ids() const { return quant ? sid : nullptr; }
};

namespace {

#define PT_PTYCHO_DETS(X) X(8) X(16) X(32) X(64) X(128)

template <int DET>
int ptycho_attrs()
{
#define PT_ATTR(K, S) PT_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(S)))
    if constexpr (DET < 16) {
        const int s = DET * (DET + 1) * sizeof(float2);
        PT_ATTR(k_ptycho_fwd_small<DET>, s);
        PT_ATTR((k_ptycho_adj_small<DET, 0>), s);
        PT_ATTR((k_ptycho_adj_small<DET, 1>), s);
        PT_ATTR((k_ptycho_adj_small<DET, 2>), s);
    } else {
        const int s = (int)PF<DET>::SMEM;
        PT_ATTR(k_ptycho_fwd<DET>, s);
        PT_ATTR((k_ptycho_adj<DET, 0>), s);
        PT_ATTR((k_ptycho_adj<DET, 1>), s);
        PT_ATTR((k_ptycho_adj<DET, 2>), s);
        PT_ATTR((k_ptycho_adj_probe<DET, 0>), s);
        PT_ATTR((k_ptycho_adj_probe<DET, 1>), s);
        PT_ATTR((k_ptycho_adj_probe<DET, 2>), s);
        PT_ATTR((k_ptycho_fwd<DET, true>), s);
        PT_ATTR((k_ptycho_adj<DET, 0, true>), s);
        PT_ATTR((k_ptycho_adj<DET, 1, true>), s);
        PT_ATTR((k_ptycho_adj<DET, 2, true>), s);
        if constexpr (DET == 128) {
            PT_ATTR((k_ptycho_fwd128<true>), P128_SMEM);
            PT_ATTR((k_ptycho_fwd128<false>), P128_SMEM);
            PT_ATTR((k_ptycho_fwd128<true, true>), P128_SMEM);
            PT_ATTR((k_ptycho_fwd128<false, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 0>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 0>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 0, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 0, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 1>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 1>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 1, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 1, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 2>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 2>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 2, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<false, 2, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 0, false, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 1, false, true>), P128_SMEM);
            PT_ATTR((k_ptycho_adj128<true, 2, false, true>), P128_SMEM);
        }
    }
#undef PT_ATTR
    return PT_OK;
}

template <int DET, int RESID>
int ptycho_adj_launch(pt_ptycho *h, float2 *out, const float2 *in, float scale, const float *data, float dscale,
                      cudaStream_t st)
{
    if constexpr (DET < 16) {
        const size_t s = DET * (DET + 1) * sizeof(float2);
        k_ptycho_adj_small<DET, RESID><<<h->ntheta, ptycho_block<DET>(), s, st>>>(
            in, out, h->corner, h->phase, h->prb, h->nz, h->n, h->nscan, h->P, h->c, scale, h->tw, data, dscale);
        PT_LAUNCHED("k_ptycho_adj_small");
        return PT_OK;
    } else {
        using F = PF<DET>;
        float2 *dst = h->parts > 1 ? h->partial : out;
        const dim3 grid(h->parts, h->ntheta);
        // the det = 128 adjoint (k_ptycho_adj128) for 16-byte aligned frames
        const bool fast128 = DET == 128 && ((uintptr_t)in % 16) == 0 && (RESID == 0 || (uintptr_t)data % 16 == 0);
        // SUB: the sub-pixel model's per-frame probe tables (a separate
        // instantiation, so the reference model's kernels are unchanged)
        auto go = [&](auto sub) {
            constexpr bool S = decltype(sub)::value;
            if (fast128 && h->P == DET)
                k_ptycho_adj128<true, RESID, S><<<grid, 512, P128_SMEM, st>>>(
                    in, dst, h->corner, h->phase_tab(), h->probe_tab(), h->nz, h->n, h->nscan, h->P, scale, h->tw128,
                    h->tw, data, dscale, h->shift_ids());
            else if (fast128)
                k_ptycho_adj128<false, RESID, S><<<grid, 512, P128_SMEM, st>>>(
                    in, dst, h->corner, h->phase_tab(), h->probe_tab(), h->nz, h->n, h->nscan, h->P, scale, h->tw128,
                    h->tw, data, dscale, h->shift_ids());
            else
                k_ptycho_adj<DET, RESID, S><<<grid, F::NT, F::SMEM, st>>>(
                    in, dst, h->corner, h->phase_tab(), h->probe_tab(), h->nz, h->n, h->nscan, h->P, scale, h->tw,
                    data, dscale, h->shift_ids());
        };
        if (h->quant)
            go(std::true_type{});
        else
            go(std::false_type{});
        PT_LAUNCHED("k_ptycho_adj");
        if (h->parts > 1) {
            const size_t slab = (size_t)h->nz * h->n, total = slab * h->ntheta;
            const unsigned blocks = (unsigned)std::min<size_t>((total + 255) / 256, 148 * 16);
            k_ptycho_reduce<<<blocks, 256, 0, st>>>(h->partial, out, slab, h->parts, total);
            PT_LAUNCHED("k_ptycho_reduce");
        }
        return PT_OK;
    }
}

template <int DET>
int ptycho_run(pt_ptycho *h, bool adj, float2 *out, const float2 *in, float scale, cudaStream_t st, int resid_mode,
               const float *data, float dscale)
{
    if (adj) {
        if (resid_mode == 1) return ptycho_adj_launch<DET, 1>(h, out, in, scale, data, dscale, st);
        if (resid_mode == 2) return ptycho_adj_launch<DET, 2>(h, out, in, scale, data, dscale, st);
        return ptycho_adj_launch<DET, 0>(h, out, in, scale, data, dscale, st);
    }
    const int nframes = h->ntheta * h->nscan;
    if constexpr (DET < 16) {
        const size_t s = DET * (DET + 1) * sizeof(float2);
        k_ptycho_fwd_small<DET><<<dim3(h->nscan, h->ntheta), ptycho_block<DET>(), s, st>>>(
            in, out, h->corner, h->phase, h->prb, h->nz, h->n, h->nscan, h->P, h->c, scale, h->tw);
    } else {
        using F = PF<DET>;
        // the det = 128 kernel writes frames with 16-byte stores; one resident
        // block per SM walks the frames (grid-stride), so the grid is one
        // block per SM (1.2 % faster than a block per frame at 256^3)
        const bool fast128 = DET == 128 && ((uintptr_t)out % 16) == 0;
        const int grid128 = std::min(nframes, h->nsm);
        auto go = [&](auto sub) {
            constexpr bool S = decltype(sub)::value;
            if (fast128 && h->P == DET)
                k_ptycho_fwd128<true, S><<<grid128, 512, P128_SMEM, st>>>(
                    in, out, h->corner, h->phase_tab(), h->probe_tab(), h->nz, h->n, h->nscan, nframes, h->P, scale,
                    h->tw128, h->tw, h->shift_ids());
            else if (fast128)
                k_ptycho_fwd128<false, S><<<grid128, 512, P128_SMEM, st>>>(
                    in, out, h->corner, h->phase_tab(), h->probe_tab(), h->nz, h->n, h->nscan, nframes, h->P, scale,
                    h->tw128, h->tw, h->shift_ids());
            else
                k_ptycho_fwd<DET, S><<<nframes, F::NT, F::SMEM, st>>>(in, out, h->corner, h->phase_tab(),
                                                                     h->probe_tab(), h->nz, h->n, h->nscan, nframes,
                                                                     h->P, scale, h->tw, h->shift_ids());
        };
        if (h->quant)
            go(std::true_type{});
        else
            go(std::false_type{});
    }
    PT_LAUNCHED("k_ptycho_fwd");
    return PT_OK;
}

bool det_supported(int d)
{
#define PT_CASE(D) \
    if (d == D) return true;
    PT_PTYCHO_DETS(PT_CASE)
#undef PT_CASE
    return false;
}

int ptycho_set_attrs(int d)
{
#define PT_CASE(D) \
    if (d == D) return ptycho_attrs<D>();
    PT_PTYCHO_DETS(PT_CASE)
#undef PT_CASE
    return PT_ERR_UNSUPPORTED;
}

int ptycho_dispatch(pt_ptycho *h, bool adj, float2 *out, const float2 *in, float scale, cudaStream_t st,
                    int resid_mode = 0, const float *data = nullptr, float dscale = 1.f)
{
#define PT_CASE(D) \
    if (h->det == D) return ptycho_run<D>(h, adj, out, in, scale, st, resid_mode, data, dscale);
    PT_PTYCHO_DETS(PT_CASE)
#undef PT_CASE
    pt::set_error("ptychofft: detector size %d not compiled", h->det);
    return PT_ERR_UNSUPPORTED;
}

template <int DET, int RESID>
int probe_adj_launch(pt_ptycho *h, float2 *gprb, const float2 *in, const float2 *psi, float scale, const float *data,
                     float dscale, cudaStream_t st)
{
    if constexpr (DET < 16) {
        pt::set_error("ptychofft.adj_probe: not compiled for detector %d (16 to 128)", DET);
        return PT_ERR_UNSUPPORTED;
    } else {
        using F = PF<DET>;
        const int nframes = h->ntheta * h->nscan;
        // det 128 with a 128 probe: the two-exchange adjoint in its probe mode;
        // smaller probes keep the generic kernel
        const bool fast128 = DET == 128 && h->P == DET && ((uintptr_t)in % 16) == 0 &&
                             (RESID == 0 || (uintptr_t)data % 16 == 0);
        if (fast128)
            k_ptycho_adj128<true, RESID, false, true><<<h->prb_blocks, 512, P128_SMEM, st>>>(
                in, h->prb_part, h->corner, h->phase, h->prbT, h->nz, h->n, h->nscan, h->P, scale, h->tw128, h->tw,
                data, dscale, nullptr, psi, nframes);
        else
            k_ptycho_adj_probe<DET, RESID><<<h->prb_blocks, F::NT, F::SMEM, st>>>(
                in, h->prb_part, psi, h->corner, h->phase, h->nz, h->n, h->nscan, nframes, h->P, scale, h->tw, data,
                dscale);
        PT_LAUNCHED("k_ptycho_adj_probe");
        k_probe_reduce<<<(h->P * h->P + 255) / 256, 256, 0, st>>>(h->prb_part, gprb, h->prb_blocks, h->P, h->c);
        PT_LAUNCHED("k_probe_reduce");
        return PT_OK;
    }
}

int probe_adj_dispatch(pt_ptycho *h, float2 *gprb, const float2 *in, const float2 *psi, float scale, int resid_mode,
                       const float *data, float dscale, cudaStream_t st)
{
#define PT_CASE(D)                                                                               \
    if (h->det == D) {                                                                           \
        if (resid_mode == 1) return probe_adj_launch<D, 1>(h, gprb, in, psi, scale, data, dscale, st); \
        if (resid_mode == 2) return probe_adj_launch<D, 2>(h, gprb, in, psi, scale, data, dscale, st); \
        return probe_adj_launch<D, 0>(h, gprb, in, psi, scale, data, dscale, st);                \
    }
    PT_PTYCHO_DETS(PT_CASE)
#undef PT_CASE
    pt::set_error("ptychofft: detector size %d not compiled", h->det);
    return PT_ERR_UNSUPPORTED;
}

void ptycho_free(pt_ptycho *h)
{
    void *bufs[] = {h->tw,     h->tw128,  h->prb,  h->prbT, h->phase, h->partial, h->corner,
                    h->prbT2,  h->prb_part, h->frac, h->prbS, h->ones, h->sid};
    for (void *p : bufs)
        if (p) cudaFree(p);
}

// D(t) of the sub-pixel model in double: 1 at multiples of P, exactly 0 at
// the other integers (a zero offset leaves the probe unchanged)
double dirichlet(double t, int P)
{
    if (t == std::floor(t)) return std::fmod(t, (double)P) == 0.0 ? 1.0 : 0.0;
    const double a = M_PI * t / P;
    return (P % 2 == 0) ? std::sin(M_PI * t) / (P * std::tan(a)) : std::sin(M_PI * t) / (P * std::sin(a));
}

void subpixel_free(pt_ptycho *h)
{
    void *bufs[] = {h->prbS, h->ones, h->sid};
    for (void *p : bufs)
        if (p) cudaFree(p);
    h->prbS = h->ones = nullptr;
    h->sid = nullptr;
    h->quant = h->nshift = 0;
}

// Builds the shifted probe tables from the handle's offsets (setobj) and
// probe.  Set-up: allocates, blocks the host.
int subpixel_build(pt_ptycho *h, int quant, cudaStream_t st)
{
    const int nf = h->ntheta * h->nscan, P = h->P;
    std::vector<float> frac(2 * (size_t)nf);
    std::vector<int> corner(2 * (size_t)nf);
    PT_CUDA(cudaMemcpyAsync(frac.data(), h->frac, frac.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaMemcpyAsync(corner.data(), h->corner, corner.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    std::map<int, int> ux, uy;                   // quantised offset -> axis table index
    std::map<std::pair<int, int>, int> up;       // (x index, y index) -> shifted table
    std::vector<int> sid(nf, 0);
    std::vector<int2> pairs;
    auto axis = [](std::map<int, int> &m, int q) {
        auto it = m.find(q);
        if (it != m.end()) return it->second;
        const int k = (int)m.size();
        m.emplace(q, k);
        return k;
    };
    for (int f = 0; f < nf; ++f) {
        if (corner[2 * f] < 0 || corner[2 * f + 1] < 0) continue;   // skipped scan
        const int qx = (int)std::lrint((double)frac[2 * f] * quant), qy = (int)std::lrint((double)frac[2 * f + 1] * quant);
        const int kx = axis(ux, qx), ky = axis(uy, qy);
        auto it = up.find({kx, ky});
        if (it == up.end()) {
            it = up.emplace(std::make_pair(kx, ky), (int)pairs.size()).first;
            pairs.push_back(make_int2(kx, ky));
        }
        sid[f] = it->second;
    }
    if (pairs.empty()) pairs.push_back(make_int2(axis(ux, 0), axis(uy, 0)));   // every scan skipped
    const size_t tab = (size_t)P * P * sizeof(float2);
    if (pairs.size() * tab > ((size_t)1 << 31)) {
        pt::set_error("ptychofft.set_subpixel: %zu distinct offsets need %zu MB of probe tables (limit 2048); "
                      "use a coarser quantisation",
                      pairs.size(), pairs.size() * tab >> 20);
        return PT_ERR_ARG;
    }
    // axis matrices: MxT[k][j][x] = D(x - dx_k - j), My[k][y][i] = D(y - dy_k - i)
    std::vector<float> mx(ux.size() * P * P), my(uy.size() * P * P);
    for (const auto &kv : ux)
        for (int j = 0; j < P; ++j)
            for (int x = 0; x < P; ++x)
                mx[((size_t)kv.second * P + j) * P + x] = (float)dirichlet(x - (double)kv.first / quant - j, P);
    for (const auto &kv : uy)
        for (int y = 0; y < P; ++y)
            for (int i = 0; i < P; ++i)
                my[((size_t)kv.second * P + y) * P + i] = (float)dirichlet(y - (double)kv.first / quant - i, P);
    float *dmx = nullptr, *dmy = nullptr;
    int2 *dpairs = nullptr;
    float2 *tmp = nullptr, *prbS = nullptr, *ones = nullptr;
    int *dsid = nullptr;
    const size_t np = pairs.size();
    bool ok = cudaMalloc((void **)&dmx, mx.size() * sizeof(float)) == cudaSuccess &&
              cudaMalloc((void **)&dmy, my.size() * sizeof(float)) == cudaSuccess &&
              cudaMalloc((void **)&dpairs, np * sizeof(int2)) == cudaSuccess &&
              cudaMalloc((void **)&tmp, np * tab) == cudaSuccess && cudaMalloc((void **)&prbS, np * tab) == cudaSuccess &&
              cudaMalloc((void **)&ones, (size_t)nf * sizeof(float2)) == cudaSuccess &&
              cudaMalloc((void **)&dsid, (size_t)nf * sizeof(int)) == cudaSuccess;
    int rc = PT_OK;
    if (!ok) {
        cudaGetLastError();
        pt::set_error("ptychofft.set_subpixel: device allocation failed");
        rc = PT_ERR_ALLOC;
    }
    if (rc == PT_OK &&
        (cudaMemcpyAsync(dmx, mx.data(), mx.size() * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess ||
         cudaMemcpyAsync(dmy, my.data(), my.size() * sizeof(float), cudaMemcpyHostToDevice, st) != cudaSuccess ||
         cudaMemcpyAsync(dpairs, pairs.data(), np * sizeof(int2), cudaMemcpyHostToDevice, st) != cudaSuccess ||
         cudaMemcpyAsync(dsid, sid.data(), (size_t)nf * sizeof(int), cudaMemcpyHostToDevice, st) != cudaSuccess)) {
        pt::set_error("ptychofft.set_subpixel: table upload failed");
        rc = PT_ERR_CUDA;
    }
    if (rc == PT_OK) {
        const size_t tot = np * P * P;
        const unsigned blocks = (unsigned)((tot + 255) / 256);
        k_probe_shift_x<<<blocks, 256, 0, st>>>(h->prbT, dmx, dpairs, tmp, P, (int)np);
        k_probe_shift_y<<<blocks, 256, 0, st>>>(tmp, dmy, dpairs, prbS, P, (int)np);
        k_fill_one<<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(ones, (size_t)nf);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
            pt::set_error("ptychofft.set_subpixel: table kernels failed");
            rc = PT_ERR_CUDA;
        }
    }
    for (void *q : {(void *)dmx, (void *)dmy, (void *)dpairs, (void *)tmp})
        if (q) cudaFree(q);
    if (rc != PT_OK) {
        for (void *q : {(void *)prbS, (void *)ones, (void *)dsid})
            if (q) cudaFree(q);
        return rc;
    }
    subpixel_free(h);
    h->prbS = prbS;
    h->ones = ones;
    h->sid = dsid;
    h->quant = quant;
    h->nshift = (int)np;
    return PT_OK;
}

}  // namespace

extern "C" int pt_ptycho_create(size_t ntheta, size_t nz, size_t n, size_t ntheta0, size_t nscan, size_t detx,
                                size_t dety, size_t nprb, pt_ptycho **out)
{
    (void)ntheta0;
    pt::clear_error();
    PT_CHECK_ARG(out != nullptr, "ptychofft: null output handle");
    *out = nullptr;
    PT_CHECK_ARG(ntheta >= 1 && nz >= 1 && n >= 1 && nscan >= 1 && nprb >= 1,
                 "ptychofft: sizes must be positive (Ntheta=%zu Nz=%zu N=%zu Nscan=%zu Nprb=%zu)", ntheta, nz, n,
                 nscan, nprb);
    PT_CHECK_ARG(ntheta * nscan < (1u << 31) && ntheta * nz * n < ((size_t)1 << 40), "ptychofft: sizes too large");
    if (detx != dety || !det_supported((int)detx)) {
        pt::set_error("ptychofft: detector %zux%zu not compiled (square 8,16,32,64,128)", detx, dety);
        return PT_ERR_UNSUPPORTED;
    }
    PT_CHECK_ARG(nprb <= detx, "ptychofft: probe %zu larger than detector %zu", nprb, detx);
    PT_CHECK_ARG(nprb <= n && nprb <= nz, "ptychofft: probe %zu larger than the object %zux%zu", nprb, nz, n);
    pt_ptycho *h = new pt_ptycho();
    h->ntheta = (int)ntheta;
    h->nz = (int)nz;
    h->n = (int)n;
    h->nscan = (int)nscan;
    h->det = (int)detx;
    h->P = (int)nprb;
    h->c = 1 / sqrtf(detx * dety);  // kernels.cuh:260
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        delete h;
        pt::set_error("ptychofft: no CUDA device");
        return PT_ERR_CUDA;
    }
    // adjoint split: enough (part, angle) blocks to fill the GPU twice
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    h->nsm = nsm;
    // waves x scans-per-block, with a 3% charge per extra part for the slab traffic;
    // PT_PTYCHO_ADJ_PARTS=<k> overrides the choice (tuning)
    h->parts = 1;
    const char *env_parts = getenv("PT_PTYCHO_ADJ_PARTS");
    if (env_parts && atoi(env_parts) >= 1) {
        h->parts = std::min<int>(atoi(env_parts), (int)nscan);
    } else if (detx >= 16) {
        double best = 1e300;
        for (int p = 1; p <= (int)std::min<size_t>(nscan, 16); ++p) {
            const double waves = std::ceil((double)ntheta * p / nsm);
            const double cost = waves * std::ceil((double)nscan / p) * (1.0 + 0.03 * (p - 1));
            if (cost < best - 1e-9) {
                best = cost;
                h->parts = p;
            }
        }
    }
    bool ok = cudaMalloc((void **)&h->tw, detx * sizeof(float2)) == cudaSuccess &&
              cudaMalloc((void **)&h->tw128, 64 * sizeof(float4)) == cudaSuccess &&
              cudaMalloc((void **)&h->prb, nprb * nprb * sizeof(float2)) == cudaSuccess &&
              cudaMalloc((void **)&h->prbT, nprb * nprb * sizeof(float2)) == cudaSuccess &&
              (h->parts == 1 || cudaMalloc((void **)&h->partial, (size_t)h->parts * ntheta * nz * n * sizeof(float2)) ==
                                    cudaSuccess) &&
              cudaMalloc((void **)&h->phase, ntheta * nscan * sizeof(float2)) == cudaSuccess &&
              cudaMalloc((void **)&h->corner, 2 * ntheta * nscan * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&h->frac, 2 * ntheta * nscan * sizeof(float)) == cudaSuccess &&
              cudaMalloc((void **)&h->prbT2, nprb * nprb * sizeof(float2)) == cudaSuccess;
    // probe adjoint: one block per SM (two below 64x64 detectors), one partial each
    h->prb_blocks = (int)std::min<size_t>((size_t)nsm * (detx >= 64 ? 1 : 2), ntheta * nscan);
    ok = ok && cudaMalloc((void **)&h->prb_part, (size_t)h->prb_blocks * nprb * nprb * sizeof(float2)) == cudaSuccess;
    if (!ok) {
        ptycho_free(h);
        delete h;
        pt::set_error("ptychofft: device allocation failed");
        return PT_ERR_ALLOC;
    }
    std::vector<float2> tw(detx);
    pt_make_twiddles(tw.data(), (int)detx);
    int rc = ptycho_set_attrs((int)detx);
    if (rc == PT_OK && cudaMemcpy(h->tw, tw.data(), detx * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess) {
        pt::set_error("ptychofft: twiddle upload failed");
        rc = PT_ERR_CUDA;
    }
    if (rc == PT_OK && detx == 128) {
        // entry q * 8 + t = (w(2q t), w((2q+1) t)), t k1 <= 105 < 128
        std::vector<float4> tw4(64);
        for (int q = 0; q < 8; ++q)
            for (int t = 0; t < 8; ++t) {
                const float2 a = tw[2 * q * t], b = tw[(2 * q + 1) * t];
                tw4[q * 8 + t] = make_float4(a.x, a.y, b.x, b.y);
            }
        if (cudaMemcpy(h->tw128, tw4.data(), 64 * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess) {
            pt::set_error("ptychofft: twiddle upload failed");
            rc = PT_ERR_CUDA;
        }
    }
    if (rc != PT_OK) {
        ptycho_free(h);
        delete h;
        return rc;
    }
    *out = h;
    return PT_OK;
}

extern "C" int pt_ptycho_destroy(pt_ptycho *h)
{
    pt::clear_error();
    if (!h) return PT_OK;
    ptycho_free(h);
    delete h;
    return PT_OK;
}

extern "C" int pt_ptycho_setobj(pt_ptycho *h, const float *scan, const void *prb, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "ptychofft.setobj: null handle");
    PT_CHECK_ARG(scan != nullptr && prb != nullptr, "ptychofft.setobj: null scan or probe");
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CHECK_ARG(dev == h->device, "ptychofft handle belongs to device %d, current device is %d", h->device, dev);
    cudaStream_t st = (cudaStream_t)stream;
    const int nf = h->ntheta * h->nscan;
    h->ready = false;
    PT_CUDA(cudaMemcpyAsync(h->prb, prb, (size_t)h->P * h->P * sizeof(float2), cudaMemcpyDefault, st));
    k_ptycho_tables<<<(nf + 255) / 256, 256, 0, st>>>(scan, h->corner, h->phase, h->frac, nf);
    PT_LAUNCHED("k_ptycho_tables");
    k_probe_t<<<(h->P * h->P + 255) / 256, 256, 0, st>>>(h->prb, h->prbT, h->P, h->c);
    PT_LAUNCHED("k_probe_t");
    std::vector<int> corner(2 * (size_t)nf);
    PT_CUDA(cudaMemcpyAsync(corner.data(), h->corner, corner.size() * sizeof(int), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < nf; ++i) {
        const int x = corner[2 * i], y = corner[2 * i + 1];
        if (x < 0 || y < 0) continue;  // sentinel: scan skipped
        if (x + h->P > h->n || y + h->P > h->nz) {
            pt::set_error("ptychofft.setobj: scan %d of angle %d at (%d,%d) puts the %dx%d probe outside the "
                          "%dx%d object",
                          i % h->nscan, i / h->nscan, x, y, h->P, h->P, h->nz, h->n);
            return PT_ERR_ARG;
        }
    }
    h->ready = true;
    if (h->quant) {   // new offsets or probe: new shifted tables (on failure the model is switched off)
        const int rc = subpixel_build(h, h->quant, st);
        if (rc != PT_OK) subpixel_free(h);
        return rc;
    }
    return PT_OK;
}

namespace {
int ptycho_call(pt_ptycho *h, bool adj, void *out, const void *in, float scale, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "ptychofft: null handle");
    PT_CHECK_ARG(out != nullptr && in != nullptr, "ptychofft.%s: null array pointer", adj ? "adj" : "fwd");
    if (!h->ready) {
        pt::set_error("ptychofft.%s: setobj(scan, prb) has not been called", adj ? "adj" : "fwd");
        return PT_ERR_STATE;
    }
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CHECK_ARG(dev == h->device, "ptychofft handle belongs to device %d, current device is %d", h->device, dev);
    return ptycho_dispatch(h, adj, (float2 *)out, (const float2 *)in, scale, (cudaStream_t)stream);
}
}  // namespace

extern "C" int pt_ptycho_fwd(pt_ptycho *h, void *g, const void *f, void *stream)
{
    return ptycho_call(h, false, g, f, 1.0f, stream);
}
// ---- autotuner: the adjoint's angle split ---------------------------------
// Times the object adjoint (the CG's dominant kernel) for each candidate
// number of parts per angle and keeps the fastest.  Setup-time: allocates the
// partial slabs of each candidate, blocks the host.
extern "C" int pt_ptycho_autotune(pt_ptycho *h, void *f, const void *g, int trials, int *parts_out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && f && g && trials >= 1, "ptychofft.autotune: bad arguments");
    if (h->det < 16) {   // the small-detector kernel has no angle split
        if (parts_out) *parts_out = h->parts;
        return PT_OK;
    }
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    PT_CUDA(cudaEventCreate(&e0));
    PT_CUDA(cudaEventCreate(&e1));
    const int cands[] = {1, 2, 3, 4, 6, 8, 12, 16};
    int best_p = h->parts;
    float best_t = 1e30f;
    int rc = PT_OK;
    for (int p : cands) {
        if (p > h->nscan) break;
        if (h->partial) {
            cudaFree(h->partial);
            h->partial = nullptr;
        }
        h->parts = p;
        if (p > 1 && cudaMalloc((void **)&h->partial, (size_t)p * h->ntheta * h->nz * h->n * sizeof(float2)) !=
                         cudaSuccess) {
            cudaGetLastError();
            h->parts = 1;
            continue;   // this split does not fit: skip it
        }
        std::vector<float> ts;
        for (int k = 0; k <= trials && rc == PT_OK; ++k) {   // the first run warms up
            cudaEventRecord(e0, st);
            rc = pt_ptycho_adj(h, f, g, stream);
            cudaEventRecord(e1, st);
            if (rc == PT_OK && cudaEventSynchronize(e1) == cudaSuccess && k > 0) {
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ts.push_back(ms);
            }
        }
        if (rc != PT_OK) break;
        std::sort(ts.begin(), ts.end());
        const float med = ts[ts.size() / 2];
        if (med < best_t) {
            best_t = med;
            best_p = p;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (h->partial) {
        cudaFree(h->partial);
        h->partial = nullptr;
    }
    h->parts = best_p;
    if (best_p > 1 &&
        cudaMalloc((void **)&h->partial, (size_t)best_p * h->ntheta * h->nz * h->n * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        h->parts = 1;
        pt::set_error("ptychofft.autotune: the chosen split's slabs could not be allocated");
        return PT_ERR_ALLOC;
    }
    if (parts_out) *parts_out = h->parts;
    return rc;
}

extern "C" int pt_ptycho_set_parts(pt_ptycho *h, int parts)
{
    pt::clear_error();
    PT_CHECK_ARG(h && parts >= 1 && (size_t)parts <= h->nscan, "ptychofft.set_parts: parts must be in [1, nscan]");
    if (h->det < 16) {
        PT_CHECK_ARG(parts == h->parts, "ptychofft.set_parts: the small-detector kernel has no angle split");
        return PT_OK;
    }
    if (h->partial) {
        cudaFree(h->partial);
        h->partial = nullptr;
    }
    h->parts = parts;
    if (parts > 1 &&
        cudaMalloc((void **)&h->partial, (size_t)parts * h->ntheta * h->nz * h->n * sizeof(float2)) != cudaSuccess) {
        cudaGetLastError();
        h->parts = 1;
        pt::set_error("ptychofft.set_parts: the split's slabs could not be allocated");
        return PT_ERR_ALLOC;
    }
    return PT_OK;
}

extern "C" int pt_ptycho_get_parts(const pt_ptycho *h, int *parts)
{
    pt::clear_error();
    PT_CHECK_ARG(h && parts, "ptychofft: null pointer");
    *parts = h->parts;
    return PT_OK;
}

extern "C" int pt_ptycho_adj(pt_ptycho *h, void *f, const void *g, void *stream)
{
    return ptycho_call(h, true, f, g, 1.0f, stream);
}
extern "C" int pt_ptycho_fwd_scaled(pt_ptycho *h, void *g, const void *f, float scale, void *stream)
{
    return ptycho_call(h, false, g, f, scale, stream);
}
extern "C" int pt_ptycho_adj_scaled(pt_ptycho *h, void *f, const void *g, float scale, void *stream)
{
    return ptycho_call(h, true, f, g, scale, stream);
}

extern "C" int pt_ptycho_adj_resid(pt_ptycho *h, void *f, const void *fpsi, const float *data, float dscale,
                                   int model, float scale, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "ptychofft: null handle");
    PT_CHECK_ARG(f != nullptr && fpsi != nullptr && data != nullptr, "ptychofft.adj_resid: null array pointer");
    PT_CHECK_ARG(model == 0 || model == 1, "ptychofft.adj_resid: model 0 (poisson) or 1 (gaussian)");
    if (!h->ready) {
        pt::set_error("ptychofft.adj_resid: setobj(scan, prb) has not been called");
        return PT_ERR_STATE;
    }
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CHECK_ARG(dev == h->device, "ptychofft handle belongs to device %d, current device is %d", h->device, dev);
    return ptycho_dispatch(h, true, (float2 *)f, (const float2 *)fpsi, scale, (cudaStream_t)stream, model + 1, data,
                           dscale);
}

// ---- probe retrieval (no counterpart in the reference) -----------------------
namespace {
int probe_checks(pt_ptycho *h, const char *what)
{
    PT_CHECK_ARG(h != nullptr, "ptychofft.%s: null handle", what);
    if (!h->ready) {
        pt::set_error("ptychofft.%s: setobj(scan, prb) has not been called", what);
        return PT_ERR_STATE;
    }
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CHECK_ARG(dev == h->device, "ptychofft handle belongs to device %d, current device is %d", h->device, dev);
    if (h->quant) {
        pt::set_error("ptychofft.%s: probe retrieval is not available with the sub-pixel scan model", what);
        return PT_ERR_STATE;
    }
    return PT_OK;
}
}  // namespace

extern "C" int pt_ptycho_adj_probe(pt_ptycho *h, void *gprb, const void *g, const void *psi, float scale,
                                   void *stream)
{
    pt::clear_error();
    const int rc = probe_checks(h, "adj_probe");
    if (rc != PT_OK) return rc;
    PT_CHECK_ARG(gprb && g && psi, "ptychofft.adj_probe: null array pointer");
    return probe_adj_dispatch(h, (float2 *)gprb, (const float2 *)g, (const float2 *)psi, scale, 0, nullptr, 1.f,
                              (cudaStream_t)stream);
}

extern "C" int pt_ptycho_adj_probe_resid(pt_ptycho *h, void *gprb, const void *psi, const void *fpsi,
                                         const float *data, float dscale, int model, float scale, void *stream)
{
    pt::clear_error();
    const int rc = probe_checks(h, "adj_probe_resid");
    if (rc != PT_OK) return rc;
    PT_CHECK_ARG(gprb && psi && fpsi && data, "ptychofft.adj_probe_resid: null array pointer");
    PT_CHECK_ARG(model == 0 || model == 1, "ptychofft.adj_probe_resid: model 0 (poisson) or 1 (gaussian)");
    return probe_adj_dispatch(h, (float2 *)gprb, (const float2 *)fpsi, (const float2 *)psi, scale, model + 1, data,
                              dscale, (cudaStream_t)stream);
}

extern "C" int pt_ptycho_fwd_probe(pt_ptycho *h, void *g, const void *psi, const void *prb, float scale,
                                   void *stream)
{
    pt::clear_error();
    const int rc = probe_checks(h, "fwd_probe");
    if (rc != PT_OK) return rc;
    PT_CHECK_ARG(g && psi && prb, "ptychofft.fwd_probe: null array pointer");
    cudaStream_t st = (cudaStream_t)stream;
    k_probe_t<<<(h->P * h->P + 255) / 256, 256, 0, st>>>((const float2 *)prb, h->prbT2, h->P, h->c);
    PT_LAUNCHED("k_probe_t");
    // the forward kernels read the handle's table: point it at this probe for one launch
    float2 *own = h->prbT;
    h->prbT = h->prbT2;
    const int rc2 = ptycho_dispatch(h, false, (float2 *)g, (const float2 *)psi, scale, st);
    h->prbT = own;
    return rc2;
}

extern "C" int pt_ptycho_set_subpixel(pt_ptycho *h, int quant, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "ptychofft.set_subpixel: null handle");
    PT_CHECK_ARG(quant >= 0 && quant <= 65536, "ptychofft.set_subpixel: quant must be in [0, 65536] (0: off)");
    if (quant == 0) {
        subpixel_free(h);
        return PT_OK;
    }
    if (h->det < 16) {
        pt::set_error("ptychofft.set_subpixel: not compiled for detector %d (16 to 128)", h->det);
        return PT_ERR_UNSUPPORTED;
    }
    if (!h->ready) {
        pt::set_error("ptychofft.set_subpixel: setobj(scan, prb) has not been called");
        return PT_ERR_STATE;
    }
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    PT_CHECK_ARG(dev == h->device, "ptychofft handle belongs to device %d, current device is %d", h->device, dev);
    return subpixel_build(h, quant, (cudaStream_t)stream);
}

extern "C" int pt_ptycho_get_subpixel(const pt_ptycho *h, int *quant, int *ntables)
{
    pt::clear_error();
    PT_CHECK_ARG(h && quant && ntables, "ptychofft.get_subpixel: null pointer");
    *quant = h->quant;
    *ntables = h->nshift;
    return PT_OK;
}
