// USFFT Radon transform (tomography operator) for sm_100a.
//
// Replaces class radonusfft of the reference (src/cuda/radonusfft.cu:1-144,
// kernels src/include/kernels.cuh:5-216).  Same mathematics, different
// machinery:
//
//  forward  R f   (radonusfft.cu:54-92)
//    K1 k_fwd_rows    pad2 edge replication + circ mask + deapodisation 1/phi
//                     + centring sign, zero-pad to 2N, row FFT (the N rows
//                     that are non-zero)                       [smem FFT]
//    K2 k_fwd_cols    column FFT of length 2N (zero rows implicit) with the
//                     post-FFT centring sign folded in          [smem FFT]
//    K3a k_fwd_gather_pts  Gaussian-kernel gather at the polar points
//                     (kernels.cuh:97-126), one 8-slice lane group per point
//    K3b k_fwd_lines  1-D centred inverse FFT along the detector, crop n of N
//  adjoint  R* g  (radonusfft.cu:94-139)
//    A1 k_adj_lines     edge-replicating pad, centred 1-D FFT, written for all
//                       slices as lines[point][slice]
//    A2 k_adj_colgather one block per (grid column, 16 slices): every cell of
//                       the column sums, in a fixed order, w * g over the polar
//                       points whose kernel window covers it (cell -> (point,
//                       weight) lists built once at setobj; no float atomics,
//                       no halo, no fold), then the column inverse FFT runs in
//                       the same block and only the n rows that survive the
//                       final crop are written
//    A4 k_adj_rows      row inverse FFT + centring sign + 1/phi + circ + crop
//
// The forward processes slices in chunks of ZC = 8 with slice-minor
// intermediates ([..][ZC]) so every gather tap and every row of the column
// kernel is a contiguous 64-byte segment, and a chunk's intermediates
// (N*2N + (2N)^2 complex per slice) stay well inside L2.  The adjoint keeps
// slice-minor full-volume buffers ([..][nzp], nzp = nz rounded up to 16).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "pt_common.cuh"
#include "pt_fft.cuh"

namespace {

constexpr int ZC = 8;   // slices per chunk (slice-minor lanes)
constexpr int RSETS = 4;   // forward chunk buffer sets (chunks in flight at most)
constexpr int CK = 2;   // grid columns per block in the column kernels
constexpr double PI_REF = 3.1415926535;  // kernels.cuh:1

template <int L>
constexpr int fft_threads() { return L >= 1024 ? 64 : 32; }

// circ, kernels.cuh:160-172 (r = 1.0f/N); evaluated without FMA contraction so
// that it equals the float32 expression (4x*x + 4y*y) < 1 - r exactly.
__device__ __forceinline__ float circ_keep(int tx, int ty, int N)
{
    const float x = (float)(tx - N / 2) / (float)N;
    const float y = (float)(ty - N / 2) / (float)N;
    const float lhs = __fadd_rn(__fmul_rn(__fmul_rn(4.f, x), x), __fmul_rn(__fmul_rn(4.f, y), y));
    const float r = 1.0f / (float)N;
    return lhs < 1.f - r ? 1.f : 0.f;
}

// phi, kernels.cuh:12 and :23 (same expression as the reference)
__device__ __forceinline__ float deapod(int tx, int ty, int N, float mu)
{
    return __expf(-mu * (tx - N / 2) * (tx - N / 2) - mu * (ty - N / 2) * (ty - N / 2));
}

// fac[ty][tx] = circ / phi / (4 N^2) on the N x N padded slice, the factor that
// unpaddivphi / divphi and circ apply (kernels.cuh:5-37, 160-172), evaluated once
// per handle with the expressions above; the row passes multiply by it.
__global__ void k_deap_table(float *__restrict__ fac, int N, float mu)
{
    const int tx = blockIdx.x * blockDim.x + threadIdx.x, ty = blockIdx.y;
    if (tx >= N) return;
    const float den = (float)(4 * N * N);
    fac[(size_t)ty * N + tx] = circ_keep(tx, ty, N) / deapod(tx, ty, N, mu) / den;
}

__device__ __forceinline__ int wrapG(int c, int G) { return c < 0 ? c + G : (c >= G ? c - G : c); }

// ---- geometry: takexy, kernels.cuh:84-95 (identical expression) -----------
__global__ void k_takexy(float *x, float *y, const float *theta, int N, int ntheta)
{
    const int tx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ty = blockIdx.y;
    if (tx >= N || ty >= ntheta) return;
    float xv = (tx - N / 2) / (float)N * __cosf(theta[ty]);
    float yv = -(tx - N / 2) / (float)N * __sinf(theta[ty]);
    if (xv >= 0.5f) xv = 0.5f - 1e-5;
    if (yv >= 0.5f) yv = 0.5f - 1e-5;
    x[tx + ty * N] = xv;
    y[tx + ty * N] = yv;
}

// ---- K1: pad2 + circ + divphi + fftshiftc + row FFT ------------------------
template <int G>
__global__ void __launch_bounds__(ZC *fft_threads<G>())
    k_fwd_rows(const float2 *__restrict__ u, float2 *__restrict__ rbuf, int nz, int z0,
               const float *__restrict__ fac, const float2 *__restrict__ tw)
{
    // the block's ZC slices are interleaved transforms: shared row X holds
    // element X of every slice (ptfft::fft_iq), so the output is a straight
    // copy into the slice-minor row buffer
    constexpr int T = fft_threads<G>(), N = G / 2, n = G / 3;
    constexpr int c0 = N / 6, c1 = 5 * N / 6 - 1;
    extern __shared__ float2 sm[];
    const int y = blockIdx.x;
    const int q = threadIdx.x % ZC, b = threadIdx.x / ZC;
    const int z = z0 + q;
    const int sr = min(max(y, c0), c1) - c0;
    const int Y = y + N / 2;
    for (int X = b; X < G; X += T) {
        float2 v = czero();
        const int tx = X - N / 2;
        if (tx >= 0 && tx < N && z < nz) {
            const int sc = min(max(tx, c0), c1) - c0;
            v = __ldg(&fac[(size_t)y * N + tx]) * u[((size_t)z * n + sr) * n + sc];
            if ((X + Y) & 1) v = -1.f * v;
        }
        sm[X * ZC + q] = v;
    }
    __syncthreads();
    ptfft::fft_iq<G, -1, T, ZC>(sm, q, b, tw);
    float2 *dst = rbuf + (size_t)y * G * ZC;
    for (int e = threadIdx.x; e < G * ZC; e += blockDim.x) dst[e] = sm[e];
}

// The forward's Fourier grid carries a halo, like the reference's (G+2M)^2
// grid (radonusfft.cu:16, wrap in kernels.cuh:50-65): rows 0..GH_ROWS-1 are
// repeated after row G-1 and column pairs 0..GH_PAIRS-1 after pair G/2-1, so
// every gather window is a plain rectangle (no index wraps) addressed from one
// base pointer.  Layout [G + GH_ROWS][G/2 + GH_PAIRS][ZC][2].
constexpr int GH_ROWS = 14;   // 2M for the largest compiled M (7)
constexpr int GH_PAIRS = 8;   // (2M + 2) / 2 column pairs for M = 7

// ---- K2: column FFT of the 2N grid, centring sign folded in ----------------
// The block's CK columns x ZC slices are NF interleaved transforms: shared
// row i holds element i of all NF (column c, slice z at c * ZC + z), so the
// input rows (one 128-byte line of the row-FFT buffer per y) and the output
// rows (one 128-byte line of the grid per ky) are straight copies, and the
// passes (ptfft::fft_iq) are free of bank conflicts.
template <int G>
__global__ void __launch_bounds__(CK *ZC *fft_threads<G>())
    k_fwd_cols(const float2 *__restrict__ rbuf, float2 *__restrict__ fg, const float2 *__restrict__ tw)
{
    constexpr int T = fft_threads<G>(), N = G / 2, NF = CK * ZC;
    extern __shared__ float2 sm[];
    const int kx0 = blockIdx.x * CK;
    const int q = threadIdx.x % NF, b = threadIdx.x / NF;
    for (int e = threadIdx.x; e < N * NF; e += blockDim.x) {
        const int y = e / NF, r = e % NF;
        sm[(N / 2 + y) * NF + r] = rbuf[((size_t)y * G + kx0) * ZC + r];
    }
    for (int e = threadIdx.x; e < N * NF; e += blockDim.x) {
        const int i = e / NF, r = e % NF;
        sm[(i < N / 2 ? i : i + N) * NF + r] = czero();
    }
    __syncthreads();
    ptfft::fft_iq<G, -1, T, NF>(sm, q, b, tw);
    // column-pair layout [ky][kx/2][z][kx&1]: one 128-byte line per (ky, pair),
    // plus the halo copies (rows < GH_ROWS again at G + ky, pairs < GH_PAIRS
    // again at G/2 + pair)
    static_assert(CK == 2, "the grid layout pairs two columns");
    constexpr int PS = G / 2 + GH_PAIRS;
    const int pr = kx0 / 2;
    for (int e = threadIdx.x; e < (G + GH_ROWS) * NF; e += blockDim.x) {
        const int kyh = e / NF, r = e % NF;
        const int ky = kyh < G ? kyh : kyh - G;
        const int z = r >> 1, c = r & 1;
        const int kx = kx0 + c;
        float2 v = sm[ky * NF + c * ZC + z];
        if ((kx + ky) & 1) v = -1.f * v;
        fg[((size_t)kyh * PS + pr) * (2 * ZC) + r] = v;
        if (pr < GH_PAIRS) fg[((size_t)kyh * PS + G / 2 + pr) * (2 * ZC) + r] = v;
    }
}

// ---- K3a: gather only, many blocks --------------------------------------------
// grid (ceil(N / GPB), ntheta); block = GPB points x ZC slice lanes.  The grid
// is in column-pair layout, so a lane reads its slice's value at two
// neighbouring window columns with one 16-byte load (the point's 8 lanes read
// one 128-byte line).  The window's 15 columns are covered by 8 column pairs;
// the one column outside the window gets weight 0.  Writes the gathered,
// 1/N- and fftshift1c-scaled samples to lines[(theta N + k) ZC + z].
// Points are visited in the order of `perm` (built at setobj): sorted by the
// 16 x 16-cell grid tile their window starts in, so the 32 points of a block
// read overlapping windows and most taps hit L1.  The order changes no
// arithmetic: every point is gathered by one group of 8 lanes as before.
constexpr int GPB = 32;
constexpr int GTILE = 16;   // grid cells per tile edge of the visiting order
template <int N, int M>
__global__ void __launch_bounds__(GPB *ZC, 3)
    k_fwd_gather_pts(const float2 *__restrict__ fg, float2 *__restrict__ lines, const float *__restrict__ xt,
                     const float *__restrict__ yt, float a, float pre, const float4 *__restrict__ ptab, int npts)
{
    constexpr int G = 2 * N, W = 2 * M + 1, NP = (W + 2) / 2;  // column pairs covering the window
    const int lane = threadIdx.x % ZC;
    const int pi = blockIdx.x * GPB + threadIdx.x / ZC;
    if (pi >= npts) return;
    const float4 q = __ldg(&ptab[pi]);   // (x, y, point index) in visiting order
    const int p = __float_as_int(q.z);
    const int th = p / N, k = p % N;
    const float x0 = q.x, y0 = q.y;
    // x0, y0 in [-1/2, 1/2) (validated at setobj); clamp keeps reads in bounds
    const int fx = min(max((int)floorf((float)G * x0), -N), N - 1);
    const int fy = min(max((int)floorf((float)G * y0), -N), N - 1);
    const int c0 = wrapG(N + fx - M, G);  // first window column
    const int odd = c0 & 1;               // window starts in the second column of a pair
    float2 wxp[NP];                       // weights of the two columns of each pair
    float wy[W];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
        float w2[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i0 = 2 * j + h - odd;
            const float w0 = (float)(fx - M + i0) / (float)G - x0;
            w2[h] = (i0 >= 0 && i0 < W) ? __expf(-a * (w0 * w0)) : 0.f;
        }
        wxp[j] = make_float2(w2[0], w2[1]);
    }
#pragma unroll
    for (int i = 0; i < W; ++i) {
        const float w1 = (float)(fy - M + i) / (float)G - y0;
        wy[i] = __expf(-a * (w1 * w1));
    }
    const int p0 = (c0 - odd) / 2;  // first column pair
    constexpr int PS = G / 2 + GH_PAIRS;
    static_assert(NP <= GH_PAIRS + 1 && 2 * M <= GH_ROWS, "the grid halo must cover the window");
    // window rows r0 .. r0 + 2M and pairs p0 .. p0 + NP - 1 lie inside the haloed grid
    const float4 *base = reinterpret_cast<const float4 *>(fg) + ((size_t)wrapG(N + fy - M, G) * PS + p0) * ZC + lane;
    float2 acc = czero();
#pragma unroll
    for (int i1 = 0; i1 < W; ++i1) {
        const float4 *rowp = base + (size_t)i1 * PS * ZC;
        float2 rs = czero();
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            const float4 v = __ldg(rowp + j * ZC);
            rs.x = fmaf(wxp[j].x, v.x, rs.x);
            rs.y = fmaf(wxp[j].x, v.y, rs.y);
            rs.x = fmaf(wxp[j].y, v.z, rs.x);
            rs.y = fmaf(wxp[j].y, v.w, rs.y);
        }
        acc.x = fmaf(wy[i1], rs.x, acc.x);
        acc.y = fmaf(wy[i1], rs.y, acc.y);
    }
    lines[((size_t)th * N + k) * ZC + lane] = ((k & 1) ? pre : -pre) * acc;
}

// The same gather with the grid staged in shared memory.  Points were sorted
// at setobj by the 16 x 16-cell tile of their window origin; a block takes a
// chunk of at most TCH points of one tile, loads the part of the haloed grid
// that their windows cover (rows ty0 .. ty0 + 16 + 2M - 1, column pairs
// tx0/2 .. tx0/2 + 7 + NP - 1, clipped to the haloed grid) once, and gathers
// from there.  Weights, loads and the order of the sums are those of
// k_fwd_gather_pts, so the results are bit-identical.
constexpr int TCH = 128;   // points per block of the tiled gather
template <int M>
constexpr int tile_rows() { return GTILE + 2 * M; }
template <int M>
constexpr int tile_pairs() { return (GTILE - 2) / 2 + (2 * M + 3) / 2; }
template <int M>
constexpr size_t tile_smem() { return (size_t)tile_rows<M>() * tile_pairs<M>() * ZC * sizeof(float4); }

// The gather of one chunk's points from its staged tile (both tiled kernels).
// Each thread's next point is loaded before the current one is gathered.
template <int N, int M>
__device__ __forceinline__ void tile_gather(const float4 *__restrict__ tsm, int4 ch, int ty0, int px0,
                                            float2 *__restrict__ lines, float a, float pre,
                                            const float4 *__restrict__ ptab)
{
    constexpr int G = 2 * N, W = 2 * M + 1, NP = (W + 2) / 2;
    constexpr int TP = tile_pairs<M>();
    const int lane = threadIdx.x % ZC;
    int t = threadIdx.x / ZC;
    float4 nq = t < ch.w ? __ldg(&ptab[ch.z + t]) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (; t < ch.w; t += GPB) {
        const float4 q = nq;
        if (t + GPB < ch.w) nq = __ldg(&ptab[ch.z + t + GPB]);
        const int p = __float_as_int(q.z);
        const int th = p / N, k = p % N;
        const float x0 = q.x, y0 = q.y;
        const int fx = min(max((int)floorf((float)G * x0), -N), N - 1);
        const int fy = min(max((int)floorf((float)G * y0), -N), N - 1);
        const int c0 = wrapG(N + fx - M, G);
        const int odd = c0 & 1;
        float2 wxp[NP];
        float wy[W];
#pragma unroll
        for (int j = 0; j < NP; ++j) {
            float w2[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int i0 = 2 * j + h - odd;
                const float w0 = (float)(fx - M + i0) / (float)G - x0;
                w2[h] = (i0 >= 0 && i0 < W) ? __expf(-a * (w0 * w0)) : 0.f;
            }
            wxp[j] = make_float2(w2[0], w2[1]);
        }
#pragma unroll
        for (int i = 0; i < W; ++i) {
            const float w1 = (float)(fy - M + i) / (float)G - y0;
            wy[i] = __expf(-a * (w1 * w1));
        }
        // window origin relative to the staged region (inside it by the tile sort)
        const int rr = wrapG(N + fy - M, G) - ty0, pp = (c0 - odd) / 2 - px0;
        const float4 *base = tsm + ((size_t)rr * TP + pp) * ZC + lane;
        float2 acc = czero();
#pragma unroll
        for (int i1 = 0; i1 < W; ++i1) {
            const float4 *rowp = base + (size_t)i1 * TP * ZC;
            float2 rs = czero();
#pragma unroll
            for (int j = 0; j < NP; ++j) {
                const float4 v = rowp[j * ZC];
                rs.x = fmaf(wxp[j].x, v.x, rs.x);
                rs.y = fmaf(wxp[j].x, v.y, rs.y);
                rs.x = fmaf(wxp[j].y, v.z, rs.x);
                rs.y = fmaf(wxp[j].y, v.w, rs.y);
            }
            acc.x = fmaf(wy[i1], rs.x, acc.x);
            acc.y = fmaf(wy[i1], rs.y, acc.y);
        }
        lines[((size_t)th * N + k) * ZC + lane] = ((k & 1) ? pre : -pre) * acc;
    }
}

template <int N, int M>
__global__ void __launch_bounds__(GPB *ZC, 3)
    k_fwd_gather_tile(const float2 *__restrict__ fg, float2 *__restrict__ lines, const float *__restrict__ xt,
                      const float *__restrict__ yt, float a, float pre, const float4 *__restrict__ ptab,
                      const int4 *__restrict__ chunks)
{
    constexpr int G = 2 * N;
    constexpr int PS = G / 2 + GH_PAIRS, NROWS = G + GH_ROWS;   // the haloed grid's pair pitch and rows
    constexpr int TR = tile_rows<M>(), TP = tile_pairs<M>();
    extern __shared__ float4 tsm[];
    const int4 ch = chunks[blockIdx.x];   // (tile row, tile column, first, count)
    const int ty0 = ch.x * GTILE, px0 = ch.y * GTILE / 2;
    const int rows = min(TR, NROWS - ty0), pairs = min(TP, PS - px0);
    const float4 *g4 = reinterpret_cast<const float4 *>(fg);
    for (int e = threadIdx.x; e < rows * pairs * ZC; e += blockDim.x) {
        const int r = e / (pairs * ZC), rem = e % (pairs * ZC), pj = rem / ZC, q = rem % ZC;
        tsm[(r * TP + pj) * ZC + q] = __ldg(&g4[((size_t)(ty0 + r) * PS + px0 + pj) * ZC + q]);
    }
    __syncthreads();
    tile_gather<N, M>(tsm, ch, ty0, px0, lines, a, pre, ptab);
}

// The same with the tile staged by the Tensor Memory Accelerator: one
// cp.async.bulk.tensor 3-D box load (32 floats = one column pair of ZC
// slices, TP pairs, TR rows) of the haloed grid into shared memory, completed
// on an mbarrier.  The box lands in exactly the layout of k_fwd_gather_tile's
// copy (and is zero-filled past the grid's end, where no window reads), so
// the results are bit-identical.  The wait is bounded: after TMA_SPIN polls
// the block records the failure in *err, waits (bounded again) for its tile
// copy and returns without writing.  The mbarriers sit after the tile in
// dynamic shared memory (no static shared memory, so the tile starts at the
// 128-byte aligned base; checked, and a misaligned base is recorded in *err
// instead of issuing the copy).
constexpr int TMA_SPIN = 1 << 24;
template <int M>
constexpr size_t tma_smem() { return tile_smem<M>() + 16; }
template <int N, int M>
__global__ void __launch_bounds__(GPB *ZC, 3)
    k_fwd_gather_tma(const __grid_constant__ CUtensorMap tmap, float2 *__restrict__ lines,
                     const float *__restrict__ xt, const float *__restrict__ yt, float a, float pre,
                     const float4 *__restrict__ ptab, const int4 *__restrict__ chunks, int *__restrict__ err,
                     int spin = TMA_SPIN, int check = 0)
{
    // check != 0 (the status test only): the blocks first wait on a second
    // barrier that nothing arrives at, so that wait runs out on purpose; the
    // failure path then waits for the tile copy itself before returning
    constexpr unsigned BYTES = (unsigned)tile_smem<M>();
    static_assert(BYTES % 128 == 0, "the mbarriers follow the tile");
    extern __shared__ __align__(128) float4 tsm_tma[];
    float4 *tsm = tsm_tma;
    const int4 ch = chunks[blockIdx.x];
    const int ty0 = ch.x * GTILE, px0 = ch.y * GTILE / 2;   // >= 0; the column coordinate is 0
    const unsigned dst = (unsigned)__cvta_generic_to_shared(tsm);
    const unsigned bar_a = dst + BYTES, bar_b = dst + BYTES + 8;
    if (dst & 127) {
        if (threadIdx.x == 0) atomicExch(err, 2);
        return;
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(BYTES) : "memory");
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
            "%4}], [%5];" ::"r"(dst),
            "l"(reinterpret_cast<unsigned long long>(&tmap)), "r"(0), "r"(px0), "r"(ty0), "r"(bar_a)
            : "memory");
    }
    auto wait = [&](unsigned bar, int limit) {
        unsigned ok = 0;
        for (int it = 0; it < limit && !ok; ++it)
            asm volatile(
                "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                : "=r"(ok)
                : "r"(bar), "r"(0)
                : "memory");
        return ok;
    };
    if (!wait(check ? bar_b : bar_a, spin)) {
        if (threadIdx.x == 0) atomicExch(err, 1);
        wait(bar_a, TMA_SPIN);   // the tile copy lands in this block's memory: let it finish first
        return;
    }
    tile_gather<N, M>(tsm, ch, ty0, px0, lines, a, pre, ptab);
}

// ---- K3b: fftshift1c / 1-D inverse FFT / fftshift1c + crop + scale --------
template <int N>
__global__ void __launch_bounds__(ZC * 32)
    k_fwd_lines(const float2 *__restrict__ lines, float2 *__restrict__ out, int nz, int z0, float scale,
                const float2 *__restrict__ tw)
{
    constexpr int n = 2 * N / 3, c0 = N / 6, T = 32;
    extern __shared__ float2 sm[];
    const int th = blockIdx.x;
    const float2 *src = lines + (size_t)th * N * ZC;   // [k][slice]: the interleaved layout already
    for (int e = threadIdx.x; e < N * ZC; e += blockDim.x) sm[e] = src[e];
    __syncthreads();
    ptfft::fft_iq<N, +1, T, ZC>(sm, threadIdx.x % ZC, threadIdx.x / ZC, tw);
    for (int e = threadIdx.x; e < ZC * n; e += blockDim.x) {
        const int q = e % ZC, j = e / ZC;
        const int z = z0 + q;
        if (z < nz) {
            const int k = c0 + j;
            out[((size_t)th * nz + z) * n + j] = ((k & 1) ? scale : -scale) * sm[k * ZC + q];
        }
    }
}

// ---- A1: pad (kernels.cuh:189-206) + fftshift1c/FFT/fftshift1c -------------
// grid (ntheta, nzp / ZC); writes lines[(theta*N + k) * nzp + z].  ZP: the
// exact adjoint's zero padding (the adjoint of the forward's crop) instead
// of the reference's edge replication.
template <int N, bool ZP = false>
__global__ void __launch_bounds__(ZC * 32)
    k_adj_lines(const float2 *__restrict__ g, float2 *__restrict__ lines, int nz, int nzp, float pre,
                const float2 *__restrict__ tw)
{
    constexpr int n = 2 * N / 3, c0 = N / 6, c1 = 5 * N / 6 - 1, T = 32;
    extern __shared__ float2 sm[];
    const int th = blockIdx.x, z0 = blockIdx.y * ZC;
    const int q = threadIdx.x % ZC, b = threadIdx.x / ZC;
    const int z = z0 + q;
    for (int k = b; k < N; k += T) {
        float2 v = czero();
        if (z < nz) {
            if (!ZP) v = g[((size_t)th * nz + z) * n + (min(max(k, c0), c1) - c0)];
            else if (k >= c0 && k <= c1) v = g[((size_t)th * nz + z) * n + (k - c0)];
        }
        sm[k * ZC + q] = (k & 1) ? v : -1.f * v;
    }
    __syncthreads();
    ptfft::fft_iq<N, -1, T, ZC>(sm, q, b, tw);
    for (int e = threadIdx.x; e < N * ZC; e += blockDim.x) {
        const int k = e / ZC, qq = e % ZC;
        lines[((size_t)th * N + k) * nzp + z0 + qq] = ((k & 1) ? pre : -pre) * sm[e];
    }
}

// ---- A2: column gather (transpose of the forward gather) + column IFFT ----
// grid (nzp / 16, G); block = 16 FFTs x T threads.  A warp owns 4 consecutive
// cells (a "cell group") of the column at a time; the group's list holds every
// polar point whose kernel window covers any of the 4 cells, with the 4
// weights (0 where the window misses a cell), in increasing point order.
// Lanes 0-15 / 16-31 = 16 slices x 2 entry streams, combined at the end in a
// fixed order -> deterministic.  Each loaded g value feeds 4 accumulators.
// ALL: write all N rows of the padded slice (rows N/2 .. N/2 + N - 1 of the
// grid, for the exact adjoint's fold) instead of the n rows of the crop.
constexpr int ZQ = 16;
constexpr int CG = 4;  // cells per group
template <int G, bool ALL = false>
__global__ void __launch_bounds__(ZQ *fft_threads<G>(), (G >= 1024 ? 1 : 2))
    k_adj_colgather(const float2 *__restrict__ lines, float2 *__restrict__ rbuf, const int *__restrict__ goff,
                    const int *__restrict__ gpt, const float4 *__restrict__ gw, const int *__restrict__ col_order,
                    int nzp, const float2 *__restrict__ tw)
{
    constexpr int T = fft_threads<G>(), N = G / 2, n = G / 3, NG4 = G / CG;
    constexpr int Y0 = N / 2 + N / 6;
    constexpr int U = 4;  // entries in flight per lane
    extern __shared__ float2 sm[];
    const int z0 = blockIdx.x * ZQ;
    const int kx = col_order[blockIdx.y];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // 4 entry streams per warp; a stream's 8 lanes hold 2 slices each (one
    // 16-byte load of a point's line covers 2 slices)
    const int s = lane >> 3, zl = lane & 7;
    const int nwarps = blockDim.x >> 5;
    const float4 *lz = reinterpret_cast<const float4 *>(lines + z0) + zl;
    const size_t lstride = (size_t)nzp / 2;  // float4 per point line
    for (int gi = warp; gi < NG4; gi += nwarps) {
        const int beg = goff[kx * NG4 + gi], end = goff[kx * NG4 + gi + 1];
        float4 acc[CG];  // (re, im) of slices 2 zl and 2 zl + 1, per cell
#pragma unroll
        for (int c = 0; c < CG; ++c) acc[c] = make_float4(0.f, 0.f, 0.f, 0.f);
        int e = beg + s;
        for (; e + 4 * (U - 1) < end; e += 4 * U) {
            int pp[U];
            float4 w[U], v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                pp[u] = __ldg(&gpt[e + 4 * u]);
                w[u] = __ldg(&gw[e + 4 * u]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) v[u] = __ldg(lz + (size_t)pp[u] * lstride);
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const float wc[CG] = {w[u].x, w[u].y, w[u].z, w[u].w};
#pragma unroll
                for (int c = 0; c < CG; ++c) {
                    acc[c].x = fmaf(wc[c], v[u].x, acc[c].x);
                    acc[c].y = fmaf(wc[c], v[u].y, acc[c].y);
                    acc[c].z = fmaf(wc[c], v[u].z, acc[c].z);
                    acc[c].w = fmaf(wc[c], v[u].w, acc[c].w);
                }
            }
        }
        for (; e < end; e += 4) {
            const int pp = __ldg(&gpt[e]);
            const float4 w = __ldg(&gw[e]);
            const float4 v = __ldg(lz + (size_t)pp * lstride);
            const float wc[CG] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                acc[c].x = fmaf(wc[c], v.x, acc[c].x);
                acc[c].y = fmaf(wc[c], v.y, acc[c].y);
                acc[c].z = fmaf(wc[c], v.z, acc[c].z);
                acc[c].w = fmaf(wc[c], v.w, acc[c].w);
            }
        }
        // streams 0+2 and 1+3, then 0+1: a fixed order
#pragma unroll
        for (int o = 16; o >= 8; o >>= 1) {
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                acc[c].x += __shfl_down_sync(0xffffffffu, acc[c].x, o);
                acc[c].y += __shfl_down_sync(0xffffffffu, acc[c].y, o);
                acc[c].z += __shfl_down_sync(0xffffffffu, acc[c].z, o);
                acc[c].w += __shfl_down_sync(0xffffffffu, acc[c].w, o);
            }
        }
        if (s == 0) {
#pragma unroll
            for (int c = 0; c < CG; ++c) {
                const int ky = gi * CG + c;
                const float sg = ((kx + ky) & 1) ? -1.f : 1.f;  // fftshiftc
                sm[ky * ZQ + 2 * zl] = make_float2(sg * acc[c].x, sg * acc[c].y);
                sm[ky * ZQ + 2 * zl + 1] = make_float2(sg * acc[c].z, sg * acc[c].w);
            }
        }
    }
    __syncthreads();
    // the 16 slices' column transforms interleaved (shared row ky = element ky of each)
    ptfft::fft_iq<G, +1, T, ZQ>(sm, threadIdx.x % ZQ, threadIdx.x / ZQ, tw);
    constexpr int ROWS = ALL ? N : n, YB = ALL ? N / 2 : Y0;
    for (int e = threadIdx.x; e < ROWS * ZQ; e += blockDim.x) {
        const int r = e / ZQ, q = e % ZQ;
        rbuf[((size_t)r * G + kx) * nzp + z0 + q] = sm[(YB + r) * ZQ + q];
    }
}

// setobj: the 4 weights of every (cell group, point) entry, with the forward
// gather's expression (wx * wy, kernels.cuh:115-119 written separably).
// key = point << 9 | i0 << 5 | (r0 + 3): window column i0, and the window row
// r0 in [-3, 2M] of the group's first cell.
template <int M>
__global__ void k_make_entries(const unsigned *__restrict__ keys, int *__restrict__ gpt, float4 *__restrict__ gw,
                               size_t total, const int *__restrict__ fxy, const float *__restrict__ xt,
                               const float *__restrict__ yt, int G, float a)
{
    constexpr int W = 2 * M + 1;
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= total) return;
    const unsigned key = keys[e];
    const int p = (int)(key >> 9), i0 = (int)((key >> 5) & 15), r0 = (int)(key & 31) - 3;
    const float w0 = (float)(fxy[2 * p] - M + i0) / (float)G - xt[p];
    const float wx = __expf(-a * (w0 * w0));
    float w[CG];
#pragma unroll
    for (int c = 0; c < CG; ++c) {
        const int i1 = r0 + c;
        w[c] = 0.f;
        if (i1 >= 0 && i1 < W) {
            const float w1 = (float)(fxy[2 * p + 1] - M + i1) / (float)G - yt[p];
            w[c] = wx * __expf(-a * (w1 * w1));
        }
    }
    gpt[e] = p;
    gw[e] = make_float4(w[0], w[1], w[2], w[3]);
}

// ---- A4: row inverse FFT + fftshiftc + unpaddivphi + circ + crop -----------
// grid (n, nzp / ZC); reads rbuf[(r * G + kx) * nzp + z]
template <int G>
__global__ void __launch_bounds__(ZC *fft_threads<G>())
    k_adj_rows(const float2 *__restrict__ rbuf, float2 *__restrict__ out, int nz, int nzp,
               const float *__restrict__ fac, float scale, const float2 *__restrict__ tw)
{
    constexpr int T = fft_threads<G>(), N = G / 2, n = G / 3, c0 = N / 6;
    extern __shared__ float2 sm[];
    const int r = blockIdx.x, z0 = blockIdx.y * ZC;
    for (int e = threadIdx.x; e < G * ZC; e += blockDim.x) {
        const int kx = e / ZC, q = e % ZC;
        sm[e] = rbuf[((size_t)r * G + kx) * nzp + z0 + q];
    }
    __syncthreads();
    ptfft::fft_iq<G, +1, T, ZC>(sm, threadIdx.x % ZC, threadIdx.x / ZC, tw);
    for (int e = threadIdx.x; e < ZC * n; e += blockDim.x) {
        const int q = e % ZC, c = e / ZC;
        const int z = z0 + q;
        if (z < nz) {
            const int tx = c0 + c, ty = c0 + r;
            const int X = N / 2 + tx, Y = N / 2 + ty;
            float2 v = sm[X * ZC + q];
            if ((X + Y) & 1) v = -1.f * v;
            out[((size_t)z * n + r) * n + c] = scale * (__ldg(&fac[(size_t)ty * N + tx]) * v);
        }
    }
}


// ---- exact adjoint: rows of the whole padded slice, then the folds ---------
// The forward's pad2 replicates the edge pixels of f into the margins of the
// N x N slice (kernels.cuh:208-216) and its last step crops n of N detector
// samples; their adjoints are a fold (every margin pixel added onto the edge
// pixel it copies) and a zero padding.  grid (N, nzp / ZC): input row ty of
// the padded slice (rbuf row ty, written by the ALL column gather): row
// inverse FFT, sign, circ / phi / (4 N^2), and the fold along x; a row inside
// the crop goes to out, a margin row (ty <= c0 or ty >= c0 + n - 1) to its
// slot of mbuf [n/2 + 2][nz][n] for the fold along y.
template <int G>
__global__ void __launch_bounds__(ZC *fft_threads<G>())
    k_adj_rows_exact(const float2 *__restrict__ rbuf, float2 *__restrict__ out, float2 *__restrict__ mbuf, int nz,
                     int nzp, const float *__restrict__ fac, float scale, const float2 *__restrict__ tw)
{
    constexpr int T = fft_threads<G>(), N = G / 2, n = G / 3, c0 = N / 6;
    extern __shared__ float2 sm[];
    const int ty = blockIdx.x, z0 = blockIdx.y * ZC;
    for (int e = threadIdx.x; e < G * ZC; e += blockDim.x) {
        const int kx = e / ZC, q = e % ZC;
        sm[e] = rbuf[((size_t)ty * G + kx) * nzp + z0 + q];
    }
    __syncthreads();
    ptfft::fft_iq<G, +1, T, ZC>(sm, threadIdx.x % ZC, threadIdx.x / ZC, tw);
    const int Y = N / 2 + ty;
    const float *facr = fac + (size_t)ty * N;
    for (int e = threadIdx.x; e < ZC * n; e += blockDim.x) {
        const int q = e % ZC, c = e / ZC;
        const int z = z0 + q;
        if (z >= nz) continue;
        // columns tx of the padded row that copy pixel c (fixed order)
        const int lo = c == 0 ? 0 : c0 + c, hi = c == n - 1 ? N - 1 : c0 + c;
        float2 acc = czero();
        for (int tx = lo; tx <= hi; ++tx) {
            const int X = N / 2 + tx;
            float2 v = sm[X * ZC + q];
            if ((X + Y) & 1) v = -1.f * v;
            acc = acc + __ldg(&facr[tx]) * v;
        }
        acc = scale * acc;
        if (ty > c0 && ty < c0 + n - 1) {
            out[((size_t)z * n + (ty - c0)) * n + c] = acc;
        } else {
            const int slot = ty <= c0 ? ty : (c0 + 1) + (ty - (c0 + n - 1));
            mbuf[((size_t)slot * nz + z) * n + c] = acc;
        }
    }
}

// out row 0 = sum of margin slots 0..c0, row n-1 = the remaining slots (fixed order)
__global__ void k_adj_fold_rows(const float2 *__restrict__ mbuf, float2 *__restrict__ out, int nz, int n, int c0,
                                int nslots)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)nz * n) return;
    const int z = (int)(i / n), c = (int)(i % n);
    float2 a = czero(), b = czero();
    for (int s = 0; s <= c0; ++s) a = a + mbuf[((size_t)s * nz + z) * n + c];
    for (int s = c0 + 1; s < nslots; ++s) b = b + mbuf[((size_t)s * nz + z) * n + c];
    out[((size_t)z * n) * n + c] = a;
    out[((size_t)z * n + (n - 1)) * n + c] = b;
}

}  // namespace

// ============================================================================
// handle
// ============================================================================
struct pt_radon {
    int ntheta = 0, nz = 0, n = 0, N = 0, G = 0, M = 0, nzp = 0;
    float mu = 0.f;
    int device = -1;
    bool ready = false;
    float2 *tw_G = nullptr, *tw_N = nullptr;
    float *theta = nullptr, *x = nullptr, *y = nullptr;
    int *fxy = nullptr;
    int *perm = nullptr;   // the forward gather's point order (grid tiles)
    float4 *ptab = nullptr;   // (x, y, point index as bits, 0) of each point in that order
    int4 *chunks = nullptr;   // the tiled gather's blocks: (tile row, tile column, first, count)
    int nchunks = 0, chunks_cap = 0;
    int gather = 2;           // 0: gather through L1 (k_fwd_gather_pts), 1: shared-memory tiles, 2: TMA-staged tiles
    // gather 2: one 3-D tensor map per grid buffer set, and a device flag the
    // TMA kernel sets if a tile load did not complete
    CUtensorMap tmap[RSETS];
    bool tma_ok = false;
    int *tma_err = nullptr;
    // forward: per chunk of ZC slices, a row-FFT buffer and a Fourier grid.
    // RSETS buffer sets and RSETS - 1 side streams: chunk c runs on set and
    // stream c % streams (set 0 on the caller's stream), so up to `streams`
    // chunks are in flight and one chunk's FFTs overlap another's gather
    // (fork/join by events)
    float2 *rbuf[RSETS] = {}, *fgrid[RSETS] = {};
    int streams = 4;   // 1, 2 or 4 (pt_radon_autotune chooses)
    cudaStream_t side[RSETS - 1] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[RSETS - 1] = {};
    // adjoint (all slices, slice-minor with nzp lanes)
    float2 *lines = nullptr, *rbuf_adj = nullptr, *mbuf = nullptr;
    int *goff = nullptr, *col_order = nullptr, *gpt = nullptr;
    float4 *gw = nullptr;
    float *deap = nullptr;  // N x N: circ / phi / (4 N^2)
    size_t entries_cap = 0;
};

namespace {

void radon_free(pt_radon *h)
{
    void *bufs[] = {h->tw_G, h->tw_N, h->theta, h->x, h->y, h->fxy, h->perm, h->ptab, h->chunks, h->tma_err,
                    h->lines, h->rbuf_adj, h->mbuf, h->goff, h->col_order, h->gpt, h->gw, h->deap};
    for (void *p : bufs)
        if (p) cudaFree(p);
    for (int k = 0; k < RSETS; ++k) {
        if (h->rbuf[k]) cudaFree(h->rbuf[k]);
        if (h->fgrid[k]) cudaFree(h->fgrid[k]);
    }
    for (int k = 0; k < RSETS - 1; ++k) {
        if (h->side[k]) cudaStreamDestroy(h->side[k]);
        if (h->ev_join[k]) cudaEventDestroy(h->ev_join[k]);
    }
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
}

// Kernel half-width for a forced M: choose -log(eps) so that the reference's
// formula (radonusfft.cu:12) yields exactly M, then mu = -log(eps)/(2N^2).
void radon_params(int n, int m_override, int *N, int *M, float *mu)
{
    *N = n * 3 / 2;
    const size_t NN = (size_t)*N;
    if (m_override <= 0) {
        float eps = 1e-6;  // radonusfft.cu:10-12, same expressions and types
        *mu = -log(eps) / (2 * NN * NN);
        *M = (int)ceil(2 * NN * 1 / PI_REF * sqrt(-*mu * log(eps) + (*mu * NN) * (*mu * NN) / 4));
    } else {
        const double L = m_override * PI_REF / 1.5 - 1e-3;  // ceil(2/pi*0.75*L) = M
        *mu = (float)(L / (2.0 * (double)NN * (double)NN));
        *M = m_override;
    }
}

typedef int (*radon_run_fn)(pt_radon *, float2 *, const float2 *, float, cudaStream_t);

// Tensor maps of the two haloed grid buffers for k_fwd_gather_tma: float32,
// dims (innermost first) {ZC * 4 floats = one column pair of the chunk's
// slices, G/2 + GH_PAIRS pairs, G + GH_ROWS rows}, row-major strides
// {ZC * 16, (G/2 + GH_PAIRS) * ZC * 16} bytes, box {ZC * 4, TP, TR}: the
// box's inner extent is 128 bytes and its first coordinate is always 0, so
// every load starts on a 16-byte boundary.  cuTensorMapEncodeTiled comes
// from the driver through the runtime's entry-point query (no link against
// libcuda); false if it or any encode fails.
bool encode_grid_maps(pt_radon *h)
{
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || fn == nullptr) {
        cudaGetLastError();
        return false;
    }
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    const int G = h->G;
    const cuuint64_t pairs = (cuuint64_t)(G / 2 + GH_PAIRS), rows = (cuuint64_t)(G + GH_ROWS);
    const cuuint64_t dims[3] = {(cuuint64_t)ZC * 4, pairs, rows};
    const cuuint64_t strides[2] = {(cuuint64_t)ZC * 16, pairs * ZC * 16};
    const cuuint32_t tr = (cuuint32_t)(GTILE + 2 * h->M), tp = (cuuint32_t)((GTILE - 2) / 2 + (2 * h->M + 3) / 2);
    const cuuint32_t box[3] = {(cuuint32_t)ZC * 4, tp, tr};
    const cuuint32_t estr[3] = {1, 1, 1};
    for (int b = 0; b < RSETS; ++b) {
        if (((uintptr_t)h->fgrid[b] & 127) != 0) return false;
        if (encode(&h->tmap[b], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, h->fgrid[b], dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

template <int G>
int set_attrs()
{
    constexpr int N = G / 2;
    const int s1 = ZC * (G + 1) * sizeof(float2);
    const int s2 = CK * ZC * (G + 1) * sizeof(float2);
    PT_CUDA(cudaFuncSetAttribute(k_fwd_rows<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    PT_CUDA(cudaFuncSetAttribute(k_fwd_cols<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
    const int s4 = ZQ * (G + 1) * sizeof(float2);
    PT_CUDA(cudaFuncSetAttribute(k_adj_colgather<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, s4));
    PT_CUDA(cudaFuncSetAttribute(k_adj_colgather<G, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s4));
    PT_CUDA(cudaFuncSetAttribute(k_adj_rows<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    PT_CUDA(cudaFuncSetAttribute(k_adj_rows_exact<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, s1));
    const int s3 = ZC * (N + 1) * sizeof(float2);
    PT_CUDA(cudaFuncSetAttribute(k_fwd_lines<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    PT_CUDA(cudaFuncSetAttribute(k_fwd_gather_tile<N, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_smem<7>()));
    PT_CUDA(cudaFuncSetAttribute(k_fwd_gather_tile<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tile_smem<4>()));
    PT_CUDA(cudaFuncSetAttribute(k_fwd_gather_tma<N, 7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tma_smem<7>()));
    PT_CUDA(cudaFuncSetAttribute(k_fwd_gather_tma<N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)tma_smem<4>()));
    PT_CUDA(cudaFuncSetAttribute(k_adj_lines<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    PT_CUDA(cudaFuncSetAttribute(k_adj_lines<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
    return PT_OK;
}

template <int G, int M>
int run_fwd(pt_radon *h, float2 *g, const float2 *f, float scale, cudaStream_t st)
{
    constexpr int N = G / 2, T = fft_threads<G>();
    const size_t s1 = ZC * (G + 1) * sizeof(float2);
    const size_t s2 = CK * ZC * (G + 1) * sizeof(float2);
    const size_t s3 = ZC * (N + 1) * sizeof(float2);
    const float a = (float)(PI_REF * PI_REF / h->mu);
    const float pre = (float)(PI_REF / std::fabs(h->mu)) / (float)N;
    const int nchunks = (h->nz + ZC - 1) / ZC;
    // buffer sets in use: at most `streams`, the chunk count, and the number
    // of ZC-slice line blocks the lines buffer holds (nzp / ZC)
    const int sets = std::max(1, std::min(std::min(h->streams, nchunks), h->nzp / ZC));
    if (sets > 1) {   // fork: the side streams start after everything queued on st so far
        PT_CUDA(cudaEventRecord(h->ev_fork, st));
        for (int k = 1; k < sets; ++k) PT_CUDA(cudaStreamWaitEvent(h->side[k - 1], h->ev_fork, 0));
    }
    for (int c = 0; c < nchunks; ++c) {
        const int z0 = c * ZC;
        // chunk buffers: set c % sets on stream c % sets (a set is reused only
        // by its own stream, in order); gathered lines at block (c % sets) of
        // the lines buffer
        const int k = c % sets;
        cudaStream_t s = k ? h->side[k - 1] : st;
        float2 *rb = h->rbuf[k], *fg = h->fgrid[k];
        float2 *ln = h->lines + (size_t)k * h->ntheta * N * ZC;
        k_fwd_rows<G><<<N, ZC * T, s1, s>>>(f, rb, h->nz, z0, h->deap, h->tw_G);
        PT_LAUNCHED("k_fwd_rows");
        k_fwd_cols<G><<<G / CK, CK * ZC * T, s2, s>>>(rb, fg, h->tw_G);
        PT_LAUNCHED("k_fwd_cols");
        const int npts = h->ntheta * N;
        if (h->gather == 2) {
            k_fwd_gather_tma<N, M><<<h->nchunks, GPB * ZC, tma_smem<M>(), s>>>(
                h->tmap[k], ln, h->x, h->y, a, pre, h->ptab, h->chunks, h->tma_err);
            PT_LAUNCHED("k_fwd_gather_tma");
        } else if (h->gather == 1) {
            k_fwd_gather_tile<N, M><<<h->nchunks, GPB * ZC, tile_smem<M>(), s>>>(fg, ln, h->x, h->y, a, pre, h->ptab,
                                                                              h->chunks);
            PT_LAUNCHED("k_fwd_gather_tile");
        } else {
            k_fwd_gather_pts<N, M><<<(npts + GPB - 1) / GPB, GPB * ZC, 0, s>>>(fg, ln, h->x, h->y, a, pre, h->ptab,
                                                                             npts);
            PT_LAUNCHED("k_fwd_gather_pts");
        }
        k_fwd_lines<N><<<h->ntheta, ZC * 32, s3, s>>>(ln, g, h->nz, z0, scale, h->tw_N);
        PT_LAUNCHED("k_fwd_lines");
    }
    for (int k = 1; k < sets; ++k) {   // join: st continues after every side stream's chunks
        PT_CUDA(cudaEventRecord(h->ev_join[k - 1], h->side[k - 1]));
        PT_CUDA(cudaStreamWaitEvent(st, h->ev_join[k - 1], 0));
    }
    return PT_OK;
}

template <int G, int M>
int run_adj(pt_radon *h, float2 *f, const float2 *g, float scale, cudaStream_t st, bool exact)
{
    constexpr int N = G / 2, n = G / 3, T = fft_threads<G>();
    const size_t s1 = ZC * (G + 1) * sizeof(float2);
    const size_t s3 = ZC * (N + 1) * sizeof(float2);
    const size_t s4 = ZQ * (G + 1) * sizeof(float2);
    const float pre = (float)(PI_REF / std::fabs(h->mu)) / (float)N;
    const int nzp = h->nzp;
    if (exact) {
        k_adj_lines<N, true><<<dim3(h->ntheta, nzp / ZC), ZC * 32, s3, st>>>(g, h->lines, h->nz, nzp, pre, h->tw_N);
        PT_LAUNCHED("k_adj_lines");
        k_adj_colgather<G, true><<<dim3(nzp / ZQ, G), ZQ * T, s4, st>>>(h->lines, h->rbuf_adj, h->goff, h->gpt,
                                                                       h->gw, h->col_order, nzp, h->tw_G);
        PT_LAUNCHED("k_adj_colgather");
        k_adj_rows_exact<G><<<dim3(N, nzp / ZC), ZC * T, s1, st>>>(h->rbuf_adj, f, h->mbuf, h->nz, nzp, h->deap,
                                                                   scale, h->tw_G);
        PT_LAUNCHED("k_adj_rows_exact");
        const size_t cnt = (size_t)h->nz * n;
        k_adj_fold_rows<<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(h->mbuf, f, h->nz, n, N / 6, n / 2 + 2);
        PT_LAUNCHED("k_adj_fold_rows");
        return PT_OK;
    }
    k_adj_lines<N><<<dim3(h->ntheta, nzp / ZC), ZC * 32, s3, st>>>(g, h->lines, h->nz, nzp, pre, h->tw_N);
    PT_LAUNCHED("k_adj_lines");
    k_adj_colgather<G><<<dim3(nzp / ZQ, G), ZQ * T, s4, st>>>(h->lines, h->rbuf_adj, h->goff, h->gpt, h->gw,
                                                             h->col_order, nzp, h->tw_G);
    PT_LAUNCHED("k_adj_colgather");
    k_adj_rows<G><<<dim3(n, nzp / ZC), ZC * T, s1, st>>>(h->rbuf_adj, f, h->nz, nzp, h->deap, scale, h->tw_G);
    PT_LAUNCHED("k_adj_rows");
    return PT_OK;
}

// Compiled grid sizes 2N = 3n (n = 8, 16, 32, 64, 128, 256, 512).
#define PT_RADON_GRIDS(X) X(24) X(48) X(96) X(192) X(384) X(768) X(1536)

bool grid_supported(int G)
{
#define PT_CASE(GG) \
    if (G == GG) return true;
    PT_RADON_GRIDS(PT_CASE)
#undef PT_CASE
    return false;
}

int radon_set_attrs(int G)
{
#define PT_CASE(GG) \
    if (G == GG) return set_attrs<GG>();
    PT_RADON_GRIDS(PT_CASE)
#undef PT_CASE
    pt::set_error("radonusfft: unsupported grid size %d", G);
    return PT_ERR_UNSUPPORTED;
}

int radon_dispatch(pt_radon *h, bool adj, float2 *out, const float2 *in, float scale, cudaStream_t st,
                   bool exact = false)
{
#define PT_CASE(GG)                                                                 \
    if (h->G == GG) {                                                               \
        if (h->M == 7) return adj ? run_adj<GG, 7>(h, out, in, scale, st, exact)    \
                                  : run_fwd<GG, 7>(h, out, in, scale, st);          \
        if (h->M == 4) return adj ? run_adj<GG, 4>(h, out, in, scale, st, exact)    \
                                  : run_fwd<GG, 4>(h, out, in, scale, st);          \
    }
    PT_RADON_GRIDS(PT_CASE)
#undef PT_CASE
    pt::set_error("radonusfft: no kernel for grid %d with half-width M=%d", h->G, h->M);
    return PT_ERR_UNSUPPORTED;
}

// The TMA gather of the first slice chunk whose blocks first wait, 256 polls
// at most, on a barrier that nothing arrives at: every block's wait runs out,
// records code 1, waits for its own tile copy and returns without writing
// (the status test of pt_radon_check_tma_wait).
template <int G, int M>
int run_tma_wait_check(pt_radon *h, cudaStream_t st)
{
    constexpr int N = G / 2;
    const float a = (float)(PI_REF * PI_REF / h->mu);
    const float pre = (float)(PI_REF / std::fabs(h->mu)) / (float)N;
    k_fwd_gather_tma<N, M><<<h->nchunks, GPB * ZC, tma_smem<M>(), st>>>(h->tmap[0], h->lines, h->x, h->y, a, pre,
                                                                        h->ptab, h->chunks, h->tma_err, 256, 1);
    PT_LAUNCHED("k_fwd_gather_tma");
    return PT_OK;
}

int radon_tma_wait_check(pt_radon *h, cudaStream_t st)
{
#define PT_CASE(GG)                                                         \
    if (h->G == GG) {                                                       \
        if (h->M == 7) return run_tma_wait_check<GG, 7>(h, st);             \
        if (h->M == 4) return run_tma_wait_check<GG, 4>(h, st);             \
    }
    PT_RADON_GRIDS(PT_CASE)
#undef PT_CASE
    pt::set_error("radonusfft: no kernel for grid %d with half-width M=%d", h->G, h->M);
    return PT_ERR_UNSUPPORTED;
}

template <typename T>
int dmalloc(T **p, size_t count)
{
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T) + 16);
    if (e != cudaSuccess) {
        *p = nullptr;
        pt::set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        return PT_ERR_ALLOC;
    }
    return PT_OK;
}

int check_device(const pt_radon *h)
{
    int dev = -1;
    PT_CUDA(cudaGetDevice(&dev));
    if (dev != h->device) {
        pt::set_error("radonusfft handle belongs to device %d, current device is %d", h->device, dev);
        return PT_ERR_ARG;
    }
    return PT_OK;
}

}  // namespace

extern "C" int pt_radon_create_ex(size_t ntheta, size_t nz, size_t n, int m_override, pt_radon **out)
{
    pt::clear_error();
    PT_CHECK_ARG(out != nullptr, "radonusfft: null output handle");
    *out = nullptr;
    PT_CHECK_ARG(ntheta >= 1 && ntheta <= (1u << 20), "radonusfft: bad Ntheta %zu", ntheta);
    PT_CHECK_ARG(nz >= 1 && nz <= (1u << 20), "radonusfft: bad Nz %zu", nz);
    PT_CHECK_ARG(n >= 8 && n % 8 == 0, "radonusfft: n=%zu must be a positive multiple of 8", n);
    PT_CHECK_ARG(ntheta * (3 * n / 2) < ((size_t)1 << 23), "radonusfft: Ntheta*3n/2 = %zu polar points exceed 2^23",
                 ntheta * (3 * n / 2));
    PT_CHECK_ARG(m_override == 0 || m_override == 4 || m_override == 7,
                 "radonusfft: kernel half-width override %d not compiled (0, 4 or 7)", m_override);
    const int G = (int)(3 * n);
    if (!grid_supported(G)) {
        pt::set_error("radonusfft: n=%zu not compiled (supported n: 8,16,32,64,128,256,512)", n);
        return PT_ERR_UNSUPPORTED;
    }
    pt_radon *h = new pt_radon();
    h->ntheta = (int)ntheta;
    h->nz = (int)nz;
    h->n = (int)n;
    radon_params((int)n, m_override, &h->N, &h->M, &h->mu);
    h->G = G;
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        delete h;
        pt::set_error("radonusfft: no CUDA device");
        return PT_ERR_CUDA;
    }
    if (h->M != 7 && h->M != 4) {
        pt::set_error("radonusfft: reference half-width M=%d has no compiled kernel", h->M);
        delete h;
        return PT_ERR_UNSUPPORTED;
    }
    int rc = PT_OK;
    const size_t N = h->N;
    if (rc == PT_OK) rc = dmalloc(&h->tw_G, (size_t)G);
    if (rc == PT_OK) rc = dmalloc(&h->tw_N, N);
    if (rc == PT_OK) rc = dmalloc(&h->theta, ntheta);
    if (rc == PT_OK) rc = dmalloc(&h->x, ntheta * N);
    if (rc == PT_OK) rc = dmalloc(&h->y, ntheta * N);
    if (rc == PT_OK) rc = dmalloc(&h->fxy, 2 * ntheta * N);
    if (rc == PT_OK) rc = dmalloc(&h->perm, ntheta * N);
    if (rc == PT_OK) rc = dmalloc(&h->ptab, ntheta * N);
    for (int k = 0; k < RSETS && rc == PT_OK; ++k) {
        rc = dmalloc(&h->rbuf[k], N * G * ZC);
        if (rc == PT_OK) rc = dmalloc(&h->fgrid[k], (size_t)(G + GH_ROWS) * (G + 2 * GH_PAIRS) * ZC);
    }
    if (rc == PT_OK) rc = dmalloc(&h->deap, (size_t)N * N);
    if (rc == PT_OK && cudaMalloc((void **)&h->tma_err, sizeof(int)) == cudaSuccess &&
        cudaMemset(h->tma_err, 0, sizeof(int)) == cudaSuccess)
        h->tma_ok = encode_grid_maps(h);   // gather 2 is offered only if every map encodes
    // default variant (the autotuner's usual choice from 128^3 up, within a
    // few percent at 64^3): four chunk pipelines, TMA-staged tiles
    h->streams = 4;
    h->gather = h->tma_ok ? 2 : 1;
    if (rc == PT_OK && cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess) rc = PT_ERR_CUDA;
    for (int k = 0; k < RSETS - 1 && rc == PT_OK; ++k)
        if (cudaStreamCreateWithFlags(&h->side[k], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&h->ev_join[k], cudaEventDisableTiming) != cudaSuccess)
            rc = PT_ERR_CUDA;
    if (rc == PT_ERR_CUDA) pt::set_error("radonusfft: stream/event creation failed");
    h->nzp = (int)((nz + ZQ - 1) / ZQ * ZQ);
    const size_t nzp = h->nzp;
    if (rc == PT_OK) rc = dmalloc(&h->lines, ntheta * N * nzp);
    // all N rows of the padded slice (the exact adjoint's fold needs them; the
    // reference adjoint uses the first n)
    if (rc == PT_OK) rc = dmalloc(&h->rbuf_adj, N * (size_t)G * nzp);
    if (rc == PT_OK) rc = dmalloc(&h->mbuf, (n / 2 + 2) * (size_t)nz * n);
    if (rc == PT_OK) rc = dmalloc(&h->goff, (size_t)G * (G / CG) + 1);
    if (rc == PT_OK) rc = dmalloc(&h->col_order, (size_t)G);
    if (rc == PT_OK) rc = radon_set_attrs(G);
    if (rc == PT_OK) {
        std::vector<float2> tw(G);
        pt_make_twiddles(tw.data(), G);
        if (cudaMemcpy(h->tw_G, tw.data(), G * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = PT_ERR_CUDA;
        pt_make_twiddles(tw.data(), (int)N);
        if (rc == PT_OK &&
            cudaMemcpy(h->tw_N, tw.data(), N * sizeof(float2), cudaMemcpyHostToDevice) != cudaSuccess)
            rc = PT_ERR_CUDA;
        if (rc != PT_OK) pt::set_error("radonusfft: twiddle upload failed");
    }
    if (rc != PT_OK) {
        radon_free(h);
        delete h;
        return rc;
    }
    *out = h;
    return PT_OK;
}

extern "C" int pt_radon_create(size_t ntheta, size_t nz, size_t n, pt_radon **out)
{
    return pt_radon_create_ex(ntheta, nz, n, 0, out);
}

extern "C" int pt_radon_destroy(pt_radon *h)
{
    pt::clear_error();
    if (!h) return PT_OK;
    radon_free(h);
    delete h;
    return PT_OK;
}

extern "C" int pt_radon_setobj(pt_radon *h, const float *theta, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "radonusfft.setobj: null handle");
    PT_CHECK_ARG(theta != nullptr, "radonusfft.setobj: null theta");
    int rc = check_device(h);
    if (rc != PT_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    h->ready = false;
    const int N = h->N, G = h->G, M = h->M, W = 2 * M + 1, ntheta = h->ntheta;
    PT_CUDA(cudaMemcpyAsync(h->theta, theta, ntheta * sizeof(float), cudaMemcpyDefault, st));
    k_takexy<<<dim3((N + 127) / 128, ntheta), 128, 0, st>>>(h->x, h->y, h->theta, N, ntheta);
    PT_LAUNCHED("k_takexy");
    k_deap_table<<<dim3((N + 127) / 128, N), 128, 0, st>>>(h->deap, N, h->mu);
    PT_LAUNCHED("k_deap_table");
    const size_t npts = (size_t)ntheta * N;
    std::vector<float> xs(npts), ys(npts);
    PT_CUDA(cudaMemcpyAsync(xs.data(), h->x, npts * sizeof(float), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaMemcpyAsync(ys.data(), h->y, npts * sizeof(float), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    // window corners floor(2N x) exactly as kernels.cuh:112-115 (float product)
    std::vector<int> fxy(2 * npts);
    for (size_t p = 0; p < npts; ++p) {
        if (!(xs[p] >= -0.5f && xs[p] < 0.5f && ys[p] >= -0.5f && ys[p] < 0.5f)) {
            pt::set_error("radonusfft.setobj: theta[%zu] is not a finite angle", p / N);
            h->ready = false;
            return PT_ERR_ARG;
        }
        fxy[2 * p] = (int)floorf((float)G * xs[p]);
        fxy[2 * p + 1] = (int)floorf((float)G * ys[p]);
    }
    PT_CUDA(cudaMemcpy(h->fxy, fxy.data(), 2 * npts * sizeof(int), cudaMemcpyHostToDevice));
    {   // the forward gather's visiting order: by the grid tile of the window origin, then point index
        std::vector<int> perm(npts);
        std::vector<unsigned> tile(npts);
        const int TPR = (G + GTILE - 1) / GTILE;
        for (size_t p = 0; p < npts; ++p) {
            perm[p] = (int)p;
            const int ox = ((N + fxy[2 * p] - M) % G + G) % G, oy = ((N + fxy[2 * p + 1] - M) % G + G) % G;
            tile[p] = (unsigned)((oy / GTILE) * TPR + ox / GTILE);
        }
        std::stable_sort(perm.begin(), perm.end(), [&](int i, int j) { return tile[i] < tile[j]; });
        PT_CUDA(cudaMemcpy(h->perm, perm.data(), npts * sizeof(int), cudaMemcpyHostToDevice));
        std::vector<float4> ptab(npts);
        for (size_t i = 0; i < npts; ++i) {
            const int q = perm[i];
            int bits;
            std::memcpy(&bits, &q, sizeof(int));
            float qf;
            std::memcpy(&qf, &bits, sizeof(float));
            ptab[i] = make_float4(xs[q], ys[q], qf, 0.f);
        }
        PT_CUDA(cudaMemcpy(h->ptab, ptab.data(), npts * sizeof(float4), cudaMemcpyHostToDevice));
        // the tiled gather's blocks: runs of one tile in perm order, at most TCH points each
        std::vector<int4> chunks;
        for (size_t i = 0; i < npts;) {
            size_t j = i;
            while (j < npts && tile[perm[j]] == tile[perm[i]]) ++j;
            const int t = (int)tile[perm[i]];
            for (size_t f = i; f < j; f += TCH)
                chunks.push_back(make_int4(t / TPR, t % TPR, (int)f, (int)std::min<size_t>(TCH, j - f)));
            i = j;
        }
        if ((int)chunks.size() > h->chunks_cap) {
            if (h->chunks) cudaFree(h->chunks);
            h->chunks = nullptr;
            h->chunks_cap = 0;
            PT_CUDA(cudaMalloc(&h->chunks, chunks.size() * sizeof(int4)));
            h->chunks_cap = (int)chunks.size();
        }
        h->nchunks = (int)chunks.size();
        PT_CUDA(cudaMemcpy(h->chunks, chunks.data(), chunks.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    // cell-group lists for the adjoint: a group is CG consecutive rows of one
    // grid column; every point is listed, in increasing point order, in each
    // group that its (2M+1)^2 window (mod G: the reference's halo fold,
    // kernels.cuh:67-82) touches, with the window column i0 and row offset r0.
    const int NG4 = G / CG;
    const size_t ngroups = (size_t)G * NG4;
    std::vector<int> off(ngroups + 1, 0);
    int cols[32], grp_first[8], ngrp = 0, oy = 0;
    auto window = [&](size_t p) {
        const int ox = ((N + fxy[2 * p] - M) % G + G) % G;
        oy = ((N + fxy[2 * p + 1] - M) % G + G) % G;
        for (int i = 0; i < W; ++i) cols[i] = (ox + i) % G;
        ngrp = 0;
        for (int i = 0; i < W; ++i) {
            const int gi = ((oy + i) % G) / CG;
            if (ngrp == 0 || grp_first[ngrp - 1] != gi) grp_first[ngrp++] = gi;
        }
    };
    for (size_t p = 0; p < npts; ++p) {
        window(p);
        for (int i0 = 0; i0 < W; ++i0)
            for (int k = 0; k < ngrp; ++k) off[(size_t)cols[i0] * NG4 + grp_first[k] + 1]++;
    }
    for (size_t c = 0; c < ngroups; ++c) off[c + 1] += off[c];
    const size_t total = (size_t)off[ngroups];
    std::vector<unsigned> keys(total);
    {
        std::vector<int> pos(off.begin(), off.end() - 1);
        for (size_t p = 0; p < npts; ++p) {
            window(p);
            for (int k = 0; k < ngrp; ++k) {
                int r0 = ((grp_first[k] * CG - oy) % G + G) % G;  // row offset of the group's first cell
                if (r0 > G - CG) r0 -= G;                          // in [-(CG-1), 2M]
                for (int i0 = 0; i0 < W; ++i0)
                    keys[pos[(size_t)cols[i0] * NG4 + grp_first[k]]++] =
                        ((unsigned)p << 9) | ((unsigned)i0 << 5) | (unsigned)(r0 + 3);
            }
        }
    }
    // columns ordered by decreasing work so the heavy centre columns start first
    std::vector<long long> colw(G, 0);
    for (int c = 0; c < G; ++c) colw[c] = off[(size_t)(c + 1) * NG4] - off[(size_t)c * NG4];
    std::vector<int> order(G);
    for (int i = 0; i < G; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return colw[i] > colw[j]; });
    if (total > h->entries_cap) {
        if (h->gpt) cudaFree(h->gpt);
        if (h->gw) cudaFree(h->gw);
        h->gpt = nullptr;
        h->gw = nullptr;
        h->entries_cap = 0;
        rc = dmalloc(&h->gpt, total);
        if (rc == PT_OK) rc = dmalloc(&h->gw, total);
        if (rc != PT_OK) return rc;
        h->entries_cap = total;
    }
    unsigned *dkeys = nullptr;
    rc = dmalloc(&dkeys, total);
    if (rc != PT_OK) return rc;
    cudaError_t e1 = cudaMemcpy(dkeys, keys.data(), total * sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e1 == cudaSuccess) {
        const float a = (float)(PI_REF * PI_REF / h->mu);
        const unsigned blocks = (unsigned)((total + 255) / 256);
        if (M == 7)
            k_make_entries<7><<<blocks, 256, 0, st>>>(dkeys, h->gpt, h->gw, total, h->fxy, h->x, h->y, G, a);
        else
            k_make_entries<4><<<blocks, 256, 0, st>>>(dkeys, h->gpt, h->gw, total, h->fxy, h->x, h->y, G, a);
        e1 = cudaGetLastError();
        if (e1 == cudaSuccess) e1 = cudaStreamSynchronize(st);
    }
    cudaFree(dkeys);
    if (e1 != cudaSuccess) {
        pt::set_error("radonusfft.setobj: building the adjoint lists failed: %s", cudaGetErrorString(e1));
        return PT_ERR_CUDA;
    }
    PT_CUDA(cudaMemcpy(h->goff, off.data(), (ngroups + 1) * sizeof(int), cudaMemcpyHostToDevice));
    PT_CUDA(cudaMemcpy(h->col_order, order.data(), G * sizeof(int), cudaMemcpyHostToDevice));
    h->ready = true;
    return PT_OK;
}

namespace {
int radon_call(pt_radon *h, bool adj, void *out, const void *in, float scale, void *stream, bool exact = false)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "radonusfft: null handle");
    PT_CHECK_ARG(out != nullptr && in != nullptr, "radonusfft.%s: null array pointer", adj ? "adj" : "fwd");
    if (!h->ready) {
        pt::set_error("radonusfft.%s: setobj(theta) has not been called", adj ? "adj" : "fwd");
        return PT_ERR_STATE;
    }
    int rc = check_device(h);
    if (rc != PT_OK) return rc;
    return radon_dispatch(h, adj, (float2 *)out, (const float2 *)in, scale, (cudaStream_t)stream, exact);
}
}  // namespace

extern "C" int pt_radon_fwd(pt_radon *h, void *g, const void *f, void *stream)
{
    return radon_call(h, false, g, f, 1.0f, stream);
}
extern "C" int pt_radon_adj(pt_radon *h, void *f, const void *g, void *stream)
{
    return radon_call(h, true, f, g, 1.0f, stream);
}
extern "C" int pt_radon_fwd_scaled(pt_radon *h, void *g, const void *f, float scale, void *stream)
{
    return radon_call(h, false, g, f, scale, stream);
}
extern "C" int pt_radon_adj_scaled(pt_radon *h, void *f, const void *g, float scale, void *stream)
{
    return radon_call(h, true, f, g, scale, stream);
}

// Autotuner: times the forward with its chunks on one stream and pipelined on
// two, each with the gather through L1 and from shared-memory tiles, and
// keeps the fastest (setup-time; blocks the host).
extern "C" int pt_radon_autotune(pt_radon *h, void *g, const void *f, int trials, int *streams_out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && g && f && trials >= 1, "radonusfft.autotune: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    PT_CUDA(cudaEventCreate(&e0));
    PT_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int best_s = h->streams, best_g = h->gather, rc = PT_OK;
    const int ngather = h->tma_ok ? 3 : 2;   // streams {1, 2, 4} x gather {L1, tiles, TMA tiles}
    for (int combo = 0; combo < 3 * ngather && rc == PT_OK; ++combo) {
        const int sc = 1 << (combo % 3);
        h->streams = sc;
        h->gather = combo / 3;
        std::vector<float> ts;
        for (int k = 0; k <= trials && rc == PT_OK; ++k) {
            cudaEventRecord(e0, st);
            rc = pt_radon_fwd(h, g, f, stream);
            cudaEventRecord(e1, st);
            if (rc == PT_OK && cudaEventSynchronize(e1) == cudaSuccess && k > 0) {
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ts.push_back(ms);
            }
        }
        if (rc != PT_OK) break;
        std::sort(ts.begin(), ts.end());
        if (ts[ts.size() / 2] < best) {
            best = ts[ts.size() / 2];
            best_s = sc;
            best_g = h->gather;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->streams = best_s;
    h->gather = best_g;
    if (streams_out) *streams_out = best_s + 8 * best_g;
    if (rc == PT_OK && h->tma_ok) {   // a TMA tile load that never completed
        int flag = 0;
        PT_CUDA(cudaMemcpy(&flag, h->tma_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) {
            h->gather = 1;
            pt::set_error("radonusfft.autotune: a TMA tile load did not complete; TMA gather disabled");
            h->tma_ok = false;
            return PT_ERR_CUDA;
        }
    }
    return rc;
}

extern "C" int pt_radon_check_tma_wait(pt_radon *h, int *code, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h && code, "radonusfft.check_tma_wait: null pointer");
    if (!h->ready || !h->tma_ok) {
        pt::set_error("radonusfft.check_tma_wait: needs setobj and the TMA gather");
        return PT_ERR_STATE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    PT_CUDA(cudaMemsetAsync(h->tma_err, 0, sizeof(int), st));
    int rc = radon_tma_wait_check(h, st);
    if (rc != PT_OK) return rc;
    PT_CUDA(cudaMemcpyAsync(code, h->tma_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    PT_CUDA(cudaMemsetAsync(h->tma_err, 0, sizeof(int), st));
    PT_CUDA(cudaStreamSynchronize(st));
    return PT_OK;
}

extern "C" int pt_radon_status(pt_radon *h, int *tma_timeouts, int *tma_available)
{
    pt::clear_error();
    PT_CHECK_ARG(h && tma_timeouts && tma_available, "radonusfft.status: null pointer");
    *tma_available = h->tma_ok ? 1 : 0;
    *tma_timeouts = 0;
    if (h->tma_err) {
        PT_CUDA(cudaMemcpy(tma_timeouts, h->tma_err, sizeof(int), cudaMemcpyDeviceToHost));
        PT_CUDA(cudaMemset(h->tma_err, 0, sizeof(int)));
    }
    return PT_OK;
}

int pt::radon_dims(const pt_radon *h, int *nz, int *ntheta)
{
    PT_CHECK_ARG(h != nullptr, "radonusfft: null handle");
    if (!h->ready) {
        pt::set_error("radonusfft: setobj(theta) has not been called");
        return PT_ERR_STATE;
    }
    *nz = h->nz;
    *ntheta = h->ntheta;
    return PT_OK;
}

extern "C" int pt_radon_set_variant(pt_radon *h, int streams, int gather)
{
    pt::clear_error();
    PT_CHECK_ARG(h && (streams == 1 || streams == 2 || streams == 4) && (gather >= 0 && gather <= 2),
                 "radonusfft.set_variant: streams 1, 2 or 4, gather 0 (L1), 1 (tiles) or 2 (TMA tiles)");
    if (gather == 2 && !h->tma_ok) {
        pt::set_error("radonusfft.set_variant: the TMA gather is not available (tensor map encoding failed)");
        return PT_ERR_UNSUPPORTED;
    }
    h->streams = streams;
    h->gather = gather;
    return PT_OK;
}

extern "C" int pt_radon_adj_exact(pt_radon *h, void *f, const void *g, float scale, void *stream)
{
    return radon_call(h, true, f, g, scale, stream, true);
}

extern "C" int pt_radon_get_params(const pt_radon *h, int *N, int *M, float *mu)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "radonusfft: null handle");
    if (N) *N = h->N;
    if (M) *M = h->M;
    if (mu) *mu = h->mu;
    return PT_OK;
}

extern "C" int pt_radon_get_xy(const pt_radon *h, float *x, float *y, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(h != nullptr, "radonusfft: null handle");
    if (!h->ready) {
        pt::set_error("radonusfft.get_xy: setobj(theta) has not been called");
        return PT_ERR_STATE;
    }
    const size_t bytes = (size_t)h->ntheta * h->N * sizeof(float);
    cudaStream_t st = (cudaStream_t)stream;
    if (x) PT_CUDA(cudaMemcpyAsync(x, h->x, bytes, cudaMemcpyDefault, st));
    if (y) PT_CUDA(cudaMemcpyAsync(y, h->y, bytes, cudaMemcpyDefault, st));
    return PT_OK;
}
