// Kernels of the learned Fourier preconditioner's network (no counterpart in
// the reference, whose tomography CG, src/ptychotomo/solver.py:180-203, is
// unpreconditioned).
//
// The network is a 3 -> 64 -> 64 -> 1 MLP with SiLU activations:
//     h1 = silu(W1 x + b1),  h2 = silu(W2 h1 + b2),  z = W3 h2 + b3.
// Parameters are one flat FP32 vector (the master copy): W1 [64][3], b1 [64],
// W2 [64][64], b2 [64], W3 [64], b3 — 4481 values.  With bf16 != 0 each
// kernel rounds the weights (not the biases) to bfloat16 when it stages them
// in shared memory, so the arithmetic uses bf16 weights; activations and
// every accumulation stay FP32.  Training is full-batch least squares
//     loss = inv_wsum * sum_p w_p (z_p - y_p)^2
// with its exact gradient with respect to the (rounded) parameters, reduced
// deterministically (fixed tiles per block, fixed block order), and Adam.
#include <cuda_bf16.h>

#include <cmath>

#include "pt_common.cuh"

namespace {

constexpr int H = 64, DIN = 3;
constexpr int OW1 = 0, OB1 = OW1 + H * DIN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H;
constexpr int NPAR = OB3 + 1;   // 4481
constexpr int TB = 256;         // threads per block = points per tile
constexpr int LD = H + 4;       // row stride of the per-point tiles (16-byte rows, conflict-free float4 writes)
constexpr int NSLOT = NPAR + 1; // gradient partials + the loss

__device__ __forceinline__ bool is_weight(int i)
{
    return i < OB1 || (i >= OW2 && i < OB2) || (i >= OW3 && i < OB3);
}

// params -> shared memory, weights rounded to bf16 (round-to-nearest-even) when asked
__device__ __forceinline__ void stage_params(float *net, const float *__restrict__ p, int bf16)
{
    for (int i = threadIdx.x; i < NPAR; i += blockDim.x) {
        float v = p[i];
        if (bf16 && is_weight(i)) v = __bfloat162float(__float2bfloat16_rn(v));
        net[i] = v;
    }
}

__device__ __forceinline__ float sigm(float s) { return 1.f / (1.f + expf(-s)); }
__device__ __forceinline__ float silu(float s) { return s * sigm(s); }
__device__ __forceinline__ float dsilu(float s)
{
    const float g = sigm(s);
    return g * (1.f + s * (1.f - g));
}

__device__ __forceinline__ float layer1(const float *net, int j, float x0, float x1, float x2)
{
    return net[OB1 + j] + net[OW1 + 3 * j] * x0 + net[OW1 + 3 * j + 1] * x1 + net[OW1 + 3 * j + 2] * x2;
}

// s2 = W2 h1 + b2 (row j of W2 read as float4s)
__device__ __forceinline__ void layer2(const float *net, const float (&h1)[H], float (&s2)[H])
{
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const float4 *w = reinterpret_cast<const float4 *>(net + OW2 + j * H);
        float a = net[OB2 + j];
#pragma unroll
        for (int q = 0; q < H / 4; ++q) {
            const float4 v = w[q];
            a = fmaf(v.x, h1[4 * q], a);
            a = fmaf(v.y, h1[4 * q + 1], a);
            a = fmaf(v.z, h1[4 * q + 2], a);
            a = fmaf(v.w, h1[4 * q + 3], a);
        }
        s2[j] = a;
    }
}

__global__ void __launch_bounds__(TB) k_mlp_forward(const float *__restrict__ params, int bf16,
                                                    const float *__restrict__ x, float *__restrict__ z, size_t npts)
{
    __shared__ __align__(16) float net[NPAR + 3];
    stage_params(net, params, bf16);
    __syncthreads();
    for (size_t p = (size_t)blockIdx.x * TB + threadIdx.x; p < npts; p += (size_t)gridDim.x * TB) {
        const float x0 = x[3 * p], x1 = x[3 * p + 1], x2 = x[3 * p + 2];
        float h1[H], s2[H];
#pragma unroll
        for (int j = 0; j < H; ++j) h1[j] = silu(layer1(net, j, x0, x1, x2));
        layer2(net, h1, s2);
        float out = net[OB3];
#pragma unroll
        for (int j = 0; j < H; ++j) out = fmaf(net[OW3 + j], silu(s2[j]), out);
        z[p] = out;
    }
}

// Loss and gradient partials.  Persistent blocks: block b walks tiles b,
// b + grid, ... of TB points; each thread owns fixed gradient entries and
// accumulates them over the block's tiles (FP32); the block writes its NSLOT
// partials to work[b * NSLOT ...].  Per tile (one point per thread):
//   1. forward; A <- h1, B <- dz2 = dz W3 silu'(s2), dzv, lossv
//   2. dW2 (each thread 16 entries: row t/4, columns 16 (t%4) ..), db2
//   3. A <- dz h2
//   4. dW3, db3, loss
//   5. dh1 = W2^T dz2 (B row of this point), dz1 = dh1 silu'(s1); A <- dz1
//   6. db1, dW1
// Points past npts take w = 0 and contribute nothing.
__global__ void __launch_bounds__(TB, 1) k_mlp_grad(const float *__restrict__ params, int bf16,
                                                    const float *__restrict__ x, const float *__restrict__ y,
                                                    const float *__restrict__ w, size_t npts, float inv_wsum,
                                                    float *__restrict__ work)
{
    extern __shared__ __align__(16) float sm[];
    float *net = sm;                                  // NPAR (+3 pad)
    float *A = sm + ((NPAR + 3) / 4) * 4;             // [TB][LD]
    float *B = A + TB * LD;                           // [TB][LD]
    float *X = B + TB * LD;                           // [TB][3]
    float *dzv = X + TB * 3;                          // [TB]
    float *lossv = dzv + TB;                          // [TB]
    stage_params(net, params, bf16);
    __syncthreads();

    const int t = threadIdx.x;
    const int rj = t >> 2, rk = (t & 3) * 16;         // this thread's dW2 entries: row rj, columns rk..rk+15
    float acc2[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) acc2[q] = 0.f;
    float accA = 0.f;   // t < 64: db2[t]; 64..127: dW3[t-64]; 128: db3; 129: loss
    float accB = 0.f;   // t < 64: db1[t]; 64..255: dW1[(t-64)/3][(t-64)%3]

    const size_t ntiles = (npts + TB - 1) / TB;
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t p = tile * TB + t;
        const bool live = p < npts;
        const float x0 = live ? x[3 * p] : 0.f, x1 = live ? x[3 * p + 1] : 0.f, x2 = live ? x[3 * p + 2] : 0.f;
        const float wp = live ? w[p] : 0.f, yp = live ? y[p] : 0.f;
        X[3 * t] = x0;
        X[3 * t + 1] = x1;
        X[3 * t + 2] = x2;
        // ---- 1. forward
        float s2[H];
        {
            float h1[H];
#pragma unroll
            for (int j = 0; j < H; ++j) h1[j] = silu(layer1(net, j, x0, x1, x2));
            float4 *a4 = reinterpret_cast<float4 *>(A + t * LD);
#pragma unroll
            for (int q = 0; q < H / 4; ++q) a4[q] = make_float4(h1[4 * q], h1[4 * q + 1], h1[4 * q + 2], h1[4 * q + 3]);
            layer2(net, h1, s2);
        }
        float z = net[OB3];
#pragma unroll
        for (int j = 0; j < H; ++j) z = fmaf(net[OW3 + j], silu(s2[j]), z);
        const float r = z - yp;
        const float dz = 2.f * wp * r * inv_wsum;
        dzv[t] = dz;
        lossv[t] = wp * r * r * inv_wsum;
        {
            float4 *b4 = reinterpret_cast<float4 *>(B + t * LD);
#pragma unroll
            for (int q = 0; q < H / 4; ++q) {
                float d[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) d[e] = dz * net[OW3 + 4 * q + e] * dsilu(s2[4 * q + e]);
                b4[q] = make_float4(d[0], d[1], d[2], d[3]);
            }
        }
        __syncthreads();
        // ---- 2. dW2, db2
        for (int pp = 0; pp < TB; ++pp) {
            const float bj = B[pp * LD + rj];
            const float4 *a4 = reinterpret_cast<const float4 *>(A + pp * LD + rk);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float4 v = a4[q];
                acc2[4 * q] = fmaf(bj, v.x, acc2[4 * q]);
                acc2[4 * q + 1] = fmaf(bj, v.y, acc2[4 * q + 1]);
                acc2[4 * q + 2] = fmaf(bj, v.z, acc2[4 * q + 2]);
                acc2[4 * q + 3] = fmaf(bj, v.w, acc2[4 * q + 3]);
            }
        }
        if (t < H) {
            for (int pp = 0; pp < TB; ++pp) accA += B[pp * LD + t];
        }
        __syncthreads();
        // ---- 3. A <- dz h2
        {
            float4 *a4 = reinterpret_cast<float4 *>(A + t * LD);
#pragma unroll
            for (int q = 0; q < H / 4; ++q)
                a4[q] = make_float4(dz * silu(s2[4 * q]), dz * silu(s2[4 * q + 1]), dz * silu(s2[4 * q + 2]),
                                    dz * silu(s2[4 * q + 3]));
        }
        __syncthreads();
        // ---- 4. dW3, db3, loss
        if (t >= H && t < 2 * H) {
            for (int pp = 0; pp < TB; ++pp) accA += A[pp * LD + (t - H)];
        } else if (t == 2 * H) {
            for (int pp = 0; pp < TB; ++pp) accA += dzv[pp];
        } else if (t == 2 * H + 1) {
            for (int pp = 0; pp < TB; ++pp) accA += lossv[pp];
        }
        __syncthreads();
        // ---- 5. dz1 = (W2^T dz2) silu'(s1)
        {
            float dh[H];
#pragma unroll
            for (int k = 0; k < H; ++k) dh[k] = 0.f;
            const float *brow = B + t * LD;
#pragma unroll 4
            for (int j = 0; j < H; ++j) {
                const float dj = brow[j];
                const float4 *w4 = reinterpret_cast<const float4 *>(net + OW2 + j * H);
#pragma unroll
                for (int q = 0; q < H / 4; ++q) {
                    const float4 v = w4[q];
                    dh[4 * q] = fmaf(v.x, dj, dh[4 * q]);
                    dh[4 * q + 1] = fmaf(v.y, dj, dh[4 * q + 1]);
                    dh[4 * q + 2] = fmaf(v.z, dj, dh[4 * q + 2]);
                    dh[4 * q + 3] = fmaf(v.w, dj, dh[4 * q + 3]);
                }
            }
            float4 *a4 = reinterpret_cast<float4 *>(A + t * LD);
#pragma unroll
            for (int q = 0; q < H / 4; ++q) {
                float d[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int k = 4 * q + e;
                    d[e] = dh[k] * dsilu(layer1(net, k, x0, x1, x2));
                }
                a4[q] = make_float4(d[0], d[1], d[2], d[3]);
            }
        }
        __syncthreads();
        // ---- 6. db1, dW1
        if (t < H) {
            for (int pp = 0; pp < TB; ++pp) accB += A[pp * LD + t];
        } else {
            const int k = (t - H) / 3, i = (t - H) % 3;
            for (int pp = 0; pp < TB; ++pp) accB = fmaf(A[pp * LD + k], X[3 * pp + i], accB);
        }
        __syncthreads();
    }
    float *out = work + (size_t)blockIdx.x * NSLOT;
#pragma unroll
    for (int q = 0; q < 16; ++q) out[OW2 + rj * H + rk + q] = acc2[q];
    if (t < H) {
        out[OB2 + t] = accA;
        out[OB1 + t] = accB;
    } else {
        const int k = (t - H) / 3, i = (t - H) % 3;
        out[OW1 + 3 * k + i] = accB;
        if (t < 2 * H) out[OW3 + (t - H)] = accA;
        else if (t == 2 * H) out[OB3] = accA;
        else if (t == 2 * H + 1) out[NPAR] = accA;
    }
}

// grad[i] = sum over blocks of work[b][i] (fixed order, FP64), loss likewise
__global__ void k_mlp_grad_finish(const float *__restrict__ work, int nblk, float *__restrict__ grad,
                                  double *__restrict__ loss)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NSLOT) return;
    double s = 0;
    for (int b = 0; b < nblk; ++b) s += work[(size_t)b * NSLOT + i];
    if (i < NPAR) grad[i] = (float)s;
    else if (loss) *loss = s;
}

// Adam (Kingma & Ba, 2015): m, v moments; bc1 = 1/(1 - b1^t), bc2 = 1/(1 - b2^t)
__global__ void k_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ g, int n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * bc1) / (sqrtf(vi * bc2) + eps);
}

constexpr size_t grad_smem_bytes()
{
    return sizeof(float) * (((NPAR + 3) / 4) * 4 + 2 * TB * LD + TB * 3 + 2 * TB);
}

int grad_blocks()
{
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return -1;
    return nsm;
}

}  // namespace

namespace {

// ---- forward on the 5th-generation tensor cores ---------------------------
// The 64 x 64 layer as one tcgen05 MMA chain per tile of 128 points: A = the
// tile's h1 (bf16, 128 x 64, K-major), B = W2 (bf16, 64 x 64, K-major), D =
// the FP32 accumulators in tensor memory (128 lanes x 64 columns), read back
// with tcgen05.ld for the epilogue (+ b2, SiLU, W3, b3) in FP32.  Layer 1 and
// the epilogue run on the CUDA cores as in k_mlp_forward; the difference is
// that h1 enters the MMA rounded to bf16 (the weights are bf16 in both).
//
// Shared-memory operands use the no-swizzle K-major canonical layout: core
// matrices of 8 rows x 16 bytes (8 bf16 of K), row group g and K chunk c at
// byte (8 g + c) * 128, row r of the group at + 16 r.  One MMA covers K = 16,
// i.e. chunks 2s and 2s + 1: leading (K) byte offset 128, stride (row group)
// byte offset 1024.  Descriptor and instruction-descriptor bit layouts follow
// the sm_100 UMMA definitions (CUTLASS cute/arch/mma_sm100_desc.hpp).
constexpr int TCM = 128;                          // points (MMA rows) per tile
constexpr int TC_A = 0, TC_B = TCM * H * 2;       // byte offsets: A 16 KB, B 8 KB
constexpr int TC_NET = TC_B + H * H * 2;          // FP32 parameters
constexpr int TC_BAR = TC_NET + ((NPAR + 3) / 4) * 16;
constexpr int TC_SMEM = TC_BAR + 32;              // + mbarrier, the TMEM address, the check's mbarrier
constexpr int TC_SPIN = 1 << 22;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    // start address >> 4 [0,14), leading byte offset >> 4 [16,30), stride byte
    // offset >> 4 [32,46), version 1 [46,48), layout SWIZZLE_NONE (0) [61,64)
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
           (1ull << 46);
}
// c_format F32 [4,6) = 1, a_format BF16 [7,10) = 1, b_format BF16 [10,13) = 1,
// K-major A and B, n_dim = N >> 3 [17,23), m_dim = M >> 4 [24,29)
constexpr uint32_t TC_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(H >> 3) << 17) | ((uint32_t)(TCM >> 4) << 24);

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);   // .x = a (low half), .y = b
    return *reinterpret_cast<const uint32_t *>(&v);
}

__global__ void __launch_bounds__(TCM) k_mlp_forward_tc(const float *__restrict__ params, const float *__restrict__ x,
                                                        float *__restrict__ z, size_t npts, int *__restrict__ err,
                                                        int spin = TC_SPIN, int check = 0)
{
    // check != 0 (the status test only): the threads first wait on a second
    // barrier that nothing arrives at, so that wait runs out on purpose; the
    // failure path then waits for the MMAs' own barrier before the tensor
    // memory is released
    extern __shared__ __align__(1024) unsigned char smc[];
    float *net = reinterpret_cast<float *>(smc + TC_NET);
    const int t = threadIdx.x, warp = t >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smc);
    const uint32_t bar = sbase + TC_BAR, slot = sbase + TC_BAR + 8, bar2 = sbase + TC_BAR + 16;
    stage_params(net, params, 1);
    // B: W2 rows (outputs) x K chunks of 8, bf16
    for (int e = t; e < H * (H / 8); e += TCM) {
        const int n = e / (H / 8), c = e % (H / 8);
        const float *w = params + OW2 + n * H + 8 * c;
        const uint4 q = make_uint4(pack_bf16x2(w[0], w[1]), pack_bf16x2(w[2], w[3]), pack_bf16x2(w[4], w[5]),
                                   pack_bf16x2(w[6], w[7]));
        *reinterpret_cast<uint4 *>(smc + TC_B + ((n / 8) * 8 + c) * 128 + (n % 8) * 16) = q;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(H));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar2) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const uint32_t tmem = *reinterpret_cast<const uint32_t *>(smc + TC_BAR + 8);
    // layer 1 for this thread's point (row t of A)
    const size_t pidx = (size_t)blockIdx.x * TCM + t;
    float x0 = 0.f, x1 = 0.f, x2 = 0.f;
    if (pidx < npts) {
        x0 = x[3 * pidx];
        x1 = x[3 * pidx + 1];
        x2 = x[3 * pidx + 2];
    }
#pragma unroll
    for (int c = 0; c < H / 8; ++c) {
        float h[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) h[i] = silu(layer1(net, 8 * c + i, x0, x1, x2));
        const uint4 q = make_uint4(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]), pack_bf16x2(h[4], h[5]),
                                   pack_bf16x2(h[6], h[7]));
        *reinterpret_cast<uint4 *>(smc + TC_A + ((t / 8) * 8 + c) * 128 + (t % 8) * 16) = q;
    }
    // the threads' shared-memory writes, then the MMAs (async proxy) that read them
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for (int s = 0; s < H / 16; ++s) {
            const uint64_t da = umma_desc(sbase + TC_A + s * 256), db = umma_desc(sbase + TC_B + s * 256);
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(TC_IDESC), "r"(s), "r"(0), "r"(0), "r"(0), "r"(0)
                : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                     : "memory");
    }
    auto wait = [&](uint32_t b, int limit) {
        unsigned ok = 0;
        for (int it = 0; it < limit && !ok; ++it)
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}\n"
                         : "=r"(ok)
                         : "r"(b)
                         : "memory");
        return ok;
    };
    const unsigned done = wait(check ? bar2 : bar, spin);
    if (done) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t row = tmem + ((uint32_t)(32 * warp) << 16);   // this warp's lane quarter
        float acc = net[OB3];
#pragma unroll
        for (int q = 0; q < H / 16; ++q) {
            uint32_t r[16];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
                         "%12, %13, %14, %15}, [%16];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                           "=r"(r[14]), "=r"(r[15])
                         : "r"(row + 16 * q));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int j = 16 * q + i;
                acc = fmaf(net[OW3 + j], silu(__uint_as_float(r[i]) + net[OB2 + j]), acc);
            }
        }
        if (pidx < npts) z[pidx] = acc;
    } else {
        if (t == 0) atomicExch(err, 1);
        wait(bar, TC_SPIN);   // the MMAs still write tensor memory: let them finish before it is released
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(H));
}

}  // namespace

extern "C" int pt_mlp_check_tc_wait(const float *params, const float *x, float *z, int *err, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(params && x && z && err, "mlp_check_tc_wait: null pointer");
    PT_CUDA(cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    k_mlp_forward_tc<<<1, TCM, TC_SMEM, (cudaStream_t)stream>>>(params, x, z, TCM, err, 256, 1);
    PT_LAUNCHED("k_mlp_forward_tc");
    return PT_OK;
}

extern "C" int pt_mlp_forward_tc(const float *params, const float *x, float *z, size_t npts, int *err, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(params && x && z && err, "mlp_forward_tc: null pointer");
    if (npts == 0) return PT_OK;
    static bool attr = false;
    if (!attr) {
        PT_CUDA(cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
        attr = true;
    }
    const size_t blocks = (npts + TCM - 1) / TCM;
    PT_CHECK_ARG(blocks < (1u << 31), "mlp_forward_tc: too many points");
    k_mlp_forward_tc<<<(unsigned)blocks, TCM, TC_SMEM, (cudaStream_t)stream>>>(params, x, z, npts, err);
    PT_LAUNCHED("k_mlp_forward_tc");
    return PT_OK;
}

extern "C" int pt_mlp_param_count(void) { return NPAR; }

extern "C" size_t pt_mlp_workspace_bytes(void) { return (size_t)1024 * NSLOT * sizeof(float); }

extern "C" int pt_mlp_forward(const float *params, int bf16, const float *x, float *z, size_t npts, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(params && x && z, "mlp_forward: null pointer");
    if (npts == 0) return PT_OK;
    size_t b = (npts + TB - 1) / TB;
    const unsigned grid = (unsigned)(b < 148 * 8 ? b : 148 * 8);
    k_mlp_forward<<<grid, TB, 0, (cudaStream_t)stream>>>(params, bf16, x, z, npts);
    PT_LAUNCHED("k_mlp_forward");
    return PT_OK;
}

extern "C" int pt_mlp_grad(const float *params, int bf16, const float *x, const float *y, const float *w, size_t npts,
                           float inv_wsum, float *grad, double *loss, void *work, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(params && x && y && w && grad && work, "mlp_grad: null pointer");
    int nblk = grad_blocks();
    if (nblk < 0) {
        pt::set_error("mlp_grad: device query failed: %s", cudaGetErrorString(cudaGetLastError()));
        return PT_ERR_CUDA;
    }
    if (nblk > 1024) nblk = 1024;   // the workspace holds 1024 partial sets
    const size_t tiles = (npts + TB - 1) / TB;
    if ((size_t)nblk > tiles) nblk = (int)(tiles ? tiles : 1);
    PT_CUDA(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem_bytes()));
    cudaStream_t st = (cudaStream_t)stream;
    k_mlp_grad<<<nblk, TB, grad_smem_bytes(), st>>>(params, bf16, x, y, w, npts, inv_wsum, (float *)work);
    PT_LAUNCHED("k_mlp_grad");
    k_mlp_grad_finish<<<(NSLOT + 255) / 256, 256, 0, st>>>((const float *)work, nblk, grad, loss);
    PT_LAUNCHED("k_mlp_grad_finish");
    return PT_OK;
}

extern "C" int pt_mlp_adam(float *params, float *m, float *v, const float *grad, int step, float lr, float beta1,
                           float beta2, float eps, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(params && m && v && grad && step >= 1, "mlp_adam: bad arguments");
    const float bc1 = (float)(1.0 / (1.0 - std::pow((double)beta1, step)));
    const float bc2 = (float)(1.0 / (1.0 - std::pow((double)beta2, step)));
    k_adam<<<(NPAR + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, m, v, grad, NPAR, lr, beta1, beta2, eps, bc1,
                                                                 bc2);
    PT_LAUNCHED("k_adam");
    return PT_OK;
}
