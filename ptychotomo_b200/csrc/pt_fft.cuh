// Block-cooperative complex64 FFTs held in shared memory.
//
// Stockham autosort formulation (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC'08): for a pass of
// radix R on a sequence of length L whose already-transformed sub-length is
// NS, butterfly j (0 <= j < L/R) reads x[j + r L/R], multiplies input r by
// W_{NS R}^{r (j mod NS)}, runs an R-point DFT and writes
// y[(j / NS) NS R + (j mod NS) + r NS].  After the last pass the output is in
// natural order.  Lengths are L = 2^a 3^b; passes run radix-3 first, then one
// radix-2 or radix-4 pass if a is not a multiple of 3, then radix-8.
//
// Unnormalised, like cuFFT C2C: DIR = -1 is exp(-2 pi i jk/L) (forward),
// DIR = +1 is exp(+2 pi i jk/L) (inverse).  Twiddles come from a table
// tw[m] = exp(-2 pi i m / L) computed in double on the host.
#pragma once

#include "pt_common.cuh"

namespace ptfft {

__host__ __device__ constexpr int pow3_of(int L) { return (L > 1 && L % 3 == 0) ? 1 + pow3_of(L / 3) : 0; }
__host__ __device__ constexpr int pow2_of(int L) { return (L > 1 && L % 2 == 0) ? 1 + pow2_of(L / 2) : 0; }
__host__ __device__ constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }
__host__ __device__ constexpr bool supported_len(int L)
{
    return L >= 2 && ipow(2, pow2_of(L)) * ipow(3, pow3_of(L)) == L;
}
__host__ __device__ constexpr int num_passes(int L)
{
    return pow3_of(L) + pow2_of(L) / 3 + (pow2_of(L) % 3 ? 1 : 0);
}
__host__ __device__ constexpr int radix_at(int L, int i)
{
    return i < pow3_of(L) ? 3
           : (pow2_of(L) % 3 && i == pow3_of(L)) ? (pow2_of(L) % 3 == 1 ? 2 : 4)
                                                  : 8;
}

// multiply by DIR * i
template <int DIR>
__device__ __forceinline__ float2 mul_i(float2 z)
{
    return DIR < 0 ? make_float2(z.y, -z.x) : make_float2(-z.y, z.x);
}

template <int R, int DIR>
struct Dft;

template <int DIR>
struct Dft<2, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <int DIR>
struct Dft<3, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float s3 = 0.86602540378443864676f;  // sin(pi/3)
        float2 t1 = v[1] + v[2];
        float2 t2 = v[0] - 0.5f * t1;
        float2 t3 = s3 * (v[1] - v[2]);
        v[0] = v[0] + t1;
        v[1] = t2 + mul_i<DIR>(t3);
        v[2] = t2 - mul_i<DIR>(t3);
    }
};

template <int DIR>
__device__ __forceinline__ void dft4(float2 &a, float2 &b, float2 &c, float2 &d)
{
    float2 t0 = a + c, t1 = a - c, t2 = b + d, t3 = mul_i<DIR>(b - d);
    a = t0 + t2;
    b = t1 + t3;
    c = t0 - t2;
    d = t1 - t3;
}

template <int DIR>
struct Dft<4, DIR> {
    static __device__ __forceinline__ void run(float2 *v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }
};

template <int DIR>
struct Dft<8, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float h = 0.70710678118654752440f;  // sqrt(2)/2
        float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<DIR>(e0, e1, e2, e3);
        dft4<DIR>(o0, o1, o2, o3);
        // W8^k o_k, W8 = exp(DIR 2 pi i / 8)
        o1 = h * (o1 + mul_i<DIR>(o1));
        o2 = mul_i<DIR>(o2);
        o3 = h * (mul_i<DIR>(o3) - o3);
        v[0] = e0 + o0;
        v[4] = e0 - o0;
        v[1] = e1 + o1;
        v[5] = e1 - o1;
        v[2] = e2 + o2;
        v[6] = e2 - o2;
        v[3] = e3 + o3;
        v[7] = e3 - o3;
    }
};

// One Stockham pass, in place in shared memory.  `buf` is this FFT's base,
// `es` the element stride, `t` the thread's index among the T threads that
// share this FFT.  All threads of the block must call it (it synchronises).
template <int L, int R, int NS, int DIR, int T>
__device__ __forceinline__ void pass(float2 *buf, int es, int t, const float2 *__restrict__ tw)
{
    constexpr int NB = L / R;
    constexpr int PER = (NB + T - 1) / T;
    float2 v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int j = t + p * T;
        if ((NB % T == 0) || j < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[p][r] = buf[(j + r * NB) * es];
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int j = t + p * T;
        if ((NB % T == 0) || j < NB) {
            const int k = j % NS;
            if (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    float2 w = __ldg(&tw[r * k * (L / (NS * R))]);
                    if (DIR > 0) w.y = -w.y;
                    v[p][r] = cmul(v[p][r], w);
                }
            }
            Dft<R, DIR>::run(v[p]);
            const int base = (j / NS) * NS * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(base + r * NS) * es] = v[p][r];
        }
    }
    __syncthreads();
}

template <int L, int DIR, int T, int I = 0, int NS = 1>
__device__ __forceinline__ void fft(float2 *buf, int es, int t, const float2 *__restrict__ tw)
{
    static_assert(supported_len(L), "FFT length must be 2^a 3^b");
    if constexpr (I < num_passes(L)) {
        constexpr int R = radix_at(L, I);
        pass<L, R, NS, DIR, T>(buf, es, t, tw);
        fft<L, DIR, T, I + 1, NS * R>(buf, es, t, tw);
    }
}

}  // namespace ptfft

// Host helper: fill tw[m] = exp(-2 pi i m / L), m < L (double precision).
void pt_make_twiddles(float2 *host_tw, int L);
