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

// 16-point DFT as 4 x 4 (n = 4 n1 + n2, k = k1 + 4 k2), natural-order output.
template <int DIR>
struct Dft<16, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float c1 = 0.92387953251128675613f;  // cos(pi/8)
        const float s1 = 0.38268343236508977173f;  // sin(pi/8)
        const float h = 0.70710678118654752440f;
        const float d = (float)DIR;
        float2 a[4][4];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
            a[n2][0] = v[n2];
            a[n2][1] = v[4 + n2];
            a[n2][2] = v[8 + n2];
            a[n2][3] = v[12 + n2];
            dft4<DIR>(a[n2][0], a[n2][1], a[n2][2], a[n2][3]);
        }
        // a[n2][k1] *= W16^(n2 k1), W16 = exp(DIR 2 pi i / 16)
        a[1][1] = cmul(a[1][1], make_float2(c1, d * s1));
        a[1][2] = cmul(a[1][2], make_float2(h, d * h));
        a[1][3] = cmul(a[1][3], make_float2(s1, d * c1));
        a[2][1] = cmul(a[2][1], make_float2(h, d * h));
        a[2][2] = mul_i<DIR>(a[2][2]);
        a[2][3] = cmul(a[2][3], make_float2(-h, d * h));
        a[3][1] = cmul(a[3][1], make_float2(s1, d * c1));
        a[3][2] = cmul(a[3][2], make_float2(-h, d * h));
        a[3][3] = cmul(a[3][3], make_float2(-c1, -d * s1));
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 b0 = a[0][k1], b1 = a[1][k1], b2 = a[2][k1], b3 = a[3][k1];
            dft4<DIR>(b0, b1, b2, b3);
            v[k1] = b0;
            v[k1 + 4] = b1;
            v[k1 + 8] = b2;
            v[k1 + 12] = b3;
        }
    }
};

// cos(j pi / 16) for j = 0..8
__host__ __device__ constexpr float cos_pi16(int j)
{
    return j == 0   ? 1.0f
           : j == 1 ? 0.98078528040323044913f
           : j == 2 ? 0.92387953251128675613f
           : j == 3 ? 0.83146961230254523708f
           : j == 4 ? 0.70710678118654752440f
           : j == 5 ? 0.55557023301960222474f
           : j == 6 ? 0.38268343236508977173f
           : j == 7 ? 0.19509032201612826785f
                    : 0.0f;
}

// z * W32^j, W32 = exp(DIR 2 pi i / 32), for a compile-time 0 <= j < 24
template <int DIR>
__device__ __forceinline__ float2 mul_w32(float2 z, int j)
{
    if (j == 0) return z;
    if (j == 8) return mul_i<DIR>(z);
    if (j == 16) return make_float2(-z.x, -z.y);
    // angle j pi / 16 by quadrant: (cos, sin)
    const float c = j < 8 ? cos_pi16(j) : j < 16 ? -cos_pi16(16 - j) : -cos_pi16(j - 16);
    const float s = j < 8 ? cos_pi16(8 - j) : j < 16 ? cos_pi16(j - 8) : -cos_pi16(24 - j);
    return cmul(z, make_float2(c, DIR * s));
}

// 32-point DFT as 4 x 8 (n = 4 n1 + n2, k = k1 + 8 k2), natural-order output.
template <int DIR>
struct Dft<32, DIR> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 a[4][8];
#pragma unroll
        for (int n2 = 0; n2 < 4; ++n2) {
#pragma unroll
            for (int n1 = 0; n1 < 8; ++n1) a[n2][n1] = v[4 * n1 + n2];
            Dft<8, DIR>::run(a[n2]);
        }
#pragma unroll
        for (int n2 = 1; n2 < 4; ++n2)
#pragma unroll
            for (int k1 = 1; k1 < 8; ++k1) a[n2][k1] = mul_w32<DIR>(a[n2][k1], n2 * k1);
#pragma unroll
        for (int k1 = 0; k1 < 8; ++k1) {
            dft4<DIR>(a[0][k1], a[1][k1], a[2][k1], a[3][k1]);
            v[k1] = a[0][k1];
            v[k1 + 8] = a[1][k1];
            v[k1 + 16] = a[2][k1];
            v[k1 + 24] = a[3][k1];
        }
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

// The same transform for NQ interleaved sequences: element i of sequence q
// at buf[i * NQ + q] (one row of NQ values per index).  Thread (q, b) of the
// block, q = t % NQ, b = t / NQ, runs butterflies b, b + TB, ... of sequence
// q, so a warp reads and writes rows of consecutive values (no bank
// conflicts) and the lanes of one row share their twiddle (one broadcast
// load).  Same butterflies, twiddles and order as pass/fft: bit-identical
// results.
template <int L, int R, int NS, int DIR, int TB, int NQ>
__device__ __forceinline__ void pass_iq(float2 *buf, int q, int b, const float2 *__restrict__ tw)
{
    constexpr int NB = L / R;
    constexpr int PER = (NB + TB - 1) / TB;
    float2 v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int j = b + p * TB;
        if ((NB % TB == 0) || j < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[p][r] = buf[(j + r * NB) * NQ + q];
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int j = b + p * TB;
        if ((NB % TB == 0) || j < NB) {
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
            for (int r = 0; r < R; ++r) buf[(base + r * NS) * NQ + q] = v[p][r];
        }
    }
    __syncthreads();
}

template <int L, int DIR, int TB, int NQ, int I = 0, int NS = 1>
__device__ __forceinline__ void fft_iq(float2 *buf, int q, int b, const float2 *__restrict__ tw)
{
    static_assert(supported_len(L), "FFT length must be 2^a 3^b");
    if constexpr (I < num_passes(L)) {
        constexpr int R = radix_at(L, I);
        pass_iq<L, R, NS, DIR, TB, NQ>(buf, q, b, tw);
        fft_iq<L, DIR, TB, NQ, I + 1, NS * R>(buf, q, b, tw);
    }
}

}  // namespace ptfft

// Host helper: fill tw[m] = exp(-2 pi i m / L), m < L (double precision).
void pt_make_twiddles(float2 *host_tw, int L);
