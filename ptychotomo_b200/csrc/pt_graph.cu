// Device-resident scalars of the ADMM iteration, so that one iteration can be
// captured as a CUDA graph and replayed with no host round trip (no
// counterpart in the reference, whose Solver, src/ptychotomo/solver.py:171-336,
// takes every step length, Dai-Yuan beta and penalty decision on the host).
//
// The scalars live in one device array of doubles (the "arena"); every
// reduction writes its result into a slot of it, and the small kernels below
// turn slots into the next step's scalars with the reference's rules:
//   * Dai-Yuan beta = ||g||^2 / <d, g - g0> (complex), solver.py:194-197;
//   * the tomography line search, solver.py:171-177 with minf of
//     solver.py:181-184: halve gamma while the decrease
//     -(2 g c1 + g^2 c2) < 0 and gamma > 1e-12 (c1, c2 of the closed form);
//   * the ptycho line search over passes of 2, 8 and 16 step lengths;
//   * takexi's background phase (solver.py:151-156) and max|t|;
//   * the penalty update, solver.py:267-282.
// Linear combinations then read their coefficients from the arena.
#include <cmath>

#include "pt_common.cuh"

namespace {

struct LinDev {
    const float2 *x[4];
};

// out = sum_{j<k} (coef[2j] + i coef[2j+1]) x_j with coefficients in device
// memory; nothing when skip_zero != null and *skip_zero == 0 (a correction
// the device found unnecessary)
__global__ void k_lincomb_dev(float2 *__restrict__ out, size_t n, int k, LinDev p, const double *__restrict__ coef,
                              const double *__restrict__ skip_zero)
{
    if (skip_zero != nullptr && *skip_zero == 0.0) return;
    float2 c[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) c[j] = j < k ? make_float2((float)coef[2 * j], (float)coef[2 * j + 1]) : czero();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 acc = czero();
        for (int j = 0; j < k; ++j) acc = acc + cmul(c[j], p.x[j][i]);
        out[i] = acc;
    }
}

// Scalar programs (one thread).  Slot layout is the caller's; every kernel
// documents the slots it reads and writes through its pointer arguments.

// d <- -g + beta d coefficients: coef = (-1, 0, beta_re, beta_im), with
// beta = ||g||^2 / (dg - dg0) (complex: dg, dg0 = <d, g>, <d, g0> as re, im
// pairs), 0 if the denominator is exactly 0 or first != 0 (first iteration)
__global__ void k_dy_beta(const double *__restrict__ g2, const double *__restrict__ dg,
                          const double *__restrict__ dg0, int first, double *__restrict__ coef)
{
    double br = 0, bi = 0;
    if (!first) {
        const double re = dg[0] - dg0[0], im = dg[1] - dg0[1];
        const double den = re * re + im * im;
        if (den != 0) {   // g2 / (re + i im)
            br = g2[0] * re / den;
            bi = -g2[0] * im / den;
        }
    }
    coef[0] = -1;
    coef[1] = 0;
    coef[2] = br;
    coef[3] = bi;
}

// tomography step: c1 = rho a_fd + tau b_gd, c2 = rho fd2 + tau gd2 (q1, q2 =
// the quad3 triples (|a|^2, Re<a, fd>, |fd|^2), (|b|^2, Re<b, gd>, |gd|^2));
// gamma halves while -(2 gamma c1 + gamma^2 c2) < 0 and gamma > 1e-12, then
// 0 if <= 1e-12.  Writes gamma (persisting) and coef = (1, 0, gamma, 0).
__global__ void k_tomo_gamma(const double *__restrict__ q1, const double *__restrict__ q2,
                             const double *__restrict__ rt, double *__restrict__ gamma, double *__restrict__ coef)
{
    const double rho = rt[0], tau = rt[1];
    const double c1 = rho * q1[1] + tau * q2[1], c2 = rho * q1[2] + tau * q2[2];
    double g = gamma[0];
    while (-(2 * g * c1 + g * g * c2) < 0 && g > 1e-12) g *= 0.5;
    if (g <= 1e-12) g = 0;
    gamma[0] = g;
    coef[0] = 1;
    coef[1] = 0;
    coef[2] = g;
    coef[3] = 0;
}

// ptycho line search over passes of J = 2, 8, 16 step lengths, as
// Solver.cg_ptycho: state = (accepted, step, gamma).  A pass's candidates
// are gamma 2^-j (j < J); once one passes, the later passes skip themselves
// (their reduction kernels read `accepted`).
__global__ void k_ls_begin(double *__restrict__ state)
{
    state[0] = 0;
    state[1] = 0;
    state[3] = state[2];   // the first pass's first step, by which it advances the frames
}

__global__ void k_ls_candidates(const double *__restrict__ state, int J, double *__restrict__ gam)
{
    const int j = threadIdx.x;
    if (j < J) gam[j] = state[2] * ldexp(1.0, -j);
}

// one pass's decision: the first j with !(dec_j < 0 && g_j > 1e-12),
// dec_j = data_j + rho (2 g_j w_d - g_j^2 d2), is taken (step 0 when
// g_j <= 1e-12); none: gamma <- g_{J-1} / 2 for the next pass.  No-op once
// a step was accepted.  quad = (|w|^2, Re<w, d>, |d|^2)
__global__ void k_ls_pass(const double *__restrict__ data, const double *__restrict__ gam, int J,
                          const double *__restrict__ quad, const double *__restrict__ rt, double *__restrict__ state)
{
    if (state[0] != 0) return;
    const double rho = rt[0], w_d = quad[1], d2 = quad[2];
    for (int j = 0; j < J; ++j) {
        const double g = gam[j];
        const double dec = data[j] + rho * (2 * g * w_d - g * g * d2);
        if (!(dec < 0 && g > 1e-12)) {
            const double step = g <= 1e-12 ? 0 : g;
            state[0] = 1;
            state[1] = step;
            state[2] = step;
            return;
        }
    }
    state[2] = gam[J - 1] * 0.5;
}

// after the first pass (which advanced the frames by gamma0 = state[3]): if
// it accepted no step, the later passes need the frames of psi itself:
// coef = (1, 0, -gamma0, 0) and state[3] <- 0; else coef = (1, 0, 0, 0),
// which the correction pass (skip_zero = &coef[2]) skips
__global__ void k_ls_unadvance(double *__restrict__ state, double *__restrict__ coef)
{
    coef[0] = 1;
    coef[1] = 0;
    coef[3] = 0;
    if (state[0] == 0) {
        coef[2] = -state[3];
        state[3] = 0;
    } else {
        coef[2] = 0;
    }
}

// coef = (1, 0, step, 0): the step taken (0 if no pass accepted one);
// corr = (1, 0, step - state[3], 0): what the frames, advanced by state[3],
// still need
__global__ void k_ls_end(const double *__restrict__ state, double *__restrict__ coef, double *__restrict__ corr)
{
    const double step = state[0] != 0 ? state[1] : 0.0;
    coef[0] = 1;
    coef[1] = 0;
    coef[2] = step;
    coef[3] = 0;
    corr[0] = 1;
    corr[1] = 0;
    corr[2] = step - state[3];
    corr[3] = 0;
}

// takexi scalars (solver.py:151-166): pshift = (m1 + m2) / 2 with
// m = band sum / cnt; coef for t = e psi - (e / rho) lamd, e = exp(-i pshift);
// pshift stored in out[0]
__global__ void k_takexi_scalars(const double *__restrict__ band1, const double *__restrict__ band2, double cnt,
                                 const double *__restrict__ rt, double *__restrict__ pshift,
                                 double *__restrict__ coef)
{
    const double p = (band1[0] / cnt + band2[0] / cnt) / 2;
    const double er = cos(-p), ei = sin(-p);
    const double rho = rt[0];
    pshift[0] = p;
    coef[0] = er;
    coef[1] = ei;
    coef[2] = -er / rho;
    coef[3] = -ei / rho;
}

// the ADMM multiplier-update coefficients: lamd + rho h - rho psi and
// mu + tau e - tau phi: coef_l = (1, 0, rho, 0, -rho, 0), coef_m likewise
__global__ void k_multiplier_coefs(const double *__restrict__ rt, double *__restrict__ coef_l,
                                   double *__restrict__ coef_m)
{
    const double rho = rt[0], tau = rt[1];
    const double cl[6] = {1, 0, rho, 0, -rho, 0}, cm[6] = {1, 0, tau, 0, -tau, 0};
    for (int i = 0; i < 6; ++i) {
        coef_l[i] = cl[i];
        coef_m[i] = cm[i];
    }
}

// penalty update (solver.py:267-282) from r1 = ||psi - h||^2, s1' = ||h - h0||^2,
// r2 = ||phi - e||^2, s2' = ||e - e0||^2: s = rho^2 s1' (tau^2 s2');
// x2 if r > 10 s, x0.5 if s > 10 r
__global__ void k_penalty(const double *__restrict__ r1, const double *__restrict__ s1,
                          const double *__restrict__ r2, const double *__restrict__ s2, double *__restrict__ rt)
{
    double rho = rt[0], tau = rt[1];
    double s = rho * rho * s1[0];
    if (r1[0] > 10 * s) rho *= 2;
    else if (s > 10 * r1[0]) rho *= 0.5;
    s = tau * tau * s2[0];
    if (r2[0] > 10 * s) tau *= 2;
    else if (s > 10 * r2[0]) tau *= 0.5;
    rt[0] = rho;
    rt[1] = tau;
}

// preconditioned CG (exact steps): beta = gz / gz0 (Fletcher-Reeves form), 0
// after a restart (restart[0] != 0) or on the first iteration; coef =
// (-1, 0, beta, 0); gz0 <- gz
__global__ void k_pcg_beta(const double *__restrict__ gz, double *__restrict__ gz0, double *__restrict__ restart,
                           int first, double *__restrict__ coef)
{
    const double b = (first || restart[0] != 0 || !(gz0[0] > 0)) ? 0.0 : gz[0] / gz0[0];
    gz0[0] = gz[0];
    restart[0] = 0;
    coef[0] = -1;
    coef[1] = 0;
    coef[2] = b;
    coef[3] = 0;
}

// exact step along d: gamma = -c1 / c2 if it descends, else 0 and restart;
// c1, c2 from the quad3 triples as k_tomo_gamma
__global__ void k_pcg_step(const double *__restrict__ q1, const double *__restrict__ q2,
                           const double *__restrict__ rt, double *__restrict__ restart, double *__restrict__ coef)
{
    const double rho = rt[0], tau = rt[1];
    const double c1 = rho * q1[1] + tau * q2[1], c2 = rho * q1[2] + tau * q2[2];
    const bool ok = c1 < 0 && c2 > 0;
    restart[0] = ok ? 0.0 : 1.0;
    coef[0] = 1;
    coef[1] = 0;
    coef[2] = ok ? -c1 / c2 : 0.0;
    coef[3] = 0;
}

// rk_tau = (rho * |K|^2 / count, tau) for the preconditioner
__global__ void k_pcg_rk(const double *__restrict__ k2, double count, const double *__restrict__ rt,
                         double *__restrict__ rk_tau)
{
    rk_tau[0] = rt[0] * k2[0] / count;
    rk_tau[1] = rt[1];
}

// coef = (a, 0, b * s[0], 0) for lincomb terms scaled by a device scalar:
// used for rho * g + tau * J^T b (s = rt) and for the ADMM's running sums
__global__ void k_coef2(const double *__restrict__ s0, double a0, const double *__restrict__ s1, double a1,
                        double *__restrict__ coef)
{
    coef[0] = s0 ? a0 * s0[0] : a0;
    coef[1] = 0;
    coef[2] = s1 ? a1 * s1[0] : a1;
    coef[3] = 0;
}

// out = (a / x[0], 0)
__global__ void k_inv(const double *__restrict__ x, double a, double *__restrict__ out)
{
    out[0] = a / x[0];
    out[1] = 0;
}

// out = exp(i s x) exp(i phi[0])  (phi from the arena)
__global__ void k_expmap_dev(float2 *__restrict__ out, const float2 *__restrict__ x, size_t n, float s,
                             const double *__restrict__ phi)
{
    float cp, sp;
    sincosf((float)phi[0], &sp, &cp);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float2 v = x[i];
        const float mag = expf(-s * v.y);
        float sn, cs;
        sincosf(s * v.x, &sn, &cs);
        out[i] = cmul(make_float2(mag * cs, mag * sn), make_float2(cp, sp));
    }
}

// takexi with 1/max|t| from the arena (k_takexi of pt_solver.cu otherwise)
__global__ void k_takexi_dev(float2 *__restrict__ K, float2 *__restrict__ xi0, const float2 *__restrict__ t, size_t n,
                             const double *__restrict__ tmax, float cxi)
{
    const float inv_tmax = (float)(1.0 / tmax[0]);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float2 v = t[i];
        const float kx = -v.y * inv_tmax, ky = v.x * inv_tmax;
        const float a = hypotf(v.x, v.y);
        if (a < 1e-32f) v = make_float2(1e-32f, 0.f);
        const float lr = logf(fmaxf(a, 1e-32f)), li = a < 1e-32f ? 0.f : atan2f(v.y, v.x);
        const float2 m = make_float2(li * cxi, -lr * cxi);
        K[i] = make_float2(kx, ky);
        xi0[i] = cmul(make_float2(kx, ky), m);
    }
}

// solve_reg (solver.py:257-264) with 1/tau and alpha/tau from the arena's tau
__global__ void k_solve_reg_dev(float2 *__restrict__ z, const float2 *__restrict__ u, const float2 *__restrict__ mu,
                                int nz, int ny, int nx, float s, const double *__restrict__ rt, float alpha)
{
    const float inv_tau = (float)(1.0 / rt[1]), thr = (float)(alpha / rt[1]);
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

extern "C" int pt_lincomb_dev_c64(void *out, size_t n, int k, const void *const *x, const double *coef,
                                  const double *skip_zero, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x && coef && k >= 1 && k <= 4, "lincomb_dev: 1..4 terms");
    LinDev p;
    for (int j = 0; j < 4; ++j) {
        p.x[j] = j < k ? (const float2 *)x[j] : nullptr;
        PT_CHECK_ARG(j >= k || p.x[j], "lincomb_dev: null term %d", j);
    }
    k_lincomb_dev<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, n, k, p, coef, skip_zero);
    PT_LAUNCHED("k_lincomb_dev");
    return PT_OK;
}

extern "C" int pt_scalar_dy_beta(const double *g2, const double *dg, const double *dg0, int first, double *coef,
                                 void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(g2 && dg && dg0 && coef, "scalar_dy_beta: null pointer");
    k_dy_beta<<<1, 1, 0, (cudaStream_t)stream>>>(g2, dg, dg0, first, coef);
    PT_LAUNCHED("k_dy_beta");
    return PT_OK;
}

extern "C" int pt_scalar_tomo_gamma(const double *q1, const double *q2, const double *rt, double *gamma, double *coef,
                                    void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(q1 && q2 && rt && gamma && coef, "scalar_tomo_gamma: null pointer");
    k_tomo_gamma<<<1, 1, 0, (cudaStream_t)stream>>>(q1, q2, rt, gamma, coef);
    PT_LAUNCHED("k_tomo_gamma");
    return PT_OK;
}

extern "C" int pt_scalar_ls_begin(double *state, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(state, "scalar_ls_begin: null pointer");
    k_ls_begin<<<1, 1, 0, (cudaStream_t)stream>>>(state);
    PT_LAUNCHED("k_ls_begin");
    return PT_OK;
}

extern "C" int pt_scalar_ls_candidates(const double *state, int J, double *gam, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(state && gam && J >= 1 && J <= 16, "scalar_ls_candidates: bad arguments");
    k_ls_candidates<<<1, 32, 0, (cudaStream_t)stream>>>(state, J, gam);
    PT_LAUNCHED("k_ls_candidates");
    return PT_OK;
}

extern "C" int pt_scalar_ls_pass(const double *data, const double *gam, int J, const double *quad, const double *rt,
                                 double *state, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(data && gam && quad && rt && state && J >= 1 && J <= 16, "scalar_ls_pass: bad arguments");
    k_ls_pass<<<1, 1, 0, (cudaStream_t)stream>>>(data, gam, J, quad, rt, state);
    PT_LAUNCHED("k_ls_pass");
    return PT_OK;
}

extern "C" int pt_scalar_ls_unadvance(double *state, double *coef, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(state && coef, "scalar_ls_unadvance: null pointer");
    k_ls_unadvance<<<1, 1, 0, (cudaStream_t)stream>>>(state, coef);
    PT_LAUNCHED("k_ls_unadvance");
    return PT_OK;
}

extern "C" int pt_scalar_ls_end(const double *state, double *coef, double *corr, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(state && coef && corr, "scalar_ls_end: null pointer");
    k_ls_end<<<1, 1, 0, (cudaStream_t)stream>>>(state, coef, corr);
    PT_LAUNCHED("k_ls_end");
    return PT_OK;
}

extern "C" int pt_scalar_takexi(const double *band1, const double *band2, double cnt, const double *rt, double *pshift,
                                double *coef, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(band1 && band2 && rt && pshift && coef && cnt > 0, "scalar_takexi: bad arguments");
    k_takexi_scalars<<<1, 1, 0, (cudaStream_t)stream>>>(band1, band2, cnt, rt, pshift, coef);
    PT_LAUNCHED("k_takexi_scalars");
    return PT_OK;
}

extern "C" int pt_scalar_multipliers(const double *rt, double *coef_l, double *coef_m, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(rt && coef_l && coef_m, "scalar_multipliers: null pointer");
    k_multiplier_coefs<<<1, 1, 0, (cudaStream_t)stream>>>(rt, coef_l, coef_m);
    PT_LAUNCHED("k_multiplier_coefs");
    return PT_OK;
}

extern "C" int pt_scalar_penalty(const double *r1, const double *s1, const double *r2, const double *s2, double *rt,
                                 void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(r1 && s1 && r2 && s2 && rt, "scalar_penalty: null pointer");
    k_penalty<<<1, 1, 0, (cudaStream_t)stream>>>(r1, s1, r2, s2, rt);
    PT_LAUNCHED("k_penalty");
    return PT_OK;
}

extern "C" int pt_scalar_pcg_beta(const double *gz, double *gz0, double *restart, int first, double *coef,
                                  void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(gz && gz0 && restart && coef, "scalar_pcg_beta: null pointer");
    k_pcg_beta<<<1, 1, 0, (cudaStream_t)stream>>>(gz, gz0, restart, first, coef);
    PT_LAUNCHED("k_pcg_beta");
    return PT_OK;
}

extern "C" int pt_scalar_pcg_step(const double *q1, const double *q2, const double *rt, double *restart, double *coef,
                                  void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(q1 && q2 && rt && restart && coef, "scalar_pcg_step: null pointer");
    k_pcg_step<<<1, 1, 0, (cudaStream_t)stream>>>(q1, q2, rt, restart, coef);
    PT_LAUNCHED("k_pcg_step");
    return PT_OK;
}

extern "C" int pt_scalar_pcg_rk(const double *k2, double count, const double *rt, double *rk_tau, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(k2 && rt && rk_tau && count > 0, "scalar_pcg_rk: bad arguments");
    k_pcg_rk<<<1, 1, 0, (cudaStream_t)stream>>>(k2, count, rt, rk_tau);
    PT_LAUNCHED("k_pcg_rk");
    return PT_OK;
}

extern "C" int pt_scalar_coef2(const double *s0, double a0, const double *s1, double a1, double *coef, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(coef, "scalar_coef2: null pointer");
    k_coef2<<<1, 1, 0, (cudaStream_t)stream>>>(s0, a0, s1, a1, coef);
    PT_LAUNCHED("k_coef2");
    return PT_OK;
}

extern "C" int pt_scalar_inv(const double *x, double a, double *out, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(x && out, "scalar_inv: null pointer");
    k_inv<<<1, 1, 0, (cudaStream_t)stream>>>(x, a, out);
    PT_LAUNCHED("k_inv");
    return PT_OK;
}

extern "C" int pt_expmap_dev_c64(void *out, const void *x, size_t n, float s, const double *phi, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(out && x && phi, "expmap_dev: null pointer");
    k_expmap_dev<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)out, (const float2 *)x, n, s, phi);
    PT_LAUNCHED("k_expmap_dev");
    return PT_OK;
}

extern "C" int pt_takexi_dev_c64(void *K, void *xi0, const void *t, size_t n, const double *tmax, float cxi,
                                 void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(K && xi0 && t && tmax, "takexi_dev: null pointer");
    k_takexi_dev<<<ew_blocks(n), 256, 0, (cudaStream_t)stream>>>((float2 *)K, (float2 *)xi0, (const float2 *)t, n,
                                                                 tmax, cxi);
    PT_LAUNCHED("k_takexi_dev");
    return PT_OK;
}

extern "C" int pt_solve_reg_dev_c64(void *z, const void *u, const void *mu, int nz, int ny, int nx, float s,
                                    const double *rt, float alpha, void *stream)
{
    pt::clear_error();
    PT_CHECK_ARG(z && u && mu && rt && nz > 0 && ny > 0 && nx > 0, "solve_reg_dev: bad arguments");
    k_solve_reg_dev<<<ew_blocks((size_t)nz * ny * nx), 256, 0, (cudaStream_t)stream>>>(
        (float2 *)z, (const float2 *)u, (const float2 *)mu, nz, ny, nx, s, rt, alpha);
    PT_LAUNCHED("k_solve_reg_dev");
    return PT_OK;
}
