// ics.cu — Zel'dovich initial conditions on the GPU (ics.rs:78-182).
//
// White noise: one N(0,1) value per cell from Philox-4x32-10 (Salmon et al., SC'11; counter =
// cell index, key = seed) and Box-Muller in double precision, rounded to f32. (The reference
// draws from rand's StdRng + rand_distr's StandardNormal; that stream is not reproduced.) The
// noise is transformed with the n^3 c2c FFT, coloured by sqrt(n^3 P(k) / V) with the BBKS
// spectrum (ics.rs:89-107), and the displacement Psi_k = i k F_k / k^2 of each axis is
// inverse-transformed (ics.rs:133-154). Positions x = (q + D Psi) mod L and momenta
// p = a^2 f E D Psi (ics.rs:156-180). Scalars follow the reference's f32 operation order.
#include <cmath>
#include <string>

#include "cpm_host.h"
#include "cpm_internal.cuh"

namespace cpm {

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(0xD2511F53u, c[0]), lo0 = 0xD2511F53u * c[0];
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c[2]), lo1 = 0xCD9E8D57u * c[2];
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n1 = lo1, n2 = hi0 ^ c[3] ^ k1, n3 = lo0;
    c[0] = n0;
    c[1] = n1;
    c[2] = n2;
    c[3] = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

__global__ void k_white_noise(float2* __restrict__ out, size_t n3, uint64_t seed) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t c[4] = {(uint32_t)i, (uint32_t)(i >> 32), 0u, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u1 = ((double)c[0] + 1.0) * (1.0 / 4294967296.0);
    const double u2 = (double)c[1] * (1.0 / 4294967296.0);
    const double g = sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
    out[i] = make_float2((float)g, 0.0f);
  }
}

struct IcParams {
  int n;
  float two_pi_over_l;
  float n3f;       // (f32) n^3
  float volume;    // L^3 (f32)
  float amplitude;
  float n_s;
  float omega_m_h; // omega_m * (h0 / 100)
};

// cosmology.rs:94-103 on the device (f32; powi expanded as x*x, x*(x*x), (x*x)*(x*x)).
__device__ __forceinline__ float bbks_dev(float k, float omega_m_h) {
  const float q = __fdiv_rn(k, omega_m_h);
  if (q == 0.0f) return 1.0f;
  const float x2 = __fmul_rn(16.1f, q), x3 = __fmul_rn(5.46f, q), x4 = __fmul_rn(6.71f, q);
  const float x4s = __fmul_rn(x4, x4);
  float poly = __fadd_rn(1.0f, __fmul_rn(3.89f, q));
  poly = __fadd_rn(poly, __fmul_rn(x2, x2));
  poly = __fadd_rn(poly, __fmul_rn(x3, __fmul_rn(x3, x3)));
  poly = __fadd_rn(poly, __fmul_rn(x4s, x4s));
  const float t = __fmul_rn(2.34f, q);
  return __fmul_rn(__fdiv_rn(log1pf(t), t), powf(poly, -0.25f));
}

// ics.rs:89-107: F_k *= sqrt(n^3 P(|k|) / V); k = 0 dropped.
__global__ void k_color(float2* __restrict__ modes, int n, IcParams p) {
  const size_t n3 = (size_t)n * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n3; idx += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(idx % n), iy = (int)((idx / n) % n), ix = (int)(idx / ((size_t)n * n));
    const float kx = wavenumber(ix, n, p.two_pi_over_l), ky = wavenumber(iy, n, p.two_pi_over_l),
                kz = wavenumber(iz, n, p.two_pi_over_l);
    float k2 = -0.0f;
    k2 = __fadd_rn(k2, __fmul_rn(kx, kx));
    k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
    k2 = __fadd_rn(k2, __fmul_rn(kz, kz));
    const float k_mag = sqrtf(k2);
    if (k_mag == 0.0f) {
      modes[idx] = make_float2(0.0f, 0.0f);
    } else {
      const float t = bbks_dev(k_mag, p.omega_m_h);
      const float pk = __fmul_rn(__fmul_rn(__fmul_rn(p.amplitude, powf(k_mag, p.n_s)), t), t);
      const float sc = sqrtf(__fdiv_rn(__fmul_rn(p.n3f, pk), p.volume));
      const float2 v = modes[idx];
      modes[idx] = make_float2(__fmul_rn(v.x, sc), __fmul_rn(v.y, sc));
    }
  }
}

// ics.rs:135-151: Psi_k[axis] = F_k * (0 + i k_axis) / k^2 (zero where k^2 = 0).
__global__ void k_psi_k(const float2* __restrict__ modes, float2* __restrict__ psi, int n, int axis, float tpl) {
  const size_t n3 = (size_t)n * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n3; idx += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(idx % n), iy = (int)((idx / n) % n), ix = (int)(idx / ((size_t)n * n));
    const float kx = wavenumber(ix, n, tpl), ky = wavenumber(iy, n, tpl), kz = wavenumber(iz, n, tpl);
    float k2 = -0.0f;
    k2 = __fadd_rn(k2, __fmul_rn(kx, kx));
    k2 = __fadd_rn(k2, __fmul_rn(ky, ky));
    k2 = __fadd_rn(k2, __fmul_rn(kz, kz));
    float2 out = make_float2(0.0f, 0.0f);
    if (k2 > 0.0f) {
      const float ka = axis == 0 ? kx : (axis == 1 ? ky : kz);
      const float2 m = modes[idx];
      // (m.re + i m.im)(0 + i ka) = (m.re*0 - m.im*ka) + i(m.re*ka + m.im*0)
      const float re = __fsub_rn(__fmul_rn(m.x, 0.0f), __fmul_rn(m.y, ka));
      const float im = __fadd_rn(__fmul_rn(m.x, ka), __fmul_rn(m.y, 0.0f));
      out = make_float2(__fdiv_rn(re, k2), __fdiv_rn(im, k2));
    }
    psi[idx] = out;
  }
}

// ics.rs:153-180 for one axis: psi = re / n^3; x = (q + D psi) mod L; p = ms psi.
__global__ void k_zeldovich_axis(const float2* __restrict__ psi_x, int n, int axis, float n3f, float h, float d,
                                 float ms, float box, float* __restrict__ x3, float* __restrict__ p3) {
  const size_t n3 = (size_t)n * n * n;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n3; idx += (size_t)gridDim.x * blockDim.x) {
    const int iz = (int)(idx % n), iy = (int)((idx / n) % n), ix = (int)(idx / ((size_t)n * n));
    const int iq = axis == 0 ? ix : (axis == 1 ? iy : iz);
    const float q = __fmul_rn((float)iq, h);
    const float psi = __fdiv_rn(psi_x[idx].x, n3f);
    x3[3 * idx + axis] = rem_euclid_f32(__fadd_rn(q, __fmul_rn(d, psi)), box);
    p3[3 * idx + axis] = __fmul_rn(ms, psi);
  }
}

cudaError_t generate_zeldovich(int n, float box, const cpm_cosmology& c, float n_s, float sigma8, float a_init,
                               uint64_t seed, float* x3_dev, float* p3_dev, DevBuf& modes, DevBuf& work,
                               FftPlan& plan, cudaStream_t s) {
  const size_t n3 = (size_t)n * n * n;
  cudaError_t e;
  if ((e = fft_plan_init(plan, n)) != cudaSuccess) return e;
  if ((e = ensure(modes, n3 * sizeof(float2))) != cudaSuccess) return e;
  if ((e = ensure(work, n3 * sizeof(float2))) != cudaSuccess) return e;
  const unsigned blocks = (unsigned)std::min<size_t>((n3 + 255) / 256, 148 * 16);
  float2* F = as<float2>(modes);
  float2* W = as<float2>(work);
  count_launch();
  k_white_noise<<<blocks, 256, 0, s>>>(F, n3, seed);
  launch_fft3_c2c(plan, F, 0, s);
  IcParams p;
  p.n = n;
  p.two_pi_over_l = 2.0f * (float)3.14159265358979323846 / box;
  p.n3f = (float)n3;
  p.volume = box * box * box;
  p.amplitude = power_amplitude(c, n_s, sigma8, 8.0f);
  p.n_s = n_s;
  p.omega_m_h = c.omega_m * (c.h0 / 100.0f);
  count_launch();
  k_color<<<blocks, 256, 0, s>>>(F, n, p);
  const float h = box / (float)n;
  const float d = growth(c, a_init);
  const float f = growth_rate(c, a_init);
  const float ee = cosmo_e(c, a_init);
  const float ms = a_init * a_init * f * ee * d;
  for (int axis = 0; axis < 3; ++axis) {
    count_launch();
    k_psi_k<<<blocks, 256, 0, s>>>(F, W, n, axis, p.two_pi_over_l);
    launch_fft3_c2c(plan, W, 1, s);
    count_launch();
    k_zeldovich_axis<<<blocks, 256, 0, s>>>(W, n, axis, p.n3f, h, d, ms, box, x3_dev, p3_dev);
  }
  return cudaGetLastError();
}

}  // namespace cpm

using namespace cpm;

extern "C" int cpm_ics_zeldovich(int n_side, float box_size, const cpm_cosmology* cosmo, float n_s, float sigma8,
                                 float a_init, uint64_t seed, float* x3, float* p3) {
  if (!cosmo || !x3 || !p3) return set_error(nullptr, CPM_E_INVALID, "cpm_ics_zeldovich: null pointer");
  if (!fft_supported(n_side))
    return set_error(nullptr, CPM_E_UNSUPPORTED,
                     "cpm_ics_zeldovich: n = " + std::to_string(n_side) + " is not one of " + fft_sizes_text());
  if (!(box_size > 0.0f) || !(a_init > 0.0f) || !(sigma8 > 0.0f))
    return set_error(nullptr, CPM_E_INVALID, "cpm_ics_zeldovich: box, a_init and sigma8 must be > 0");
  int rc = check_device_once(nullptr);
  if (rc) return rc;
  const size_t n3 = (size_t)n_side * n_side * n_side;
  cudaStream_t s = nullptr;
  DevBuf modes, work, xd, pd;
  FftPlan plan;
  auto cleanup = [&]() {
    release(modes);
    release(work);
    release(xd);
    release(pd);
    fft_plan_free(plan);
    if (s) cudaStreamDestroy(s);
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = ensure(xd, 3 * n3 * sizeof(float));
  if (e == cudaSuccess) e = ensure(pd, 3 * n3 * sizeof(float));
  if (e == cudaSuccess)
    e = generate_zeldovich(n_side, box_size, *cosmo, n_s, sigma8, a_init, seed, as<float>(xd), as<float>(pd), modes,
                           work, plan, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(x3, xd.p, 3 * n3 * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(p3, pd.p, 3 * n3 * sizeof(float), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cleanup();
  if (e != cudaSuccess)
    return set_error(nullptr, e == cudaErrorMemoryAllocation ? CPM_E_NOMEM : CPM_E_CUDA,
                     std::string("cpm_ics_zeldovich: ") + cudaGetErrorString(e));
  return CPM_OK;
}
