// pk.cu — matter power spectrum of a particle set (no reference counterpart: the reference bins
// the power of its initial modes only inside a test, ics.rs:213-266, whose estimator is restated
// here: P = V |delta_k|^2 / M^2 in integer shells round(|m|), ics.rs:229-243).
//
// The density comes from the CIC deposit (the simulation's u64 fixed-point mesh), delta =
// rho/mean - 1 is formed while the R2C transform loads it, and the padded half spectrum
// [n][n][n/2+2] is binned here. Each mode with 0 < kz < n/2 stands for itself and its
// Hermitian mirror (-m, same |m|, same |F|), so the sums equal those over the full spectrum;
// the kz = 0 and kz = n/2 planes hold each of their modes once. Nyquist modes are included, as in
// the oracle's estimator. Sums are FP64: per-block shared-memory histograms flushed with FP64
// atomics, so the last bits of a shell sum depend on the order the blocks finish in.
#include <cmath>
#include <cstring>

#include "cpm_internal.cuh"

namespace cpm {

constexpr int PK_THREADS = 256;
constexpr int PK_RUN = 8;  // consecutive kz of one line per thread, merged while in one shell

__global__ void __launch_bounds__(PK_THREADS) k_pk_bin(const float2* __restrict__ spec, int n, int n_shells,
                                                       PkSums* sums) {
  extern __shared__ double pk_sh[];
  double* sp = pk_sh;                   // [n_shells + 1]
  double* sk = pk_sh + (n_shells + 1);  // [n_shells + 1]
  unsigned int* sc = reinterpret_cast<unsigned int*>(pk_sh + 2 * (n_shells + 1));
  for (int s = threadIdx.x; s <= n_shells; s += blockDim.x) {
    sp[s] = 0.0;
    sk[s] = 0.0;
    sc[s] = 0u;
  }
  __syncthreads();
  const int nh = n / 2 + 1, nhp = n / 2 + 2;
  const int runs = (nh + PK_RUN - 1) / PK_RUN;
  const long long items = (long long)n * n * runs;
  const double smax = (double)n_shells + 0.5;
  auto flush = [&](int shell, double p, double k, unsigned c) {
    if (shell >= 1 && shell <= n_shells && c) {
      atomicAdd(&sp[shell], p);
      atomicAdd(&sk[shell], k);
      atomicAdd(&sc[shell], c);
    }
  };
  for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < items;
       it += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(it % runs);
    const long long line = it / runs;
    const int ix = (int)(line / n), iy = (int)(line % n);
    const long long mx = ix <= n / 2 ? ix : ix - n, my = iy <= n / 2 ? iy : iy - n;
    const long long mp2 = mx * mx + my * my;
    if ((double)mp2 > smax * smax) continue;
    int cur = -1;
    double ps = 0.0, ks = 0.0;
    unsigned c = 0;
    for (int q = 0; q < PK_RUN; ++q) {
      const int kz = r * PK_RUN + q;
      if (kz >= nh) break;
      const long long m2 = mp2 + (long long)kz * kz;
      const double mabs = sqrt((double)m2);
      const int shell = (int)rint(mabs);  // sqrt of an integer is never exactly half-integer
      if (shell > n_shells) break;        // shells grow with kz along a line
      const float2 F = spec[line * nhp + kz];
      const unsigned w = (kz == 0 || 2 * kz == n) ? 1u : 2u;
      if (shell != cur) {
        flush(cur, ps, ks, c);
        cur = shell;
        ps = ks = 0.0;
        c = 0;
      }
      ps += (double)w * ((double)F.x * (double)F.x + (double)F.y * (double)F.y);
      ks += (double)w * mabs;
      c += w;
    }
    flush(cur, ps, ks, c);
  }
  __syncthreads();
  for (int s = threadIdx.x; s <= n_shells; s += blockDim.x) {
    if (sc[s]) {
      atomicAdd(&sums->power[s], sp[s]);
      atomicAdd(&sums->kabs[s], sk[s]);
      atomicAdd(&sums->count[s], (unsigned long long)sc[s]);
    }
  }
}

void launch_pk_bin(const float2* spec, int n, int n_shells, PkSums* sums, cudaStream_t s) {
  cudaMemsetAsync(sums, 0, sizeof(PkSums), s);
  const size_t smem = (size_t)(n_shells + 1) * (2 * sizeof(double) + sizeof(unsigned int));
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_pk_bin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long items = (long long)n * n * ((n / 2 + 1 + PK_RUN - 1) / PK_RUN);
  const long long want = (items + PK_THREADS - 1) / PK_THREADS;
  const int grid = (int)std::max(1LL, std::min(want, (long long)sms * 4));
  count_launch();
  k_pk_bin<<<grid, PK_THREADS, smem, s>>>(spec, n, n_shells, sums);
}

void pk_finish(const PkSums& sums, int n, float box, int n_shells, double* k_mean, double* p_mean, uint64_t* counts) {
  const double m = (double)n * (double)n * (double)n;
  const double volume = (double)box * (double)box * (double)box;
  const double kf = 6.283185307179586476925286766559 / (double)box;
  for (int s = 1; s <= n_shells; ++s) {
    const unsigned long long c = sums.count[s];
    k_mean[s - 1] = c ? kf * sums.kabs[s] / (double)c : 0.0;
    p_mean[s - 1] = c ? volume * sums.power[s] / (m * m * (double)c) : 0.0;
    counts[s - 1] = c;
  }
}

}  // namespace cpm
