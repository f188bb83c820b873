// FP64 direct sum on the GPU (Examples/DirectComputation.cpp:104-142, pair math FP2PR::NonMutualParticles,
// Src/Kernels/P2P/FP2PR.hpp:45-69): every listed target against all n sources, i != j.  Used to score FMM
// results at sizes where the CPU direct sum is too slow.
#include "common.cuh"

namespace b200 {

namespace {

constexpr int DIRECT_THREADS = 256;

__global__ void direct_kernel(long long n, const double *__restrict__ x, const double *__restrict__ y,
                              const double *__restrict__ z, const double *__restrict__ q, long long nt,
                              const long long *__restrict__ targets, double *__restrict__ phi,
                              double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz) {
  __shared__ double sx[DIRECT_THREADS], sy[DIRECT_THREADS], sz[DIRECT_THREADS], sq[DIRECT_THREADS];
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = k < nt;
  const long long i = active ? (targets ? targets[k] : k) : -1;
  const double tx = active ? x[i] : 0, ty = active ? y[i] : 0, tz = active ? z[i] : 0, tq = active ? q[i] : 0;
  double pv = 0, gx = 0, gy = 0, gz = 0;
  for (long long b = 0; b < n; b += DIRECT_THREADS) {
    __syncthreads();
    const long long j = b + threadIdx.x;
    if (j < n) {
      sx[threadIdx.x] = x[j];
      sy[threadIdx.x] = y[j];
      sz[threadIdx.x] = z[j];
      sq[threadIdx.x] = q[j];
    }
    __syncthreads();
    const int cnt = (int)min((long long)DIRECT_THREADS, n - b);
    if (active)
      for (int s = 0; s < cnt; ++s) {
        if (b + s == i) continue;
        const double dx = tx - sx[s], dy = ty - sy[s], dz = tz - sz[s];
        double inv2 = 1.0 / (dx * dx + dy * dy + dz * dz);
        const double inv = sqrt(inv2);
        inv2 *= inv;
        inv2 *= tq * sq[s];
        gx += -dx * inv2;
        gy += -dy * inv2;
        gz += -dz * inv2;
        pv += inv * sq[s];
      }
  }
  if (active) {
    phi[k] = pv;
    fx[k] = gx;
    fy[k] = gy;
    fz[k] = gz;
  }
}

}  // namespace

b200fmm_status run_direct(long long n, const double *x, const double *y, const double *z, const double *q,
                          long long nt, const long long *targets, double *phi, double *fx, double *fy, double *fz,
                          cudaStream_t s) {
  direct_kernel<<<grid_for(nt, DIRECT_THREADS), DIRECT_THREADS, 0, s>>>(n, x, y, z, q, nt, targets, phi, fx, fy, fz);
  B200_CUDA(cudaGetLastError());
  return B200FMM_OK;
}

}  // namespace b200
