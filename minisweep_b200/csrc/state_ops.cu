// state_ops.cu -- device versions of the reference's state helpers:
// initialize_state and get_state_norms (array_operations.c:26-110).
//
// The norms are FP64 sums in a fixed tree order (deterministic run to run).
// The reference adds sequentially; both are exact whenever every term is an
// integer below 2^53, which holds for the built-in problem.
#include <cuda_runtime.h>

#include "internal.h"
#include "sweep_common.cuh"

namespace msb {

constexpr int kNormThreads = 256;
constexpr int kNormBlocks = 1184;  // 8 x 148 SMs

__global__ void __launch_bounds__(kNormThreads) norms_partial_kernel(const double* __restrict__ vi,
                                                                     const double* __restrict__ vo, size_t n,
                                                                     double* __restrict__ part) {
  double s = 0.0, d = 0.0;
  const size_t stride = (size_t)gridDim.x * blockDim.x * 2;
  for (size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 2; i < n; i += stride) {
    if (i + 1 < n) {
      const double2 a = __ldcs(reinterpret_cast<const double2*>(vi + i));
      const double2 b = __ldcs(reinterpret_cast<const double2*>(vo + i));
      const double d0 = a.x - b.x, d1 = a.y - b.y;
      s = __fma_rn(b.x, b.x, s);
      s = __fma_rn(b.y, b.y, s);
      d = __fma_rn(d0, d0, d);
      d = __fma_rn(d1, d1, d);
    } else {
      const double a = vi[i], b = vo[i], d0 = a - b;
      s = __fma_rn(b, b, s);
      d = __fma_rn(d0, d0, d);
    }
  }
  __shared__ double ss[kNormThreads], sd[kNormThreads];
  ss[threadIdx.x] = s;
  sd[threadIdx.x] = d;
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      ss[threadIdx.x] += ss[threadIdx.x + w];
      sd[threadIdx.x] += sd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ss[0];
    part[2 * blockIdx.x + 1] = sd[0];
  }
}

__global__ void norms_final_kernel(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  __shared__ double ss[kNormThreads], sd[kNormThreads];
  double s = 0.0, d = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) {
    s += part[2 * i];
    d += part[2 * i + 1];
  }
  ss[threadIdx.x] = s;
  sd[threadIdx.x] = d;
  __syncthreads();
  for (int w = kNormThreads / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      ss[threadIdx.x] += ss[threadIdx.x + w];
      sd[threadIdx.x] += sd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = ss[0];
    out[1] = sd[0];
  }
}

// Built-in initial state (quantities_testing.h:60-90), one thread per element
// pair in the reference layout; group ie of the array is global group
// ie_base + ie (an energy-group slice of a larger problem).
__global__ void init_state_kernel(double* __restrict__ v, int nx, int ny, int nz, int ne, int nm, int ie_base) {
  const size_t n = (size_t)nx * ny * nz * ne * nm * NU;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    size_t k = i;
    const int im = (int)(k % nm); k /= nm;
    const int iu = (int)(k % NU); k /= NU;
    const int ix = (int)(k % nx); k /= nx;
    const int iy = (int)(k % ny); k /= ny;
    const int ie = (int)(k % ne); k /= ne;
    const int iz = (int)k;
    v[i] = (double)(1 + im) * (double)d_scale_space(ix, iy, iz) * (double)d_scale_energy(ie_base + ie) *
           (double)d_scale_unknown(iu);
  }
}

}  // namespace msb

extern "C" int msb_state_norms_device(const double* vi_d, const double* vo_d, size_t n, double* normsq,
                                      double* normsqdiff, Env* env) {
  cudaStream_t st = env ? (cudaStream_t)env->stream_kernel_faces_ : nullptr;
  double* buf = nullptr;
  int rc;
  if ((rc = msb::cuda_check(cudaMallocAsync(&buf, sizeof(double) * (2 * msb::kNormBlocks + 2), st), "norms alloc")))
    return rc;
  msb::norms_partial_kernel<<<msb::kNormBlocks, msb::kNormThreads, 0, st>>>(vi_d, vo_d, n, buf);
  msb::norms_final_kernel<<<1, msb::kNormThreads, 0, st>>>(buf, msb::kNormBlocks, buf + 2 * msb::kNormBlocks);
  double out[2] = {0, 0};
  rc = msb::cuda_check(cudaMemcpyAsync(out, buf + 2 * msb::kNormBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, st),
                       "norms copy");
  cudaFreeAsync(buf, st);
  if (!rc) rc = msb::cuda_check(cudaStreamSynchronize(st), "norms");
  if (rc) return rc;
  *normsq = out[0];
  *normsqdiff = out[1];
  return MSB_OK;
}

extern "C" int msb_initialize_state_slice_device(double* v_d, Dimensions dims, int ie_base, Env* env) {
  cudaStream_t st = env ? (cudaStream_t)env->stream_kernel_faces_ : nullptr;
  if (dims.nm <= 0) return msb::set_error(MSB_ERR_ARG, "invalid nm");
  if (ie_base < 0) return msb::set_error(MSB_ERR_ARG, "ie_base must be >= 0");
  msb::init_state_kernel<<<148 * 8, 256, 0, st>>>(v_d, dims.ncell_x, dims.ncell_y, dims.ncell_z, dims.ne, dims.nm,
                                                 ie_base);
  return msb::cuda_check(cudaGetLastError(), "init state launch");
}

extern "C" int msb_initialize_state_device(double* v_d, Dimensions dims, Env* env) {
  return msb_initialize_state_slice_device(v_d, dims, 0, env);
}

extern "C" long long msb_schedule_tasks(int nx, int ny, int nz, int ne, int tx, int ty, int gp_block, int* out,
                                        long long max_tasks) {
  msb::Schedule s;
  const int rc = msb::build_schedule(nx, ny, nz, (ne + 1) / 2, tx, ty, gp_block, s);
  if (rc) return rc;
  const long long n = s.ntask();
  if (out) memcpy(out, s.rec.data(), (size_t)(n < max_tasks ? n : max_tasks) * MSB_TASK_INTS * sizeof(int));
  return n;
}
