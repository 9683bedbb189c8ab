// esg_probe.cu -- integer-pipe peak probe for the roofline of the scorer.
//
// The scorer's kernels run on the integer ALUs (PRMT, the DPX
// VIADDMNMX/VIMNMX family, packed 16-bit adds), not on tensor cores or HBM,
// so their roofline is the chip's integer lane-op rate.  That rate is not in
// any vendor table we can read here, so it is measured: each probe kernel
// runs a dependency-free, unrolled stream of one instruction kind (eight
// independent chains per thread, 64 warps per SM) over every SM, timed with
// CUDA events and with the SM clock counter so rates can be quoted per
// second and per SM clock.
#include <cstdint>
#include <cuda_runtime.h>

namespace {

enum Op { kIadd = 0, kImax, kLop3, kPrmt, kAdd16x2, kMax16x2, kViaddmax16x2, kVimax3_16x2,
          kViaddmax32, kNumOps };

template <int OP>
__device__ __forceinline__ uint32_t op(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t d;
  if constexpr (OP == kIadd) {
    asm volatile("add.s32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(y));
  } else if constexpr (OP == kImax) {
    asm volatile("max.s32 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(y));
  } else if constexpr (OP == kLop3) {
    asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(d) : "r"(x), "r"(y), "r"(z));
  } else if constexpr (OP == kPrmt) {
    asm volatile("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(x), "r"(y), "r"(z));
  } else if constexpr (OP == kAdd16x2) {
    asm volatile("add.s16x2 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(y));
  } else if constexpr (OP == kMax16x2) {
    asm volatile("max.s16x2 %0, %1, %2;" : "=r"(d) : "r"(x), "r"(y));
  } else if constexpr (OP == kViaddmax16x2) {
    d = __viaddmax_s16x2(x, y, z);
  } else if constexpr (OP == kVimax3_16x2) {
    d = __vimax3_s16x2(x, y, z);
  } else {
    d = (uint32_t)__viaddmax_s32((int)x, (int)y, (int)z);
  }
  return d;
}

constexpr int kChains = 8;
constexpr int kUnroll = 32;

template <int OP>
__global__ void __launch_bounds__(256) probe(uint32_t* out, int iters, uint32_t seed,
                                             unsigned long long* cycles) {
  uint32_t c[kChains];
  const uint32_t y = seed ^ threadIdx.x, z = seed * 3u + blockIdx.x;
#pragma unroll
  for (int k = 0; k < kChains; ++k) c[k] = seed + (uint32_t)(k * 7919) + threadIdx.x;
  const long long t0 = clock64();
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
#pragma unroll
      for (int k = 0; k < kChains; ++k) c[k] = op<OP>(c[k], y, z);
    }
  }
  const long long t1 = clock64();
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) acc ^= c[k];
  if (acc == 0x12345679u) out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
  if (threadIdx.x == 0) atomicMax(cycles, (unsigned long long)(t1 - t0));
}

template <int OP>
cudaError_t run_one(int blocks, int iters, float* ms, unsigned long long* cyc, uint32_t* d_out,
                    unsigned long long* d_cyc, cudaStream_t st) {
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  probe<OP><<<blocks, 256, 0, st>>>(d_out, 2, 1u, d_cyc);  // warm-up
  cudaMemsetAsync(d_cyc, 0, 8, st);
  cudaEventRecord(a, st);
  probe<OP><<<blocks, 256, 0, st>>>(d_out, iters, 1u, d_cyc);
  cudaEventRecord(b, st);
  cudaError_t e = cudaEventSynchronize(b);
  cudaEventElapsedTime(ms, a, b);
  cudaMemcpy(cyc, d_cyc, 8, cudaMemcpyDeviceToHost);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

}  // namespace

extern "C" {

// Runs every probe on `device`; per op k writes lane_ops_per_s[k] (32-bit
// lane operations per second over the whole GPU) and lane_ops_per_clk_sm[k]
// (per SM per SM-clock cycle, from clock64).  Returns 0 or a cudaError_t.
int esg_probe_int_peak(int device, int iters, double* lane_ops_per_s,
                       double* lane_ops_per_clk_sm, int* n_ops, int* sm_count) {
  if (cudaSetDevice(device) != cudaSuccess) return (int)cudaGetLastError();
  cudaDeviceProp p{};
  cudaGetDeviceProperties(&p, device);
  *sm_count = p.multiProcessorCount;
  *n_ops = kNumOps;
  const int blocks = p.multiProcessorCount * 8;  // 64 warps per SM
  uint32_t* d_out = nullptr;
  unsigned long long* d_cyc = nullptr;
  cudaMalloc(&d_out, (size_t)blocks * 256 * 4);
  cudaMalloc(&d_cyc, 8);
  cudaStream_t st;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  float ms[kNumOps] = {};
  unsigned long long cyc[kNumOps] = {};
  cudaError_t e = cudaSuccess;
  if (!e) e = run_one<kIadd>(blocks, iters, &ms[0], &cyc[0], d_out, d_cyc, st);
  if (!e) e = run_one<kImax>(blocks, iters, &ms[1], &cyc[1], d_out, d_cyc, st);
  if (!e) e = run_one<kLop3>(blocks, iters, &ms[2], &cyc[2], d_out, d_cyc, st);
  if (!e) e = run_one<kPrmt>(blocks, iters, &ms[3], &cyc[3], d_out, d_cyc, st);
  if (!e) e = run_one<kAdd16x2>(blocks, iters, &ms[4], &cyc[4], d_out, d_cyc, st);
  if (!e) e = run_one<kMax16x2>(blocks, iters, &ms[5], &cyc[5], d_out, d_cyc, st);
  if (!e) e = run_one<kViaddmax16x2>(blocks, iters, &ms[6], &cyc[6], d_out, d_cyc, st);
  if (!e) e = run_one<kVimax3_16x2>(blocks, iters, &ms[7], &cyc[7], d_out, d_cyc, st);
  if (!e) e = run_one<kViaddmax32>(blocks, iters, &ms[8], &cyc[8], d_out, d_cyc, st);
  const double ops = (double)blocks * 256 * (double)iters * kUnroll * kChains;
  for (int k = 0; k < kNumOps; ++k) {
    lane_ops_per_s[k] = ms[k] > 0 ? ops / (ms[k] * 1e-3) : 0;
    // cycles is the slowest block's span; blocks per SM run concurrently
    lane_ops_per_clk_sm[k] = cyc[k] ? ops / ((double)cyc[k] * p.multiProcessorCount) : 0;
  }
  cudaFree(d_out);
  cudaFree(d_cyc);
  cudaStreamDestroy(st);
  return (int)e;
}

const char* esg_probe_op_name(int k) {
  static const char* names[kNumOps] = {"iadd32", "imax32", "lop3", "prmt", "add16x2",
                                       "max16x2", "viaddmax16x2", "vimax3_16x2", "viaddmax32"};
  return (k >= 0 && k < kNumOps) ? names[k] : "";
}

}  // extern "C"
