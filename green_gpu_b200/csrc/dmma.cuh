// Device helpers of the FP64 tensor-core kernels: the DMMA instruction (mma.sync m8n8k4 f64)
// and 16-byte asynchronous global->shared copies.
//
// Fragment layouts of m8n8k4 .row.col f64 (lane = 4 g + k, g = lane / 4, k = lane % 4):
//   A (8 x 4): one element, A[g][k];   B (4 x 8): one element, B[k][g];
//   C (8 x 8): two elements, C[g][2k] and C[g][2k + 1].
#pragma once

namespace gg {

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// 16-byte copy; with valid = false the destination is zero-filled and nothing is read
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid = true) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

}  // namespace gg
