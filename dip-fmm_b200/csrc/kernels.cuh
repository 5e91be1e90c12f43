// Device helpers shared by the evaluator kernels.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cdfmm_b200 {

// 1 / (4 pi) in FP32 (the kernel constant of G(r) = 1 / (4 pi |r|)).
constexpr float kInvFourPiF = 0.0795774715459476678844418816862571810F;

// 1/k for k = 0..15 (entry 0 unused), correctly rounded FP32: monomial
// recurrences d^(k+1)/(k+1)! = d^k/k! * d * (1/(k+1)) multiply instead of divide.
__constant__ constexpr float kInvInt[16] = {
    0.0F,         1.0F,        0.5F,         1.0F / 3.0F,  0.25F,       0.2F,        1.0F / 6.0F, 1.0F / 7.0F,
    0.125F,       1.0F / 9.0F, 0.1F,         1.0F / 11.0F, 1.0F / 12.0F, 1.0F / 13.0F, 1.0F / 14.0F, 1.0F / 15.0F};

__host__ __device__ inline int basis_size_d(int p) { return p < 0 ? 0 : (p + 1) * (p + 2) * (p + 3) / 6; }

// Position of multi-index (a, b, c) in the total-degree basis.
__host__ __device__ inline int rank3(int a, int b, int c) {
  const int d = a + b + c;
  return d * (d + 1) * (d + 2) / 6 + a * (d + 1) - a * (a - 1) / 2 + b;
}

__host__ __device__ inline int level_offset_d(int level) { return ((1 << (3 * level)) - 1) / 7; }

// Bit dilation of a 10-bit coordinate: bit b moves to bit 3b (the
// shift-and-mask "part 1 by 2" construction), and its inverse.
__host__ __device__ inline uint32_t dilate3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}
__host__ __device__ inline uint32_t undilate3(uint32_t v) {
  v &= 0x09249249u;
  v = (v | (v >> 2)) & 0x030c30c3u;
  v = (v | (v >> 4)) & 0x0300f00fu;
  v = (v | (v >> 8)) & 0x030000ffu;
  v = (v | (v >> 16)) & 0x000003ffu;
  return v;
}

__host__ __device__ inline uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return dilate3(x) | (dilate3(y) << 1) | (dilate3(z) << 2);
}

// Lets `kernel` use all opt-in shared memory left after its static shared
// memory.  Returns false (and clears the runtime's last error) on failure.
template <typename Kernel> inline bool allow_dynamic_smem(Kernel *kernel, size_t optin) {
  cudaFuncAttributes attr{};
  if (cudaFuncGetAttributes(&attr, kernel) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const size_t room = optin > attr.sharedSizeBytes ? optin - attr.sharedSizeBytes : 0;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(room)) !=
      cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return true;
}

// Asks for the largest shared-memory carve-out of the unified L1 / shared
// memory whenever `kernel` runs: kernels that share an SM must run under one
// carve-out, and one sized for a smaller footprint would leave no room for
// the other kernel's CTA.
template <typename Kernel> inline void prefer_max_shared_carveout(Kernel *kernel) {
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           static_cast<int>(cudaSharedmemCarveoutMaxShared)) != cudaSuccess)
    cudaGetLastError();
}

__host__ __device__ inline void demorton3(uint32_t m, int &x, int &y, int &z) {
  x = static_cast<int>(undilate3(m));
  y = static_cast<int>(undilate3(m >> 1));
  z = static_cast<int>(undilate3(m >> 2));
}

#ifdef __CUDACC__
// 16-byte asynchronous global -> shared copy (bypasses registers, so many
// copies of one thread are in flight at once), its commit and wait.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem))),
               "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Monomials d^mu / mu! for every |mu| <= q, written into out[rank(mu)].
__device__ inline void monomials(float dx, float dy, float dz, int q, float *out) {
  float xa = 1.0F;
  for (int a = 0; a <= q; ++a) {
    float xb = xa;
    for (int b = 0; a + b <= q; ++b) {
      float xc = xb;
      for (int c = 0; a + b + c <= q; ++c) {
        out[rank3(a, b, c)] = xc;
        xc = xc * dz * kInvInt[c + 1];
      }
      xb = xb * dy * kInvInt[b + 1];
    }
    xa = xa * dx * kInvInt[a + 1];
  }
}

// The monomials of monomials() whose x-degree a belongs to part r of 4:
// a = r, 7 - r, 8 + r, 15 - r, ... (part 0 takes a = 0, the largest group;
// for q = 6 the parts hold 28, 22, 18 and 16 of the 84 monomials).  Four
// threads per point share the work; each runs the serial recurrences, so the
// values are bit-identical to monomials().  zero: store zeros instead.
__device__ inline void monomials_part(float dx, float dy, float dz, int q, float *out, int stride, int r, bool zero) {
  for (int a0 = 0; a0 <= q; a0 += 8) {
    for (int h = 0; h < 2; ++h) {
      const int a = a0 + (h == 0 ? r : 7 - r);
      if (a > q) continue;
      float xa = 1.0F;
      for (int i = 0; i < a; ++i) xa = xa * dx * kInvInt[i + 1];
      float xb = xa;
      for (int b = 0; a + b <= q; ++b) {
        float xc = xb;
        for (int c = 0; a + b + c <= q; ++c) {
          out[rank3(a, b, c) * stride] = zero ? 0.0F : xc;
          xc = xc * dz * kInvInt[c + 1];
        }
        xb = xb * dy * kInvInt[b + 1];
      }
    }
  }
}

#endif

} // namespace cdfmm_b200
