// Padded internal layout of the PCG fields, and the TMA bulk-copy / mbarrier
// primitives the stencil pipeline uses.
//
// Every nodal or element field a solve touches lives, inside the workspace, as
// columns of P "slots" (P a multiple of 16): node (c, y) is slot c*P + y + LEAD,
// element (ex, ey) is slot ex*P + ey + LEAD. Slots outside the grid rows are
// zero, so stencils need no y-boundary tests, and every column window a CTA
// stages starts on a 16-byte boundary, as cp.async.bulk requires.
// The caller's arrays keep the reference's compact numbering; they are packed
// into this layout once per solve and unpacked at the end.
#pragma once

#include "common.cuh"

namespace tpo {

constexpr int LEAD = 16;                  // zero slots before row 0 of every column
constexpr int RPW = 30;                   // output rows per warp (lanes 1..30)
constexpr int WPC = 4;                    // warps per stencil CTA
constexpr int RPC = RPW * WPC;            // output rows per stencil CTA (120)
constexpr int N_WIN = 124;                // node slots staged per column
constexpr int N_OFF = LEAD - 2;           // node window = slots [Y0+N_OFF, +N_WIN)
constexpr int M_WIN = 144;                // mask bytes staged per column

// element window per storage type: slots [Y0 + E_OFF, + E_WIN)
template <typename T> struct EWin;
template <> struct EWin<double> { static constexpr int OFF = LEAD - 2, N = 124; };
template <> struct EWin<float> { static constexpr int OFF = LEAD - 4, N = 128; };

__host__ __device__ inline int pad_pitch(int ny) {
  const int nbx = (ny + 1 + RPC - 1) / RPC;
  const int y0_last = RPC * (nbx - 1);
  // largest slot any CTA stages: the mask window, start <= Y0+LEAD-8, 144 bytes
  return ((y0_last + LEAD + 136 + 16) + 15) / 16 * 16;
}
__device__ __forceinline__ size_t pslot(int c, int y, int P) { return (size_t)c * P + y + LEAD; }

// -------------------------------------------------------------- pack / unpack
// compact node vector (reference numbering, FP64) -> padded T (zero pads)
template <typename T>
__global__ void k_pack_nodes(int nx, int ny, int P, const double *__restrict__ src,
                             T *__restrict__ dst) {
  const size_t total = (size_t)(nx + 1) * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / P), j = (int)(i % P) - LEAD;
    double vx = 0.0, vy = 0.0;
    if (j >= 0 && j <= ny) {
      const size_t n = (size_t)c * (ny + 1) + j;
      vx = src[2 * n];
      vy = src[2 * n + 1];
    }
    dst[2 * i] = (T)vx;
    dst[2 * i + 1] = (T)vy;
  }
}

__device__ __forceinline__ void unpack_nodes_run(int nx, int ny, int P,
                                                 const double *__restrict__ src,
                                                 double *__restrict__ dst, int bx, int gx) {
  const size_t total = (size_t)(nx + 1) * (ny + 1);
  for (size_t n = bx * (size_t)blockDim.x + threadIdx.x; n < total;
       n += (size_t)gx * blockDim.x) {
    const int c = (int)(n / (ny + 1)), y = (int)(n % (ny + 1));
    const size_t i = (size_t)c * P + y + LEAD;
    dst[2 * n] = src[2 * i];
    dst[2 * n + 1] = src[2 * i + 1];
  }
}
__global__ void k_unpack_nodes(int nx, int ny, int P, const double *__restrict__ src,
                               double *__restrict__ dst) {
  unpack_nodes_run(nx, ny, P, src, dst, blockIdx.x, gridDim.x);
}

template <typename T>
__global__ void k_unpack_nodes_t(int nx, int ny, int P, const T *__restrict__ src,
                                 T *__restrict__ dst) {
  const size_t total = (size_t)(nx + 1) * (ny + 1);
  for (size_t n = blockIdx.x * (size_t)blockDim.x + threadIdx.x; n < total;
       n += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(n / (ny + 1)), y = (int)(n % (ny + 1));
    const size_t i = (size_t)c * P + y + LEAD;
    dst[2 * n] = src[2 * i];
    dst[2 * n + 1] = src[2 * i + 1];
  }
}

template <typename T>
__global__ void k_pack_nodes_t(int nx, int ny, int P, const T *__restrict__ src,
                               T *__restrict__ dst) {
  const size_t total = (size_t)(nx + 1) * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / P), j = (int)(i % P) - LEAD;
    T vx = T(0), vy = T(0);
    if (j >= 0 && j <= ny) {
      const size_t n = (size_t)c * (ny + 1) + j;
      vx = src[2 * n];
      vy = src[2 * n + 1];
    }
    dst[2 * i] = vx;
    dst[2 * i + 1] = vy;
  }
}

__global__ void k_pack_mask(int nx, int ny, int P, const uint8_t *__restrict__ src,
                            uint8_t *__restrict__ dst) {
  const size_t total = (size_t)(nx + 1) * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
       i += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / P), j = (int)(i % P) - LEAD;
    dst[i] = (j >= 0 && j <= ny) ? src[(size_t)c * (ny + 1) + j] : (uint8_t)0;
  }
}

// ------------------------------------------------------------ TMA primitives
__device__ __forceinline__ unsigned smem_u32(const void *p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// one arrival, announcing `bytes` of incoming transaction traffic
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// One poll of a phase. A thread whose phase is not complete is suspended until
// it completes or kSuspendNs elapse, so waiting warps do not spin through
// issue slots that the other warps of the SM need.
constexpr unsigned kSuspendNs = 20000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendNs)
      : "memory");
  return ok != 0;
}
// TMA bulk copy global -> shared (non-tensor, no multicast); completion is
// signalled on `bar` as transaction bytes. dst, src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes,
                                         uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase. Returns false (and records the failure
// in *err) if the phase has not completed after kLimit polls of at most
// kSuspendNs each (about 1.3 s in all).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *err,
                                                  int code) {
  constexpr int kLimit = 1 << 16;
  for (int i = 0; i < kLimit; ++i)
    if (mbar_try_wait(bar, parity)) return true;
  if (err) atomicExch(err, code);
  return false;
}

}  // namespace tpo
